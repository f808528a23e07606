// Launches of the pressure-Poisson axis transforms (the device code is in transform.cuh).
#include "transform.cuh"

namespace aero {


template <typename T, int N, int LOG2L_>
cudaError_t launch_pow2_tile(const TransformParams<T> &P, cudaStream_t s) {
  using G = Pow2Tile<T, N, LOG2L_>;
  static bool configured = false;
  if (!configured) {
    const cudaError_t e = cudaFuncSetAttribute(pow2_transform_kernel<T, N, LOG2L_>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::SMEM);
    if (e != cudaSuccess) return e;
    configured = true;
  }
  dim3 grid;
  if (P.axis == 0)
    grid = dim3((unsigned)(((size_t)P.nz * P.ny + G::L - 1) / G::L), 1, 1);
  else
    grid = dim3((unsigned)((P.nx + G::L - 1) / G::L), (unsigned)(P.axis == 1 ? P.nz : P.ny), 1);
  (void)aero::launch_k(pow2_transform_kernel<T, N, LOG2L_>, grid, 256, G::SMEM, s, P);
  return cudaGetLastError();
}

// The widest tile, unless that leaves the pass a handful of blocks (a 2D grid of 256 x 128
// gets 8): then two-line tiles spread its lines over more SMs.  Larger grids keep a wide
// tile, whose blocks do more work each (and concurrent solves fill the GPU anyway); for axes
// of 64..256 cells half the widest one: the passes wait on their tile loads, and twice the
// blocks (half the shared memory each) overlap more of them (256 x 128 x 128: 0.124 -> 0.119 ms
// per solve, the step 2.7 % faster; a quarter of the widest tile was slower, 0.132 ms).
template <typename T, int N>
cudaError_t launch_pow2(const TransformParams<T> &P, cudaStream_t s) {
  const size_t lines = P.axis == 0 ? (size_t)P.nz * P.ny : (size_t)P.nx * (P.axis == 1 ? P.nz : P.ny);
  const size_t blocks = (lines + Pow2Tile<T, N>::L - 1) / Pow2Tile<T, N>::L;
  if (blocks < 32 && Pow2Tile<T, N>::L > 2) return launch_pow2_tile<T, N, 1>(P, s);
  if constexpr (N >= 64 && N <= 256) return launch_pow2_tile<T, N, Pow2Tile<T, N>::LOG2L - 1>(P, s);
  return launch_pow2_tile<T, N, -1>(P, s);
}

bool transform_tiled(int n) { return fft::tile_len(n); }

// Tables: twiddles e^{-2 pi i m / n}, DCT post-twiddles s_k e^{-i pi k / 2n}, cos / sin of
// pi k / 2n, eigenvalues (2 cos(pi k / n) - 2) / h^2 or (2 cos(2 pi k / n) - 2) / h^2,
// and the dense orthonormal matrix of poisson.py:74-90 for lengths the FFT does not take.
template <typename T>
__global__ void axis_tables_kernel(int n, int kind, int dense, double h, T *tw, T *post, T *cs, double *lam, T *mat) {
  aero::pdl_wait();
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nthr = gridDim.x * blockDim.x;
  for (int m = tid; m < n; m += nthr) {
    double s, c;
    sincospi(2.0 * m / n, &s, &c);
    tw[2 * m] = T(c);
    tw[2 * m + 1] = T(-s);
    sincospi(0.5 * m / n, &s, &c);
    const double sk = (m == 0) ? sqrt(1.0 / n) : sqrt(2.0 / n);
    post[2 * m] = T(sk * c);
    post[2 * m + 1] = T(-sk * s);
    cs[2 * m] = T(c);
    cs[2 * m + 1] = T(s);
    const double arg = kind == 1 ? 2.0 * m / n : (double)m / n;
    lam[m] = (2.0 * cospi(arg) - 2.0) / (h * h);
  }
  if (dense) {
    for (int e = tid; e < n * n; e += nthr) {
      const int k = e / n, j = e % n;
      double v;
      if (kind == 1) {
        double s, c;
        sincospi(2.0 * (double)(((long long)k * j) % n) / n, &s, &c);
        v = (c + s) / sqrt((double)n);
      } else {
        v = cospi((double)k * (j + 0.5) / n) * sqrt(2.0 / n);
        if (k == 0) v *= sqrt(0.5);
      }
      mat[e] = T(v);
    }
  }
}

template <typename T>
size_t transform_smem_bytes(int n, int L) {
  return (((size_t)n * (L + 1) * sizeof(T) + 15) & ~size_t(15)) + 2 * (size_t)n * (L / 2) * 2 * sizeof(T);
}

template <typename T>
cudaError_t launch_transform(const TransformParams<T> &P, cudaStream_t s) {
  if (P.A.method == 0 && transform_tiled(P.A.n)) {
    switch (P.A.n) {
      case 8: return launch_pow2<T, 8>(P, s);
      case 16: return launch_pow2<T, 16>(P, s);
      case 32: return launch_pow2<T, 32>(P, s);
      case 64: return launch_pow2<T, 64>(P, s);
      case 128: return launch_pow2<T, 128>(P, s);
      case 256: return launch_pow2<T, 256>(P, s);
      case 512: return launch_pow2<T, 512>(P, s);
      case 1024: return launch_pow2<T, 1024>(P, s);
      case 2048: return launch_pow2<T, 2048>(P, s);
      case 12: return launch_pow2<T, 12>(P, s);
      case 24: return launch_pow2<T, 24>(P, s);
      case 48: return launch_pow2<T, 48>(P, s);
      case 96: return launch_pow2<T, 96>(P, s);
      case 192: return launch_pow2<T, 192>(P, s);
      case 384: return launch_pow2<T, 384>(P, s);
      case 768: return launch_pow2<T, 768>(P, s);
      default: return launch_pow2<T, 1536>(P, s);
    }
  }
  if (P.fuse_div || P.p_acc) return cudaErrorInvalidValue;  // fusions exist on tiled axes only
  const size_t smem = transform_smem_bytes<T>(P.A.n, P.L);
  static size_t set_to = 0;
  if (smem > set_to) {
    cudaError_t e = cudaFuncSetAttribute(line_transform_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)std::max<size_t>(smem, 48 * 1024));
    if (e != cudaSuccess) return e;
    set_to = std::max<size_t>(smem, 48 * 1024);
  }
  dim3 grid;
  if (P.axis == 0) {
    grid = dim3((unsigned)(((size_t)P.nz * P.ny + P.L - 1) / P.L), 1, 1);
  } else {
    grid = dim3((unsigned)((P.nx + P.L - 1) / P.L), (unsigned)(P.axis == 1 ? P.nz : P.ny), 1);
  }
  (void)aero::launch_k(line_transform_kernel<T>, grid, 256, smem, s, P);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_axis_tables(int n, int kind, int dense, double h, T *tw, T *post, T *cs, double *lam, T *mat,
                               cudaStream_t s) {
  (void)aero::launch_k(axis_tables_kernel<T>, 64, 256, 0, s, n, kind, dense, h, tw, post, cs, lam, mat);
  return cudaGetLastError();
}

template size_t transform_smem_bytes<float>(int, int);
template size_t transform_smem_bytes<double>(int, int);
template cudaError_t launch_transform<float>(const TransformParams<float> &, cudaStream_t);
template cudaError_t launch_transform<double>(const TransformParams<double> &, cudaStream_t);
template cudaError_t launch_axis_tables<float>(int, int, int, double, float *, float *, float *, double *, float *,
                                               cudaStream_t);
template cudaError_t launch_axis_tables<double>(int, int, int, double, double *, double *, double *, double *,
                                                double *, cudaStream_t);

}  // namespace aero
