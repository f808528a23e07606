// Device code of the pressure-Poisson axis transforms (used by poisson.cu for the plans' launches
// and by the batched 2D sweep's persistent kernel in ns2d.cu): the runtime-table line
// transform and the compile-time power-of-two tile transform, each as a body over an explicit
// tile (bx, by) with its shared memory, and as a kernel.
#pragma once
// Exact pressure-Poisson solve on the cell-centred grid (Aerolume ns3d/poisson.py:93-157).
//
// The reference applies dense orthonormal eigenbases per axis with IEEE FP32 GEMMs:
// DCT-II for homogeneous Neumann axes (poisson.py:74-81), the discrete Hartley
// transform for periodic ones (poisson.py:84-90), divides by the eigenvalue sum and
// transforms back.  Here each axis transform is an O(n log n) shared-memory FFT:
//
//   DCT-II   Makhoul's even/odd reordering, a length-n complex FFT carrying two real
//            lines at once (real and imaginary parts), then X_k = s_k Re(e^{-i pi k/2n} V_k)
//   DCT-III  the transpose: V_k = e^{i pi k/2n} (Y_k - i Y_{n-k}) / 2 (V_0 = Y_0), inverse
//            FFT, un-reordering
//   DHT      H_k = (Re F_k - Im F_k) / sqrt(n) (an involution: forward = inverse)
//
// The FFT is a Stockham autosort with radix 4, 2 and 3 passes (n = 2^a 3^b): compile-time
// tiles for n = 2^a and 3 * 2^a, run-time stage tables for the other 2^a 3^b; any other
// length falls back to the dense orthonormal matrix in shared memory.  The z pass runs
// forward transform, division by lambda_x + lambda_y + lambda_z (zero mode dropped) and
// inverse transform in one kernel.
#include "fft_tile.cuh"
#include "ns3d.cuh"

namespace aero {

template <typename T>
struct Cx {
  T x, y;
};

template <typename T>
__device__ __forceinline__ Cx<T> cmul(Cx<T> a, Cx<T> b) {
  return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}

// Stockham passes over P interleaved complex lines of length n (element m of line p at
// m * P + p).  Returns the buffer holding the result.
template <typename T>
__device__ Cx<T> *fft_lines(Cx<T> *a, Cx<T> *b, int n, int P, const AxisTables<T> &A, bool inverse) {
  const int nthr = blockDim.x, tid = threadIdx.x;
  const Cx<T> *tw = reinterpret_cast<const Cx<T> *>(A.tw);
  Cx<T> *in = a, *out = b;
  int Ns = 1;
  const T sgn = inverse ? T(1) : T(-1);
  for (int s = 0; s < A.nfac; ++s) {
    const int r = A.fac[s], m = n / r, stride = n / (Ns * r);
    for (int item = tid; item < m * P; item += nthr) {
      const int p = item % P, jj = item / P;
      const int k = jj % Ns;
      Cx<T> v[4];
#pragma unroll
      for (int t = 0; t < 4; ++t)
        if (t < r) v[t] = in[(jj + t * m) * P + p];
#pragma unroll
      for (int t = 1; t < 4; ++t)
        if (t < r) {
          Cx<T> w = tw[t * k * stride];
          if (inverse) w.y = -w.y;
          v[t] = cmul(v[t], w);
        }
      Cx<T> V[4];
      if (r == 4) {
        const Cx<T> a0 = {v[0].x + v[2].x, v[0].y + v[2].y}, a1 = {v[0].x - v[2].x, v[0].y - v[2].y};
        const Cx<T> a2 = {v[1].x + v[3].x, v[1].y + v[3].y};
        const Cx<T> d = {v[1].x - v[3].x, v[1].y - v[3].y};
        const Cx<T> a3 = {-sgn * d.y, sgn * d.x};  // sgn * i * d
        V[0] = {a0.x + a2.x, a0.y + a2.y};
        V[2] = {a0.x - a2.x, a0.y - a2.y};
        V[1] = {a1.x + a3.x, a1.y + a3.y};
        V[3] = {a1.x - a3.x, a1.y - a3.y};
      } else if (r == 2) {
        V[0] = {v[0].x + v[1].x, v[0].y + v[1].y};
        V[1] = {v[0].x - v[1].x, v[0].y - v[1].y};
      } else {  // r == 3
        const T h3 = T(0.866025403784438646763723170752936183);
        const Cx<T> t1 = {v[1].x + v[2].x, v[1].y + v[2].y};
        const Cx<T> t2 = {v[0].x - T(0.5) * t1.x, v[0].y - T(0.5) * t1.y};
        const Cx<T> d = {v[1].x - v[2].x, v[1].y - v[2].y};
        const Cx<T> t3 = {-sgn * h3 * d.y, sgn * h3 * d.x};  // sgn * i * (sqrt3/2) * d
        V[0] = {v[0].x + t1.x, v[0].y + t1.y};
        V[1] = {t2.x + t3.x, t2.y + t3.y};
        V[2] = {t2.x - t3.x, t2.y - t3.y};
      }
      const int base = (jj / Ns) * Ns * r + k;
#pragma unroll
      for (int t = 0; t < 4; ++t)
        if (t < r) out[(base + t * Ns) * P + p] = V[t];
    }
    __syncthreads();
    Cx<T> *tmp = in;
    in = out;
    out = tmp;
    Ns *= r;
  }
  return in;
}

// Makhoul reordering: v[m] = x[perm(m)]
__device__ __forceinline__ int makhoul(int m, int n) { return (2 * m < n) ? 2 * m : 2 * (n - 1 - m) + 1; }

// In place on the real tile R[m * ld + l] (n x L): forward (DCT-II / DHT) or inverse
// (DCT-III / DHT) orthonormal transform of each of the L lines.
template <typename T>
__device__ void transform_tile(T *R, int ld, Cx<T> *C0, Cx<T> *C1, int n, int L, const AxisTables<T> &A,
                               bool inverse) {
  const int nthr = blockDim.x, tid = threadIdx.x;
  const int P = L / 2;
  if (A.method == 1) {  // dense orthonormal matrix
    T *tmp = reinterpret_cast<T *>(C0);
    for (int item = tid; item < n * L; item += nthr) {
      const int l = item % L, k = item / L;
      T s = T(0);
      if (!inverse) {
        for (int m = 0; m < n; ++m) s += __ldg(A.dense + (size_t)k * n + m) * R[m * ld + l];
      } else {
        for (int m = 0; m < n; ++m) s += __ldg(A.dense + (size_t)m * n + k) * R[m * ld + l];
      }
      tmp[k * L + l] = s;
    }
    __syncthreads();
    for (int item = tid; item < n * L; item += nthr) {
      const int l = item % L, k = item / L;
      R[k * ld + l] = tmp[k * L + l];
    }
    __syncthreads();
    return;
  }
  const Cx<T> *post = reinterpret_cast<const Cx<T> *>(A.post);  // DCT: s_k e^{-i pi k / 2n}
  // ---- build the complex input
  for (int item = tid; item < n * P; item += nthr) {
    const int p = item % P, m = item / P;
    Cx<T> z;
    if (A.kind == 1) {  // Hartley: natural order
      z = {R[m * ld + 2 * p], R[m * ld + 2 * p + 1]};
    } else if (!inverse) {  // DCT-II: reorder
      const int src = makhoul(m, n);
      z = {R[src * ld + 2 * p], R[src * ld + 2 * p + 1]};
    } else {  // DCT-III: V_k = e^{i pi k/2n} (Y_k - i Y_{n-k}) / 2, V_0 = Y_0, Y = s X
      const int k = m;
      const Cx<T> e = {A.cs[2 * k], A.cs[2 * k + 1]};  // cos, sin of pi k / 2n
      Cx<T> va, vb;
      if (k == 0) {
        va = {A.s0 * R[2 * p], T(0)};
        vb = {A.s0 * R[2 * p + 1], T(0)};
      } else {
        const T ya = A.s1 * R[k * ld + 2 * p], yra = A.s1 * R[(n - k) * ld + 2 * p];
        const T yb = A.s1 * R[k * ld + 2 * p + 1], yrb = A.s1 * R[(n - k) * ld + 2 * p + 1];
        va = cmul(e, Cx<T>{T(0.5) * ya, -T(0.5) * yra});
        vb = cmul(e, Cx<T>{T(0.5) * yb, -T(0.5) * yrb});
      }
      z = {va.x - vb.y, va.y + vb.x};  // va + i vb
    }
    C0[m * P + p] = z;
  }
  __syncthreads();
  Cx<T> *Z = fft_lines<T>(C0, C1, n, P, A, inverse && A.kind == 0);
  // ---- unpack into R
  for (int item = tid; item < n * P; item += nthr) {
    const int p = item % P, k = item / P;
    if (A.kind == 0 && inverse) {
      const Cx<T> z = Z[k * P + p];  // v_a[k] + i v_b[k]
      const int dst = makhoul(k, n);
      R[dst * ld + 2 * p] = z.x;
      R[dst * ld + 2 * p + 1] = z.y;
    } else {
      const Cx<T> z = Z[k * P + p];
      const Cx<T> zr = Z[((n - k) % n) * P + p];
      const T ar = T(0.5) * (z.x + zr.x), ai = T(0.5) * (z.y - zr.y);   // F_a = (Z_k + conj Z_{n-k}) / 2
      const T br = T(0.5) * (z.y + zr.y), bi = -T(0.5) * (z.x - zr.x);  // F_b = (Z_k - conj Z_{n-k}) / 2i
      T xa, xb;
      if (A.kind == 1) {
        xa = (ar - ai) * A.rsqrt_n;
        xb = (br - bi) * A.rsqrt_n;
      } else {
        const Cx<T> w = post[k];
        xa = w.x * ar - w.y * ai;
        xb = w.x * br - w.y * bi;
      }
      // R is read by other threads (k and n - k) in this loop: write to C1/C0 scratch first
      reinterpret_cast<T *>(Z == C0 ? C1 : C0)[k * L + 2 * p] = xa;
      reinterpret_cast<T *>(Z == C0 ? C1 : C0)[k * L + 2 * p + 1] = xb;
    }
  }
  __syncthreads();
  if (!(A.kind == 0 && inverse)) {
    const T *tmp = reinterpret_cast<const T *>(Z == C0 ? C1 : C0);
    for (int item = tid; item < n * L; item += nthr) {
      const int l = item % L, k = item / L;
      R[k * ld + l] = tmp[k * L + l];
    }
    __syncthreads();
  }
}

// The pass of tile (bx, by) with its shared memory given: line_transform_kernel runs it as
// its own launch, the batched sweep's persistent kernel (sweep2d.cu) as one work item.
template <typename T>
__device__ __forceinline__ void line_transform_body(const TransformParams<T> &P, int bx, int by,
                                                    unsigned char *smem_raw) {
  const int n = P.A.n, L = P.L, ld = L + 1;
  T *R = reinterpret_cast<T *>(smem_raw);
  size_t roff = ((size_t)n * ld * sizeof(T) + 15) & ~size_t(15);
  Cx<T> *C0 = reinterpret_cast<Cx<T> *>(smem_raw + roff);
  Cx<T> *C1 = C0 + (size_t)n * (L / 2);
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  const int tid = threadIdx.x, nthr = blockDim.x;
  // line addressing
  size_t base;
  size_t lstride, estride;
  int nl;
  if (P.axis == 0) {
    const size_t r0 = (size_t)bx * L;
    const size_t rows = (size_t)nz * ny;
    nl = (int)min((size_t)L, rows - r0);
    base = r0 * nx;
    lstride = nx;
    estride = 1;
  } else {
    const int i0 = bx * L;
    nl = min(L, nx - i0);
    if (P.axis == 1) {
      base = (size_t)by * ny * nx + i0;
      estride = nx;
    } else {
      base = (size_t)by * nx + i0;
      estride = (size_t)ny * nx;
    }
    lstride = 1;
  }
  // load (coalesced along whichever index is contiguous)
  for (int e = tid; e < n * L; e += nthr) {
    int m, l;
    if (P.axis == 0) {
      m = e % n;
      l = e / n;
    } else {
      l = e % L;
      m = e / L;
    }
    R[m * ld + l] = (l < nl) ? P.in[base + (size_t)l * lstride + (size_t)m * estride] : T(0);
  }
  __syncthreads();
  if (P.mode == 2) {  // forward, divide by the eigenvalue sum, inverse (z axis)
    transform_tile<T>(R, ld, C0, C1, n, L, P.A, false);
    const int j = by, i0 = bx * L;
    for (int e = tid; e < n * L; e += nthr) {
      const int l = e % L, k = e / L;
      const int i = i0 + l;
      double inv = 0.0;
      if (l < nl) {
        const double lam = P.A.lam[k] + P.lam_y[j] + P.lam_x[i];
        inv = (lam != 0.0) ? 1.0 / lam : 0.0;
        if (k == 0 && j == 0 && i == 0) inv = 0.0;
      }
      R[k * ld + l] = R[k * ld + l] * T(inv);
    }
    __syncthreads();
    transform_tile<T>(R, ld, C0, C1, n, L, P.A, true);
  } else {
    transform_tile<T>(R, ld, C0, C1, n, L, P.A, P.mode == 1);
  }
  for (int e = tid; e < n * L; e += nthr) {
    int m, l;
    if (P.axis == 0) {
      m = e % n;
      l = e / n;
    } else {
      l = e % L;
      m = e / L;
    }
    if (l < nl) P.out[base + (size_t)l * lstride + (size_t)m * estride] = R[m * ld + l];
  }
}

template <typename T>
__global__ void __launch_bounds__(256) line_transform_kernel(const TransformParams<T> P) {
  aero::pdl_wait();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  line_transform_body<T>(P, blockIdx.x, blockIdx.y, smem_raw);
}

// --------------------------------------------------------------------------------------
// Axes of 2^a or 3 * 2^a cells: the compile-time tile transform of fft_tile.cuh
// --------------------------------------------------------------------------------------

struct BlockExec {
  template <class F>
  __device__ __forceinline__ void operator()(F &&f) {
    f((int)threadIdx.x, 256);  // every launch of the transform kernel uses 256 threads
    __syncthreads();
  }
};

// Tile of L = 2^LOG2L_ lines of N cells, N = 2^a or 3 * 2^a (LOG2L_ < 0: the widest tile
// within ~48 KiB).
template <typename T, int N, int LOG2L_ = -1>
struct Pow2Tile {
  static constexpr int LOG2L = LOG2L_ >= 0 ? LOG2L_ : fft::tile_log2L(N, (int)sizeof(T)), L = 1 << LOG2L, LD = L + 1;
  static constexpr size_t TW = (size_t)N * 2 * sizeof(T);                        // twiddles
  static constexpr size_t RB = ((size_t)N * LD * sizeof(T) + 15) & ~size_t(15);  // real tile
  static constexpr size_t CB = (size_t)N * (L / 2) * 2 * sizeof(T);              // one complex buffer
  static constexpr size_t SMEM = TW + RB + 2 * CB;
};

// One axis pass over L lines of N = 2^a or 3 * 2^a cells: x lines are rows (r = k ny + j), y / z lines
// are L consecutive x at fixed k / j.  Mode 0 forward, 1 inverse, 2 forward, division by
// lambda_x + lambda_y + lambda_z (zero mode dropped) and inverse (z axis).
template <typename T, int N, int LOG2L_>
__device__ __forceinline__ void pow2_transform_body(const TransformParams<T> &P, int bx, int by,
                                                    unsigned char *smem_raw) {
  using G = Pow2Tile<T, N, LOG2L_>;
  constexpr int L = G::L, LD = G::LD, LOG2L = G::LOG2L;
  fft::Cx<T> *tw = reinterpret_cast<fft::Cx<T> *>(smem_raw);
  T *R = reinterpret_cast<T *>(smem_raw + G::TW);
  fft::Cx<T> *C0 = reinterpret_cast<fft::Cx<T> *>(smem_raw + G::TW + G::RB);
  fft::Cx<T> *C1 = reinterpret_cast<fft::Cx<T> *>(smem_raw + G::TW + G::RB + G::CB);
  __shared__ long long rowoff[5][L];  // fused divergence: u row, v rows j / j+1, w planes k / k+1
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  const int tid = threadIdx.x;
  constexpr int nthr = 256;  // the launch's block size: loop trip counts are compile-time
  for (int m = tid; m < N; m += nthr) tw[m] = {P.A.tw[2 * m], P.A.tw[2 * m + 1]};
  int nl;
  size_t base, estride;
  if (P.axis == 0) {
    const size_t r0 = (size_t)bx << LOG2L, rows = (size_t)nz * ny;
    nl = (int)min((size_t)L, rows - r0);
    base = r0 * N;
    estride = 1;
    if (P.fuse_div == 2 && tid < nl) {  // 2D: rows r of u (nx + 1 faces) and v (nx cells)
      const long long r = (long long)r0 + tid;
      rowoff[0][tid] = r * (nx + 1);
      rowoff[1][tid] = r * nx;
      rowoff[2][tid] = (r + 1) * nx;
    } else if (P.fuse_div && tid < nl) {
      const long long r = (long long)r0 + tid;
      const int k = (int)(r / ny), j = (int)(r - (long long)k * ny);
      rowoff[0][tid] = r * (nx + 1);
      rowoff[1][tid] = ((long long)k * (ny + 1) + j) * nx;
      rowoff[2][tid] = (P.py && j == ny - 1) ? (long long)k * (ny + 1) * nx : rowoff[1][tid] + nx;
      rowoff[3][tid] = ((long long)k * ny + j) * nx;
      rowoff[4][tid] = (P.pz && k == nz - 1) ? (long long)j * nx : rowoff[3][tid] + (long long)ny * nx;
    }
  } else {
    const int i0 = bx << LOG2L;
    nl = min(L, nx - i0);
    base = P.axis == 1 ? (size_t)by * ny * nx + i0 : (size_t)by * nx + i0;
    estride = P.axis == 1 ? (size_t)nx : (size_t)ny * nx;
  }
  __syncthreads();
  // ---- load (coalesced along whichever index is contiguous)
  if (P.axis == 0) {
    for (int e = tid; e < N * L; e += nthr) {
      const int m = e % N, l = e / N;  // constant N: shifts / multiplications
      T val = T(0);
      if (l < nl) {
        if (P.fuse_div == 2) {  // 2D: ((u_{i+1} - u_i) + v_{j+1}) - v_j (ns2d/core.py:620-622)
          const T *ur = P.uh + rowoff[0][l];
          val = (((ur[m + 1] - ur[m]) + P.vh[rowoff[2][l] + m]) - P.vh[rowoff[1][l] + m]) * P.inv_h;
        } else if (P.fuse_div) {  // div(uh) of the stage velocity (ns3d/core.py:577-579)
          const T *ur = P.uh + rowoff[0][l];
          const T u1 = (P.px && m == N - 1) ? ur[0] : ur[m + 1];
          val = ((u1 - ur[m]) + (P.vh[rowoff[2][l] + m] - P.vh[rowoff[1][l] + m]) +
                 (P.wh[rowoff[4][l] + m] - P.wh[rowoff[3][l] + m])) *
                P.inv_h;
        } else {
          val = P.in[base + (size_t)l * N + m];
        }
      }
      R[m * LD + l] = val;
    }
  } else {
    for (int e = tid; e < N * L; e += nthr) {
      const int l = e & (L - 1), m = e >> LOG2L;
      R[m * LD + l] = (l < nl) ? P.in[base + l + (size_t)m * estride] : T(0);
    }
  }
  __syncthreads();
  const fft::AxisView<T> A{tw, reinterpret_cast<const fft::Cx<T> *>(P.A.post),
                           reinterpret_cast<const fft::Cx<T> *>(P.A.cs), P.A.s0, P.A.s1, P.A.rsqrt_n, P.A.kind};
  BlockExec ex;
  if (P.mode == 2) {
    fft::transform_tile<T, N, LOG2L>(R, C0, C1, tw, A, false, ex);
    const int j = by, i0 = bx << LOG2L;
    for (int e = tid; e < N * L; e += nthr) {
      const int l = e & (L - 1), k = e >> LOG2L;
      const int i = i0 + l;
      double inv = 0.0;
      if (l < nl) {
        const double lam = P.A.lam[k] + P.lam_y[j] + P.lam_x[i];
        inv = (lam != 0.0) ? 1.0 / lam : 0.0;
        if (k == 0 && j == 0 && i == 0) inv = 0.0;
      }
      R[k * LD + l] = R[k * LD + l] * T(inv);
    }
    __syncthreads();
    fft::transform_tile<T, N, LOG2L>(R, C0, C1, tw, A, true, ex);
  } else {
    fft::transform_tile<T, N, LOG2L>(R, C0, C1, tw, A, P.mode == 1, ex);
  }
  // ---- store
  if (P.axis == 0) {
    const T rdt = (P.p_acc && P.acc_mode == 2) ? T(1) / *P.dt : T(1);
    for (int e = tid; e < N * L; e += nthr) {
      const int m = e % N, l = e / N;  // constant N: shifts / multiplications
      if (l >= nl) continue;
      const size_t g = base + (size_t)l * N + m;
      const T psi = R[m * LD + l];
      P.out[g] = psi;
      if (P.p_acc) {  // step-averaged pressure (core.py:874-875)
        if (P.acc_mode == 0) {
          P.p_acc[g] = psi * P.wgt;
        } else {
          const T sum = P.p_acc[g] + P.wgt * psi;
          P.p_acc[g] = P.acc_mode == 2 ? sum * rdt : sum;
        }
      }
    }
  } else {
    for (int e = tid; e < N * L; e += nthr) {
      const int l = e & (L - 1), m = e >> LOG2L;
      if (l < nl) P.out[base + l + (size_t)m * estride] = R[m * LD + l];
    }
  }
}

// FP32: registers capped for 8 blocks per SM (32, no spills; half-width tiles also fit 8 in
// shared memory): the passes wait on their tile loads, and more blocks in flight hide more of
// that (the 3D step 0.5 % faster than at the 40-42 registers the compiler picks unbounded)
template <typename T, int N, int LOG2L_>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 8 : 1) pow2_transform_kernel(const __grid_constant__ TransformParams<T> P) {
  aero::pdl_wait();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  pow2_transform_body<T, N, LOG2L_>(P, blockIdx.x, blockIdx.y, smem_raw);
}

}  // namespace aero
