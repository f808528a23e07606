// Output fields of a 3D state (Aerolume ns3d/fields.py:24-102, ns3d/solver.py:1374-1416):
// cell-centred velocity and speed, vorticity magnitude, Q-criterion and eddy viscosity from the
// velocity-gradient tensor, and trilinear sampling of any (staggered) field at points.  These
// are outputs (per frame, not per step): one thread per cell, the 3 x 3 x 3 neighbourhood
// staged per block in shared memory with the ghost rules applied while staging.
#include "ns3d.cuh"
#include "stencil.cuh"

namespace aero {

// g[i][j] = du_i / dx_j at the cell (ns3d/core.py:400-434: edge differences averaged over the
// four edges around the cell, in the reference's order), from a loader L(c, dz, dy, dx)
template <typename T, class Load>
__device__ __forceinline__ void cell_gradient(const Load &L, T inv, T g[3][3]) {
  const T qq = T(0.25);
  g[0][0] = (L(0, 0, 0, 1) - L(0, 0, 0, 0)) * inv;
  g[1][1] = (L(1, 0, 1, 0) - L(1, 0, 0, 0)) * inv;
  g[2][2] = (L(2, 1, 0, 0) - L(2, 0, 0, 0)) * inv;
  g[0][1] = ((((L(0, 0, 0, 0) - L(0, 0, -1, 0)) * inv + (L(0, 0, 1, 0) - L(0, 0, 0, 0)) * inv) +
              (L(0, 0, 0, 1) - L(0, 0, -1, 1)) * inv) +
             (L(0, 0, 1, 1) - L(0, 0, 0, 1)) * inv) *
            qq;
  g[0][2] = ((((L(0, 0, 0, 0) - L(0, -1, 0, 0)) * inv + (L(0, 1, 0, 0) - L(0, 0, 0, 0)) * inv) +
              (L(0, 0, 0, 1) - L(0, -1, 0, 1)) * inv) +
             (L(0, 1, 0, 1) - L(0, 0, 0, 1)) * inv) *
            qq;
  g[1][0] = ((((L(1, 0, 0, 0) - L(1, 0, 0, -1)) * inv + (L(1, 0, 1, 0) - L(1, 0, 1, -1)) * inv) +
              (L(1, 0, 0, 1) - L(1, 0, 0, 0)) * inv) +
             (L(1, 0, 1, 1) - L(1, 0, 1, 0)) * inv) *
            qq;
  g[1][2] = ((((L(1, 0, 0, 0) - L(1, -1, 0, 0)) * inv + (L(1, 1, 0, 0) - L(1, 0, 0, 0)) * inv) +
              (L(1, 0, 1, 0) - L(1, -1, 1, 0)) * inv) +
             (L(1, 1, 1, 0) - L(1, 0, 1, 0)) * inv) *
            qq;
  g[2][0] = ((((L(2, 0, 0, 0) - L(2, 0, 0, -1)) * inv + (L(2, 1, 0, 0) - L(2, 1, 0, -1)) * inv) +
              (L(2, 0, 0, 1) - L(2, 0, 0, 0)) * inv) +
             (L(2, 1, 0, 1) - L(2, 1, 0, 0)) * inv) *
            qq;
  g[2][1] = ((((L(2, 0, 0, 0) - L(2, 0, -1, 0)) * inv + (L(2, 1, 0, 0) - L(2, 1, -1, 0)) * inv) +
              (L(2, 0, 1, 0) - L(2, 0, 0, 0)) * inv) +
             (L(2, 1, 1, 0) - L(2, 1, 0, 0)) * inv) *
            qq;
}

template <typename T>
__device__ __forceinline__ void write_fields(const FieldsParams<T> &P, const T g[3][3], size_t c, int k, int j, int i,
                                             T uc, T vc, T wc) {
  if (P.out[0]) P.out[0][c] = uc;
  if (P.out[1]) P.out[1][c] = vc;
  if (P.out[2]) P.out[2][c] = wc;
  if (P.out[3]) P.out[3][c] = sqrt((uc * uc + vc * vc) + wc * wc);
  if (P.out[4]) {  // |curl u|
    const T ox = g[2][1] - g[1][2], oy = g[0][2] - g[2][0], oz = g[1][0] - g[0][1];
    P.out[4][c] = sqrt((ox * ox + oy * oy) + oz * oz);
  }
  if (P.out[5]) {  // Q = -g_ij g_ji / 2, summed in (i, j) order
    T s = g[0][0] * g[0][0];
    s = s + g[0][1] * g[1][0];
    s = s + g[0][2] * g[2][0];
    s = s + g[1][0] * g[0][1];
    s = s + g[1][1] * g[1][1];
    s = s + g[1][2] * g[2][1];
    s = s + g[2][0] * g[0][2];
    s = s + g[2][1] * g[1][2];
    s = s + g[2][2] * g[2][2];
    P.out[5][c] = T(-0.5) * s;
  }
  if (P.out[6]) {  // eddy viscosity of the traceless gradient, off inside solids
    T nu = T(0);
    if (P.les != AERO_LES_NONE) {
      T gt[3][3];
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) gt[a][b] = g[a][b];
      gt[2][2] = -(g[0][0] + g[1][1]);
      nu = eddy_viscosity<T>(gt, P.les, P.cd2);
      T chi = T(0);
      if (P.has_win && k >= P.win[0] && k < P.win[1] && j >= P.win[2] && j < P.win[3] && i >= P.win[4] &&
          i < P.win[5])
        chi = P.chi_c[((size_t)(k - P.win[0]) * P.wny + (j - P.win[2])) * P.wnx + (i - P.win[4])];
      nu = nu * (T(1) - chi);
    }
    P.out[6][c] = nu;
  }
}

// One block per 32 x 8 cells of a z-plane.  The block first stages the three face arrays on
// the tile's neighbourhood -- entries (k-1..k+1, j0-1..j0+8, i0-1..i0+32) of each -- in shared
// memory, reading in-range entries directly and applying the ghost rules only to the entries
// outside an array, so no thread diverges into the rules while the fields are computed.
constexpr int FTX = 32, FTY = 8, FSX = FTX + 2, FSY = FTY + 2;

template <typename T>
__global__ void __launch_bounds__(FTX *FTY) fields_kernel(const __grid_constant__ FieldsParams<T> P) {
  aero::pdl_wait();
  __shared__ T sm[3][3][FSY][FSX];  // [component][dz + 1][y][x]
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  const int i0 = blockIdx.x * FTX, j0 = blockIdx.y * FTY, k = blockIdx.z;
  const int tid = threadIdx.y * FTX + threadIdx.x;
  for (int e = tid; e < 3 * 3 * FSY * FSX; e += FTX * FTY) {
    const int x = e % FSX, y = (e / FSX) % FSY, z = (e / (FSX * FSY)) % 3, comp = e / (FSX * FSY * 3);
    const int gi = i0 - 1 + x, gj = j0 - 1 + y, gk = k - 1 + z;
    T val;
    if (comp == 0) {
      val = (gi >= 0 && gi <= nx && gj >= 0 && gj < ny && gk >= 0 && gk < nz)
                ? __ldg(P.u + ((size_t)gk * ny + gj) * (nx + 1) + gi)
                : padded<T>(P.u, P.ru, gk, gj, gi);
    } else if (comp == 1) {
      val = (gi >= 0 && gi < nx && gj >= 0 && gj <= ny && gk >= 0 && gk < nz)
                ? __ldg(P.v + ((size_t)gk * (ny + 1) + gj) * nx + gi)
                : padded<T>(P.v, P.rv, gk, gj, gi);
    } else {
      val = (gi >= 0 && gi < nx && gj >= 0 && gj < ny && gk >= 0 && gk <= nz)
                ? __ldg(P.w + ((size_t)gk * ny + gj) * nx + gi)
                : padded<T>(P.w, P.rw, gk, gj, gi);
    }
    sm[comp][z][y][x] = val;
  }
  __syncthreads();
  const int tx = threadIdx.x, ty = threadIdx.y, i = i0 + tx, j = j0 + ty;
  if (i >= nx || j >= ny) return;
  auto L = [&](int comp, int dz, int dy, int dx) -> T { return sm[comp][1 + dz][1 + ty + dy][1 + tx + dx]; };
  const T uc = T(0.5) * (L(0, 0, 0, 1) + L(0, 0, 0, 0)), vc = T(0.5) * (L(1, 0, 1, 0) + L(1, 0, 0, 0)),
          wc = T(0.5) * (L(2, 1, 0, 0) + L(2, 0, 0, 0));
  const size_t c = ((size_t)k * ny + j) * nx + i;
  T g[3][3] = {{T(0), T(0), T(0)}, {T(0), T(0), T(0)}, {T(0), T(0), T(0)}};
  if (P.gradient) cell_gradient<T>(L, P.inv_h, g);
  write_fields<T>(P, g, c, k, j, i, uc, vc, wc);
}

// Trilinear sampling (ns3d/fields.py:78-102): points outside are clamped to the edge.
template <typename T>
__global__ void probe_kernel(const T *__restrict__ f, int fnx, int fny, int fnz, T x0, T y0, T z0, T h, T ox, T oy,
                             T oz, const T *__restrict__ pts, long long npts, T *__restrict__ out) {
  aero::pdl_wait();
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= npts) return;
  auto axis = [&](T x, T origin, T off, int n, int &i0, T &t, int &s) {
    T fv = (x - origin) / h - off;
    const T hi = T(n - 1 > 0 ? n - 1 : 0);
    fv = fv < T(0) ? T(0) : (fv > hi ? hi : fv);  // NaN stays NaN, as the reference's clamp
    int ii = (int)floor(fv);
    const int top = n - 2 > 0 ? n - 2 : 0;
    ii = ii > top ? top : ii;
    ii = ii < 0 ? 0 : ii;
    i0 = ii;
    t = fv - T(ii);
    s = n - 1 < 1 ? n - 1 : 1;
  };
  int i0, j0, k0, sx, sy, sz;
  T tx, ty, tz;
  axis(pts[3 * p + 0], x0, ox, fnx, i0, tx, sx);
  axis(pts[3 * p + 1], y0, oy, fny, j0, ty, sy);
  axis(pts[3 * p + 2], z0, oz, fnz, k0, tz, sz);
  auto at = [&](int dk, int dj, int di) {
    return __ldg(f + ((size_t)(k0 + dk * sz) * fny + (j0 + dj * sy)) * fnx + (i0 + di * sx));
  };
  const T one = T(1);
  const T c00 = at(0, 0, 0) * (one - tx) + at(0, 0, 1) * tx;
  const T c01 = at(0, 1, 0) * (one - tx) + at(0, 1, 1) * tx;
  const T c10 = at(1, 0, 0) * (one - tx) + at(1, 0, 1) * tx;
  const T c11 = at(1, 1, 0) * (one - tx) + at(1, 1, 1) * tx;
  out[p] = (c00 * (one - ty) + c01 * ty) * (one - tz) + (c10 * (one - ty) + c11 * ty) * tz;
}

template <typename T>
cudaError_t launch_fields(const FieldsParams<T> &P, cudaStream_t s) {
  (void)aero::launch_k(fields_kernel<T>, dim3((P.nx + FTX - 1) / FTX, (P.ny + FTY - 1) / FTY, P.nz), dim3(FTX, FTY), 0, s, P);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_probe(const T *f, int fnx, int fny, int fnz, const double origin[3], double h, const double off[3],
                         const T *pts, long long npts, T *out, cudaStream_t s) {
  if (npts <= 0) return cudaSuccess;
  const unsigned blocks = (unsigned)((npts + 255) / 256);
  (void)aero::launch_k(probe_kernel<T>, blocks, 256, 0, s, f, fnx, fny, fnz, T(origin[0]), T(origin[1]), T(origin[2]), T(h), T(off[0]),
                                         T(off[1]), T(off[2]), pts, npts, out);
  return cudaGetLastError();
}

template cudaError_t launch_fields<float>(const FieldsParams<float> &, cudaStream_t);
template cudaError_t launch_fields<double>(const FieldsParams<double> &, cudaStream_t);
template cudaError_t launch_probe<float>(const float *, int, int, int, const double *, double, const double *,
                                         const float *, long long, float *, cudaStream_t);
template cudaError_t launch_probe<double>(const double *, int, int, int, const double *, double, const double *,
                                          const double *, long long, double *, cudaStream_t);

}  // namespace aero
