// Shared device helpers of the B200 Navier-Stokes kernels.
#pragma once

#include <cstdint>
#include <utility>
#include <cuda_runtime.h>

#include "../../include/aero_b200.h"

namespace aero {

// Programmatic dependent launch: every kernel of the library is launched with programmatic
// stream serialisation, so its launch and block scheduling overlap the tail of the kernel
// before it, and every kernel's first statement waits (griddepcontrol.wait) until that kernel
// has completed and its writes are visible.  Launched without the attribute, the wait returns
// at once.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <typename... KArgs, typename... Args>
inline cudaError_t launch_k(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                            Args &&...args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// Bounds checks of the checked build (-DAERO_BOUNDS_CHECK, libaero_b200_checked.so): a failed
// check records (code, index, bound) once in aero_check_word and the access is skipped.  In the
// release build every check is `true` and compiles away.
#ifdef AERO_BOUNDS_CHECK
extern __device__ long long aero_check_word[4];
__device__ __forceinline__ bool aero_check(bool ok, int code, long long idx, long long bound) {
  if (ok) return true;
  if (atomicCAS(reinterpret_cast<unsigned long long *>(&aero_check_word[0]), 0ull, (unsigned long long)code) == 0ull) {
    aero_check_word[1] = idx;
    aero_check_word[2] = bound;
    aero_check_word[3] = ((long long)blockIdx.x << 32) | threadIdx.x;
  }
  return false;
}
#define AERO_IN(idx, bound, code) \
  aero::aero_check((long long)(idx) >= 0 && (long long)(idx) < (long long)(bound), (code), (long long)(idx), (long long)(bound))
#else
#define AERO_IN(idx, bound, code) true
#endif

// Ghost-cell rules of Aerolume ns3d/core.py:147-246 as index maps.  A ghost entry g
// (g < 0 or g >= n along an axis of n entries) takes the value s * x[map(g)] + c.
// Rules of the three axes compose in the order x, then y, then z (core.py:249-272):
//   value = sz * (sy * (sx * x + cx) + cy) + cz.
template <typename T>
__device__ __forceinline__ int ghost_map(int g, int n, int kind_lo, int kind_hi, T val_lo, T val_hi, T &s, T &c) {
  s = T(1);
  c = T(0);
  if (g >= 0 && g < n) return g;
  const bool lo = g < 0;
  if (lo) {
    if (g < -2) g = -2;
  } else if (g > n + 1) {
    g = n + 1;
  }
  const int kind = lo ? kind_lo : kind_hi;
  int m;
  switch (kind) {
    case AERO_GHOST_EDGE: m = lo ? 0 : n - 1; break;
    case AERO_GHOST_EVEN: m = lo ? -1 - g : 2 * n - 1 - g; break;
    case AERO_GHOST_ODD: m = lo ? -1 - g : 2 * n - 1 - g; s = T(-1); break;
    case AERO_GHOST_AFFINE:
      m = lo ? -1 - g : 2 * n - 1 - g;
      s = T(-1);
      c = T(2) * (lo ? val_lo : val_hi);
      break;
    case AERO_GHOST_FACE_ODD: m = lo ? -g : 2 * (n - 1) - g; s = T(-1); break;
    case AERO_GHOST_PERIODIC_CELL: m = lo ? g + n : g - n; break;
    default: m = lo ? g + n - 1 : g - n + 1; break;  // periodic_face
  }
  if (m < 0) m = 0;
  if (m > n - 1) m = n - 1;
  return m;
}

// The rules of one staggered component on its (n2, n1, n0) = (z, y, x) array.
template <typename T>
struct CompRules {
  int n0, n1, n2;  // entries along x, y, z
  int p0;          // row pitch (elements) of the array, >= n0
  int kind[3][2];
  T val[3][2];
};

// Value of the ghost-padded component at (k, j, i) (each index may lie up to two
// entries outside the array).
template <typename T>
__device__ __forceinline__ T padded(const T *__restrict__ f, const CompRules<T> &r, int k, int j, int i) {
  T sx, cx, sy, cy, sz, cz;
  const int mi = ghost_map<T>(i, r.n0, r.kind[0][0], r.kind[0][1], r.val[0][0], r.val[0][1], sx, cx);
  const int mj = ghost_map<T>(j, r.n1, r.kind[1][0], r.kind[1][1], r.val[1][0], r.val[1][1], sy, cy);
  const int mk = ghost_map<T>(k, r.n2, r.kind[2][0], r.kind[2][1], r.val[2][0], r.val[2][1], sz, cz);
  const T x = __ldg(f + ((size_t)mk * r.n1 + mj) * r.p0 + mi);
  return sz * (sy * (sx * x + cx) + cy) + cz;
}

// Temperature ghosts of ns3d/physics.py:589-621: one side's rule on the six faces; edge
// and corner ghosts are never read (the MUSCL stencil runs along one axis at a time).
struct ThetaSides {
  int kind[6];
  double val[6];
};

template <typename T>
__device__ __forceinline__ T theta_padded(const T *__restrict__ c, int nz, int ny, int nx, const ThetaSides &sd,
                                          T h, int k, int j, int i) {
  const bool ox = i < 0 || i >= nx, oy = j < 0 || j >= ny, oz = k < 0 || k >= nz;
  if (!ox && !oy && !oz) return __ldg(c + ((size_t)k * ny + j) * nx + i);
  if ((int)ox + (int)oy + (int)oz > 1) return T(0);
  int g, n, side;
  if (ox) {
    g = i; n = nx; side = i < 0 ? 0 : 1;
  } else if (oy) {
    g = j; n = ny; side = j < 0 ? 2 : 3;
  } else {
    g = k; n = nz; side = k < 0 ? 4 : 5;
  }
  const bool lo = (side & 1) == 0;
  if (lo && g < -2) g = -2;
  if (!lo && g > n + 1) g = n + 1;
  auto at = [&](int m) -> T {
    if (m < 0) m = 0;
    if (m > n - 1) m = n - 1;
    if (ox) return __ldg(c + ((size_t)k * ny + j) * nx + m);
    if (oy) return __ldg(c + ((size_t)k * ny + m) * nx + i);
    return __ldg(c + ((size_t)m * ny + j) * nx + i);
  };
  const int kind = sd.kind[side];
  const T val = T(sd.val[side]);
  if (kind == AERO_TH_PERIODIC) return at(lo ? g + n : g - n);
  if (kind == AERO_TH_OUTFLOW) return at(lo ? 0 : n - 1);
  const T mirror = at(lo ? -1 - g : 2 * n - 1 - g);
  switch (kind) {
    case AERO_TH_ADIABATIC: return mirror;
    case AERO_TH_INFLOW: return val;
    case AERO_TH_TEMPERATURE: return T(2) * val - mirror;
    default: {  // heat flux: + G h on the first layer, + 3 G h on the second
      const T w = (lo ? (g == -2) : (g == n + 1)) ? T(3) : T(1);
      return mirror + val * (w * h);
    }
  }
}

// torch.lerp's two-branch formula (the reference blends RK stages with it).
template <typename T>
__device__ __forceinline__ T lerp_t(T s, T e, T w) {
  return (w < T(0.5)) ? s + w * (e - s) : e - (e - s) * (T(1) - w);
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Non-negative maxima through the ordered bit patterns of IEEE doubles (NaN wins,
// which the status check then reports).
__device__ __forceinline__ void atomic_max_nonneg(unsigned long long *addr, double v) {
  atomicMax(addr, (unsigned long long)__double_as_longlong(v));
}

// Block-wide max of a non-negative value (NaN wins), then one atomic for the block.
template <typename T>
__device__ __forceinline__ void block_max_atomic(T m, unsigned long long *out) {
  __shared__ double red[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const T other = __shfl_xor_sync(0xffffffffu, m, o);
    m = (other > m || other != other) ? other : m;
  }
  const int nw = (blockDim.x * blockDim.y * blockDim.z + 31) >> 5;
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  if ((tid & 31) == 0) red[tid >> 5] = (double)m;
  __syncthreads();
  if (tid == 0) {
    double r = 0.0;
    for (int w = 0; w < nw; ++w) r = (red[w] > r || red[w] != red[w]) ? red[w] : r;
    atomic_max_nonneg(out, r);
  }
}

__device__ __forceinline__ double as_double(unsigned long long bits) { return __longlong_as_double((long long)bits); }

}  // namespace aero
