// Host-side pieces shared by the 3D and 2D plans of the C ABI: the thread-local error
// message, CUDA error propagation, workspace alignment and the per-axis transform tables
// of the Poisson solve.
#pragma once

#include <algorithm>
#include <cmath>
#include <string>

#include "ns3d.cuh"

namespace aero_host {

// Stores msg as the calling thread's aero_last_error() and returns code (defined in capi.cu).
int set_error(int code, const std::string &msg);

// The learned closure's eddy-viscosity pass of the 3D step (closure.cu): over the padded
// (nzp, nyp, pitch) cells whose gradient and window factor the eddy-viscosity kernel left in
// grad (9 components, `plane` apart), nu_t of the learned stress where it applies.
int closure_nu(const AeroClosureModel *m, const float *grad, int64_t plane, int nxp, int nyp, int nzp, int pitch,
               double delta, float *nu, unsigned long long *nut_max, unsigned long long *counts, int *status,
               cudaStream_t s);

constexpr size_t ALIGN = 256;
inline size_t align_up(size_t x) { return (x + ALIGN - 1) & ~(ALIGN - 1); }

// radix sequence (4s, then 2, then 3s) for n = 2^a 3^b, else -1
inline int factor(int n, int *fac) {
  int k = 0;
  while (n % 4 == 0) { fac[k++] = 4; n /= 4; }
  while (n % 2 == 0) { fac[k++] = 2; n /= 2; }
  while (n % 3 == 0) { fac[k++] = 3; n /= 3; }
  return n == 1 ? k : -1;
}

// One axis of the Poisson solve: its transform (FFT or dense), the lines per tile of the
// generic transform kernel and where its tables live in the workspace.
struct AxisInfo {
  int n, kind, method, nfac, L;
  int fac[16];
  size_t off_tw, off_post, off_cs, off_lam, off_dense;
};

// Fills everything but the table offsets for an axis of n cells (kind 1: periodic).
inline void axis_setup(AxisInfo &x, int n, bool periodic, size_t e) {
  x.n = n;
  x.kind = periodic ? 1 : 0;
  x.nfac = factor(x.n, x.fac);
  x.method = x.nfac < 0 ? 1 : 0;
  if (x.nfac < 0) x.nfac = 0;
  // lines per block: keep the tile (3 n L elements) within ~48 KiB, even, 2..64
  int L = (int)((48 * 1024) / (3 * e * (size_t)x.n));
  L = std::max(2, std::min(64, L));
  L &= ~1;
  if (x.method == 1) L = std::max(2, std::min(L, 16));
  x.L = L;
}

// Places the axis tables with `take(bytes) -> offset`.
template <class Take>
void axis_place(AxisInfo &x, size_t e, Take &&take) {
  x.off_tw = take(2 * x.n * e);
  x.off_post = take(2 * x.n * e);
  x.off_cs = take(2 * x.n * e);
  x.off_lam = take(sizeof(double) * x.n);
  x.off_dense = take(x.method == 1 ? (size_t)x.n * x.n * e : 0);
}

template <typename T>
aero::AxisTables<T> axis_view(const AxisInfo &x, unsigned char *ws) {
  aero::AxisTables<T> A{};
  A.n = x.n;
  A.method = x.method;
  A.kind = x.kind;
  A.nfac = x.nfac;
  for (int i = 0; i < x.nfac; ++i) A.fac[i] = x.fac[i];
  A.tw = reinterpret_cast<const T *>(ws + x.off_tw);
  A.post = reinterpret_cast<const T *>(ws + x.off_post);
  A.cs = reinterpret_cast<const T *>(ws + x.off_cs);
  A.lam = reinterpret_cast<const double *>(ws + x.off_lam);
  A.dense = x.method == 1 ? reinterpret_cast<const T *>(ws + x.off_dense) : nullptr;
  A.s0 = T(std::sqrt(1.0 / x.n));
  A.s1 = T(std::sqrt(2.0 / x.n));
  A.rsqrt_n = T(1.0 / std::sqrt((double)x.n));
  return A;
}

template <typename T>
cudaError_t axis_init(const AxisInfo &x, double h, unsigned char *ws, cudaStream_t s) {
  return aero::launch_axis_tables<T>(x.n, x.kind, x.method == 1, h, reinterpret_cast<T *>(ws + x.off_tw),
                                     reinterpret_cast<T *>(ws + x.off_post), reinterpret_cast<T *>(ws + x.off_cs),
                                     reinterpret_cast<double *>(ws + x.off_lam),
                                     x.method == 1 ? reinterpret_cast<T *>(ws + x.off_dense) : nullptr, s);
}

}  // namespace aero_host

#define AERO_CUDA_TRY(expr)                                                                                  \
  do {                                                                                                       \
    cudaError_t e__ = (expr);                                                                                \
    if (e__ != cudaSuccess)                                                                                  \
      return aero_host::set_error(AERO_ECUDA, std::string(#expr) + ": " + cudaGetErrorString(e__));        \
  } while (0)
