// Point stencils shared by the 3D kernels (arithmetic of Aerolume ns3d/core.py and dye.py).
#pragma once

#include "common.cuh"

namespace aero {

// 24/7 x the upwind3 flux, or 4 x the central flux (core.py:331-345).
template <typename T>
__device__ __forceinline__ T face_flux(T vsum, T a, T b, T c, T d, bool upwind) {
  const T s = b + c;
  if (!upwind) return vsum * s;
  const T cen = s + T(-1.0 / 7.0) * (a + d);
  const T dis = (b - c) + T(-1.0 / 3.0) * (a - d);
  return vsum * cen + T(3.0 / 7.0) * fabs(vsum) * dis;
}

// MUSCL / van Leer upwind face value times the velocity (dye.py:266-277).
// FP64 divides exactly.  FP32 uses the hardware reciprocal (__fdividef, within 2 ulp of the
// rounded quotient): wherever pq > 0 holds in FP32, |p| |q| >= 2^-149 and so
// |p + q| >= max(|p|, |q|) >= 2^-75, inside the range where that division is accurate, and
// the select is branch-free.
template <typename T>
__device__ __forceinline__ T van_leer(T p, T q) {
  const T pq = p * q;
  if constexpr (sizeof(T) == 4) {
    const T r = __fdividef(T(2) * pq, p + q);
    return pq > T(0) ? r : T(0);
  } else {
    return pq > T(0) ? T(2) * pq / (p + q) : T(0);
  }
}

template <typename T>
__device__ __forceinline__ T muscl_flux(T a, T b, T c, T d, T vel) {
  // the upwind side's slope only (the reference evaluates both sides and selects; the
  // selected value is the same)
  const bool pos = vel > T(0);
  const T p = pos ? b - a : c - b;
  const T q = pos ? c - b : d - c;
  const T base = pos ? b : c;
  const T s = van_leer(p, q);
  return vel * (pos ? base + T(0.5) * s : base - T(0.5) * s);
}

// Square root and quotient for the eddy viscosity: exact in FP64; in FP32 the hardware
// approximations (sqrt.approx: relative error within 2^-23 on the non-negative inputs used
// here; __fdividef: 2 ulp for divisors in [2^-126, 2^126], and every divisor below is at
// least 1e-30)
template <typename T>
__device__ __forceinline__ T nut_sqrt(T x) {
  if constexpr (sizeof(T) == 4) {
    float r;
    asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
  } else {
    return sqrt(x);
  }
}

template <typename T>
__device__ __forceinline__ T nut_div(T a, T b) {
  if constexpr (sizeof(T) == 4)
    return __fdividef(a, b);
  else
    return a / b;
}

// Eddy viscosity from the traceless gradient (core.py:448-482); g[i][j] = du_i/dx_j.
template <typename T>
__device__ __forceinline__ T eddy_viscosity(const T g[3][3], int model, T cd2) {
  T s[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) s[i][j] = T(0.5) * (g[i][j] + g[j][i]);
  T ss = T(0);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) ss = ss + s[i][j] * s[i][j];
  if (model == AERO_LES_SMAGORINSKY) return cd2 * nut_sqrt(T(2) * ss + T(1e-30));
  if (model == AERO_LES_WALE) {
    T g2[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) g2[i][j] = (g[i][0] * g[0][j] + g[i][1] * g[1][j]) + g[i][2] * g[2][j];
    const T tr3 = (g2[0][0] + g2[1][1] + g2[2][2]) * T(1.0 / 3.0);
    T sd = T(0);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        T sdij = T(0.5) * (g2[i][j] + g2[j][i]);
        if (i == j) sdij = sdij - tr3;
        sd = sd + sdij * sdij;
      }
    const T sdp = sd > T(0) ? sd : T(0);
    const T ssp = ss > T(0) ? ss : T(0);
    // x^1.5 = x sqrt(x), x^2.5 = x^2 sqrt(x), x^1.25 = x sqrt(sqrt(x))
    const T rsd = nut_sqrt(sdp);
    const T num = sdp * rsd;
    const T den = (ssp * ssp) * nut_sqrt(ssp) + sdp * nut_sqrt(rsd) + T(1e-30);
    return nut_div(cd2 * num, den);
  }
  // Vreman: beta_ij = sum_m g[i][m] g[j][m]
  T b[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) b[i][j] = (g[i][0] * g[j][0] + g[i][1] * g[j][1]) + g[i][2] * g[j][2];
  T bb = b[0][0] * b[1][1] - b[0][1] * b[0][1] + b[0][0] * b[2][2] - b[0][2] * b[0][2] + b[1][1] * b[2][2] -
         b[1][2] * b[1][2];
  bb = bb > T(0) ? bb : T(0);
  T aa = T(0);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) aa = aa + g[i][j] * g[i][j];
  return cd2 * nut_sqrt(nut_div(bb, aa + T(1e-30)) + T(1e-30));
}

}  // namespace aero
