// Kernel parameter blocks and launchers of the 3D step (internal to libaero_b200.so).
#pragma once

#include <algorithm>
#include <cstddef>

#include <cuda.h>

#include "common.cuh"

namespace aero {

// scalar slots of the workspace's double block
enum : int {
  SC_MAXU = 0,
  SC_MAXV = 1,
  SC_MAXW = 2,
  SC_MAXT = 3,
  SC_NUTMAX = 4,
  SC_DT = 5,
  SC_SUM_INLET = 6,
  SC_SUM_U0 = 7,       // sum u0[..., nx]
  SC_SUMS = 8,         // 3 stages x (sum up[nx], sum up[nx-1], spare)
  SC_TOT = 20,         // reduced force / heat sums (AERO_MAX_BODIES * 10)
  SC_COUNT = 20 + AERO_MAX_BODIES * 10
};

template <typename T>
struct NuParams {
  CUtensorMap map_u, map_v, map_w;  // TMA views of the stage-start velocity (use_tma)
  int use_tma;
  int *status;
  // polls of a plane's barrier before the CTA gives up (status bit 1), drains its copies in
  // flight and returns; wait_extra_tx > 0 only in the test of that bound (bytes that never arrive)
  int wait_limit, wait_extra_tx;
  int nu_pitch;
  int nx, ny, nz, zc, les;
  T inv_h, cd2;
  CompRules<T> ru, rv, rw;
  const T *up, *vp, *wp;
  int has_win, win[6], wnx, wny;
  const T *chi_c;
  T *nu;                      // (nz+2, ny+2, nx+2): cells -1..n of every axis
  unsigned long long *nut_max;  // or NULL
  // learned closure: the eight gradient components and the window factor (1 - chi_c) of every
  // cell, at the nu array's index, components grad_plane apart (FP32; NULL: not written)
  float *grad;
  int64_t grad_plane;
};

// An actuator disc as the stage kernel sees it: its window, force and swirl weights on the
// window's u, v, w faces, and its thrust / swirl amplitude (device scalars of this step).
template <typename T>
struct FanForce {
  int win[6];
  const T *f[3], *s[3];
  const T *thrust, *swirl_amp;
};

// A jet or vent as the stage kernel sees it (physics.py:1033-1072).
template <typename T>
struct PortSource {
  int win[6], vent;
  T theta;
  const T *f[3], *m;
};

template <typename T>
struct PortParamsBlock {
  PortSource<T> port[AERO_MAX_PORTS];
};

// The fans' begin-of-step update (physics.py:922-942): disc velocities and the PI thrust.
template <typename T>
struct FanBeginParams {
  int nfan, any_swirl, nx, ny, nz;
  const T *u0, *v0, *w0, *dt;
  struct {
    int win[6], velocity_mode;
    double target, kp, ki, tmax, swirl;
    const T *m[3];
    T *thrust, *ud, *e_prev, *swirl_amp;
  } fan[AERO_MAX_FANS];
};

template <typename T>
struct StageParams {
  CUtensorMap map_u, map_v, map_w, map_th, map_nu;  // TMA views (use_tma)
  int use_tma;
  int *status;
  int wait_limit, wait_extra_tx;  // as in NuParams
  int forcing;                    // the verification cases' uniform body force (core.py:565-566)
  T force[3];
  int nu_pitch;
  int nx, ny, nz, zc;
  T h, inv_h;
  CompRules<T> ru, rv, rw;
  int px, py, pz, closed;
  int upwind, les;
  T kadv, nu_h2;
  const T *nu;                // eddy viscosity of the stage-start velocity (nu_kernel)
  // stage
  T a, bdt_scale, wgt;
  const T *dt;
  const T *up, *vp, *wp;      // stage-start velocity (ghosts by rule)
  const T *u0, *v0, *w0;      // step-start velocity (RK blend)
  T *uh, *vh, *wh;            // stage value out
  const T *u_inlet;
  const T *outlet_corr;       // device scalar: the outlet mass-balance correction
  // window
  int has_win, win[6], wnx, wny, nbody, nq;
  T eta;
  const T *chi_u, *chi_v, *chi_w, *chi_c, *a_u, *a_v, *a_w, *k_u, *k_v, *k_w;
  double *partials;           // [block][nq] (this stage's slice)
  // heat
  int thermal, has_adia, n_tbody;
  ThetaSides sides;
  T kh, kprt, kappa, ri, eta_t;
  const T *thp, *th0;
  T *thh;
  const T *chi_t, *a_t, *w_t, *adia_u, *adia_v, *adia_w, *vol_w, *skin;
  const T *paint_u, *paint_v, *paint_w;  // painted solid fractions (whole grid) or NULL
  int nfan, fan_swirl;
  FanForce<T> fan[AERO_MAX_FANS];
  int nport;
  T port_leak;
  PortSource<T> port[AERO_MAX_PORTS];
  int nheat;                        // volumetric heaters: cell window and source density
  struct {
    int win[6];
    const T *q;
  } heat[AERO_MAX_HEATERS];
};

struct DtParams {
  double *scalars;
  const void *dt_in;
  void *dt_out;
  int *status;
  int has_dt_fixed, les, thermal, has_heat_max;
  double dt_fixed, cfl, h, nu, viscous_dt, kappa, prt, ri, heat_max;
  double u_floor;             // sources' speed scale (0: none)
  int pid;                    // PID controller on the rule's dt
  double pid_target;
  void *pid_dt_prev, *pid_e1, *pid_e2;  // its state (plan dtype), updated in place
};

template <typename T>
struct CorrectParams {
  int nx, ny, nz, px, py, pz;
  int pu_out;                 // row pitch of the u output
  T inv_h;
  const T *uh, *vh, *wh, *psi;
  T *u, *v, *w;
};

template <typename T>
struct SmokeParams {
  int nx, ny, nz, px, py, pz;
  T inv_h;
  const T *c0, *u, *v, *w, *dt, *t0, *t_new;  // t_new NULL: t0 + dt
  T *c;
  const T *chi_c;
  int win[6];
  const T *weight;
  int dwin[6];
  double pulse_on, pulse_period;
  const T *paint_c;           // painted solid fraction of the cells (whole grid) or NULL
};

template <typename T>
struct FinalizeParams {
  size_t ncell;
  int nbody, nq, nblocks, n_tbody, symmetry;
  const double *partials;
  double *tot;                // nq reduced sums (workspace)
  double h, pe, y0, moment_ref_y, ref_area, span_ref, length_ref;
  int t_index[AERO_MAX_BODIES];
  double flux_rate[AERO_MAX_BODIES];
  const T *dt, *t0;
  T *t_out, *dt_out, *coeffs, *heat_rate, *p;
  int *status;
};

template <typename T>
struct AxisTables {
  int n, method, kind, nfac;
  int fac[16];
  const T *tw, *post, *cs, *dense;
  const double *lam;
  T s0, s1, rsqrt_n;
};

template <typename T>
struct TransformParams {
  const T *in;
  T *out;
  int nx, ny, nz, axis, mode, L;  // mode: 0 forward, 1 inverse, 2 forward-solve-inverse
  AxisTables<T> A;
  const double *lam_x, *lam_y;
  // power-of-two x passes only: the forward pass may form div(uh, vh, wh) itself instead of
  // reading `in` (fuse_div 1: 3D; 2: the 2D grid viewed as (ny, 1, nx)); the inverse pass may
  // also fold psi into the step-averaged pressure
  // (acc_mode 0: p = wgt psi; 1: p += wgt psi; 2: p = (p + wgt psi) / dt)
  int fuse_div, px, py, pz;
  const T *uh, *vh, *wh;
  T inv_h;
  T *p_acc;
  T wgt;
  int acc_mode;
  const T *dt;
};

// output fields (fields3d.cu): out[0..6] = centred u, v, w, speed, vorticity, Q, nu_t (or NULL)
template <typename T>
struct FieldsParams {
  int nx, ny, nz, les, gradient;
  T inv_h, cd2;
  CompRules<T> ru, rv, rw;
  const T *u, *v, *w;
  int has_win, win[6], wnx, wny;
  const T *chi_c;
  T *out[7];
};

template <typename T> size_t stage_smem_bytes();
template <typename T> cudaError_t launch_stage(const StageParams<T> &, cudaStream_t);
template <typename T> cudaError_t launch_nu(const NuParams<T> &, cudaStream_t);
template <typename T> cudaError_t launch_absmax(const T *, size_t, unsigned long long *, cudaStream_t);
template <typename T>
cudaError_t launch_copy_u(const T *, T *, int, int, int, int, unsigned long long *, cudaStream_t);
template <typename T> cudaError_t launch_dt(const DtParams &, cudaStream_t);
template <typename T>
struct MaxJob {
  const T *a;
  size_t n;
  unsigned long long *out;
};
template <typename T>
struct MaxJobs {
  MaxJob<T> job[3];
  int vec;
};
// max |a| of up to three arrays (ordered bit patterns, atomics), one launch
template <typename T> cudaError_t launch_absmax_multi(const MaxJobs<T> &, int njobs, cudaStream_t);
template <typename T> cudaError_t launch_fan_begin(const FanBeginParams<T> &, cudaStream_t);
// div -= m on every port's cells (physics.py:1043-1047)
template <typename T>
cudaError_t launch_port_continuity(T *div, int nx, int ny, int nport, const PortSource<T> *ports, cudaStream_t s);
template <typename T> cudaError_t launch_outlet_sum(const T *, const T *, int, int, double *, cudaStream_t);
template <typename T>
cudaError_t launch_outlet_corr(const double *, const double *, const double *, const double *, int, const T *, double,
                               double, double, double, double, T *, cudaStream_t);
template <typename T>
cudaError_t launch_divergence(const T *, const T *, const T *, int, int, int, int, int, int, T, T *, cudaStream_t);
// sum of squares of a[0, n) into the device scalar out (FP64 partials of SUMSQ_PARTS blocks)
constexpr int SUMSQ_PARTS = 2 * 148;
template <typename T>
cudaError_t launch_sumsq(const T *a, size_t n, double *part, T *out, cudaStream_t s);
template <typename T> cudaError_t launch_correct(const CorrectParams<T> &, cudaStream_t);
template <typename T> cudaError_t launch_smoke(const SmokeParams<T> &, cudaStream_t);
template <typename T> cudaError_t launch_finalize(const FinalizeParams<T> &, cudaStream_t);
template <typename T> cudaError_t launch_psi_accumulate(const T *, T *, size_t, T, int, const T *, cudaStream_t);
template <typename T> size_t transform_smem_bytes(int, int);
template <typename T> cudaError_t launch_transform(const TransformParams<T> &, cudaStream_t);
// true when an axis of n cells runs the compile-time tile transform (n = 2^a or 3 * 2^a,
// 8 <= n <= 2048), which also takes the divergence / pressure fusions of TransformParams
bool transform_tiled(int n);
template <typename T> cudaError_t launch_fields(const FieldsParams<T> &, cudaStream_t);
template <typename T>
cudaError_t launch_probe(const T *, int, int, int, const double *, double, const double *, const T *, long long, T *,
                         cudaStream_t);
template <typename T>
cudaError_t launch_axis_tables(int, int, int, double, T *, T *, T *, double *, T *, cudaStream_t);

}  // namespace aero
