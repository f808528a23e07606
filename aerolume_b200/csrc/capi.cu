// C ABI of libaero_b200.so: plans, workspace layout and the launch sequence of a step.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include <cudaTypedefs.h>

#include "host_common.cuh"
#include "ns3d.cuh"

#ifdef AERO_BOUNDS_CHECK
namespace aero {
__device__ long long aero_check_word[4];
}
#endif

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string &msg) {
  g_last_error = msg;
  return code;
}

using aero_host::align_up;
using aero_host::ALIGN;
using aero_host::AxisInfo;
using aero_host::factor;

#define CUDA_TRY(expr)                                                                              \
  do {                                                                                              \
    cudaError_t e__ = (expr);                                                                       \
    if (e__ != cudaSuccess) return fail(AERO_ECUDA, std::string(#expr) + ": " + cudaGetErrorString(e__)); \
  } while (0)


// cuTensorMapEncodeTiled through the runtime's driver entry point (no libcuda link)
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// 3D tiled view (x, y, z extents, row pitch in elements) with a (bx, by, 1) box; false when
// the view cannot be described (alignment) -- the kernels then load synchronously.
bool encode3d(CUtensorMap *m, bool f64, const void *base, size_t nx, size_t ny, size_t nz, size_t pitch, int bx,
              int by) {
  auto fn = encode_fn();
  if (!fn || !base) return false;
  const size_t e = f64 ? 8 : 4;
  if (reinterpret_cast<uintptr_t>(base) % 16 || (pitch * e) % 16 || (bx * e) % 16) return false;
  cuuint64_t dims[3] = {nx, ny, nz};
  cuuint64_t strides[2] = {pitch * e, pitch * ny * e};
  cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(m, f64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<void *>(base),
                  dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

}  // namespace

int aero_host::set_error(int code, const std::string &msg) { return fail(code, msg); }

struct AeroNs3dPlan {
  AeroNs3dConfig cfg;
  size_t esz;                     // bytes per element
  size_t nu, nv, nw, nc;          // element counts of u, v, w and cell arrays
  size_t off_uh, off_vh, off_wh, off_up, off_vp, off_wp, off_tha, off_thb, off_pa, off_nu;
  size_t off_small, off_scalars, off_status, off_partials, off_psum, off_grad, off_counts, off_sumsq, total;
  AxisInfo ax[3];
  int zc, zc_nu, nblocks, nq;    // z-planes per CTA of the stage and eddy-viscosity kernels
  int pu, pn;                     // row pitches of the stage-start u copy and of nu
  int wait_limit = 0, wait_extra_tx = 0;  // plane-wait bound (0: default) and its test hook
};

namespace {

template <typename T>
aero::AxisTables<T> axis_tables(const AeroNs3dPlan *p, int a, unsigned char *ws) {
  return aero_host::axis_view<T>(p->ax[a], ws);
}

// psi = L^{-1} f through five passes: x, y forward; z forward-solve-inverse; y, x inverse.
// Every pass owns whole lines per block, so after the first pass the solve runs in place.
// `fuse` (x axes of 2^a or 3 * 2^a cells only) supplies the divergence fusion fields for the first
// pass and the pressure-accumulation fields for the last one.
template <typename T>
int poisson_passes(const AeroNs3dPlan *p, const T *f, T *psi, unsigned char *ws, cudaStream_t s,
                   const aero::TransformParams<T> *fuse = nullptr) {
  const AeroNs3dConfig &c = p->cfg;
  const int axes[5] = {0, 1, 2, 1, 0}, modes[5] = {0, 0, 2, 1, 1};
  for (int q = 0; q < 5; ++q) {
    aero::TransformParams<T> P{};
    if (fuse && q == 0) {
      P.fuse_div = fuse->fuse_div;
      P.px = fuse->px;
      P.py = fuse->py;
      P.pz = fuse->pz;
      P.uh = fuse->uh;
      P.vh = fuse->vh;
      P.wh = fuse->wh;
      P.inv_h = fuse->inv_h;
    }
    if (fuse && q == 4) {
      P.p_acc = fuse->p_acc;
      P.wgt = fuse->wgt;
      P.acc_mode = fuse->acc_mode;
      P.dt = fuse->dt;
    }
    P.nx = c.nx;
    P.ny = c.ny;
    P.nz = c.nz;
    P.lam_x = reinterpret_cast<const double *>(ws + p->ax[0].off_lam);
    P.lam_y = reinterpret_cast<const double *>(ws + p->ax[1].off_lam);
    P.axis = axes[q];
    P.mode = modes[q];
    P.in = q == 0 ? f : psi;
    P.out = psi;
    P.L = p->ax[axes[q]].L;
    P.A = axis_tables<T>(p, axes[q], ws);
    CUDA_TRY(aero::launch_transform<T>(P, s));
  }
  return AERO_OK;
}

template <typename T>
aero::CompRules<T> comp_rules(const AeroNs3dConfig &c, int comp, int pitch = 0) {
  aero::CompRules<T> r{};
  r.n0 = c.nx + (comp == 0);
  r.n1 = c.ny + (comp == 1);
  r.n2 = c.nz + (comp == 2);
  r.p0 = pitch > 0 ? pitch : r.n0;
  for (int a = 0; a < 3; ++a)
    for (int s = 0; s < 2; ++s) {
      r.kind[a][s] = c.ghost_kind[comp][a][s];
      r.val[a][s] = T(c.ghost_val[comp][a][s]);
    }
  return r;
}

// Block b of the grid sums a[r * stride + off] over its contiguous slice of the rows, in a
// fixed order, into out[b] (double); the consumer adds the PLANE_PARTS partials in order, so
// the total is the same on every run.
constexpr int PLANE_PARTS = 64;

template <typename T>
__global__ void __launch_bounds__(256) plane_sum_kernel(const T *a0, size_t stride0, size_t off0, double *out0,
                                                        const T *a1, size_t stride1, size_t off1, double *out1,
                                                        int rows) {
  aero::pdl_wait();
  __shared__ double red[2][8];
  const int per = (rows + gridDim.x - 1) / gridDim.x;
  const int r0 = blockIdx.x * per, r1 = min(rows, r0 + per);
  double s0 = 0.0, s1 = 0.0;
  for (int r = r0 + (int)threadIdx.x; r < r1; r += blockDim.x) {
    if (a0) s0 += (double)a0[(size_t)r * stride0 + off0];
    if (a1) s1 += (double)a1[(size_t)r * stride1 + off1];
  }
  s0 = aero::warp_sum(s0);
  s1 = aero::warp_sum(s1);
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = s0;
    red[1][threadIdx.x >> 5] = s1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double x = 0.0, y = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) {
      x += red[0][q];
      y += red[1][q];
    }
    if (a0) out0[blockIdx.x] = x;
    if (a1) out1[blockIdx.x] = y;
  }
}

template <typename T>
int smoke_impl(const AeroNs3dPlan *p, const AeroNs3dFields *f, const AeroNs3dGeom *g, const T *dt, const T *t_new,
               cudaStream_t s) {
  const AeroNs3dConfig &c = p->cfg;
  const bool has_win = !(c.window[1] <= c.window[0] || c.window[3] <= c.window[2] || c.window[5] <= c.window[4]) &&
                       c.nbody > 0;
  aero::SmokeParams<T> M{};
  M.nx = c.nx;
  M.ny = c.ny;
  M.nz = c.nz;
  M.px = c.periodic[0];
  M.py = c.periodic[1];
  M.pz = c.periodic[2];
  M.inv_h = T(1.0 / c.h);
  M.c0 = static_cast<const T *>(f->dye0);
  M.u = static_cast<const T *>(f->u);
  M.v = static_cast<const T *>(f->v);
  M.w = static_cast<const T *>(f->w);
  M.dt = dt;
  M.t0 = static_cast<const T *>(f->t0);
  M.t_new = t_new;
  M.c = static_cast<T *>(f->dye);
  M.chi_c = has_win ? static_cast<const T *>(g->chi_c) : nullptr;
  for (int q = 0; q < 6; ++q) {
    M.win[q] = has_win ? c.window[q] : 0;
    M.dwin[q] = c.dye_window[q];
  }
  const bool dye_src = !(c.dye_window[1] <= c.dye_window[0] || c.dye_window[3] <= c.dye_window[2] ||
                         c.dye_window[5] <= c.dye_window[4]);
  M.weight = dye_src ? static_cast<const T *>(g->dye_weight) : nullptr;
  M.pulse_on = c.pulse_on;
  M.pulse_period = c.pulse_period;
  M.paint_c = c.paint ? static_cast<const T *>(g->paint_c) : nullptr;
  CUDA_TRY(aero::launch_smoke<T>(M, s));
  return AERO_OK;
}

template <typename T>
int step_impl(const AeroNs3dPlan *p, const AeroNs3dFields *f, const AeroNs3dGeom *g, const void *dt_in,
              unsigned char *ws, cudaStream_t s, void *const *events = nullptr, int nevents = 0) {
  auto mark = [&](int i) -> cudaError_t {
    if (!events || i >= nevents || !events[i]) return cudaSuccess;
    return cudaEventRecordWithFlags(static_cast<cudaEvent_t>(events[i]), s, cudaEventRecordExternal);
  };
  const AeroNs3dConfig &c = p->cfg;
  const int nx = c.nx, ny = c.ny, nz = c.nz;
  T *uh = reinterpret_cast<T *>(ws + p->off_uh), *vh = reinterpret_cast<T *>(ws + p->off_vh),
    *wh = reinterpret_cast<T *>(ws + p->off_wh);
  T *upb = reinterpret_cast<T *>(ws + p->off_up), *vpb = reinterpret_cast<T *>(ws + p->off_vp),
    *wpb = reinterpret_cast<T *>(ws + p->off_wp);
  T *tha = reinterpret_cast<T *>(ws + p->off_tha), *thb = reinterpret_cast<T *>(ws + p->off_thb);
  T *pa = reinterpret_cast<T *>(ws + p->off_pa);
  T *small = reinterpret_cast<T *>(ws + p->off_small);  // [0] dt, [1] outlet corr
  double *sc = reinterpret_cast<double *>(ws + p->off_scalars);
  int *status = reinterpret_cast<int *>(ws + p->off_status);
  double *partials = reinterpret_cast<double *>(ws + p->off_partials);
  unsigned long long *bits = reinterpret_cast<unsigned long long *>(sc);

  const T *u0 = static_cast<const T *>(f->u0), *v0 = static_cast<const T *>(f->v0),
          *w0 = static_cast<const T *>(f->w0);
  const bool thermal = c.thermal != 0;
  const bool les = c.les != AERO_LES_NONE;
  const bool has_win = !(c.window[1] <= c.window[0] || c.window[3] <= c.window[2] || c.window[5] <= c.window[4]) &&
                       c.nbody > 0;
  const bool tunnel = !c.periodic[0] && !c.closed;
  const T *th0 = thermal ? static_cast<const T *>(f->theta0) : nullptr;

  CUDA_TRY(mark(0));
  CUDA_TRY(cudaMemsetAsync(sc, 0, sizeof(double) * aero::SC_COUNT, s));
  CUDA_TRY(cudaMemsetAsync(status, 0, sizeof(int), s));

  // ---- time step
  const bool need_max = dt_in == nullptr && !c.has_dt_fixed;
  // the stage-start u copy with a 16-byte row pitch (TMA), and max |u0| on the way
  CUDA_TRY(aero::launch_copy_u<T>(u0, upb, nx, ny, nz, p->pu, need_max ? bits + aero::SC_MAXU : nullptr, s));
  if (need_max) {  // max |v0|, |w0| (and |theta0|) in one launch
    aero::MaxJobs<T> J{};
    J.job[0] = {v0, p->nv, bits + aero::SC_MAXV};
    J.job[1] = {w0, p->nw, bits + aero::SC_MAXW};
    if (thermal) J.job[2] = {th0, p->nc, bits + aero::SC_MAXT};
    CUDA_TRY(aero::launch_absmax_multi<T>(J, thermal ? 3 : 2, s));
  }

  aero::StageParams<T> S{};
  S.nx = nx;
  S.ny = ny;
  S.nz = nz;
  S.zc = p->zc;
  S.h = T(c.h);
  S.inv_h = T(1.0 / c.h);
  S.ru = comp_rules<T>(c, 0, p->pu);
  S.rv = comp_rules<T>(c, 1);
  S.rw = comp_rules<T>(c, 2);
  S.status = status;
  S.wait_limit = p->wait_limit;
  S.wait_extra_tx = p->wait_extra_tx;
  S.forcing = c.forcing;
  for (int q = 0; q < 3; ++q) S.force[q] = T(c.force[q]);
  S.nu_pitch = p->pn;
  S.px = c.periodic[0];
  S.py = c.periodic[1];
  S.pz = c.periodic[2];
  S.closed = c.closed;
  S.upwind = c.advection == AERO_ADV_UPWIND3;
  S.les = c.les;
  S.kadv = T((c.advection == AERO_ADV_UPWIND3 ? 7.0 / 24.0 : 0.25) / c.h);
  S.nu_h2 = T(T(c.nu) * T(1.0 / (c.h * c.h)));
  T *nu_buf = reinterpret_cast<T *>(ws + p->off_nu);
  S.nu = nu_buf;
  aero::NuParams<T> NP{};
  NP.nx = nx;
  NP.ny = ny;
  NP.nz = nz;
  NP.zc = p->zc_nu;
  NP.les = c.les;
  NP.inv_h = T(1.0 / c.h);
  NP.cd2 = T(c.les == AERO_LES_VREMAN ? c.les_c * c.h * c.h : c.les_c * c.les_c * c.h * c.h);
  NP.ru = comp_rules<T>(c, 0, p->pu);
  NP.rv = comp_rules<T>(c, 1);
  NP.rw = comp_rules<T>(c, 2);
  NP.status = status;
  NP.wait_limit = p->wait_limit;
  NP.wait_extra_tx = p->wait_extra_tx;
  NP.nu_pitch = p->pn;
  const bool f64 = sizeof(T) == 8;
  // TMA views: stage-start u copy and nu are fixed workspace buffers; v, w, theta change by stage
  CUtensorMap map_u_stage, map_u_nu, map_nu;
  bool tma_ok = encode3d(&map_u_stage, f64, upb, nx + 1, ny, nz, p->pu, 40, 12) &&
                encode3d(&map_u_nu, f64, upb, nx + 1, ny, nz, p->pu, 36, 10);
  if (les) tma_ok = tma_ok && encode3d(&map_nu, f64, nu_buf, nx + 2, ny + 2, nz + 2, p->pn, 36, 10);
  auto stage_views = [&](const T *vp, const T *wp, const T *thp, aero::StageParams<T> &P) {
    P.use_tma = tma_ok && encode3d(&P.map_v, f64, vp, nx, ny + 1, nz, nx, 40, 12) &&
                encode3d(&P.map_w, f64, wp, nx, ny, nz + 1, nx, 40, 12) &&
                (!thermal || encode3d(&P.map_th, f64, thp, nx, ny, nz, nx, 40, 12));
    P.map_u = map_u_stage;
    if (les) P.map_nu = map_nu;
  };
  auto nu_views = [&](const T *vp, const T *wp, aero::NuParams<T> &N) {
    N.use_tma = tma_ok && encode3d(&N.map_v, f64, vp, nx, ny + 1, nz, nx, 36, 10) &&
                encode3d(&N.map_w, f64, wp, nx, ny, nz + 1, nx, 36, 10);
    N.map_u = map_u_nu;
  };
  NP.has_win = has_win;
  for (int q = 0; q < 6; ++q) NP.win[q] = has_win ? c.window[q] : 0;
  NP.wnx = c.window[5] - c.window[4];
  NP.wny = c.window[3] - c.window[2];
  NP.chi_c = static_cast<const T *>(g->chi_c);
  NP.nu = nu_buf;
  // the learned closure: the eddy-viscosity kernel leaves the gradients for the closure's pass,
  // which replaces WALE's nu_t where the learned stress applies (FP32 plans only)
  const int64_t grad_plane = (int64_t)(nz + 2) * (ny + 2) * p->pn;
  if (c.closure) {
    NP.grad = reinterpret_cast<float *>(ws + p->off_grad);
    NP.grad_plane = grad_plane;
  }
  auto closure_pass = [&](unsigned long long *nut_max) -> int {
    return aero_host::closure_nu(g->closure, reinterpret_cast<const float *>(ws + p->off_grad), grad_plane, nx + 2,
                                 ny + 2, nz + 2, p->pn, c.h, reinterpret_cast<float *>(nu_buf), nut_max,
                                 reinterpret_cast<unsigned long long *>(ws + p->off_counts), status, s);
  };
  S.dt = small;
  S.u0 = u0;
  S.v0 = v0;
  S.w0 = w0;
  S.uh = uh;
  S.vh = vh;
  S.wh = wh;
  S.u_inlet = static_cast<const T *>(g->u_inlet);
  S.outlet_corr = small + 1;
  S.has_win = has_win;
  for (int q = 0; q < 6; ++q) S.win[q] = has_win ? c.window[q] : 0;
  S.wnx = c.window[5] - c.window[4];
  S.wny = c.window[3] - c.window[2];
  S.nbody = has_win ? c.nbody : 0;
  S.nq = p->nq;
  S.eta = T(c.eta);
  S.chi_u = static_cast<const T *>(g->chi_u);
  S.chi_v = static_cast<const T *>(g->chi_v);
  S.chi_w = static_cast<const T *>(g->chi_w);
  S.chi_c = static_cast<const T *>(g->chi_c);
  if (c.paint) {
    S.paint_u = static_cast<const T *>(g->paint_u);
    S.paint_v = static_cast<const T *>(g->paint_v);
    S.paint_w = static_cast<const T *>(g->paint_w);
  }
  S.nfan = c.nfan;
  S.fan_swirl = c.fan_swirl;
  for (int q = 0; q < c.nfan; ++q) {
    const AeroNs3dFan &F = g->fans[q];
    auto &d = S.fan[q];
    for (int e = 0; e < 6; ++e) d.win[e] = F.window[e];
    d.f[0] = static_cast<const T *>(F.f_u);
    d.f[1] = static_cast<const T *>(F.f_v);
    d.f[2] = static_cast<const T *>(F.f_w);
    d.s[0] = static_cast<const T *>(F.s_u);
    d.s[1] = static_cast<const T *>(F.s_v);
    d.s[2] = static_cast<const T *>(F.s_w);
    d.thrust = static_cast<const T *>(F.thrust);
    d.swirl_amp = static_cast<const T *>(F.swirl_amp);
  }
  S.nport = c.nport;
  S.port_leak = T(c.port_leak);
  for (int q = 0; q < c.nport; ++q) {
    const AeroNs3dPort &Q = g->ports[q];
    auto &d = S.port[q];
    for (int e = 0; e < 6; ++e) d.win[e] = Q.window[e];
    d.vent = Q.vent;
    d.theta = T(Q.theta);
    d.f[0] = static_cast<const T *>(Q.f_u);
    d.f[1] = static_cast<const T *>(Q.f_v);
    d.f[2] = static_cast<const T *>(Q.f_w);
    d.m = static_cast<const T *>(Q.m);
  }
  S.nheat = thermal ? c.nheat : 0;
  for (int q = 0; q < S.nheat; ++q) {
    for (int e = 0; e < 6; ++e) S.heat[q].win[e] = g->heaters[q].window[e];
    S.heat[q].q = static_cast<const T *>(g->heaters[q].q);
  }
  S.a_u = static_cast<const T *>(g->a_u);
  S.a_v = static_cast<const T *>(g->a_v);
  S.a_w = static_cast<const T *>(g->a_w);
  S.k_u = static_cast<const T *>(g->k_u);
  S.k_v = static_cast<const T *>(g->k_v);
  S.k_w = static_cast<const T *>(g->k_w);
  S.thermal = thermal;
  if (thermal) {
    S.has_adia = c.has_adia;
    S.n_tbody = has_win ? c.n_tbody : 0;
    for (int q = 0; q < 6; ++q) {
      S.sides.kind[q] = c.side_kind[q];
      S.sides.val[q] = c.side_val[q];
    }
    S.kh = T(c.kappa / c.h);
    S.kprt = T(0.5 / (c.prt * c.h));
    S.kappa = T(c.kappa);
    S.ri = T(c.ri);
    S.eta_t = T(c.eta_t);
    S.th0 = th0;
    S.chi_t = static_cast<const T *>(g->chi_t);
    S.a_t = static_cast<const T *>(g->a_t);
    S.w_t = static_cast<const T *>(g->w_t);
    S.adia_u = static_cast<const T *>(g->adia_u);
    S.adia_v = static_cast<const T *>(g->adia_v);
    S.adia_w = static_cast<const T *>(g->adia_w);
    S.vol_w = static_cast<const T *>(g->vol_w);
    S.skin = static_cast<const T *>(g->skin);
    if (!has_win) {
      S.chi_t = S.a_t = S.w_t = S.adia_u = S.adia_v = S.adia_w = S.vol_w = S.skin = nullptr;
      S.has_adia = 0;
    }
  }

  if (les) {  // eddy viscosity of u0: the first stage's, and its maximum for the time step
    aero::NuParams<T> N = NP;
    N.up = upb;
    N.vp = v0;
    N.wp = w0;
    nu_views(v0, w0, N);
    N.nut_max = need_max && !c.closure ? bits + aero::SC_NUTMAX : nullptr;
    CUDA_TRY(aero::launch_nu<T>(N, s));
    if (c.closure) {
      const int rc = closure_pass(need_max ? bits + aero::SC_NUTMAX : nullptr);
      if (rc) return rc;
    }
  }

  aero::DtParams D{};
  D.scalars = sc;
  D.dt_in = dt_in;
  D.dt_out = small;
  D.status = status;
  D.has_dt_fixed = c.has_dt_fixed;
  D.dt_fixed = c.dt_fixed;
  D.les = les;
  D.thermal = thermal;
  D.has_heat_max = c.has_heat_max;
  D.cfl = c.cfl;
  D.h = c.h;
  D.nu = c.nu;
  D.viscous_dt = 1.0 / 6.0;
  D.kappa = c.kappa;
  D.prt = c.prt;
  D.ri = c.ri;
  D.heat_max = c.heat_max;
  D.u_floor = c.u_floor;
  D.pid = c.pid;
  D.pid_target = c.pid_target;
  D.pid_dt_prev = f->pid_dt_prev;
  D.pid_e1 = f->pid_e1;
  D.pid_e2 = f->pid_e2;
  CUDA_TRY(aero::launch_dt<T>(D, s));

  // fans: disc velocities of the step-start state and the PI thrust, before any stage
  if (c.nfan > 0) {
    aero::FanBeginParams<T> FB{};
    FB.nfan = c.nfan;
    FB.any_swirl = c.fan_swirl;
    FB.nx = nx;
    FB.ny = ny;
    FB.nz = nz;
    FB.u0 = u0;
    FB.v0 = v0;
    FB.w0 = w0;
    FB.dt = small;
    for (int q = 0; q < c.nfan; ++q) {
      const AeroNs3dFan &F = g->fans[q];
      auto &d = FB.fan[q];
      for (int e = 0; e < 6; ++e) d.win[e] = F.window[e];
      d.velocity_mode = F.velocity_mode;
      d.target = F.target;
      d.kp = F.kp;
      d.ki = F.ki;
      d.tmax = F.tmax;
      d.swirl = F.swirl;
      d.m[0] = static_cast<const T *>(F.m_u);
      d.m[1] = static_cast<const T *>(F.m_v);
      d.m[2] = static_cast<const T *>(F.m_w);
      d.thrust = static_cast<T *>(F.thrust);
      d.ud = static_cast<T *>(F.ud);
      d.e_prev = static_cast<T *>(F.e_prev);
      d.swirl_amp = static_cast<T *>(F.swirl_amp);
    }
    CUDA_TRY(aero::launch_fan_begin<T>(FB, s));
  }

  const int rows = nz * ny;
  double *psum = reinterpret_cast<double *>(ws + p->off_psum);  // [u0 outlet | inlet | 3 stages x 2] x parts
  if (tunnel) {
    (void)aero::launch_k(plane_sum_kernel<T>, PLANE_PARTS, 256, 0, s, upb, p->pu, nx, psum, S.u_inlet, 1, 0, psum + PLANE_PARTS,
                                                    rows);
    CUDA_TRY(cudaGetLastError());
  }

  CUDA_TRY(mark(1));
  static const double RK[3][3] = {{0.0, 1.0, 1.0 / 6.0}, {0.75, 0.25, 2.0 / 3.0}, {1.0 / 3.0, 2.0 / 3.0, 1.0}};
  T *p_out = static_cast<T *>(f->p);
  for (int st = 0; st < 3; ++st) {
    const T *up = upb, *vp = st == 0 ? v0 : vpb, *wp = st == 0 ? w0 : wpb;
    if (tunnel) {
      double *sums = psum + (2 + 2 * st) * PLANE_PARTS;  // outlet column, the one before it
      (void)aero::launch_k(plane_sum_kernel<T>, PLANE_PARTS, 256, 0, s, up, p->pu, nx, sums, up, p->pu, nx - 1, sums + PLANE_PARTS,
                                                      rows);
      CUDA_TRY(cudaGetLastError());
      CUDA_TRY(aero::launch_outlet_corr<T>(sums, sums + PLANE_PARTS, psum, psum + PLANE_PARTS, PLANE_PARTS, small,
                                           RK[st][0], RK[st][1], 1.0 / c.h, 1.0 / rows,
                                           c.nport > 0 ? c.port_source : 0.0, small + 1, s));
    }
    if (les && st > 0) {
      aero::NuParams<T> N = NP;
      N.up = up;
      N.vp = vp;
      N.wp = wp;
      nu_views(vp, wp, N);
      N.nut_max = nullptr;
      CUDA_TRY(aero::launch_nu<T>(N, s));
      if (c.closure) {
        const int rc = closure_pass(nullptr);
        if (rc) return rc;
      }
    }
    CUDA_TRY(mark(2 + 5 * st));
    aero::StageParams<T> P = S;
    P.a = T(RK[st][0]);
    P.bdt_scale = T(RK[st][1]);
    P.wgt = T(RK[st][2]);
    P.up = up;
    P.vp = vp;
    P.wp = wp;
    P.partials = has_win ? partials + (size_t)st * p->nblocks * p->nq : nullptr;
    if (thermal) {
      P.thp = st == 0 ? th0 : (st == 1 ? tha : thb);
      P.thh = st == 0 ? tha : (st == 1 ? thb : static_cast<T *>(f->theta));
    }
    stage_views(vp, wp, thermal ? P.thp : nullptr, P);
    CUDA_TRY(aero::launch_stage<T>(P, s));
    CUDA_TRY(mark(3 + 5 * st));
    const int acc_mode = st == 0 ? 0 : (st == 1 ? 1 : 2);
    // a diagnostics row needs the last stage's right-hand side as an array: that stage then
    // takes the unfused projection
    const bool want_div_sq = f->div_sq != nullptr && st == 2;
    if (p->ax[0].method == 0 && aero::transform_tiled(nx) && c.nport == 0 && !want_div_sq) {
      // the first x pass forms div(u_hat) itself, the last one folds psi into p
      aero::TransformParams<T> F{};
      F.fuse_div = 1;
      F.px = c.periodic[0];
      F.py = c.periodic[1];
      F.pz = c.periodic[2];
      F.uh = uh;
      F.vh = vh;
      F.wh = wh;
      F.inv_h = T(1.0 / c.h);
      F.p_acc = p_out;
      F.wgt = T(RK[st][2]);
      F.acc_mode = acc_mode;
      F.dt = small;
      CUDA_TRY(mark(4 + 5 * st));
      const int rc = poisson_passes<T>(p, nullptr, pa, ws, s, &F);
      if (rc) return rc;
    } else {
      CUDA_TRY(aero::launch_divergence<T>(uh, vh, wh, nx, ny, nz, c.periodic[0], c.periodic[1], c.periodic[2],
                                          T(1.0 / c.h), pa, s));
      CUDA_TRY(aero::launch_port_continuity<T>(pa, nx, ny, S.nport, S.port, s));  // div - m (jets, vents)
      if (want_div_sq)
        CUDA_TRY(aero::launch_sumsq<T>(pa, p->nc, reinterpret_cast<double *>(ws + p->off_sumsq),
                                       static_cast<T *>(f->div_sq), s));
      CUDA_TRY(mark(4 + 5 * st));
      const int rc = poisson_passes<T>(p, pa, pa, ws, s);
      if (rc) return rc;
      CUDA_TRY(aero::launch_psi_accumulate<T>(pa, p_out, p->nc, T(RK[st][2]), acc_mode, small, s));
    }
    CUDA_TRY(mark(5 + 5 * st));
    aero::CorrectParams<T> C{};
    C.nx = nx;
    C.ny = ny;
    C.nz = nz;
    C.px = c.periodic[0];
    C.py = c.periodic[1];
    C.pz = c.periodic[2];
    C.inv_h = T(1.0 / c.h);
    C.uh = uh;
    C.vh = vh;
    C.wh = wh;
    C.psi = pa;
    C.u = st == 2 ? static_cast<T *>(f->u) : upb;
    C.pu_out = st == 2 ? nx + 1 : p->pu;
    C.v = st == 2 ? static_cast<T *>(f->v) : vpb;
    C.w = st == 2 ? static_cast<T *>(f->w) : wpb;
    CUDA_TRY(aero::launch_correct<T>(C, s));
    CUDA_TRY(mark(6 + 5 * st));
  }

  const T *t0 = static_cast<const T *>(f->t0);
  if (c.smoke) {
    const int rc = smoke_impl<T>(p, f, g, small, nullptr, s);
    if (rc) return rc;
  }
  CUDA_TRY(mark(17));

  aero::FinalizeParams<T> F{};
  F.ncell = p->nc;
  F.nbody = has_win ? c.nbody : 0;
  F.nq = p->nq;
  F.nblocks = p->nblocks;
  F.n_tbody = thermal && has_win ? c.n_tbody : 0;
  F.symmetry = c.symmetry;
  F.partials = partials;
  F.tot = sc + aero::SC_TOT;
  F.h = c.h;
  F.pe = c.pe;
  F.y0 = c.y0;
  F.moment_ref_y = c.moment_ref[1];
  F.ref_area = c.ref_area;
  F.span_ref = c.span_ref;
  F.length_ref = c.length_ref;
  for (int q = 0; q < AERO_MAX_BODIES; ++q) {
    F.t_index[q] = c.t_index[q];
    F.flux_rate[q] = c.flux_rate[q];
  }
  F.dt = small;
  F.t0 = t0;
  F.t_out = static_cast<T *>(f->t);
  F.dt_out = static_cast<T *>(f->dt);
  F.coeffs = static_cast<T *>(f->coeffs);
  F.heat_rate = thermal ? static_cast<T *>(f->heat_rate) : nullptr;
  F.p = p_out;
  F.status = status;
  CUDA_TRY(aero::launch_finalize<T>(F, s));
  CUDA_TRY(mark(18));
  return AERO_OK;
}

template <typename T>
int init_impl(const AeroNs3dPlan *p, unsigned char *ws, cudaStream_t s) {
  CUDA_TRY(cudaMemsetAsync(ws, 0, p->total, s));
  for (int a = 0; a < 3; ++a) CUDA_TRY(aero_host::axis_init<T>(p->ax[a], p->cfg.h, ws, s));
  return AERO_OK;
}

template <typename T>
int poisson_impl(const AeroNs3dPlan *p, const void *f, void *psi, unsigned char *ws, cudaStream_t s) {
  return poisson_passes<T>(p, static_cast<const T *>(f), static_cast<T *>(psi), ws, s);
}

template <typename T>
int project_impl(const AeroNs3dPlan *p, void *u, void *v, void *w, void *psi, unsigned char *ws, cudaStream_t s) {
  const AeroNs3dConfig &c = p->cfg;
  T *pa = reinterpret_cast<T *>(ws + p->off_pa);
  T *upb = reinterpret_cast<T *>(ws + p->off_uh), *vpb = reinterpret_cast<T *>(ws + p->off_vh),
    *wpb = reinterpret_cast<T *>(ws + p->off_wh);
  CUDA_TRY(aero::launch_divergence<T>(static_cast<T *>(u), static_cast<T *>(v), static_cast<T *>(w), c.nx, c.ny, c.nz,
                                      c.periodic[0], c.periodic[1], c.periodic[2], T(1.0 / c.h), pa, s));
  const int rc = poisson_passes<T>(p, pa, static_cast<T *>(psi), ws, s);
  if (rc) return rc;
  aero::CorrectParams<T> C{};
  C.nx = c.nx;
  C.ny = c.ny;
  C.nz = c.nz;
  C.px = c.periodic[0];
  C.py = c.periodic[1];
  C.pz = c.periodic[2];
  C.inv_h = T(1.0 / c.h);
  C.uh = static_cast<T *>(u);
  C.vh = static_cast<T *>(v);
  C.wh = static_cast<T *>(w);
  C.psi = static_cast<T *>(psi);
  C.u = upb;
  C.v = vpb;
  C.w = wpb;
  C.pu_out = c.nx + 1;
  CUDA_TRY(aero::launch_correct<T>(C, s));
  CUDA_TRY(cudaMemcpyAsync(u, upb, p->nu * sizeof(T), cudaMemcpyDeviceToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(v, vpb, p->nv * sizeof(T), cudaMemcpyDeviceToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(w, wpb, p->nw * sizeof(T), cudaMemcpyDeviceToDevice, s));
  return AERO_OK;
}

// ---- allocation-free Poisson solve -------------------------------------------------
// The per-axis transform tables (twiddles, DCT post-twiddles, cos/sin, eigenvalues, dense
// matrices) normally live in the caller's workspace.  aero_ns3d_poisson_solve_static keeps
// them in this file-scope device array instead: every GPU that loads the library holds its
// AERO_STATIC_SCRATCH_BYTES until the process exits, and no call allocates anything.  Every
// call rewrites all of the tables it reads before reading them, so nothing in the array has
// to start at zero; calls that overlap on the GPU (two streams, two host threads) share the
// array and race.
static __device__ __align__(256) unsigned char g_static_scratch[AERO_STATIC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
void *g_scratch_addr[kMaxDevices];  // device address of g_static_scratch, per device ordinal

// Set-up, once per device and with that device current: g_static_scratch is a host-side
// stand-in for the symbol, so its device address comes from cudaGetSymbolAddress.  On a
// device's first call this may load the library's device code (lazy module loading).
int static_scratch(unsigned char **out) {
  int dev = -1;
  CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return fail(AERO_EUNSUPPORTED, "device ordinal beyond 63");
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_addr[dev]) {
    void *ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_static_scratch);
    if (e != cudaSuccess || !ptr)
      return fail(AERO_ECUDA, std::string("cudaGetSymbolAddress(static scratch): ") + cudaGetErrorString(e));
    g_scratch_addr[dev] = ptr;
  }
  *out = static_cast<unsigned char *>(g_scratch_addr[dev]);
  return AERO_OK;
}

// The plan's tables re-laid out back to back (256-byte aligned) from offset 0; returns the bytes.
size_t compact_tables(AeroNs3dPlan *q) {
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t at = off;
    off += (bytes + ALIGN - 1) / ALIGN * ALIGN;
    return at;
  };
  for (int a = 0; a < 3; ++a) aero_host::axis_place(q->ax[a], q->esz, take);
  return off;
}

template <typename T>
int poisson_static_impl(const AeroNs3dPlan *plan, const void *f, void *psi, cudaStream_t s) {
  AeroNs3dPlan q = *plan;  // host copy whose table offsets point into the static scratch
  const size_t need = compact_tables(&q);
  if (need > AERO_STATIC_SCRATCH_BYTES)
    return fail(AERO_EINVAL, "the transform tables of this grid need " + std::to_string(need) +
                                 " bytes; the static scratch holds " + std::to_string(AERO_STATIC_SCRATCH_BYTES) +
                                 " (use aero_ns3d_poisson_solve with a workspace)");
  unsigned char *scratch = nullptr;
  const int rc = static_scratch(&scratch);
  if (rc) return rc;
  for (int a = 0; a < 3; ++a) CUDA_TRY(aero_host::axis_init<T>(q.ax[a], q.cfg.h, scratch, s));
  return poisson_passes<T>(&q, static_cast<const T *>(f), static_cast<T *>(psi), scratch, s);
}

template <typename T>
int fields_impl(const AeroNs3dPlan *p, const void *u, const void *v, const void *w, const AeroNs3dGeom *g,
                void *const *out, cudaStream_t s) {
  const AeroNs3dConfig &c = p->cfg;
  aero::FieldsParams<T> F{};
  F.nx = c.nx;
  F.ny = c.ny;
  F.nz = c.nz;
  F.les = c.les;
  F.inv_h = T(1.0 / c.h);
  F.cd2 = T(c.les == AERO_LES_VREMAN ? c.les_c * c.h * c.h : c.les_c * c.les_c * c.h * c.h);
  F.ru = comp_rules<T>(c, 0);
  F.rv = comp_rules<T>(c, 1);
  F.rw = comp_rules<T>(c, 2);
  F.u = static_cast<const T *>(u);
  F.v = static_cast<const T *>(v);
  F.w = static_cast<const T *>(w);
  const bool has_win = !(c.window[1] <= c.window[0] || c.window[3] <= c.window[2] || c.window[5] <= c.window[4]) &&
                       c.nbody > 0 && g && g->chi_c;
  F.has_win = has_win;
  for (int q = 0; q < 6; ++q) F.win[q] = has_win ? c.window[q] : 0;
  F.wnx = c.window[5] - c.window[4];
  F.wny = c.window[3] - c.window[2];
  F.chi_c = has_win ? static_cast<const T *>(g->chi_c) : nullptr;
  for (int q = 0; q < AERO_FIELD_COUNT; ++q) F.out[q] = static_cast<T *>(out[q]);
  F.gradient = out[4] || out[5] || out[6];
  CUDA_TRY(aero::launch_fields<T>(F, s));
  return AERO_OK;
}

bool window_empty(const int32_t *w) { return w[1] <= w[0] || w[3] <= w[2] || w[5] <= w[4]; }

}  // namespace

extern "C" {

int aero_abi_version(void) { return AERO_ABI_VERSION; }

const char *aero_last_error(void) { return g_last_error.c_str(); }

int aero_ns3d_plan_create(const AeroNs3dConfig *cfg, AeroNs3dPlan **plan) {
  if (!cfg || !plan) return fail(AERO_EINVAL, "null argument");
  *plan = nullptr;
  const AeroNs3dConfig &c = *cfg;
  if (c.abi_version != AERO_ABI_VERSION) return fail(AERO_EINVAL, "ABI version mismatch");
  if (c.dtype != AERO_F32 && c.dtype != AERO_F64) return fail(AERO_EINVAL, "dtype must be float32 or float64");
  if (c.nx < 4 || c.ny < 4 || c.nz < 4) return fail(AERO_EINVAL, "the grid needs at least 4 x 4 x 4 cells");
  if (!(c.h > 0) || !std::isfinite(c.h)) return fail(AERO_EINVAL, "cell size h must be positive");
  if (c.advection != AERO_ADV_UPWIND3 && c.advection != AERO_ADV_CENTRAL) return fail(AERO_EINVAL, "unknown advection");
  if (c.les < AERO_LES_NONE || c.les > AERO_LES_VREMAN) return fail(AERO_EINVAL, "unknown turbulence model");
  if (c.closure && (c.les != AERO_LES_WALE || c.dtype != AERO_F32))
    return fail(AERO_EINVAL, "the learned closure runs on WALE (its fallback) in FP32 plans");
  if (c.nbody < 0 || c.nbody > AERO_MAX_BODIES)
    return fail(AERO_EUNSUPPORTED, "at most " + std::to_string(AERO_MAX_BODIES) + " bodies");
  for (int comp = 0; comp < 3; ++comp)
    for (int a = 0; a < 3; ++a)
      for (int sd = 0; sd < 2; ++sd)
        if (c.ghost_kind[comp][a][sd] < AERO_GHOST_EDGE || c.ghost_kind[comp][a][sd] > AERO_GHOST_PERIODIC_FACE)
          return fail(AERO_EINVAL, "unknown ghost rule");
  if (!window_empty(c.window)) {
    if (c.window[0] < 0 || c.window[1] > c.nz || c.window[2] < 0 || c.window[3] > c.ny || c.window[4] < 0 ||
        c.window[5] > c.nx)
      return fail(AERO_EINVAL, "body window outside the domain");
  }
  if (c.thermal) {
    if (c.n_tbody < 0 || c.n_tbody > c.nbody) return fail(AERO_EINVAL, "bad temperature-body count");
    for (int q = 0; q < 6; ++q)
      if (c.side_kind[q] < AERO_TH_PERIODIC || c.side_kind[q] > AERO_TH_HEAT_FLUX)
        return fail(AERO_EINVAL, "unknown thermal side condition");
    if (!(c.prt > 0) || !(c.eta_t > 0)) return fail(AERO_EINVAL, "bad thermal constants");
  }
  if (c.smoke && !window_empty(c.dye_window)) {
    if (c.dye_window[0] < 0 || c.dye_window[1] > c.nz || c.dye_window[2] < 0 || c.dye_window[3] > c.ny ||
        c.dye_window[4] < 0 || c.dye_window[5] > c.nx)
      return fail(AERO_EINVAL, "smoke nozzle window outside the domain");
  }
  if (!(c.eta > 0)) return fail(AERO_EINVAL, "eta must be positive");
  if (!(c.u_floor >= 0) || !std::isfinite(c.u_floor)) return fail(AERO_EINVAL, "u_floor must be >= 0");
  if (c.pid && !(c.pid_target >= 0.1 && c.pid_target <= 1.0)) return fail(AERO_EINVAL, "pid_target must be in [0.1, 1]");
  if (c.nfan < 0 || c.nfan > AERO_MAX_FANS)
    return fail(AERO_EUNSUPPORTED, "at most " + std::to_string(AERO_MAX_FANS) + " fans");
  if (c.nheat < 0 || c.nheat > AERO_MAX_HEATERS)
    return fail(AERO_EUNSUPPORTED, "at most " + std::to_string(AERO_MAX_HEATERS) + " volumetric heaters");
  if (c.nheat > 0 && !c.thermal) return fail(AERO_EINVAL, "heaters need heat transfer");
  if (c.nport < 0 || c.nport > AERO_MAX_PORTS)
    return fail(AERO_EUNSUPPORTED, "at most " + std::to_string(AERO_MAX_PORTS) + " jets and vents");
  if (c.nport > 0 && c.smoke)
    return fail(AERO_EUNSUPPORTED, "jets and vents with the smoke update inside the step: run the step without "
                                   "smoke and apply their smoke sources after aero_ns3d_smoke");
  AeroNs3dPlan *p = new AeroNs3dPlan();
  p->cfg = c;
  p->esz = c.dtype == AERO_F64 ? 8 : 4;
  const size_t nx = c.nx, ny = c.ny, nz = c.nz;
  p->nu = nz * ny * (nx + 1);
  p->nv = nz * (ny + 1) * nx;
  p->nw = (nz + 1) * ny * nx;
  p->nc = nz * ny * nx;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off = align_up(off + bytes);
    return o;
  };
  const size_t e = p->esz;
  p->off_uh = take(p->nu * e);
  p->off_vh = take(p->nv * e);
  p->off_wh = take(p->nw * e);
  p->pu = (int)((nx + 1 + 3) / 4 * 4);
  p->pn = (int)((nx + 2 + 3) / 4 * 4);
  p->off_up = take(nz * ny * (size_t)p->pu * e);
  p->off_vp = take(p->nv * e);
  p->off_wp = take(p->nw * e);
  p->off_tha = take(c.thermal ? p->nc * e : 0);
  p->off_thb = take(c.thermal ? p->nc * e : 0);
  p->off_pa = take(p->nc * e);
  p->off_nu = take(c.les != AERO_LES_NONE ? (nz + 2) * (ny + 2) * (size_t)p->pn * e : 0);
  p->off_grad = take(c.closure ? 9 * (nz + 2) * (ny + 2) * (size_t)p->pn * sizeof(float) : 0);
  p->off_counts = take(c.closure ? 2 * sizeof(unsigned long long) : 0);
  p->off_small = take(8 * e);
  p->off_scalars = take(sizeof(double) * aero::SC_COUNT);
  p->off_status = take(sizeof(int) * 4);
  // planes per CTA: the stage kernel in chunks of about 19 planes (at 256 x 128 x 128: 896
  // CTAs, two full waves at 3 CTAs per SM on 148 SMs; 16 planes gave 1024 CTAs, 2.3 waves, and
  // a 4 % slower stage), the eddy-viscosity kernel (5 CTAs per SM) in chunks of 16
  const int nch = std::max(1, (int)std::lround(c.nz / 19.0));
  p->zc = (c.nz + nch - 1) / nch;
  p->zc_nu = c.nz <= 16 ? c.nz : 16;
  p->nblocks = (int)(((nx + 31) / 32) * ((ny + 7) / 8) * ((nz + p->zc - 1) / p->zc));
  p->nq = c.nbody * 9 + (c.thermal ? c.n_tbody : 0);
  p->off_partials = take(sizeof(double) * 3 * (size_t)p->nblocks * std::max(p->nq, 1));
  p->off_psum = take(sizeof(double) * 8 * PLANE_PARTS);
  p->off_sumsq = take(sizeof(double) * aero::SUMSQ_PARTS);
  const int ns[3] = {c.nx, c.ny, c.nz};
  for (int a = 0; a < 3; ++a) {
    AxisInfo &x = p->ax[a];
    aero_host::axis_setup(x, ns[a], c.periodic[a] != 0, e);
    aero_host::axis_place(x, e, take);
  }
  p->total = off;
  *plan = p;
  return AERO_OK;
}

void aero_ns3d_plan_destroy(AeroNs3dPlan *plan) { delete plan; }

size_t aero_ns3d_workspace_bytes(const AeroNs3dPlan *plan) { return plan ? plan->total : 0; }

int aero_ns3d_workspace_init(const AeroNs3dPlan *plan, void *workspace, void *stream) {
  if (!plan || !workspace) return fail(AERO_EINVAL, "null argument");
  if (reinterpret_cast<uintptr_t>(workspace) % ALIGN) return fail(AERO_EINVAL, "workspace must be 256-byte aligned");
  auto s = static_cast<cudaStream_t>(stream);
  auto ws = static_cast<unsigned char *>(workspace);
  return plan->cfg.dtype == AERO_F64 ? init_impl<double>(plan, ws, s) : init_impl<float>(plan, ws, s);
}

int aero_ns3d_step(const AeroNs3dPlan *plan, const AeroNs3dFields *f, const AeroNs3dGeom *g, const void *dt_in,
                   void *workspace, void *stream) {
  return aero_ns3d_step_traced(plan, f, g, dt_in, workspace, stream, nullptr, 0);
}

int aero_ns3d_step_traced(const AeroNs3dPlan *plan, const AeroNs3dFields *f, const AeroNs3dGeom *g,
                          const void *dt_in, void *workspace, void *stream, void *const *events, int32_t nevents) {
  if (!plan || !f || !g || !workspace) return fail(AERO_EINVAL, "null argument");
  if (reinterpret_cast<uintptr_t>(workspace) % ALIGN) return fail(AERO_EINVAL, "workspace must be 256-byte aligned");
  const AeroNs3dConfig &c = plan->cfg;
  if (!f->u0 || !f->v0 || !f->w0 || !f->u || !f->v || !f->w || !f->p || !f->t0 || !f->t || !f->dt)
    return fail(AERO_EINVAL, "missing state pointer");
  if (c.thermal && (!f->theta0 || !f->theta)) return fail(AERO_EINVAL, "heat transfer needs theta pointers");
  if (c.smoke && (!f->dye0 || !f->dye)) return fail(AERO_EINVAL, "smoke needs dye pointers");
  if (c.smoke && f->dye0 == f->dye) return fail(AERO_EINVAL, "dye output must not alias dye input");
  if (!c.periodic[0] && !c.closed && !g->u_inlet) return fail(AERO_EINVAL, "missing inlet profile");
  if (!window_empty(c.window) && c.nbody > 0) {
    if (!g->chi_u || !g->chi_v || !g->chi_w || !g->chi_c || !g->a_u || !g->a_v || !g->a_w || !g->k_u || !g->k_v ||
        !g->k_w || !f->coeffs)
      return fail(AERO_EINVAL, "missing body masks");
    if (c.thermal && c.n_tbody > 0 && (!g->chi_t || !g->a_t || !g->w_t)) return fail(AERO_EINVAL, "missing thermal masks");
    if (c.thermal && c.has_adia && (!g->adia_u || !g->adia_v || !g->adia_w))
      return fail(AERO_EINVAL, "missing adiabatic masks");
    if (c.thermal && c.has_skin && !g->skin) return fail(AERO_EINVAL, "missing heat-flux skin");
  }
  if (c.thermal && !f->heat_rate && c.nbody > 0) return fail(AERO_EINVAL, "missing heat-rate output");
  if (c.closure && (!g->closure || !g->closure->params || !g->closure->params_bf16))
    return fail(AERO_EINVAL, "the learned closure needs its model");
  if (c.paint && (!g->paint_u || !g->paint_v || !g->paint_w || (c.smoke && !g->paint_c)))
    return fail(AERO_EINVAL, "missing paint masks");
  if (c.pid && (!f->pid_dt_prev || !f->pid_e1 || !f->pid_e2)) return fail(AERO_EINVAL, "missing PID state");
  if (c.nheat > 0) {
    if (!g->heaters) return fail(AERO_EINVAL, "missing heater descriptors");
    for (int q = 0; q < c.nheat; ++q) {
      const AeroNs3dHeater &Hq = g->heaters[q];
      if (window_empty(Hq.window) || Hq.window[0] < 0 || Hq.window[1] > c.nz || Hq.window[2] < 0 ||
          Hq.window[3] > c.ny || Hq.window[4] < 0 || Hq.window[5] > c.nx)
        return fail(AERO_EINVAL, "heater window empty or outside the domain");
      if (!Hq.q) return fail(AERO_EINVAL, "missing heater density");
    }
  }
  if (c.nport > 0) {
    if (!g->ports) return fail(AERO_EINVAL, "missing port descriptors");
    for (int q = 0; q < c.nport; ++q) {
      const AeroNs3dPort &Q = g->ports[q];
      if (window_empty(Q.window) || Q.window[0] < 0 || Q.window[1] > c.nz || Q.window[2] < 0 || Q.window[3] > c.ny ||
          Q.window[4] < 0 || Q.window[5] > c.nx)
        return fail(AERO_EINVAL, "port window empty or outside the domain");
      if (!Q.f_u || !Q.f_v || !Q.f_w || !Q.m) return fail(AERO_EINVAL, "missing port weights");
    }
  }
  if (c.nfan > 0) {
    if (!g->fans) return fail(AERO_EINVAL, "missing fan descriptors");
    for (int q = 0; q < c.nfan; ++q) {
      const AeroNs3dFan &F = g->fans[q];
      if (window_empty(F.window) || F.window[0] < 0 || F.window[1] > c.nz || F.window[2] < 0 || F.window[3] > c.ny ||
          F.window[4] < 0 || F.window[5] > c.nx)
        return fail(AERO_EINVAL, "fan window empty or outside the domain");
      if (!F.f_u || !F.f_v || !F.f_w || !F.m_u || !F.m_v || !F.m_w || !F.thrust || !F.ud || !F.e_prev ||
          !F.swirl_amp || (c.fan_swirl && (!F.s_u || !F.s_v || !F.s_w)))
        return fail(AERO_EINVAL, "missing fan weights or state");
    }
  }
  auto s = static_cast<cudaStream_t>(stream);
  auto ws = static_cast<unsigned char *>(workspace);
  return c.dtype == AERO_F64 ? step_impl<double>(plan, f, g, dt_in, ws, s, events, nevents)
                             : step_impl<float>(plan, f, g, dt_in, ws, s, events, nevents);
}

int aero_ns3d_smoke(const AeroNs3dPlan *plan, const AeroNs3dFields *f, const AeroNs3dGeom *g, void *stream) {
  if (!plan || !f || !g) return fail(AERO_EINVAL, "null argument");
  if (!plan->cfg.smoke) return fail(AERO_EINVAL, "the plan has no smoke");
  if (!f->dye0 || !f->dye || !f->u || !f->v || !f->w || !f->t || !f->dt) return fail(AERO_EINVAL, "missing pointer");
  if (f->dye0 == f->dye) return fail(AERO_EINVAL, "dye output must not alias dye input");
  auto s = static_cast<cudaStream_t>(stream);
  return plan->cfg.dtype == AERO_F64
             ? smoke_impl<double>(plan, f, g, static_cast<const double *>(f->dt), static_cast<const double *>(f->t), s)
             : smoke_impl<float>(plan, f, g, static_cast<const float *>(f->dt), static_cast<const float *>(f->t), s);
}

int aero_ns3d_poisson_solve(const AeroNs3dPlan *plan, const void *f, void *psi, void *workspace, void *stream) {
  if (!plan || !f || !psi || !workspace) return fail(AERO_EINVAL, "null argument");
  auto s = static_cast<cudaStream_t>(stream);
  auto ws = static_cast<unsigned char *>(workspace);
  return plan->cfg.dtype == AERO_F64 ? poisson_impl<double>(plan, f, psi, ws, s)
                                     : poisson_impl<float>(plan, f, psi, ws, s);
}

int aero_ns3d_poisson_solve_static(const AeroNs3dPlan *plan, const void *f, void *psi, void *stream) {
  if (!plan || !f || !psi) return fail(AERO_EINVAL, "null argument");
  auto s = static_cast<cudaStream_t>(stream);
  return plan->cfg.dtype == AERO_F64 ? poisson_static_impl<double>(plan, f, psi, s)
                                     : poisson_static_impl<float>(plan, f, psi, s);
}

int aero_ns3d_closure_counts(const AeroNs3dPlan *plan, const void *workspace, uint64_t out[2], void *stream) {
  if (!plan || !workspace || !out) return fail(AERO_EINVAL, "null argument");
  if (!plan->cfg.closure) return fail(AERO_EINVAL, "the plan has no learned closure");
  uint64_t h[2] = {0, 0};
  auto s = static_cast<cudaStream_t>(stream);
  CUDA_TRY(cudaMemcpyAsync(h, static_cast<const unsigned char *>(workspace) + plan->off_counts, sizeof(h),
                           cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  out[0] = h[0];
  out[1] = h[1];
  return AERO_OK;
}

int aero_ns3d_fields(const AeroNs3dPlan *plan, const void *u, const void *v, const void *w, const AeroNs3dGeom *g,
                     void *const *out, void *stream) {
  if (!plan || !u || !v || !w || !out) return fail(AERO_EINVAL, "null argument");
  auto s = static_cast<cudaStream_t>(stream);
  return plan->cfg.dtype == AERO_F64 ? fields_impl<double>(plan, u, v, w, g, out, s)
                                     : fields_impl<float>(plan, u, v, w, g, out, s);
}

int aero_ns3d_probe(const AeroNs3dPlan *plan, const void *field, const int32_t shape[3], const double origin[3],
                    const double off[3], const void *pts, int64_t npts, void *out, void *stream) {
  if (!plan || !field || !shape || !origin || !off || (npts > 0 && (!pts || !out)))
    return fail(AERO_EINVAL, "null argument");
  if (npts < 0 || shape[0] < 1 || shape[1] < 1 || shape[2] < 1) return fail(AERO_EINVAL, "bad shape or point count");
  auto s = static_cast<cudaStream_t>(stream);
  if (plan->cfg.dtype == AERO_F64)
    CUDA_TRY(aero::launch_probe<double>(static_cast<const double *>(field), shape[2], shape[1], shape[0], origin,
                                        plan->cfg.h, off, static_cast<const double *>(pts), npts,
                                        static_cast<double *>(out), s));
  else
    CUDA_TRY(aero::launch_probe<float>(static_cast<const float *>(field), shape[2], shape[1], shape[0], origin,
                                       plan->cfg.h, off, static_cast<const float *>(pts), npts,
                                       static_cast<float *>(out), s));
  return AERO_OK;
}

int aero_ns3d_project(const AeroNs3dPlan *plan, void *u, void *v, void *w, void *psi, void *workspace, void *stream) {
  if (!plan || !u || !v || !w || !psi || !workspace) return fail(AERO_EINVAL, "null argument");
  auto s = static_cast<cudaStream_t>(stream);
  auto ws = static_cast<unsigned char *>(workspace);
  return plan->cfg.dtype == AERO_F64 ? project_impl<double>(plan, u, v, w, psi, ws, s)
                                     : project_impl<float>(plan, u, v, w, psi, ws, s);
}

int aero_debug_check(int64_t *out4) {
#ifdef AERO_BOUNDS_CHECK
  long long w[4];
  CUDA_TRY(cudaMemcpyFromSymbol(w, aero::aero_check_word, sizeof(w)));
  for (int q = 0; q < 4; ++q) out4[q] = w[q];
  const long long zero[4] = {0, 0, 0, 0};
  CUDA_TRY(cudaMemcpyToSymbol(aero::aero_check_word, zero, sizeof(zero)));
  return AERO_OK;
#else
  (void)out4;
  return fail(AERO_EUNSUPPORTED, "bounds checks are compiled only into libaero_b200_checked.so");
#endif
}

int aero_ns3d_read_status(const AeroNs3dPlan *plan, const void *workspace, int32_t *status, void *stream) {
  if (!plan || !workspace || !status) return fail(AERO_EINVAL, "null argument");
  auto s = static_cast<cudaStream_t>(stream);
  int v = 0;
  CUDA_TRY(cudaMemcpyAsync(&v, static_cast<const unsigned char *>(workspace) + plan->off_status, sizeof(int),
                           cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  *status = v;
  return AERO_OK;
}

int aero_ns3d_set_wait_bound(AeroNs3dPlan *plan, int32_t spin_limit, int32_t test_extra_bytes) {
  if (!plan || spin_limit < 0 || test_extra_bytes < 0 || test_extra_bytes > 4096)
    return fail(AERO_EINVAL, "bad wait bound");
  plan->wait_limit = spin_limit;
  plan->wait_extra_tx = test_extra_bytes;
  return AERO_OK;
}

}  // extern "C"
