// The 2D step of the C ABI: Aerolume ns2d/core.py:815-969 (step_full) with heat transfer as
// its only placed physics (physics.py:623-884, core.py:774-813, 974-995), and the dye update
// of its lines 959-962.
//
// Arithmetic follows the reference's plain-torch step operation by operation, so float64
// runs agree with it to round-off:
//   ghosts     core.py:284-325     advection  core.py:366-383   diffusion core.py:417-424
//   LES        core.py:427-525     boundaries core.py:571-613, 337-359
//   penalty    core.py:663-682     projection core.py:620-660   dt        core.py:685-696
//   dye        core.py:703-735, 779-792
//
// Layout: C-contiguous (y, x) arrays, u (ny, nx+1), v (ny+1, nx), cells (ny, nx).  One
// launch per stage computes the tendencies of a 32 x 8 tile of u- and v-faces from shared-
// memory tiles of the stage-start velocity (ghost values from the index maps of
// common.cuh), the eddy viscosity and stresses of the tile's cells and corners, the RK
// blend, the inlet / outlet balance, the implicit Brinkman penalisation and the bodies'
// force partials.  The Poisson solve runs the transform kernels of poisson.cu on the grid
// as (nz, ny, nx) = (ny, 1, nx): x forward, y forward-solve-inverse, x inverse.
#include <cstring>
#include <type_traits>
#include <vector>

#include "host_common.cuh"
#include "ns3d.cuh"
#include "stencil.cuh"
#include "transform.cuh"

namespace aero {
namespace ns2d {

constexpr int TX = 32, TY = 8, NT = TX * TY;
constexpr int UX = TX + 5, UY = TY + 4;  // u tile: faces i0-2 .. i0+TX+2, rows j0-2 .. j0+TY+1
constexpr int VX = TX + 4, VY = TY + 5;  // v tile: columns i0-2 .. i0+TX+1, faces j0-2 .. j0+TY+2
constexpr int CX = TX + 2, CY = TY + 2;  // cells i0-1 .. i0+TX, j0-1 .. j0+TY
constexpr int KX = TX + 1, KY = TY + 1;  // corners i0 .. i0+TX, j0 .. j0+TY
constexpr int MAXQ = 4 * AERO_MAX_BODIES;

// Ghost rules of one component on its (n1, n0) = (y, x) array; rules compose x, then y.
template <typename T>
struct Rules2 {
  int n0, n1, p0;  // entries along x and y (face arrays: with the periodic duplicate), row pitch
  int kind[2][2];
  T val[2][2];
};

// value at (j, i) of a field with its ghost rules; load(mj, mi) gives the in-range entries
template <typename T, class Load>
__device__ __forceinline__ T padded2f(const Rules2<T> &r, int j, int i, const Load &load) {
  T sx, cx, sy, cy;
  const int mi = ghost_map<T>(i, r.n0, r.kind[0][0], r.kind[0][1], r.val[0][0], r.val[0][1], sx, cx);
  const int mj = ghost_map<T>(j, r.n1, r.kind[1][0], r.kind[1][1], r.val[1][0], r.val[1][1], sy, cy);
  const T x = load(mj, mi);
  return sy * (sx * x + cx) + cy;
}

// NC: read through the non-coherent read-only path (__ldg), right for a launch that does not
// write the array; the batched sweep's persistent kernel, which rewrites psi and the stage
// values between its phases, reads them with coherent loads (NC = false).
template <bool NC, typename T>
__device__ __forceinline__ T ldx(const T *p) {
  if constexpr (NC) return __ldg(p);
  else return *p;
}

template <typename T, bool NC = true>
__device__ __forceinline__ T padded2(const T *__restrict__ f, const Rules2<T> &r, int j, int i) {
  return padded2f<T>(r, j, i, [&](int mj, int mi) { return ldx<NC>(f + (size_t)mj * r.p0 + mi); });
}

// The projected velocity u = u_hat - grad psi on the u-face (j, fi) and the v-face (fj, i),
// the correction of ns2d/core.py:632-646 (boundary-normal faces of a bounded domain keep
// u_hat; a periodic domain wraps psi); correct2d_kernel writes the same values.
template <typename T, bool NC = true>
__device__ __forceinline__ T projected_u(const T *__restrict__ uh, const T *__restrict__ psi, int nx, int periodic,
                                         T inv_h, int j, int fi) {
  const size_t c = (size_t)j * nx;
  const T x = ldx<NC>(uh + (size_t)j * (nx + 1) + fi);
  if (periodic) {
    const int ii = fi == nx ? 0 : fi, il = ii == 0 ? nx - 1 : ii - 1;
    return x - (ldx<NC>(psi + c + ii) - ldx<NC>(psi + c + il)) * inv_h;
  }
  if (fi == 0 || fi == nx) return x;
  return x - (ldx<NC>(psi + c + fi) - ldx<NC>(psi + c + fi - 1)) * inv_h;
}

template <typename T, bool NC = true>
__device__ __forceinline__ T projected_v(const T *__restrict__ vh, const T *__restrict__ psi, int nx, int ny,
                                         int periodic, T inv_h, int fj, int i) {
  const T x = ldx<NC>(vh + (size_t)fj * nx + i);
  if (periodic) {
    const int jj = fj == ny ? 0 : fj, jl = jj == 0 ? ny - 1 : jj - 1;
    return x - (ldx<NC>(psi + (size_t)jj * nx + i) - ldx<NC>(psi + (size_t)jl * nx + i)) * inv_h;
  }
  if (fj == 0 || fj == ny) return x;
  return x - (ldx<NC>(psi + (size_t)fj * nx + i) - ldx<NC>(psi + (size_t)(fj - 1) * nx + i)) * inv_h;
}

// Eddy viscosity of the 2D gradient (core.py:469-500); cfac = c^2 h^2 (Smagorinsky, WALE)
// or c h^2 (Vreman).
template <typename T>
__device__ __forceinline__ T eddy2d(T g11, T g12, T g21, T g22, int model, T cfac) {
  const T s12 = T(0.5) * (g12 + g21);
  const T ss = (g11 * g11 + g22 * g22) + T(2) * s12 * s12;
  if (model == AERO_LES_SMAGORINSKY) return cfac * sqrt(T(2) * ss + T(1e-30));
  if (model == AERO_LES_WALE) {
    const T q11 = g11 * g11 + g12 * g21;
    const T q22 = g21 * g12 + g22 * g22;
    const T q12 = T(0.5) * (((g11 * g12 + g12 * g22) + g21 * g11) + g22 * g21);
    const T tr3 = (q11 + q22) * T(1.0 / 3.0);
    const T d1 = q11 - tr3, d2 = q22 - tr3;
    const T sd = ((d1 * d1 + d2 * d2) + T(2) * q12 * q12) + tr3 * tr3;
    const T sdp = sd > T(0) ? sd : T(0), ssp = ss > T(0) ? ss : T(0);
    const T num = pow(sdp, T(1.5));
    const T den = (pow(ssp, T(2.5)) + pow(sdp, T(1.25))) + T(1e-30);
    return cfac * num / den;
  }
  // Vreman
  const T b11 = g11 * g11 + g12 * g12;
  const T b22 = g21 * g21 + g22 * g22;
  const T b12 = g11 * g21 + g12 * g22;
  T bb = b11 * b22 - b12 * b12;
  bb = bb > T(0) ? bb : T(0);
  const T aa = ((g11 * g11 + g12 * g12) + g21 * g21) + g22 * g22;
  return cfac * sqrt(bb / (aa + T(1e-30)) + T(1e-30));
}

// The step's dt (ns2d/core.py:686-695): given (mode 2), fixed (mode 1), or the CFL / viscous rule
// on the maxima in the scalar block (mode 0), rounded through the field type as the reference.
// Heat transfer's limits on dt (physics.py:851-884): the bounded temperature step and the
// buoyant free-fall limit; on == 0 leaves dt alone.
struct Dt2dThermal {
  int on;
  double kappa, inv_prt, two_over_h, diff_over_h2, abs_ri, cfl, h;
};

// placed physics in the step bound (physics.py:851-884): fans (and jets) put their speed
// scale u_floor into the CFL bound and the temperature bound; heaters add the two bounds of a
// parcel heated from rest (heat_max > 0: present)
template <typename T>
struct Dt2dPlaced {
  int fans;
  T u_floor, heat_max;
};

template <typename T, bool HEAT>
__device__ __forceinline__ T dt2d_value(int mode, const T *dt_in, double dt_fixed, const unsigned long long *bits,
                                        double cfl_h, double nu, double visc_h2, int les, const Dt2dThermal &th,
                                        const Dt2dPlaced<T> &pl = Dt2dPlaced<T>{0, T(0), T(-1)}) {
  if (mode == 2) return *dt_in;
  if (mode == 1) return T(dt_fixed);
  const T usum = T(as_double(bits[SC_MAXU])) + T(as_double(bits[SC_MAXV]));
  T umax = usum;
  umax = umax > T(1e-6) || umax != umax ? umax : T(1e-6);
  T dt = T(cfl_h) / umax;
  const T nut_max = T(as_double(bits[SC_NUTMAX]));
  const T nut = les ? T(nu) + nut_max : T(nu);
  const T dv = T(visc_h2) / nut;
  dt = dv < dt ? dv : dt;
  if (pl.fans) {
    const T uf = pl.u_floor > T(1e-6) ? pl.u_floor : T(1e-6);
    const T l0 = T(cfl_h) / uf;
    dt = l0 < dt ? l0 : dt;
  }
  if (HEAT && th.on) {
    const T kap = les ? T(th.kappa) + nut_max * T(th.inv_prt) : T(th.kappa);
    const T speed = usum > pl.u_floor || usum != usum ? usum : pl.u_floor;
    const T rate = speed * T(th.two_over_h) + kap * T(th.diff_over_h2);
    const T l1 = T(1) / rate;
    dt = l1 < dt ? l1 : dt;
    T acc = T(th.abs_ri) * T(as_double(bits[SC_MAXT]));
    acc = acc > T(1e-12) || acc != acc ? acc : T(1e-12);
    const T l2 = T(th.cfl) * sqrt(T(th.h) / acc);
    dt = l2 < dt ? l2 : dt;
    if (pl.heat_max >= T(0)) {
      const T sm = pl.heat_max > T(1e-12) ? pl.heat_max : T(1e-12);
      const T l3 = T(1) / sm;
      dt = l3 < dt ? l3 : dt;
      T den = T(th.abs_ri) * sm;
      den = den > T(1e-12) ? den : T(1e-12);
      const T l4 = pow(T(6.0 * th.cfl * th.h) / den, T(1.0 / 3.0));
      dt = l4 < dt ? l4 : dt;
    }
  }
  return dt;
}

template <typename T>
struct StageParams {
  int nx, ny, periodic, closed, upwind, les;
  T inv_h, kadv, nuh2, cfac;
  Rules2<T> ru, rv;
  const T *up, *vp, *u0, *v0;  // stage start (or, with psi, the previous stage value), step start
  const T *psi;                // non-NULL: the stage start is up / vp projected with this psi
  T *uh, *vh;                  // stage value (after BCs and penalisation)
  T a, b, w;                   // RK blend weight, tendency weight, force weight
  const T *dt;
  const T *u_inlet;
  int has_win, win[4];         // j0, j1, i0, i1
  const T *chi_u, *chi_v, *chi_c, *a_u, *a_v, *k_u, *k_v;
  T eta;
  // the caller's 0-d device scalars nu and eta (NULL: the plan's constants), read at every
  // launch so that a live Re change reaches a captured graph; inv_h2 = 1 / h^2
  const T *live_nu, *live_eta, *live_kappa;
  T inv_h2;
  // heat transfer: buoyancy -Ri theta g on the faces from the stage-start theta, after the
  // penalisation (core.py:774-813), with the solids' share (vol_u / vol_v, else chi) booked
  // against the body force; nut_out (ny, nx) receives nu_t of the stage for the heat equation
  const T *thp;
  T ri_gx, ri_gy;              // Ri (-g_x), Ri (-g_y); 0: no buoyancy on that component
  int buoy_u, buoy_v;
  const T *vol_u, *vol_v;
  T *nut_out;
  T *up_out, *vp_out;          // the stage-start (projected) face velocities, for the theta stage
  int nbody;
  double *partials;            // this stage's [block][4 nbody]
  unsigned long long *nut_max; // nu-only pass: max nu_t (ordered bits)
  // first stage: every block derives the step's dt (dt2d_value) and block (0, 0) stores it
  // in *dt_store for the kernels after it; otherwise dt is read from *dt
  int dt_here, dt_mode, dt_les;
  Dt2dThermal dt_th;
  const T *dt_in;
  const unsigned long long *dt_bits;
  double dt_fixed, dt_cfl_h, dt_nu, dt_visc_h2;
  T *dt_store;
  // placed physics (PLACED instantiations only): the fans' forces per unit thrust and this
  // step's thrusts (core.py:875-882); the paint layer's implicit penalisation after the bodies,
  // its force weights and the paint's per-block impulse sums [u, v] of this stage
  // (physics.py:675-683, core.py:807-811)
  int nfan;
  const T *fan_gu, *fan_gv, *fan_thrust;
  const T *paint_u, *paint_v, *paint_wu, *paint_wv;
  double *paint_part;
  // the combined penalisation of jets / vents and paint, (u + k xa) / (1 + k xchi) (xa NULL:
  // paint alone), and the ports' net volume flow joining the outlet balance (core.py:352-356)
  const T *xchi_u, *xa_u, *xchi_v, *xa_v, *q_net;
  // the Werner-Wengle wall shear (bit 0 bottom, 1 top, 2 left, 3 right), the floor's speed and
  // the constant nu when no live scalar is given
  int wall_model;
  T wall_ground, nu_c, h_c;
  int forcing;                 // the verification cases' uniform body force (core.py:597-599)
  T force_u, force_v;
};

// core.py:510-533: the Werner-Wengle shear above the resolved one at distance y, signed like us
template <typename T>
__device__ __forceinline__ T wall_shear_excess(T us, T nu_over_y) {
  const T a = us < T(0) ? -us : us;
  const T lam = a * nu_over_y;
  const T ww = pow((a * pow(nu_over_y, T(1.0 / 7.0))) * T(1.0 / 8.3), T(2.0 / (1.0 + 1.0 / 7.0)));
  const T d = ww - lam > T(0) ? ww - lam : T(0);
  const T sg = us > T(0) ? T(1) : (us < T(0) ? T(-1) : T(0));
  return sg * d;
}

// One RK stage of the u- and v-faces of a 32 x 8 tile; NU_ONLY: only the maximum eddy
// viscosity of the tile's cells (the first stage's dt needs it before the update); HEAT: the
// heat-transfer instantiation (thermal dt limits, buoyancy and its force share, nu_t and the
// stage-start face velocities handed to the theta stage), so the plain step carries none of it.
//
// The body takes its tile (bx, by) of a gx-wide grid and its thread tid (0 .. NT-1)
// explicitly: stage2d_kernel runs it as one launch per instance, the batched sweep's
// persistent kernel (sweep2d.cu) as one work item among every instance's tiles.
template <typename T, bool NU_ONLY, bool HEAT, bool NC = true, bool PLACED = false>
__device__ __forceinline__ void stage2d_body(const StageParams<T> &P, int bx, int by, int gx, int tid_) {
  __shared__ T U[UY][UX];
  __shared__ T V[VY][VX];
  __shared__ T NU[CY][CX], TXX[CY][CX], TYY[CY][CX];
  __shared__ T TXY[KY][KX];
  __shared__ double red[NT / 32][MAXQ];
  __shared__ T corr_s;
  const int nx = P.nx, ny = P.ny;
  const int tid = tid_, tx = tid % TX, ty = tid / TX;
  const int i0 = bx * TX, j0 = by * TY;
  const bool tunnel = !P.periodic && !P.closed;
  const T nuh2 = P.live_nu ? __ldg(P.live_nu) * P.inv_h2 : P.nuh2;
  const T eta = P.live_eta ? __ldg(P.live_eta) : P.eta;
  T dt;
  if (P.dt_here) {
    Dt2dThermal dth = P.dt_th;
    if (HEAT && P.live_kappa) dth.kappa = (double)__ldg(P.live_kappa);
    dt = dt2d_value<T, HEAT>(P.dt_mode, P.dt_in, P.dt_fixed, P.dt_bits, P.dt_cfl_h,
                             P.live_nu ? (double)__ldg(P.live_nu) : P.dt_nu, P.dt_visc_h2, P.dt_les, dth);
  } else {
    dt = *P.dt;
  }
  if (P.dt_here && bx == 0 && by == 0 && tid == 0) *P.dt_store = dt;
  const T bdt = dt * P.b;
  // outlet balance (core.py:352-359): every block with outlet faces sums the whole outlet
  // column of the stage value in the same fixed order, so all agree
  if (!NU_ONLY && tunnel && i0 + TX >= nx && tid < 32) {
    double s_in = 0.0, s_out = 0.0;
    for (int j = tid; j < ny; j += 32) {
      const T un = P.psi ? projected_u<T, NC>(P.up, P.psi, nx, P.periodic, P.inv_h, j, nx) : P.up[(size_t)j * (nx + 1) + nx];
      const T un1 = P.psi ? projected_u<T, NC>(P.up, P.psi, nx, P.periodic, P.inv_h, j, nx - 1)
                          : P.up[(size_t)j * (nx + 1) + nx - 1];
      const T lu = (un1 - un) * P.inv_h;
      const T uo = P.a == T(0) ? un : lerp_t<T>(un, P.u0[(size_t)j * (nx + 1) + nx], P.a);
      s_out += (double)(uo + lu * bdt);
      s_in += (double)P.u_inlet[j];
    }
    s_in = warp_sum(s_in);
    s_out = warp_sum(s_out);
    if (PLACED && P.q_net) s_in = s_in + (double)(*P.q_net * P.inv_h);
    if (tid == 0) corr_s = T((s_in - s_out) / (double)ny);
  }
  if (P.psi) {  // the previous stage's projection, applied while staging the tile
    for (int e = tid; e < UY * UX; e += NT) {
      const int r = e / UX, c = e - r * UX;
      U[r][c] = padded2f<T>(P.ru, j0 - 2 + r, i0 - 2 + c, [&](int mj, int mi) {
        return projected_u<T, NC>(P.up, P.psi, nx, P.periodic, P.inv_h, mj, mi);
      });
    }
    for (int e = tid; e < VY * VX; e += NT) {
      const int r = e / VX, c = e - r * VX;
      V[r][c] = padded2f<T>(P.rv, j0 - 2 + r, i0 - 2 + c, [&](int mj, int mi) {
        return projected_v<T, NC>(P.vp, P.psi, nx, ny, P.periodic, P.inv_h, mj, mi);
      });
    }
  } else {
    for (int e = tid; e < UY * UX; e += NT) {
      const int r = e / UX, c = e - r * UX;
      U[r][c] = padded2<T, NC>(P.up, P.ru, j0 - 2 + r, i0 - 2 + c);
    }
    for (int e = tid; e < VY * VX; e += NT) {
      const int r = e / VX, c = e - r * VX;
      V[r][c] = padded2<T, NC>(P.vp, P.rv, j0 - 2 + r, i0 - 2 + c);
    }
  }
  __syncthreads();
  // tile coordinates: u[j][i] -> U[j - j0 + 2][i - i0 + 2], v likewise in V
  if (P.les) {
    T mx = T(0);
    const T q = T(0.25);
    for (int e = tid; e < CY * CX; e += NT) {
      const int r = e / CX, c = e - r * CX;  // cell (j0 - 1 + r, i0 - 1 + c)
      const int jc = j0 - 1 + r, ic = i0 - 1 + c;
      const int ju = r + 1, iu = c + 1;      // U / V index of u[jc][ic], v[jc][ic]
      const T g11 = (U[ju][iu + 1] - U[ju][iu]) * P.inv_h;
      const T g22 = (V[ju + 1][iu] - V[ju][iu]) * P.inv_h;
      // du/dy and dv/dx at the corners (jc .. jc+1, ic .. ic+1), averaged in the
      // reference's order: (c[j, i] + c[j+1, i]) + c[j, i+1] + c[j+1, i+1]
      auto dudy = [&](int kr, int kc) { return (U[kr][kc] - U[kr - 1][kc]) * P.inv_h; };
      auto dvdx = [&](int kr, int kc) { return (V[kr][kc] - V[kr][kc - 1]) * P.inv_h; };
      const T g12 = (((dudy(ju, iu) + dudy(ju + 1, iu)) + dudy(ju, iu + 1)) + dudy(ju + 1, iu + 1)) * q;
      const T g21 = (((dvdx(ju, iu) + dvdx(ju + 1, iu)) + dvdx(ju, iu + 1)) + dvdx(ju + 1, iu + 1)) * q;
      T nu = eddy2d<T>(g11, g12, g21, g22, P.les, P.cfac);
      if (P.has_win && jc >= P.win[0] && jc < P.win[1] && ic >= P.win[2] && ic < P.win[3]) {
        const T chi = P.chi_c[(size_t)(jc - P.win[0]) * (P.win[3] - P.win[2]) + (ic - P.win[2])];
        nu = nu * (T(1) - chi);
      }
      NU[r][c] = nu;
      if (HEAT && !NU_ONLY && P.nut_out && r >= 1 && r <= TY && c >= 1 && c <= TX && jc < ny && ic < nx)
        P.nut_out[(size_t)jc * nx + ic] = nu;
      TXX[r][c] = T(2) * nu * g11;
      TYY[r][c] = T(2) * nu * g22;
      if (jc >= -1 && jc <= ny && ic >= -1 && ic <= nx) mx = (nu > mx || nu != nu) ? nu : mx;
    }
    if (NU_ONLY) {
      block_max_atomic<T>(mx, P.nut_max);
      return;
    }
    __syncthreads();
    for (int e = tid; e < KY * KX; e += NT) {
      const int r = e / KX, c = e - r * KX;  // corner (j0 + r, i0 + c)
      const T nk = (((NU[r][c] + NU[r + 1][c]) + NU[r][c + 1]) + NU[r + 1][c + 1]) * q;
      const int kr = r + 2, kc = c + 2;      // U / V index of the corner's u[j][i], v[j][i]
      const T shear = (U[kr][kc] - U[kr - 1][kc]) * P.inv_h + (V[kr][kc] - V[kr][kc - 1]) * P.inv_h;
      TXY[r][c] = nk * shear;
    }
    __syncthreads();
  }
  if (NU_ONLY) return;
  const int j = j0 + ty, i = i0 + tx;
  const bool in = j < ny && i < nx;
  const T k_pen = bdt / eta;
  const bool wblock = P.has_win && P.nbody > 0;
  double fq[4] = {0.0, 0.0, 0.0, 0.0};  // this thread's force sums of body `bsel`
  double pimp = 0.0, pimp_v = 0.0;      // this thread's paint impulse (weighted) of u and v faces
  // ---- u-faces (j, i) and, for the last column, (j, nx)
  auto u_face = [&](int fi, T &out, bool &pen, T &du, int &widx, T &sh) {
    const int r = j - j0 + 2, c = fi - i0 + 2;
    const T *row = U[r];
    const T fxl = face_flux<T>(row[c - 1] + row[c], row[c - 2], row[c - 1], row[c], row[c + 1], P.upwind != 0);
    const T fxr = face_flux<T>(row[c] + row[c + 1], row[c - 1], row[c], row[c + 1], row[c + 2], P.upwind != 0);
    const T vsb = V[r][c - 1] + V[r][c], vst = V[r + 1][c - 1] + V[r + 1][c];
    const T gyb = face_flux<T>(vsb, U[r - 2][c], U[r - 1][c], U[r][c], U[r + 1][c], P.upwind != 0);
    const T gyt = face_flux<T>(vst, U[r - 1][c], U[r][c], U[r + 1][c], U[r + 2][c], P.upwind != 0);
    T lu = (((fxl - fxr) + gyb) - gyt) * P.kadv;
    T ring = ((row[c + 1] + row[c - 1]) + U[r + 1][c]) + U[r - 1][c];
    ring = ring + T(-4) * row[c];
    lu = lu + ring * nuh2;
    if (P.les) {
      const int cc = fi - i0 + 1, cr = j - j0 + 1;  // cell fi in TXX, corner row j in TXY
      lu = lu + (((TXX[cr][cc] - TXX[cr][cc - 1]) + TXY[cr][fi - i0]) - TXY[cr - 1][fi - i0]) * P.inv_h;
    }
    if (PLACED && P.forcing) lu = lu + P.force_u;
    if (PLACED && P.wall_model && (j == 0 || j == ny - 1)) {   // the walls' excess shear, tau / h
      const T nuy = (P.live_nu ? __ldg(P.live_nu) : P.nu_c) / (T(0.5) * P.h_c);
      T f = T(0);
      if (j == 0 && (P.wall_model & 1)) f = -wall_shear_excess<T>(row[c] - P.wall_ground, nuy) * P.inv_h;
      if (j == ny - 1 && (P.wall_model & 2)) f = -wall_shear_excess<T>(row[c], nuy) * P.inv_h;
      lu = lu + f;
    }
    if (!P.periodic) {
      if (fi == 0) lu = T(0);
      if (fi == nx) lu = P.closed ? T(0) : (row[c - 1] - row[c]) * P.inv_h;
    }
    if (PLACED && P.nfan) {   // + sum_f thrust_f g_f (physics.py:671-672, core.py:880-882)
      const size_t gg = (size_t)j * (nx + 1) + fi, nfu = (size_t)ny * (nx + 1);
      T ff = P.fan_thrust[0] * P.fan_gu[gg];
      for (int q = 1; q < P.nfan; ++q) ff = ff + P.fan_thrust[q] * P.fan_gu[q * nfu + gg];
      lu = lu + ff;
    }
    const T up = row[c];
    const size_t g = (size_t)j * (nx + 1) + fi;
    T uh = (P.a == T(0) ? up : lerp_t<T>(up, P.u0[g], P.a)) + lu * bdt;
    if (!P.periodic) {
      if (P.closed) {
        if (fi == 0 || fi == nx) uh = T(0);
      } else {
        if (fi == 0) uh = P.u_inlet[j];
        if (fi == nx) uh = uh + corr_s;
      }
    }
    pen = false;
    if (P.has_win && j >= P.win[0] && j < P.win[1] && fi >= P.win[2] && fi <= P.win[3]) {
      widx = (j - P.win[0]) * (P.win[3] - P.win[2] + 1) + (fi - P.win[2]);
      const T un = (uh + k_pen * P.a_u[widx]) / (T(1) + k_pen * P.chi_u[widx]);
      du = un - uh;
      uh = un;
      pen = true;
    }
    if (PLACED && P.xchi_u) {   // jets / vents and paint, after the bodies (physics.py:675-683)
      const T un = (uh + k_pen * (P.xa_u ? P.xa_u[g] : T(0))) / (T(1) + k_pen * P.xchi_u[g]);
      if (P.paint_wu) pimp += (double)((un - uh) * P.paint_wu[g]) * (double)P.w;
      uh = un;
    }
    if (HEAT && P.buoy_u) {  // face average of theta (0 on boundary faces of a bounded domain)
      T tf;
      const size_t tr = (size_t)j * nx;
      if (fi > 0 && fi < nx) tf = T(0.5) * (P.thp[tr + fi] + P.thp[tr + fi - 1]);
      else tf = P.periodic ? T(0.5) * (P.thp[tr] + P.thp[tr + nx - 1]) : T(0);
      const T fu = tf * P.ri_gx;
      uh = uh + bdt * fu;
      if (pen) sh = fu * (P.vol_u ? P.vol_u[widx] : P.chi_u[widx]) * (bdt * P.w);
      if (PLACED && P.paint_u) pimp += (double)((fu * P.paint_u[g]) * P.paint_wu[g]) * (double)(bdt * P.w);
    }
    out = uh;
  };
  auto v_face = [&](int fj, T &out, bool &pen, T &dv, int &widx, T &sh) {
    const int r = fj - j0 + 2, c = i - i0 + 2;
    const T usl = U[r - 1][c] + U[r][c], usr = U[r - 1][c + 1] + U[r][c + 1];
    const T *row = V[r];
    const T fxl = face_flux<T>(usl, row[c - 2], row[c - 1], row[c], row[c + 1], P.upwind != 0);
    const T fxr = face_flux<T>(usr, row[c - 1], row[c], row[c + 1], row[c + 2], P.upwind != 0);
    const T gyb = face_flux<T>(V[r - 1][c] + V[r][c], V[r - 2][c], V[r - 1][c], V[r][c], V[r + 1][c], P.upwind != 0);
    const T gyt = face_flux<T>(V[r][c] + V[r + 1][c], V[r - 1][c], V[r][c], V[r + 1][c], V[r + 2][c], P.upwind != 0);
    T lv = (((fxl - fxr) + gyb) - gyt) * P.kadv;
    T ring = ((row[c + 1] + row[c - 1]) + V[r + 1][c]) + V[r - 1][c];
    ring = ring + T(-4) * row[c];
    lv = lv + ring * nuh2;
    if (P.les) {
      const int cc = i - i0 + 1, cr = fj - j0 + 1;  // cell row fj in TYY, corner row fj in TXY
      lv = lv + (((TXY[cr - 1][i - i0 + 1] - TXY[cr - 1][i - i0]) + TYY[cr][cc]) - TYY[cr - 1][cc]) * P.inv_h;
    }
    if (PLACED && P.forcing) lv = lv + P.force_v;
    if (PLACED && (P.wall_model & 12) && (i == 0 || i == nx - 1)) {
      const T nuy = (P.live_nu ? __ldg(P.live_nu) : P.nu_c) / (T(0.5) * P.h_c);
      T f = T(0);
      if (i == 0 && (P.wall_model & 4)) f = -wall_shear_excess<T>(row[c], nuy) * P.inv_h;
      if (i == nx - 1 && (P.wall_model & 8)) f = -wall_shear_excess<T>(row[c], nuy) * P.inv_h;
      lv = lv + f;
    }
    if (!P.periodic && (fj == 0 || fj == ny)) lv = T(0);
    if (PLACED && P.nfan) {
      const size_t gg = (size_t)fj * nx + i, nfv = (size_t)(ny + 1) * nx;
      T ff = P.fan_thrust[0] * P.fan_gv[gg];
      for (int q = 1; q < P.nfan; ++q) ff = ff + P.fan_thrust[q] * P.fan_gv[q * nfv + gg];
      lv = lv + ff;
    }
    const T vp = row[c];
    const size_t g = (size_t)fj * nx + i;
    T vh = (P.a == T(0) ? vp : lerp_t<T>(vp, P.v0[g], P.a)) + lv * bdt;
    pen = false;
    if (P.has_win && fj >= P.win[0] && fj <= P.win[1] && i >= P.win[2] && i < P.win[3]) {
      widx = (fj - P.win[0]) * (P.win[3] - P.win[2]) + (i - P.win[2]);
      const T vn = (vh + k_pen * P.a_v[widx]) / (T(1) + k_pen * P.chi_v[widx]);
      dv = vn - vh;
      vh = vn;
      pen = true;
    }
    if (PLACED && P.xchi_v) {
      const T vn = (vh + k_pen * (P.xa_v ? P.xa_v[g] : T(0))) / (T(1) + k_pen * P.xchi_v[g]);
      if (P.paint_wv) pimp_v += (double)((vn - vh) * P.paint_wv[g]) * (double)P.w;
      vh = vn;
    }
    if (HEAT && P.buoy_v) {
      T tf;
      if (fj > 0 && fj < ny) tf = T(0.5) * (P.thp[(size_t)fj * nx + i] + P.thp[(size_t)(fj - 1) * nx + i]);
      else tf = P.periodic ? T(0.5) * (P.thp[i] + P.thp[(size_t)(ny - 1) * nx + i]) : T(0);
      const T fv = tf * P.ri_gy;
      vh = vh + bdt * fv;
      if (pen) sh = fv * (P.vol_v ? P.vol_v[widx] : P.chi_v[widx]) * (bdt * P.w);
      if (PLACED && P.paint_v) pimp_v += (double)((fv * P.paint_v[g]) * P.paint_wv[g]) * (double)(bdt * P.w);
    }
    out = vh;
  };
  // u faces of this thread: i, plus nx for the thread of i = nx - 1 (non-periodic)
  T uv[2], du[2], ush[2] = {T(0), T(0)};
  bool upen[2] = {false, false};
  int uidx[2] = {0, 0}, nuf = 0;
  T vv[2], dv[2], vsh[2] = {T(0), T(0)};
  bool vpen[2] = {false, false};
  int vidx[2] = {0, 0}, nvf = 0;
  if (in) {
    // the last face of a row / column is computed everywhere; in a periodic domain its
    // penalisation increment counts towards the force, but the face itself then takes the
    // value of face 0 (core.py:330-331, 923-924)
    u_face(i, uv[0], upen[0], du[0], uidx[0], ush[0]);
    nuf = 1;
    if (i == nx - 1) {
      u_face(nx, uv[1], upen[1], du[1], uidx[1], ush[1]);
      nuf = 2;
    }
    v_face(j, vv[0], vpen[0], dv[0], vidx[0], vsh[0]);
    nvf = 1;
    if (j == ny - 1) {
      v_face(ny, vv[1], vpen[1], dv[1], vidx[1], vsh[1]);
      nvf = 2;
    }
    if (HEAT && P.up_out) {  // tile coordinates: u[j][i] -> U[j - j0 + 2][i - i0 + 2], v likewise
      P.up_out[(size_t)j * (nx + 1) + i] = U[ty + 2][tx + 2];
      if (i == nx - 1) P.up_out[(size_t)j * (nx + 1) + nx] = U[ty + 2][tx + 3];
      P.vp_out[(size_t)j * nx + i] = V[ty + 2][tx + 2];
      if (j == ny - 1) P.vp_out[(size_t)ny * nx + i] = V[ty + 3][tx + 2];
    }
    P.uh[(size_t)j * (nx + 1) + i] = uv[0];
    if (nuf == 2 && !P.periodic) P.uh[(size_t)j * (nx + 1) + nx] = uv[1];
    if (P.periodic && i == 0) P.uh[(size_t)j * (nx + 1) + nx] = uv[0];
    P.vh[(size_t)j * nx + i] = vv[0];
    if (nvf == 2 && !P.periodic) P.vh[(size_t)ny * nx + i] = vv[1];
    if (P.periodic && j == 0) P.vh[(size_t)ny * nx + i] = vv[0];
  }
  // ---- force partials of the bodies (core.py:943-949): per warp, then per block in order
  if (wblock) {
    const int warp = tid >> 5, lane = tid & 31;
    const T wq = P.w;
    const int wx = P.win[3] - P.win[2], wy = P.win[1] - P.win[0];
    const size_t su = (size_t)wy * (wx + 1), sv = (size_t)(wy + 1) * wx;
    for (int b = 0; b < P.nbody; ++b) {
      fq[0] = fq[1] = fq[2] = fq[3] = 0.0;
      for (int q = 0; q < nuf; ++q)
        if (upen[q]) {
          const double d = (double)(du[q] * wq) + (double)ush[q];
          fq[0] += (double)P.k_u[(size_t)(2 * b) * su + uidx[q]] * d;
          fq[1] += (double)P.k_u[(size_t)(2 * b + 1) * su + uidx[q]] * d;
        }
      for (int q = 0; q < nvf; ++q)
        if (vpen[q]) {
          const double d = (double)(dv[q] * wq) + (double)vsh[q];
          fq[2] += (double)P.k_v[(size_t)(2 * b) * sv + vidx[q]] * d;
          fq[3] += (double)P.k_v[(size_t)(2 * b + 1) * sv + vidx[q]] * d;
        }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const double s = warp_sum(fq[q]);
        if (lane == 0) red[warp][4 * b + q] = s;
      }
    }
    __syncthreads();
    const int nq = 4 * P.nbody;
    if (tid < nq) {
      double s = 0.0;
      for (int wv = 0; wv < NT / 32; ++wv) s += red[wv][tid];
      P.partials[(size_t)(by * gx + bx) * nq + tid] = s;
    }
  }
  // ---- the paint's impulse sums of this block (per warp, then in order)
  if (PLACED && P.paint_part) {
    __shared__ double pred[NT / 32][2];
    const int warp = tid >> 5, lane = tid & 31;
    const double a = warp_sum(pimp), b = warp_sum(pimp_v);
    if (lane == 0) {
      pred[warp][0] = a;
      pred[warp][1] = b;
    }
    __syncthreads();
    if (tid < 2) {
      double t = 0.0;
      for (int wv = 0; wv < NT / 32; ++wv) t += pred[wv][tid];
      P.paint_part[(size_t)(by * gx + bx) * 2 + tid] = t;
    }
  }
}

template <typename T, bool NU_ONLY, bool HEAT, bool PLACED = false>
__global__ void __launch_bounds__(NT) stage2d_kernel(const __grid_constant__ StageParams<T> P) {
  aero::pdl_wait();
  stage2d_body<T, NU_ONLY, HEAT, true, PLACED>(P, blockIdx.x, blockIdx.y, gridDim.x, threadIdx.y * TX + threadIdx.x);
}

// u <- uh - grad psi (core.py:643-660); one thread per cell column, the thread of the last
// column also does the last u-face and the thread of the last row the last v-face
template <typename T>
__device__ __forceinline__ void correct2d_body(int nx, int ny, int periodic, T inv_h, const T *__restrict__ uh,
                                               const T *__restrict__ vh, const T *__restrict__ psi, T *__restrict__ u,
                                               T *__restrict__ v, int i, int j) {
  if (i >= nx || j >= ny) return;
  const size_t c = (size_t)j * nx;
  for (int fi = i; fi <= (i == nx - 1 ? nx : i); ++fi) {
    const size_t e = (size_t)j * (nx + 1) + fi;
    T val;
    if (periodic) {
      const int ii = fi == nx ? 0 : fi, il = ii == 0 ? nx - 1 : ii - 1;
      val = uh[e] - (psi[c + ii] - psi[c + il]) * inv_h;
    } else if (fi == 0 || fi == nx) {
      val = uh[e];
    } else {
      val = uh[e] - (psi[c + fi] - psi[c + fi - 1]) * inv_h;
    }
    u[e] = val;
  }
  for (int fj = j; fj <= (j == ny - 1 ? ny : j); ++fj) {
    const size_t e = (size_t)fj * nx + i;
    T val;
    if (periodic) {
      const int jj = fj == ny ? 0 : fj, jl = jj == 0 ? ny - 1 : jj - 1;
      val = vh[e] - (psi[(size_t)jj * nx + i] - psi[(size_t)jl * nx + i]) * inv_h;
    } else if (fj == 0 || fj == ny) {
      val = vh[e];
    } else {
      val = vh[e] - (psi[(size_t)fj * nx + i] - psi[(size_t)(fj - 1) * nx + i]) * inv_h;
    }
    v[e] = val;
  }
}

template <typename T>
__global__ void correct2d_kernel(int nx, int ny, int periodic, T inv_h, const T *__restrict__ uh,
                                 const T *__restrict__ vh, const T *__restrict__ psi, T *__restrict__ u,
                                 T *__restrict__ v) {
  aero::pdl_wait();
  correct2d_body<T>(nx, ny, periodic, inv_h, uh, vh, psi, u, v, blockIdx.x * blockDim.x + threadIdx.x, blockIdx.y);
}

// ((u_{i+1} - u_i) + v_{j+1}) - v_j, over h (core.py:620-622)
template <typename T>
__device__ __forceinline__ void divergence2d_body(int nx, int ny, T inv_h, const T *__restrict__ u,
                                                  const T *__restrict__ v, T *__restrict__ div, int i, int j) {
  if (i >= nx || j >= ny) return;
  const size_t ru = (size_t)j * (nx + 1);
  div[(size_t)j * nx + i] =
      (((u[ru + i + 1] - u[ru + i]) + v[(size_t)(j + 1) * nx + i]) - v[(size_t)j * nx + i]) * inv_h;
}

template <typename T>
__global__ void divergence2d_kernel(int nx, int ny, T inv_h, const T *__restrict__ u, const T *__restrict__ v,
                                    T *__restrict__ div) {
  aero::pdl_wait();
  divergence2d_body<T>(nx, ny, inv_h, u, v, div, blockIdx.x * blockDim.x + threadIdx.x, blockIdx.y);
}

template <typename T>
struct DyeParams {
  int nx, ny, periodic;
  T inv_h;
  const T *c0, *u, *v, *dt, *inlet;  // inlet may be NULL (zeros)
  T *c;
  int has_win, win[4];
  const T *chi_c;
  const T *paint_c;                  // painted cells hold no smoke (core.py:958-959; NULL: none)
};

template <typename T>
__device__ __forceinline__ T dye2d_at(const DyeParams<T> &P, int j, int i) {
  // ghosts of core.py:716-721: inlet comb / zero-gradient outlet in x, zero gradient in y
  if (P.periodic) {
    i = i < 0 ? i + P.nx : (i >= P.nx ? i - P.nx : i);
    j = j < 0 ? j + P.ny : (j >= P.ny ? j - P.ny : j);
  } else {
    j = j < 0 ? 0 : (j >= P.ny ? P.ny - 1 : j);
    if (i < 0) return P.inlet ? P.inlet[j] : T(0);
    if (i >= P.nx) i = P.nx - 1;
  }
  return __ldg(P.c0 + (size_t)j * P.nx + i);
}

// One forward-Euler MUSCL / van Leer step of the dye (core.py:703-735), cut below 1e-6,
// clamped at 1, zero inside solids (core.py:779-792)
template <typename T>
__global__ void dye2d_kernel(const __grid_constant__ DyeParams<T> P) {
  aero::pdl_wait();
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
  const int nx = P.nx, ny = P.ny;
  if (i >= nx || j >= ny) return;
  auto C = [&](int dj, int di) { return dye2d_at<T>(P, j + dj, i + di); };
  const T c = C(0, 0);
  const T fx0 = muscl_flux<T>(C(0, -2), C(0, -1), c, C(0, 1), P.u[(size_t)j * (nx + 1) + i]);
  const T fx1 = muscl_flux<T>(C(0, -1), c, C(0, 1), C(0, 2), P.u[(size_t)j * (nx + 1) + i + 1]);
  const T fy0 = muscl_flux<T>(C(-2, 0), C(-1, 0), c, C(1, 0), P.v[(size_t)j * nx + i]);
  const T fy1 = muscl_flux<T>(C(-1, 0), c, C(1, 0), C(2, 0), P.v[(size_t)(j + 1) * nx + i]);
  T out = c - (*P.dt * P.inv_h) * (((fx1 - fx0) + fy1) - fy0);
  out = out > T(1e-6) ? out : T(0);
  out = out < T(1) ? out : T(1);
  if (P.has_win && j >= P.win[0] && j < P.win[1] && i >= P.win[2] && i < P.win[3]) {
    const T chi = P.chi_c[(size_t)(j - P.win[0]) * (P.win[3] - P.win[2]) + (i - P.win[2])];
    out = out * (chi <= T(0.5) ? T(1) : T(0));
  }
  if (P.paint_c) out = out * (P.paint_c[(size_t)j * nx + i] <= T(0.5) ? T(1) : T(0));
  P.c[(size_t)j * nx + i] = out;
}

// ---------------------------------------------------------------------------------------
// smoke channels with emitter groups and smoking jets (physics.py:795-830): every channel one
// forward-Euler step of the bounded (MUSCL / van Leer) advection with the end-of-step velocity
// (scalar.py:42-88: the channel's inlet value left of a tunnel), the vents' sink, the emitter
// groups relaxing their footprint to their concentration while on, the jets relaxing theirs to
// 1, solids and paint cleared, the floor and the cap
// ---------------------------------------------------------------------------------------

constexpr int MAX_DYE_CH = AERO_MAX_DYE_CHANNELS, MAX_DYE_GRP = AERO_MAX_DYE_GROUPS;

template <typename T>
struct DyeChannelsParams {
  int nx, ny, periodic, closed, nch, ngroup;
  T inv_h;
  const T *c0[MAX_DYE_CH];
  T *c[MAX_DYE_CH];
  const T *u, *v, *dt, *t0;          // the emitters' clock is the new time t0 + dt
  const T *inflow;                   // (nch, ny) inlet values, or NULL (zeros)
  const T *src_neg;                  // vents' sinks (ny, nx), or NULL
  int gch[MAX_DYE_GRP];
  const T *gw[MAX_DYE_GRP], *gtarget[MAX_DYE_GRP], *gtiming[MAX_DYE_GRP];
  const T *port_w[MAX_DYE_CH];
  int has_win, win[4];
  const T *chi_c, *paint_c;
};

// 1 while an emitter group releases at time t (physics.py:795-802; the remainder with the
// divisor's sign)
template <typename T>
__device__ __forceinline__ T emitter_on(T t, const T *timing) {
  const T start = timing[0], stop = timing[1], period = timing[2], duty = timing[3];
  const bool active = t >= start && t < stop;
  const T safe = period > T(0) ? period : T(1);
  T r = fmod(t - start, safe);
  if (r != T(0) && ((safe < T(0)) != (r < T(0)))) r = r + safe;
  const T phase = r / safe;
  return (active && (period <= T(0) || phase < duty)) ? T(1) : T(0);
}

template <typename T>
__global__ void dye_channels2d_kernel(const __grid_constant__ DyeChannelsParams<T> P) {
  aero::pdl_wait();
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
  const int nx = P.nx, ny = P.ny;
  if (i >= nx || j >= ny) return;
  const size_t g = (size_t)j * nx + i;
  const T dt = *P.dt;
  T out[MAX_DYE_CH];
  for (int ch = 0; ch < P.nch; ++ch) {
    const T *c0 = P.c0[ch];
    auto at = [&](int jj, int ii) -> T {
      if (P.periodic) {
        ii = ii < 0 ? ii + nx : (ii >= nx ? ii - nx : ii);
        jj = jj < 0 ? jj + ny : (jj >= ny ? jj - ny : jj);
      } else {
        jj = jj < 0 ? 0 : (jj >= ny ? ny - 1 : jj);
        if (ii < 0) {
          if (!P.closed) return P.inflow ? P.inflow[(size_t)ch * ny + jj] : T(0);
          ii = 0;
        }
        if (ii >= nx) ii = nx - 1;
      }
      return __ldg(c0 + (size_t)jj * nx + ii);
    };
    const T c = at(j, i);
    const T fx0 = muscl_flux<T>(at(j, i - 2), at(j, i - 1), c, at(j, i + 1), P.u[(size_t)j * (nx + 1) + i]);
    const T fx1 = muscl_flux<T>(at(j, i - 1), c, at(j, i + 1), at(j, i + 2), P.u[(size_t)j * (nx + 1) + i + 1]);
    const T fy0 = muscl_flux<T>(at(j - 2, i), at(j - 1, i), c, at(j + 1, i), P.v[g]);
    const T fy1 = muscl_flux<T>(at(j - 1, i), c, at(j + 1, i), at(j + 2, i), P.v[(size_t)(j + 1) * nx + i]);
    T cn = c + dt * ((((fx0 - fx1) + fy0) - fy1) * P.inv_h);
    if (P.src_neg) cn = cn + (dt * P.src_neg[g]) * cn;
    out[ch] = cn;
  }
  if (P.ngroup) {
    const T t = *P.t0 + dt;
    for (int q = 0; q < P.ngroup; ++q) {
      const int ch = P.gch[q];
      const T w = P.gw[q][g] * emitter_on<T>(t, P.gtiming[q]);
      out[ch] = out[ch] + w * (P.gtarget[q][g] - out[ch]);
    }
  }
  for (int ch = 0; ch < P.nch; ++ch)
    if (P.port_w[ch]) out[ch] = out[ch] + P.port_w[ch][g] * (T(1) - out[ch]);
  bool keep = true;
  if (P.has_win && j >= P.win[0] && j < P.win[1] && i >= P.win[2] && i < P.win[3])
    keep = P.chi_c[(size_t)(j - P.win[0]) * (P.win[3] - P.win[2]) + (i - P.win[2])] <= T(0.5);
  const bool paint_keep = !P.paint_c || P.paint_c[g] <= T(0.5);
  for (int ch = 0; ch < P.nch; ++ch) {
    T x = out[ch] * (keep ? T(1) : T(0));
    x = x * (paint_keep ? T(1) : T(0));
    x = x > T(1e-6) ? x : T(0);
    P.c[ch][g] = x < T(1) ? x : T(1);
  }
}

// ---------------------------------------------------------------------------------------
// placed physics before the first stage: the step (with the fans' and heaters' bounds and the
// PID controller) and the fans' PI controllers (core.py:856-878, physics.py:640-672, 851-884,
// diagnostics.py:104-124), one block
// ---------------------------------------------------------------------------------------

template <typename T>
struct Control2dParams {
  int nx, ny, nfan, pid, dt_mode, les, heat, ports;
  const T *dt_in;
  double dt_fixed, cfl_h, nu, visc_h2;
  const unsigned long long *bits;
  const T *live_nu, *live_kappa;
  Dt2dThermal th;
  const T *u_floor, *heat_max;        // 0-d (heat_max NULL: no heaters)
  const T *dt_prev, *ctrl0;           // the previous step (<= 0: first) and the controller memory
  T *ctrl;                            // new memory (2 + 2 nfan)
  const T *u0, *v0;
  const T *fan_phi, *fan_dir, *fan_value, *fan_width, *fan_kp, *fan_ki, *fan_dpmax, *fan_isvel, *fan_isthrust;
  T *thrust, *thrust_out, *ud_out;    // this step's thrusts (for the stages), the reported ones, disc speeds
  T *dt_out;
};

constexpr double PID_TARGET = 0.9, PID_KP = 0.10, PID_KI = 0.25, PID_KD = 0.02, PID_MAX_GROWTH = 1.03;

template <typename T, bool HEAT>
__global__ void __launch_bounds__(1024) control2d_kernel(const __grid_constant__ Control2dParams<T> P) {
  aero::pdl_wait();
  __shared__ double red[32][2 * AERO_MAX_FANS];
  const int tid = threadIdx.x, nx = P.nx, ny = P.ny;
  const size_t nc = (size_t)nx * ny;
  // disc velocities: the footprint-weighted cell-centred velocity of every fan, each thread a
  // fixed set of cells, then the warps and the block in order
  for (int f = 0; f < P.nfan; ++f) {
    const T *phi = P.fan_phi + (size_t)f * nc;
    double su = 0.0, sv = 0.0;
    for (size_t e = tid; e < nc; e += blockDim.x) {
      const T wgt = phi[e];
      if (wgt != T(0)) {
        const int j = (int)(e / nx), i = (int)(e - (size_t)j * nx);
        const T uc = T(0.5) * (P.u0[(size_t)j * (nx + 1) + i + 1] + P.u0[(size_t)j * (nx + 1) + i]);
        const T vc = T(0.5) * (P.v0[(size_t)(j + 1) * nx + i] + P.v0[(size_t)j * nx + i]);
        su += (double)(wgt * uc);
        sv += (double)(wgt * vc);
      }
    }
    su = warp_sum(su);
    sv = warp_sum(sv);
    if ((tid & 31) == 0) {
      red[tid >> 5][2 * f] = su;
      red[tid >> 5][2 * f + 1] = sv;
    }
  }
  __syncthreads();
  if (tid != 0) return;
  T dt;
  if (P.dt_mode == 2) {
    dt = *P.dt_in;
  } else if (P.dt_mode == 1) {
    dt = T(P.dt_fixed);
  } else {
    const Dt2dPlaced<T> pl{P.nfan > 0 || P.ports, *P.u_floor, P.heat_max ? *P.heat_max : T(-1)};
    Dt2dThermal th = P.th;
    if (HEAT && P.live_kappa) th.kappa = (double)*P.live_kappa;
    dt = dt2d_value<T, HEAT>(0, nullptr, 0.0, P.bits, P.cfl_h, P.live_nu ? (double)*P.live_nu : P.nu, P.visc_h2,
                             P.les, th, pl);
  }
  const int nctrl = 2 + 2 * P.nfan;
  if (P.ctrl)
    for (int q = 0; q < nctrl; ++q) P.ctrl[q] = P.ctrl0[q];
  if (P.pid && P.dt_mode == 0) {   // e = log(target / dt_prev); the first step takes the target
    const T target = T(PID_TARGET) * dt;
    const T prev = *P.dt_prev;
    const bool first = prev <= T(0);
    const T safe = first ? target : prev;
    T e = log(target / safe);
    const T e1 = P.ctrl0[0], e2 = P.ctrl0[1];
    T step = (T(PID_KI) * e + T(PID_KP) * (e - e1)) + T(PID_KD) * ((e - T(2) * e1) + e2);
    const T cap = T(log(PID_MAX_GROWTH));
    step = step < cap ? step : cap;
    const T grown = safe * exp(step);
    dt = first ? target : (grown < dt ? grown : dt);
    P.ctrl[0] = first ? T(0) : e;
    P.ctrl[1] = e1;
  }
  *P.dt_out = dt;
  for (int f = 0; f < P.nfan; ++f) {
    double ua = 0.0, va = 0.0;
    for (int w = 0; w < 32; ++w) {
      ua += red[w][2 * f];
      va += red[w][2 * f + 1];
    }
    const T ud = T(ua) * P.fan_dir[2 * f] + T(va) * P.fan_dir[2 * f + 1];
    const T value = P.fan_value[f], width = P.fan_width[f], ki = P.fan_ki[f], dpmax = P.fan_dpmax[f];
    const T err = value - ud, ilim = dpmax / ki;
    T integ = P.ctrl0[2 + 2 * f] + (err * dt) * P.fan_isvel[f];
    integ = integ < ilim ? integ : ilim;
    integ = integ > -ilim ? integ : -ilim;
    T dp = P.fan_kp[f] * err + ki * integ;
    dp = dp < dpmax ? dp : dpmax;
    dp = dp > -dpmax ? dp : -dpmax;
    const T fixed = P.fan_isthrust[f] > T(0) ? value : value * width;
    const T thrust = P.fan_isvel[f] > T(0) ? dp * width : fixed;
    P.thrust[f] = thrust;
    if (P.thrust_out) P.thrust_out[f] = thrust;
    if (P.ud_out) P.ud_out[f] = ud;
    if (P.ctrl) {
      P.ctrl[2 + 2 * f] = integ;
      P.ctrl[3 + 2 * f] = thrust / width;
    }
  }
}

// The projection's right-hand side with the ports' mass source: div - src (core.py:636-638)
template <typename T>
__global__ void port_source2d_kernel(T *__restrict__ rhs, const T *__restrict__ src, size_t n) {
  aero::pdl_wait();
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
    rhs[e] = rhs[e] - src[e];
}

// The painted obstacles' force coefficients [Cd, Cl] from the stages' impulse sums
// (core.py:1001-1002): one warp per component, a fixed lane order.
template <typename T>
__global__ void paint_force2d_kernel(const double *__restrict__ part, int nblocks, double h2, double force_ref,
                                     const T *dt, T *out) {
  aero::pdl_wait();
  const int c = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (c >= 2) return;
  double s = 0.0;
  for (int q = lane; q < 3 * nblocks; q += 32) s += part[(size_t)q * 2 + c];
  s = warp_sum(s);
  if (lane == 0) out[c] = T(s) * (T(-h2) / ((*dt * T(0.5)) * T(force_ref)));
}


// ---------------------------------------------------------------------------------------
// heat transfer (ns2d/physics.py:623-923 with scalar.py:34-146)
// ---------------------------------------------------------------------------------------
constexpr int MAXR = 2 * AERO_MAX_BODIES + 3;  // per-block partials: heat, then sums, wall weights, vent sum

template <typename T>
struct ThetaParams {
  int nx, ny, periodic, closed;
  T inv_h, inv_half;          // 1 / h, 2 / h
  T kappa, inv_prt, theta_in, eta_t;
  const T *live_kappa, *live_eta_t;  // the caller's device kappa / thermal eta (NULL: the constants)
  const T *thp, *th0;         // stage-start and step-start theta (ny, nx)
  T *th;                      // the stage's theta
  const T *upf, *vpf;         // stage-start face velocities (ny, nx+1), (ny+1, nx)
  const T *nut;               // (ny, nx) nu_t of the stage, NULL without LES
  int mode[4];                // AERO_TH2_* of left, right, bottom, top
  T wval[4];
  int has_win, win[4];
  const T *ins_u, *ins_v, *q_skin, *chi_t, *a_t, *w_t, *w_f;  // NULL: absent
  int n_temp, n_flux;
  T a, b;
  const T *dt;
  double *heat_part;          // (nblocks, n_temp) of this stage
  double *rep_part;           // last stage: (nblocks, 2 + n_flux) = sum theta, sum theta0, wall weights
  // placed physics: the heaters' density (ny, nx), added after the diffusion (physics.py:721-722),
  // and the paint's face fractions, which scale the face diffusivity by 1 - chi (:715-717)
  const T *heat, *paint_u, *paint_v;
  // jets and vents: the vents' sinks src_neg (ny, nx), whose fluid leaves with its heat
  // (physics.py:727-728); the jets' penalisation toward their temperature (:753-756) with the
  // stage's per-block sums of the increments (jet_part); the last stage also sums
  // src_neg theta for the vent heat (one more rep_part entry)
  const T *src_neg, *pt_chi, *pt_a;
  double *jet_part;
};

// theta at (j, i) with the ghosts of scalar.py:63-78: periodic wrap; else the first / last
// cell repeated, except the inflow value left of a tunnel.  The tile staging reaches up to
// TX + 2 cells past the last one, more than a period of a small grid: the wrap is a modulo.
template <typename T>
__device__ __forceinline__ T theta_at(const ThetaParams<T> &P, int j, int i) {
  if (P.periodic) {
    i = ((i % P.nx) + P.nx) % P.nx;
    j = ((j % P.ny) + P.ny) % P.ny;
  } else {
    j = j < 0 ? 0 : (j >= P.ny ? P.ny - 1 : j);
    if (i < 0) {
      if (!P.closed) return P.theta_in;
      i = 0;
    }
    if (i >= P.nx) i = P.nx - 1;
  }
  return __ldg(P.thp + (size_t)j * P.nx + i);
}

// diffusivity on the x-face (j, f): kappa (+ the face average of nu_t / Pr_t), times the
// insulation factor inside the window (physics.py:700-718)
template <typename T>
__device__ __forceinline__ T kappa_of(const ThetaParams<T> &P) {
  return P.live_kappa ? __ldg(P.live_kappa) : P.kappa;
}

template <typename T>
__device__ __forceinline__ T kx_face(const ThetaParams<T> &P, int j, int f) {
  const T kap = kappa_of<T>(P);
  T k = kap;
  const int nx = P.nx;
  if (P.nut) {
    const T *row = P.nut + (size_t)j * nx;
    T avg;
    if (f > 0 && f < nx) avg = T(0.5) * (__ldg(row + f) * P.inv_prt + __ldg(row + f - 1) * P.inv_prt);
    else if (P.periodic) avg = T(0.5) * (__ldg(row) * P.inv_prt + __ldg(row + nx - 1) * P.inv_prt);
    else avg = __ldg(row + (f == 0 ? 0 : nx - 1)) * P.inv_prt;
    k = kap + avg;
  }
  if (P.paint_u) k = k * (T(1) - __ldg(P.paint_u + (size_t)j * (nx + 1) + f));   // painted solids insulate
  if (P.ins_u && j >= P.win[0] && j < P.win[1] && f >= P.win[2] && f <= P.win[3])
    k = k * __ldg(P.ins_u + (size_t)(j - P.win[0]) * (P.win[3] - P.win[2] + 1) + (f - P.win[2]));
  return k;
}

template <typename T>
__device__ __forceinline__ T ky_face(const ThetaParams<T> &P, int f, int i) {
  const T kap = kappa_of<T>(P);
  T k = kap;
  const int nx = P.nx, ny = P.ny;
  if (P.nut) {
    T avg;
    if (f > 0 && f < ny)
      avg = T(0.5) * (__ldg(P.nut + (size_t)f * nx + i) * P.inv_prt + __ldg(P.nut + (size_t)(f - 1) * nx + i) * P.inv_prt);
    else if (P.periodic)
      avg = T(0.5) * (__ldg(P.nut + i) * P.inv_prt + __ldg(P.nut + (size_t)(ny - 1) * nx + i) * P.inv_prt);
    else
      avg = __ldg(P.nut + (size_t)(f == 0 ? 0 : ny - 1) * nx + i) * P.inv_prt;
    k = kap + avg;
  }
  if (P.paint_v) k = k * (T(1) - __ldg(P.paint_v + (size_t)f * nx + i));
  if (P.ins_v && f >= P.win[0] && f <= P.win[1] && i >= P.win[2] && i < P.win[3])
    k = k * __ldg(P.ins_v + (size_t)(f - P.win[0]) * (P.win[3] - P.win[2]) + (i - P.win[2]));
  return k;
}

// diffusive flux -k dtheta/dn of a boundary face (scalar.py:112-146); sign +1 on the low side
template <typename T>
__device__ __forceinline__ T wall_flux(int mode, T k, T inner, T value, T inv_half, T sign) {
  if (mode == AERO_TH2_TEMPERATURE || mode == AERO_TH2_INLET) return ((-sign * inv_half) * k) * (inner - value);
  if (mode == AERO_TH2_HEAT_FLUX) return (sign * k) * value;
  return T(0);
}

// One RK stage of theta on a 32 x 8 tile of cells: bounded advection with the stage-start
// velocity, diffusion with the wall conditions, heat-flux skins, the RK blend and the
// implicit penalisation toward the temperature bodies with their heat partials.
template <typename T>
__global__ void __launch_bounds__(NT) theta2d_kernel(const __grid_constant__ ThetaParams<T> P) {
  aero::pdl_wait();
  __shared__ T S[TY + 4][TX + 4];
  __shared__ double red[NT / 32][MAXR];
  const int nx = P.nx, ny = P.ny;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
  for (int e = tid; e < (TY + 4) * (TX + 4); e += NT) {
    const int r = e / (TX + 4), c = e - r * (TX + 4);
    S[r][c] = theta_at<T>(P, j0 - 2 + r, i0 - 2 + c);
  }
  __syncthreads();
  const int j = j0 + ty, i = i0 + tx;
  const bool in = j < ny && i < nx;
  const int nh = P.n_temp, nr = P.rep_part ? 2 + P.n_flux + (P.src_neg ? 1 : 0) : 0;
  double jet = 0.0;
  double acc[MAXR];
#pragma unroll
  for (int q = 0; q < MAXR; ++q) acc[q] = 0.0;
  if (in) {
    const int r = ty + 2, c = tx + 2;
    const T ctr = S[r][c];
    auto uface = [&](int f) { return __ldg(P.upf + (size_t)j * (nx + 1) + f); };
    auto vface = [&](int f) { return __ldg(P.vpf + (size_t)f * nx + i); };
    const T fx0 = muscl_flux<T>(S[r][c - 2], S[r][c - 1], ctr, S[r][c + 1], uface(i));
    const T fx1 = muscl_flux<T>(S[r][c - 1], ctr, S[r][c + 1], S[r][c + 2], uface(i + 1));
    const T fy0 = muscl_flux<T>(S[r - 2][c], S[r - 1][c], ctr, S[r + 1][c], vface(j));
    const T fy1 = muscl_flux<T>(S[r - 1][c], ctr, S[r + 1][c], S[r + 2][c], vface(j + 1));
    T lt = (((fx0 - fx1) + fy0) - fy1) * P.inv_h;
    // diffusive fluxes of the four faces
    auto dfx = [&](int f) {
      if (f > 0 && f < nx) return -(kx_face<T>(P, j, f) * (S[r][f - i0 + 2] - S[r][f - i0 + 1])) * P.inv_h;
      if (P.periodic)   // both ends carry the wrap flux with the first face's diffusivity
        return -(kx_face<T>(P, j, 0) * (__ldg(P.thp + (size_t)j * nx) - __ldg(P.thp + (size_t)j * nx + nx - 1))) *
               P.inv_h;
      const int side = f == 0 ? 0 : 1;
      const T inner = __ldg(P.thp + (size_t)j * nx + (f == 0 ? 0 : nx - 1));
      return wall_flux<T>(P.mode[side], kx_face<T>(P, j, f), inner, P.wval[side], P.inv_half,
                          side == 0 ? T(1) : T(-1));
    };
    auto dfy = [&](int f) {
      if (f > 0 && f < ny) return -(ky_face<T>(P, f, i) * (S[f - j0 + 2][c] - S[f - j0 + 1][c])) * P.inv_h;
      if (P.periodic)
        return -(ky_face<T>(P, 0, i) * (__ldg(P.thp + i) - __ldg(P.thp + (size_t)(ny - 1) * nx + i))) * P.inv_h;
      const int side = f == 0 ? 2 : 3;
      const T inner = __ldg(P.thp + (size_t)(f == 0 ? 0 : ny - 1) * nx + i);
      return wall_flux<T>(P.mode[side], ky_face<T>(P, f, i), inner, P.wval[side], P.inv_half,
                          side == 2 ? T(1) : T(-1));
    };
    const T ld = (((dfx(i) - dfx(i + 1)) + dfy(j)) - dfy(j + 1)) * P.inv_h;
    lt = lt + ld;
    if (P.heat) lt = lt + __ldg(P.heat + (size_t)j * nx + i);
    const bool inwin = P.has_win && j >= P.win[0] && j < P.win[1] && i >= P.win[2] && i < P.win[3];
    const size_t widx = inwin ? (size_t)(j - P.win[0]) * (P.win[3] - P.win[2]) + (i - P.win[2]) : 0;
    const size_t wsz = (size_t)(P.win[1] - P.win[0]) * (P.win[3] - P.win[2]);
    if (inwin && P.q_skin) lt = lt + kappa_of<T>(P) * __ldg(P.q_skin + widx);
    if (P.src_neg) lt = lt + __ldg(P.src_neg + (size_t)j * nx + i) * ctr;
    const T bdt = *P.dt * P.b;
    const size_t g = (size_t)j * nx + i;
    const T t0 = __ldg(P.th0 + g);
    T th = (P.a == T(0) ? ctr : lerp_t<T>(ctr, t0, P.a)) + lt * bdt;
    if (inwin && nh > 0) {
      const T kt = bdt / (P.live_eta_t ? __ldg(P.live_eta_t) : P.eta_t);
      const T tn = (th + kt * __ldg(P.a_t + widx)) / (T(1) + kt * __ldg(P.chi_t + widx));
      const double d = (double)(tn - th);
      for (int b = 0; b < nh; ++b) acc[b] = (double)__ldg(P.w_t + (size_t)b * wsz + widx) * d;
      th = tn;
    }
    if (P.pt_chi) {
      const T kt = bdt / (P.live_eta_t ? __ldg(P.live_eta_t) : P.eta_t);
      const T tn = (th + kt * __ldg(P.pt_a + g)) / (T(1) + kt * __ldg(P.pt_chi + g));
      jet = (double)(tn - th);
      th = tn;
    }
    if (nr) {
      acc[nh] = (double)th;
      acc[nh + 1] = (double)t0;
      if (inwin)
        for (int b = 0; b < P.n_flux; ++b) acc[nh + 2 + b] = (double)__ldg(P.w_f + (size_t)b * wsz + widx) * (double)th;
      if (P.src_neg) acc[nh + 2 + P.n_flux] = (double)(__ldg(P.src_neg + g) * th);
    }
    P.th[g] = th;
  }
  if (P.jet_part) {   // the jets' heat of this stage: per warp, then the block in order
    __shared__ double jred[NT / 32];
    const double js = warp_sum(jet);
    if ((tid & 31) == 0) jred[tid >> 5] = js;
    __syncthreads();
    if (tid == 0) {
      double t = 0.0;
      for (int w = 0; w < NT / 32; ++w) t += jred[w];
      P.jet_part[(size_t)blockIdx.y * gridDim.x + blockIdx.x] = t;
    }
  }
  const int nq = nh + nr;
  if (nq == 0) return;
  const int warp = tid >> 5, lane = tid & 31;
  for (int q = 0; q < nq; ++q) {
    const double v = warp_sum(acc[q]);
    if (lane == 0) red[warp][q] = v;
  }
  __syncthreads();
  if (tid < nq) {
    double t = 0.0;
    for (int w = 0; w < NT / 32; ++w) t += red[w][tid];
    const size_t blk = (size_t)blockIdx.y * gridDim.x + blockIdx.x;
    if (tid < nh) P.heat_part[blk * nh + tid] = t;
    else P.rep_part[blk * nr + (tid - nh)] = t;
  }
}

template <typename T>
struct ReportParams {
  int nx, ny, periodic, closed, nblocks, n_temp, n_flux;
  T h, h2, kappa, theta_in;
  const T *live_kappa;        // the caller's device kappa (NULL: the constant)
  double hd;
  int mode[4];
  T wval[4];
  T wgt[3];
  const double *heat_part;    // (3, nblocks, n_temp)
  const double *rep_part;     // (nblocks, 2 + n_flux (+1 with ports))
  const T *theta, *u, *dt;
  double *heat, *theta_wall, *wall_heat, *heat_storage, *flow_heat;
  int ports;                  // jets and vents: the vent heat, and (jet_part) the jets' heat
  const double *jet_part;     // (3, nblocks) or NULL
  double *jet_heat, *vent_heat;
};

// The step's heat report (core.py:974-995, physics.py:760-794): one block, each warp takes
// whole sums (a body's heat over the three stages, the two grid sums of the heat storage, a
// heat-flux body's wall temperature, one side's wall heat, the two flow-heat sums) in a fixed
// lane order, so the sums are deterministic and no block barrier is needed.
template <typename T>
__global__ void heat_report2d_kernel(const __grid_constant__ ReportParams<T> P) {
  aero::pdl_wait();
  const int nx = P.nx, ny = P.ny, lane = threadIdx.x & 31, nwarp = blockDim.x >> 5;
  const T dt = *P.dt;
  const double per_dt = (double)(P.h2 / dt);
  const int nh = P.n_temp, nr = 2 + P.n_flux + (P.ports ? 1 : 0), nb = P.nblocks;
  const int ntask = nh + 1 + P.n_flux + 4 + 1 + (P.ports ? 2 : 0);
  for (int task = threadIdx.x >> 5; task < ntask; task += nwarp) {
    if (P.ports && task >= ntask - 2) {
      if (task == ntask - 2) {   // heat leaving with the vents' fluid: -sum src_neg theta h^2
        double s = 0.0;
        for (int e = lane; e < nb; e += 32) s += P.rep_part[(size_t)e * nr + 2 + P.n_flux];
        s = warp_sum(s);
        if (lane == 0 && P.vent_heat) P.vent_heat[0] = -s * (double)P.h2;
      } else if (P.jet_part) {   // the jets' heat: the weighted stage sums times h^2 / dt
        double tot = 0.0;
        for (int st = 0; st < 3; ++st) {
          double s = 0.0;
          for (int e = lane; e < nb; e += 32) s += P.jet_part[(size_t)st * nb + e];
          s = warp_sum(s);
          tot = st == 0 ? s * (double)P.wgt[0] : tot + s * (double)P.wgt[st];
        }
        if (lane == 0 && P.jet_heat) P.jet_heat[0] = tot * per_dt;
      }
      continue;
    }
    if (task < nh) {  // heat of temperature body `task`
      const int b = task;
      double tot = 0.0;
      for (int st = 0; st < 3; ++st) {
        double s = 0.0;
        for (int e = lane; e < nb; e += 32) s += P.heat_part[((size_t)st * nb + e) * nh + b];
        s = warp_sum(s);
        tot = st == 0 ? s * (double)P.wgt[0] : tot + s * (double)P.wgt[st];
      }
      if (lane == 0) P.heat[b] = tot * per_dt;
      continue;
    }
    int t = task - nh;
    if (t == 0) {  // heat storage: (sum theta - sum theta0) h^2 / dt
      double s1 = 0.0, s0 = 0.0;
      for (int e = lane; e < nb; e += 32) {
        s1 += P.rep_part[(size_t)e * nr];
        s0 += P.rep_part[(size_t)e * nr + 1];
      }
      s1 = warp_sum(s1);
      s0 = warp_sum(s0);
      if (lane == 0) P.heat_storage[0] = (s1 - s0) * per_dt;
      continue;
    }
    t -= 1;
    if (t < P.n_flux) {  // wall temperature of heat-flux body t
      double s = 0.0;
      for (int e = lane; e < nb; e += 32) s += P.rep_part[(size_t)e * nr + 2 + t];
      s = warp_sum(s);
      if (lane == 0) P.theta_wall[t] = s;
      continue;
    }
    t -= P.n_flux;
    if (t < 4) {  // wall heat of side t (left, right, bottom, top)
      const int side = t, mode = P.mode[side];
      const int n = side < 2 ? ny : nx;
      double rate = 0.0;
      if (mode == AERO_TH2_TEMPERATURE || mode == AERO_TH2_INLET) {
        double s = 0.0;
        for (int e = lane; e < n; e += 32) {
          const size_t g = side == 0 ? (size_t)e * nx : side == 1 ? (size_t)e * nx + nx - 1
                                                      : side == 2 ? (size_t)e : (size_t)(ny - 1) * nx + e;
          s += (double)(P.wval[side] - P.theta[g]);
        }
        rate = (double)(T(2) * (P.live_kappa ? __ldg(P.live_kappa) : P.kappa)) * warp_sum(s);
      } else if (mode == AERO_TH2_HEAT_FLUX) {
        rate = (double)(((P.live_kappa ? __ldg(P.live_kappa) : P.kappa) * P.wval[side]) * T((double)n * P.hd));
      }
      if (lane == 0) P.wall_heat[side] = rate;
      continue;
    }
    // flow heat in at the inlet and out at the outlet of a tunnel
    double fin = 0.0, fout = 0.0;
    if (!P.periodic && !P.closed) {
      for (int e = lane; e < ny; e += 32) {
        fin += (double)(P.u[(size_t)e * (nx + 1)] * P.theta_in);
        fout += (double)(P.u[(size_t)e * (nx + 1) + nx] * P.theta[(size_t)e * nx + nx - 1]);
      }
      fin = warp_sum(fin) * (double)P.h;
      fout = warp_sum(fout) * (double)P.h;
    }
    if (lane == 0) {
      P.flow_heat[0] = fin;
      P.flow_heat[1] = fout;
    }
  }
}

// Coefficients [Cd, Cl, Cm] per body from the stage partials in a fixed order, t + dt, dt
template <typename T>
__device__ __forceinline__ void finalize2d_body(const double *__restrict__ partials, int nblocks, int nbody, double h,
                                                double force_ref, const T *dt, const T *t0, T *t_out, T *dt_out,
                                                T *coeffs, int tid, int nthr) {
  __shared__ double tot[MAXQ];
  const int nq = 4 * nbody;
  for (int q = tid >> 5; q < nq; q += nthr >> 5) {
    double s = 0.0;
    for (int e = tid & 31; e < 3 * nblocks; e += 32) s += partials[(size_t)e * nq + q];
    s = warp_sum(s);
    if ((tid & 31) == 0) tot[q] = s;
  }
  __syncthreads();
  if (tid == 0) {
    const T d = *dt;
    *t_out = *t0 + d;
    *dt_out = d;
    const double denom = (double)((d * T(0.5)) * T(force_ref));
    const double scale = -(h * h) / denom;
    for (int b = 0; b < nbody; ++b) {
      coeffs[3 * b + 0] = T(tot[4 * b + 0] * scale);
      coeffs[3 * b + 1] = T(tot[4 * b + 2] * scale);
      coeffs[3 * b + 2] = T((tot[4 * b + 1] + tot[4 * b + 3]) * scale);
    }
  }
}

template <typename T>
__global__ void finalize2d_kernel(const double *__restrict__ partials, int nblocks, int nbody, double h,
                                  double force_ref, const T *dt, const T *t0, T *t_out, T *dt_out, T *coeffs) {
  aero::pdl_wait();
  finalize2d_body<T>(partials, nblocks, nbody, h, force_ref, dt, t0, t_out, dt_out, coeffs, threadIdx.x, blockDim.x);
}

// ---------------------------------------------------------------------------------------
// The batched sweep: every instance's step as one persistent launch
// ---------------------------------------------------------------------------------------
//
// aero_ns2d_step of each instance is recorded as its sequence of operations (the launches it
// would make: zeroing the maxima, the maxima, the three stage kernels with their transform
// passes, the correction, the finalisation), each with its parameters and its grid of work
// items.  Phase p of the sweep is operation p of every instance; one persistent kernel runs
// the phases in order, its CTAs taking the work items of all instances' operations of the
// phase (a grid-stride loop over their concatenation), with a grid barrier between phases.
// Every work item runs the same device body as the single-instance launch (stage2d_body,
// the transform bodies, correct2d_body, ...) on the same tile, so each instance's result is
// bit-identical to stepping it alone.

namespace sweep {

enum Kind : int { ZERO = 0, MAXABS = 1, STAGE = 2, POW2 = 3, LINE = 4, DIV = 5, PSIACC = 6, CORRECT = 7, FINAL = 8 };

struct ZeroArgs { double *p; int n; };
struct MaxArgs { MaxJobs<float> J; int njobs; long long chunk; };
struct DivArgs { int nx, ny; float inv_h; const float *u, *v; float *div; };
struct PsiArgs { const float *psi; float *pw; long long n; float wgt; int mode; const float *dt; };
struct CorrArgs { int nx, ny, periodic; float inv_h; const float *uh, *vh, *psi; float *u, *v; };
struct FinalArgs {
  const double *partials;
  int nblocks, nbody;
  double h, force_ref;
  const float *dt, *t0;
  float *t_out, *dt_out, *coeffs;
};

struct alignas(16) Op {
  int kind, gx, gy, n;   // n: the transform length of POW2
  // the instance, and how many of its work items (of its earlier operations) end before this
  // operation may start: the dependency the schedules without grid barriers wait for
  int inst, need;
  // tiled operations (stage, transforms): tiles along x of the single-instance grid, and how
  // many consecutive ones a work item runs (gx = ceil(tgx / tiles) work items along x)
  int tgx, tiles;
  union Args {
    StageParams<float> st;
    TransformParams<float> tr;
    ZeroArgs zero;
    MaxArgs mx;
    DivArgs dv;
    PsiArgs pa;
    CorrArgs co;
    FinalArgs fi;
  } a;
};

// the recording of one instance's step (host)
struct Recorder {
  std::vector<Op> ops;
  int lcap;    // log2 of the widest compile-time transform tile (lines)
  int tiles;   // tiles per work item of the stage and transform operations
};

// Schedules: BARRIER runs phase p (operation p of every instance) between grid barriers;
// COUNTERS and QUEUE drop the barriers: a work item waits only until its own instance has
// finished the items of its earlier operations (a per-instance counter of finished items),
// COUNTERS with the items dealt round robin to the CTAs, QUEUE with the CTAs taking the next
// item from a global counter.  Items are numbered phase by phase, so every item an item waits
// for has a smaller number and was taken earlier by a CTA that is running (all CTAs are
// co-resident): the smallest unfinished item can always go on, and nothing deadlocks.
enum Schedule : int { BARRIER = 0, COUNTERS = 1, QUEUE = 2 };

struct Tables {
  const Op *ops;
  const int *item_op;                       // operation of every work item (phase by phase)
  const long long *op_first;                // first work item of every operation
  const long long *phase_base, *phase_items;
  long long total;                          // work items of one step
  int nphase, sched;
  unsigned int *bar;         // [0] arrivals, [1] generation (BARRIER)
  unsigned long long *queue; // next work item (QUEUE)
  unsigned int *done;        // finished work items of every instance (COUNTERS, QUEUE)
  int *status;               // bit 0: a wait ran out (the launch then stopped)
  int spin_limit, extra;
};

constexpr int NTHR = 256;
constexpr int EW = 8;   // elements per thread of an elementwise work item (divergence, psi, correction)
constexpr long long MAX_CHUNK = 2048;   // elements of one work item of the maxima

// Wait (thread 0 for the CTA) until instance `inst` has finished `need` work items; bounded,
// and cut short once another CTA has given up (bit 0 of the status word).
__device__ __forceinline__ bool await_instance(const Tables &T, int inst, int need) {
  __shared__ int ok_s;
  if (threadIdx.x == 0) {
    int ok = 1, it = 0;
    const unsigned int target = (unsigned int)need + (unsigned int)T.extra;
    unsigned int got;
    for (;;) {
      asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(got) : "l"(T.done + inst) : "memory");
      if (got >= target) break;
      if (++it >= T.spin_limit || *(volatile int *)T.status & 1) {
        ok = 0;
        atomicOr(T.status, 1);
        break;
      }
      __nanosleep(32);
    }
    ok_s = ok;
  }
  __syncthreads();
  return ok_s != 0;
}

// Grid-wide barrier between phases: arrivals counted atomically, the last one bumps the
// generation; the others poll it (bounded: after spin_limit polls bit 0 of the status is set
// and every CTA returns).  extra > 0 asks for more arrivals than CTAs (a test of the bound).
__device__ __forceinline__ bool grid_barrier(const Tables &T) {
  __shared__ int ok_s;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned int *gen = T.bar + 1;
    const unsigned int g0 = *gen;
    __threadfence();
    const unsigned int expect = gridDim.x + (unsigned int)T.extra;
    int ok = 1;
    if (atomicAdd(T.bar, 1u) == expect - 1u) {
      atomicExch(T.bar, 0u);
      __threadfence();
      atomicAdd(T.bar + 1, 1u);
    } else {
      int it = 0;
      while (*gen == g0) {
        if (++it >= T.spin_limit) {
          ok = 0;
          atomicOr(T.status, 1);
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    ok_s = ok;
  }
  __syncthreads();
  return ok_s != 0;
}

// Dynamic shared memory of a compile-time transform tile of 2^l2 lines of n cells (FP32):
// twiddles, the real tile, two complex buffers.
constexpr size_t tile_smem(int n, int l2) {
  return (size_t)n * 8 + ((((size_t)n * ((1u << l2) + 1) * 4) + 15) & ~size_t(15)) + (size_t)n * (1u << l2) * 8;
}
// Lines per transform tile of the persistent kernel: the widest tile for n, at most 2^lcap lines,
// and no more shared memory than lets 4 CTAs share an SM beside the stage body's static tile
// (with 8-line tiles unbounded, 3 CTAs per SM fit: 5.48 against 4.65 ms per sweep step).
constexpr size_t TILE_SMEM_4CTA = 44 * 1024;
constexpr int tile_l2(int n, int lcap) {
  int l = fft::tile_log2L(n, 4) < lcap ? fft::tile_log2L(n, 4) : lcap;
  while (l > 1 && tile_smem(n, l) > TILE_SMEM_4CTA) --l;
  return l;
}

template <int N, int LCAP>
struct Cap {
  static constexpr int L2 = tile_l2(N, LCAP);
};

template <int LCAP>
__device__ __forceinline__ void run_pow2(const TransformParams<float> &P, int n, int bx, int by, unsigned char *sm) {
  switch (n) {
    case 64: pow2_transform_body<float, 64, Cap<64, LCAP>::L2>(P, bx, by, sm); break;
    case 128: pow2_transform_body<float, 128, Cap<128, LCAP>::L2>(P, bx, by, sm); break;
    case 256: pow2_transform_body<float, 256, Cap<256, LCAP>::L2>(P, bx, by, sm); break;
    case 512: pow2_transform_body<float, 512, Cap<512, LCAP>::L2>(P, bx, by, sm); break;
    case 1024: pow2_transform_body<float, 1024, Cap<1024, LCAP>::L2>(P, bx, by, sm); break;
    case 192: pow2_transform_body<float, 192, Cap<192, LCAP>::L2>(P, bx, by, sm); break;
    case 384: pow2_transform_body<float, 384, Cap<384, LCAP>::L2>(P, bx, by, sm); break;
    case 768: pow2_transform_body<float, 768, Cap<768, LCAP>::L2>(P, bx, by, sm); break;
    default: pow2_transform_body<float, 2048, Cap<2048, LCAP>::L2>(P, bx, by, sm); break;
  }
}

// MINB: CTAs per SM the register allocation is capped for (2: up to 128 registers, no spills;
// 3: up to 80, a few spills); the autotuner measures both.  LINE_ITEMS: the sweep has transform
// passes on run-time stage tables (lengths other than 2^a and 3 * 2^a); without them that body
// is left out, and with it the registers it needs.
template <int LCAP, int MINB, bool LINE_ITEMS>
__global__ void __launch_bounds__(NTHR, MINB) sweep2d_kernel(const __grid_constant__ Tables T) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // the current operation in shared memory: the bodies then read its parameters from a space
  // their global stores cannot alias, so they stay in registers instead of being reloaded
  // after every store; restaged only when the operation changes
  __shared__ Op op_s;
  __shared__ long long item_s;
  const int tid = threadIdx.x;
  int ph = 0, cur = -1;
  long long l = blockIdx.x, next = blockIdx.x;
  // QUEUE: thread 0 claims the item after the current one while the current one runs (claims
  // stay in queue order, so the argument against deadlock holds for claimed items)
  unsigned long long pending = 0;
  if (T.sched == QUEUE && tid == 0) pending = atomicAdd(T.queue, 1ull);
  for (;;) {
    long long g;
    if (T.sched == BARRIER) {
      while (ph < T.nphase && l >= T.phase_items[ph]) {
        if (!grid_barrier(T)) return;
        ++ph;
        l = blockIdx.x;
      }
      if (ph >= T.nphase) return;
      g = T.phase_base[ph] + l;
      l += gridDim.x;
    } else {
      if (T.sched == QUEUE) {
        if (tid == 0) {
          item_s = (long long)pending;
          pending = atomicAdd(T.queue, 1ull);
        }
        __syncthreads();
        next = item_s;
      }
      g = next;
      if (g >= T.total) return;
      next += gridDim.x;
    }
    const int o = T.item_op[g];
    if (o != cur) {
      const uint4 *src = reinterpret_cast<const uint4 *>(T.ops + o);
      for (int q = tid; q < (int)(sizeof(Op) / 16); q += NTHR) reinterpret_cast<uint4 *>(&op_s)[q] = src[q];
      cur = o;
      __syncthreads();
    }
    const Op &op = op_s;
    const int inst = op.inst;   // read before the next item may restage op_s
    if (T.sched != BARRIER && !await_instance(T, inst, op.need)) return;
    {
      const long long b = g - T.op_first[o];
      const int bx = (int)(b % op.gx), by = (int)(b / op.gx);
      switch (op.kind) {
        case ZERO:
          if (tid < op.a.zero.n) op.a.zero.p[tid] = 0.0;
          break;
        case MAXABS: {
          const MaxJob<float> &q = op.a.mx.J.job[by];
          const long long e0 = (long long)bx * op.a.mx.chunk, e1 = min(e0 + op.a.mx.chunk, (long long)q.n);
          float m = 0.f;
          for (long long e = e0 + tid; e < e1; e += NTHR) {   // coherent loads: written in this launch
            const float v = fabsf(q.a[e]);
            m = (v > m || v != v) ? v : m;
          }
          // block maximum (NaN wins), one atomic on the ordered bits of the double
          for (int sh = 16; sh > 0; sh >>= 1) {
            const float other = __shfl_xor_sync(0xffffffffu, m, sh);
            m = (other > m || other != other) ? other : m;
          }
          if ((tid & 31) == 0) atomic_max_nonneg(q.out, (double)m);
          break;
        }
        case STAGE:
          for (int t = 0, tb = bx * op.tiles; t < op.tiles && tb < op.tgx; ++t, ++tb) {
            if (t) __syncthreads();   // the previous tile's shared memory is free
            stage2d_body<float, false, false, false>(op.a.st, tb, by, op.tgx, tid);
          }
          break;
        case POW2:
          for (int t = 0, tb = bx * op.tiles; t < op.tiles && tb < op.tgx; ++t, ++tb) {
            if (t) __syncthreads();
            run_pow2<LCAP>(op.a.tr, op.n, tb, by, smem_raw);
          }
          break;
        case LINE:
          if constexpr (LINE_ITEMS) {
            for (int t = 0, tb = bx * op.tiles; t < op.tiles && tb < op.tgx; ++t, ++tb) {
              if (t) __syncthreads();
              line_transform_body<float>(op.a.tr, tb, by, smem_raw);
            }
          }
          break;
        case DIV: {
          const DivArgs &a = op.a.dv;
#pragma unroll
          for (int k = 0; k < EW; ++k)
            divergence2d_body<float>(a.nx, a.ny, a.inv_h, a.u, a.v, a.div, (bx * EW + k) * NTHR + tid, by);
          break;
        }
        case PSIACC: {
          const PsiArgs &a = op.a.pa;
          const float rdt = a.mode == 2 ? 1.f / *a.dt : 1.f;
#pragma unroll
          for (int k = 0; k < EW; ++k) {
            const long long e = (b * EW + k) * NTHR + tid;
            if (e < a.n) {
              if (a.mode == 0) {
                a.pw[e] = a.psi[e] * a.wgt;
              } else {
                const float sum = a.pw[e] + a.wgt * a.psi[e];
                a.pw[e] = a.mode == 2 ? sum * rdt : sum;
              }
            }
          }
          break;
        }
        case CORRECT: {
          const CorrArgs &a = op.a.co;
#pragma unroll
          for (int k = 0; k < EW; ++k)
            correct2d_body<float>(a.nx, a.ny, a.periodic, a.inv_h, a.uh, a.vh, a.psi, a.u, a.v,
                                  (bx * EW + k) * NTHR + tid, by);
          break;
        }
        default: {
          const FinalArgs &a = op.a.fi;
          finalize2d_body<float>(a.partials, a.nblocks, a.nbody, a.h, a.force_ref, a.dt, a.t0, a.t_out, a.dt_out,
                                 a.coeffs, tid, NTHR);
          break;
        }
      }
    }
    __syncthreads();   // the item's shared memory is free for the next one
    if (T.sched != BARRIER && tid == 0) {   // publish: the item's writes, then the count
      __threadfence();
      atomicAdd(T.done + inst, 1u);
    }
  }
}


}  // namespace sweep

}  // namespace ns2d
}  // namespace aero

// ---------------------------------------------------------------------------------------
// plan and C ABI
// ---------------------------------------------------------------------------------------

using aero_host::AxisInfo;

struct AeroNs2dPlan {
  AeroNs2dConfig cfg;
  size_t esz;
  size_t nu, nv, nc;          // element counts of u, v and cells
  size_t off_uh, off_vh, off_up, off_vp, off_pa, off_small, off_scalars, off_zero, off_partials, total;
  size_t off_nut, off_tb0, off_tb1, off_hpart, off_rpart, off_upf, off_vpf;  // heat transfer only
  size_t off_thrust = 0, off_ppart = 0, off_jpart = 0;   // fans' thrusts, paint's impulse and jets' heat sums
  // heat transfer: each theta stage runs on a side stream, forked after its stage kernel and
  // joined before the next one, so it overlaps the stage's pressure solve
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork[3] = {}, ev_join[3] = {};
  AxisInfo ax[2];             // x (n = nx), y (n = ny)
  int gx, gy, nblocks, nq;
};

namespace {

using aero_host::set_error;

template <typename T>
aero::ns2d::Rules2<T> rules2(const AeroNs2dConfig &c, int comp) {
  aero::ns2d::Rules2<T> r{};
  r.n0 = c.nx + (comp == 0);
  r.n1 = c.ny + (comp == 1);
  r.p0 = c.nx + (comp == 0);
  for (int a = 0; a < 2; ++a)
    for (int s = 0; s < 2; ++s) {
      r.kind[a][s] = c.ghost_kind[comp][a][s];
      r.val[a][s] = T(c.ghost_val[comp][a][s]);
    }
  return r;
}

// psi = L^{-1} f: x forward, y forward-solve-inverse, x inverse on the (ny, 1, nx) view
using aero::ns2d::sweep::Op;
using aero::ns2d::sweep::Recorder;

Op new_op(int kind, long long gx, int gy) {
  Op o;
  std::memset(&o, 0, sizeof(o));
  o.kind = kind;
  o.gx = (int)std::max<long long>(gx, 1);
  o.gy = std::max(gy, 1);
  return o;
}

// a tiled operation: tgx tiles along x, `tiles` of them per work item
Op new_tiled_op(int kind, long long tgx, int gy, int tiles) {
  Op o = new_op(kind, (tgx + tiles - 1) / tiles, gy);
  o.tgx = (int)std::max<long long>(tgx, 1);
  o.tiles = tiles;
  return o;
}

// compile-time tiles inside the persistent sweep kernel: every power of two from 8 and the 3 * 2^a
// lengths of the sweep's grids (each further length is another inlined body competing for the
// kernel's registers); other lengths take the run-time stage tables
bool sweep_tiled(int n) { return aero::transform_tiled(n) && (aero::fft::pow2_len(n) || n == 192 || n == 384 || n == 768); }

// one transform pass as a sweep operation (compile-time tiles of 2^a or 3 * 2^a cells no wider
// than 2^lcap lines; run-time stage tables for other lengths)
int record_transform(Recorder *rec, const aero::TransformParams<float> &P) {
  namespace sw = aero::ns2d::sweep;
  const int n = P.A.n;
  const size_t lines_x = (size_t)P.nz * P.ny;
  const int gy = P.axis == 0 ? 1 : (P.axis == 1 ? P.nz : P.ny);
  if (P.A.method == 0 && sweep_tiled(n)) {
    if (n < 64) return set_error(AERO_EUNSUPPORTED, "the persistent sweep needs transform lengths of at least 64");
    const int l2 = sw::tile_l2(n, rec->lcap), L = 1 << l2;
    Op o = new_tiled_op(sw::POW2, P.axis == 0 ? (long long)((lines_x + L - 1) / L) : (P.nx + L - 1) / L, gy,
                        rec->tiles);
    o.n = n;
    o.a.tr = P;
    rec->ops.push_back(o);
    return AERO_OK;
  }
  if (P.fuse_div || P.p_acc) return set_error(AERO_EINVAL, "fused transform passes need axes of 2^a or 3 * 2^a cells");
  const int L = P.L;
  Op o = new_tiled_op(sw::LINE, P.axis == 0 ? (long long)((lines_x + L - 1) / L) : (P.nx + L - 1) / L, gy,
                      rec->tiles);
  o.n = n;
  o.a.tr = P;
  rec->ops.push_back(o);
  return AERO_OK;
}

template <typename T>
int poisson2d_passes(const AeroNs2dPlan *p, const T *f, T *psi, unsigned char *ws, cudaStream_t s,
                     const aero::TransformParams<T> *fuse = nullptr, Recorder *rec = nullptr) {
  const AeroNs2dConfig &c = p->cfg;
  const int axes[3] = {0, 2, 0}, modes[3] = {0, 2, 1};
  for (int q = 0; q < 3; ++q) {
    aero::TransformParams<T> P{};
    if (fuse && q == 0) {
      P.fuse_div = fuse->fuse_div;
      P.uh = fuse->uh;
      P.vh = fuse->vh;
      P.inv_h = fuse->inv_h;
    }
    if (fuse && q == 2) {
      P.p_acc = fuse->p_acc;
      P.wgt = fuse->wgt;
      P.acc_mode = fuse->acc_mode;
      P.dt = fuse->dt;
    }
    P.nx = c.nx;
    P.ny = 1;
    P.nz = c.ny;
    P.lam_x = reinterpret_cast<const double *>(ws + p->ax[0].off_lam);
    P.lam_y = reinterpret_cast<const double *>(ws + p->off_zero);
    P.axis = axes[q];
    P.mode = modes[q];
    P.in = q == 0 ? f : psi;
    P.out = psi;
    const AxisInfo &x = p->ax[axes[q] == 0 ? 0 : 1];
    P.L = x.L;
    P.A = aero_host::axis_view<T>(x, ws);
    if (rec) {
      if constexpr (std::is_same<T, float>::value) {
        const int rc = record_transform(rec, P);
        if (rc) return rc;
      }
      continue;
    }
    AERO_CUDA_TRY(aero::launch_transform<T>(P, s));
  }
  return AERO_OK;
}

template <typename T>
int init2d_impl(const AeroNs2dPlan *p, unsigned char *ws, cudaStream_t s) {
  AERO_CUDA_TRY(cudaMemsetAsync(ws, 0, p->total, s));
  for (int a = 0; a < 2; ++a) AERO_CUDA_TRY(aero_host::axis_init<T>(p->ax[a], p->cfg.h, ws, s));
  return AERO_OK;
}

// One step of the plan, launched on s; with rec (FP32 plans of the batched sweep: no LES,
// heat transfer or dye, the CFL time step) the launches are recorded instead of made.
template <typename T>
int step2d_impl(const AeroNs2dPlan *p, const AeroNs2dFields *f, const AeroNs2dGeom *g, const void *dt_in,
                unsigned char *ws, cudaStream_t s, Recorder *rec = nullptr) {
  using namespace aero::ns2d;
  namespace sw = aero::ns2d::sweep;
  const AeroNs2dConfig &c = p->cfg;
  const int nx = c.nx, ny = c.ny;
  const T *u0 = static_cast<const T *>(f->u0), *v0 = static_cast<const T *>(f->v0);
  T *uh = reinterpret_cast<T *>(ws + p->off_uh), *vh = reinterpret_cast<T *>(ws + p->off_vh);
  T *upb = reinterpret_cast<T *>(ws + p->off_up), *vpb = reinterpret_cast<T *>(ws + p->off_vp);
  T *pa = reinterpret_cast<T *>(ws + p->off_pa);
  T *small = reinterpret_cast<T *>(ws + p->off_small);
  double *sc = reinterpret_cast<double *>(ws + p->off_scalars);
  auto *bits = reinterpret_cast<unsigned long long *>(sc);
  double *partials = reinterpret_cast<double *>(ws + p->off_partials);
  const bool has_win = c.nbody > 0 && c.window[1] > c.window[0] && c.window[3] > c.window[2];
  const bool les = c.les != AERO_LES_NONE;
  const bool thermal = c.thermal != 0;
  // ---- dt
  int dt_mode = dt_in ? 2 : (c.has_dt_fixed ? 1 : 0);
  StageParams<T> S{};
  S.nx = nx;
  S.ny = ny;
  S.periodic = c.periodic;
  S.closed = c.closed;
  S.upwind = c.advection == AERO_ADV_UPWIND3;
  S.les = les ? c.les : 0;
  S.inv_h = T(1.0 / c.h);
  S.kadv = T((c.advection == AERO_ADV_UPWIND3 ? 7.0 / 24.0 : 0.25) / c.h);
  S.nuh2 = T(c.nu) * T(1.0 / (c.h * c.h));
  S.inv_h2 = T(1.0 / (c.h * c.h));
  S.live_nu = static_cast<const T *>(g->nu);
  S.live_eta = static_cast<const T *>(g->eta);
  S.live_kappa = c.thermal ? static_cast<const T *>(g->kappa) : nullptr;
  S.cfac = T(c.les == AERO_LES_VREMAN ? c.les_c * c.h * c.h : c.les_c * c.les_c * c.h * c.h);
  S.ru = rules2<T>(c, 0);
  S.rv = rules2<T>(c, 1);
  S.u0 = u0;
  S.v0 = v0;
  S.uh = uh;
  S.vh = vh;
  S.dt = small;
  S.u_inlet = static_cast<const T *>(g->u_inlet);
  S.has_win = has_win;
  for (int q = 0; q < 4; ++q) S.win[q] = c.window[q];
  S.chi_u = static_cast<const T *>(g->chi_u);
  S.chi_v = static_cast<const T *>(g->chi_v);
  S.chi_c = static_cast<const T *>(g->chi_c);
  S.a_u = static_cast<const T *>(g->a_u);
  S.a_v = static_cast<const T *>(g->a_v);
  S.k_u = static_cast<const T *>(g->k_u);
  S.k_v = static_cast<const T *>(g->k_v);
  S.eta = T(c.eta);
  S.nbody = has_win ? c.nbody : 0;
  const dim3 grid(p->gx, p->gy), block(TX, TY);
  const bool placed =
      c.nfan || c.pid || c.paint || c.heaters || c.ports || c.dye_channels || c.wall_model || c.forcing;
  S.forcing = c.forcing;
  S.force_u = T(c.force[0]);
  S.force_v = T(c.force[1]);
  S.wall_model = c.wall_model;
  S.wall_ground = T(c.wall_ground_speed);
  S.nu_c = T(c.nu);
  S.h_c = T(c.h);
  if (c.dye_channels > 0 && c.dye && c.dye_channels > 1 && !(f->dye_extra0 && f->dye_extra))
    return set_error(AERO_EINVAL, "smoke channels 1.. need dye_extra0 / dye_extra");
  if (rec && (!std::is_same<T, float>::value || les || thermal || c.dye || dt_mode != 0 || placed))
    return set_error(AERO_EUNSUPPORTED, "the persistent sweep runs FP32 plans without LES, heat transfer, dye or "
                                        "placed physics, with the CFL time step");
  if ((c.nfan || c.pid) && (!f->ctrl0 || !f->ctrl || (c.pid && !f->dt_prev)))
    return set_error(AERO_EINVAL, "fans and the PID step need the controller memory (ctrl0, ctrl) and dt_prev");
  // fans, the PID controller and the heaters' bounds act on the step before the first stage:
  // the control kernel computes dt (and the thrusts) and the stages read it
  const bool control = c.nfan || (dt_mode == 0 && (c.pid || c.heaters || c.ports));
  if (placed) {
    S.nfan = c.nfan;
    S.fan_gu = static_cast<const T *>(g->fan_gu);
    S.fan_gv = static_cast<const T *>(g->fan_gv);
    S.fan_thrust = c.nfan ? reinterpret_cast<const T *>(ws + p->off_thrust) : nullptr;
    if (c.paint) {
      S.paint_u = static_cast<const T *>(g->paint_u);
      S.paint_v = static_cast<const T *>(g->paint_v);
      S.paint_wu = static_cast<const T *>(g->paint_wu);
      S.paint_wv = static_cast<const T *>(g->paint_wv);
    }
    if (c.ports) {   // the combined port / paint penalisation
      S.xchi_u = static_cast<const T *>(g->xchi_u);
      S.xa_u = static_cast<const T *>(g->xa_u);
      S.xchi_v = static_cast<const T *>(g->xchi_v);
      S.xa_v = static_cast<const T *>(g->xa_v);
      S.q_net = static_cast<const T *>(g->q_net);
      if (!(S.xchi_u && S.xa_u && S.xchi_v && S.xa_v && S.q_net && g->src && g->src_neg))
        return set_error(AERO_EINVAL, "a jets / vents array is missing");
    } else if (c.paint) {
      S.xchi_u = S.paint_u;
      S.xchi_v = S.paint_v;
    }
  }
  if (dt_mode == 0) {
    aero::MaxJobs<T> J{};
    J.job[0] = {u0, p->nu, bits + aero::SC_MAXU};
    J.job[1] = {v0, p->nv, bits + aero::SC_MAXV};
    if (thermal) J.job[2] = {static_cast<const T *>(f->theta0), p->nc, bits + aero::SC_MAXT};
    if (rec) {
      if constexpr (std::is_same<T, float>::value) {
        Op z = new_op(sw::ZERO, 1, 1);
        z.a.zero = {sc, 8};
        rec->ops.push_back(z);
        const long long nmax = (long long)std::max(p->nu, p->nv);
        Op m = new_op(sw::MAXABS, (nmax + sw::MAX_CHUNK - 1) / sw::MAX_CHUNK, 2);
        m.a.mx.J = J;
        m.a.mx.njobs = 2;
        m.a.mx.chunk = sw::MAX_CHUNK;
        rec->ops.push_back(m);
      }
    } else {
      AERO_CUDA_TRY(cudaMemsetAsync(sc, 0, 8 * sizeof(double), s));
      AERO_CUDA_TRY(aero::launch_absmax_multi<T>(J, thermal ? 3 : 2, s));
    }
    if (les) {
      StageParams<T> N = S;
      N.up = u0;
      N.vp = v0;
      N.nut_max = bits + aero::SC_NUTMAX;
      (void)aero::launch_k(stage2d_kernel<T, true, false>, grid, block, 0, s, N);
      AERO_CUDA_TRY(cudaGetLastError());
    }
  }
  // the time step itself is derived by the first stage kernel (dt2d_value), which stores it
  S.dt_mode = dt_mode;
  S.dt_in = static_cast<const T *>(dt_in);
  S.dt_bits = bits;
  S.dt_fixed = c.dt_fixed;
  S.dt_cfl_h = c.cfl * c.h;
  S.dt_nu = c.nu;
  S.dt_visc_h2 = 0.25 * c.h * c.h;
  S.dt_les = les ? 1 : 0;
  S.dt_store = small;
  if (thermal && dt_mode == 0)
    S.dt_th = Dt2dThermal{1, c.kappa, 1.0 / c.prt, 2.0 / c.h, c.diff_coef / (c.h * c.h), std::fabs(c.ri), c.cfl, c.h};
  if (control) {
    Control2dParams<T> K{};
    K.nx = nx;
    K.ny = ny;
    K.nfan = c.nfan;
    K.pid = c.pid;
    K.ports = c.ports;
    K.dt_mode = dt_mode;
    K.les = les ? 1 : 0;
    K.dt_in = static_cast<const T *>(dt_in);
    K.dt_fixed = c.dt_fixed;
    K.cfl_h = c.cfl * c.h;
    K.nu = c.nu;
    K.visc_h2 = 0.25 * c.h * c.h;
    K.bits = bits;
    K.live_nu = static_cast<const T *>(g->nu);
    K.live_kappa = thermal ? static_cast<const T *>(g->kappa) : nullptr;
    K.th = S.dt_th;
    K.u_floor = static_cast<const T *>(g->u_floor);
    K.heat_max = c.heaters ? static_cast<const T *>(g->heat_max) : nullptr;
    K.dt_prev = static_cast<const T *>(f->dt_prev);
    K.ctrl0 = static_cast<const T *>(f->ctrl0);
    K.ctrl = static_cast<T *>(f->ctrl);
    K.u0 = u0;
    K.v0 = v0;
    K.fan_phi = static_cast<const T *>(g->fan_phi);
    K.fan_dir = static_cast<const T *>(g->fan_dir);
    K.fan_value = static_cast<const T *>(g->fan_value);
    K.fan_width = static_cast<const T *>(g->fan_width);
    K.fan_kp = static_cast<const T *>(g->fan_kp);
    K.fan_ki = static_cast<const T *>(g->fan_ki);
    K.fan_dpmax = static_cast<const T *>(g->fan_dpmax);
    K.fan_isvel = static_cast<const T *>(g->fan_isvel);
    K.fan_isthrust = static_cast<const T *>(g->fan_isthrust);
    K.thrust = c.nfan ? reinterpret_cast<T *>(ws + p->off_thrust) : nullptr;
    K.thrust_out = static_cast<T *>(f->fan_thrust);
    K.ud_out = static_cast<T *>(f->fan_ud);
    K.dt_out = small;
    if (!K.u_floor) return set_error(AERO_EINVAL, "placed physics needs the u_floor scalar");
    if (c.nfan && !(K.fan_phi && K.fan_dir && K.fan_value && K.fan_width && K.fan_kp && K.fan_ki && K.fan_dpmax &&
                    K.fan_isvel && K.fan_isthrust && S.fan_gu && S.fan_gv))
      return set_error(AERO_EINVAL, "a fan array is missing");
    if (c.heaters && !K.heat_max) return set_error(AERO_EINVAL, "heaters need heat_max");
    if (thermal)
      (void)aero::launch_k(control2d_kernel<T, true>, 1, 1024, 0, s, K);
    else
      (void)aero::launch_k(control2d_kernel<T, false>, 1, 1024, 0, s, K);
    AERO_CUDA_TRY(cudaGetLastError());
  }
  if (c.paint && !(S.paint_u && S.paint_v && S.paint_wu && S.paint_wv && g->paint_c))
    return set_error(AERO_EINVAL, "a paint array is missing");
  // heat transfer: buoyancy in the stage kernel, theta in its own kernel after it
  T *nutb = thermal ? reinterpret_cast<T *>(ws + p->off_nut) : nullptr;
  T *tb[2] = {thermal ? reinterpret_cast<T *>(ws + p->off_tb0) : nullptr,
              thermal ? reinterpret_cast<T *>(ws + p->off_tb1) : nullptr};
  ThetaParams<T> TP{};
  if (thermal) {
    S.ri_gx = T(T(c.ri) * T(-c.gravity[0]));
    S.ri_gy = T(T(c.ri) * T(-c.gravity[1]));
    S.buoy_u = c.ri != 0.0 && c.gravity[0] != 0.0;
    S.buoy_v = c.ri != 0.0 && c.gravity[1] != 0.0;
    S.vol_u = c.has_vol ? static_cast<const T *>(g->vol_u) : nullptr;
    S.vol_v = c.has_vol ? static_cast<const T *>(g->vol_v) : nullptr;
    S.nut_out = les ? nutb : nullptr;
    S.up_out = reinterpret_cast<T *>(ws + p->off_upf);
    S.vp_out = reinterpret_cast<T *>(ws + p->off_vpf);
    TP.nx = nx;
    TP.ny = ny;
    TP.periodic = c.periodic;
    TP.closed = c.closed;
    TP.inv_h = T(1.0 / c.h);
    TP.inv_half = T(2.0 / c.h);
    TP.kappa = T(c.kappa);
    TP.inv_prt = T(1.0 / c.prt);
    TP.theta_in = T(c.theta_in);
    TP.eta_t = T(c.eta_t);
    TP.live_kappa = static_cast<const T *>(g->kappa);
    TP.live_eta_t = static_cast<const T *>(g->eta_t);
    TP.th0 = static_cast<const T *>(f->theta0);
    TP.nut = les ? nutb : nullptr;
    for (int q = 0; q < 4; ++q) {
      TP.mode[q] = c.wall_mode[q];
      TP.wval[q] = T(c.wall_value[q]);
      TP.win[q] = c.window[q];
    }
    TP.has_win = has_win;
    TP.ins_u = c.has_ins ? static_cast<const T *>(g->ins_u) : nullptr;
    TP.ins_v = c.has_ins ? static_cast<const T *>(g->ins_v) : nullptr;
    TP.q_skin = c.n_flux ? static_cast<const T *>(g->q_skin) : nullptr;
    TP.chi_t = static_cast<const T *>(g->chi_t);
    TP.a_t = static_cast<const T *>(g->a_t);
    TP.w_t = static_cast<const T *>(g->w_t);
    TP.w_f = static_cast<const T *>(g->w_f);
    TP.n_temp = has_win ? c.n_temp : 0;
    TP.n_flux = has_win ? c.n_flux : 0;
    TP.dt = small;
  }
  // ---- stages
  static const double RK[3][3] = {{0.0, 1.0, 1.0 / 6.0}, {0.75, 0.25, 2.0 / 3.0}, {1.0 / 3.0, 2.0 / 3.0, 1.0}};
  T *p_out = static_cast<T *>(f->p);
  // the fused projection on the x lengths the persistent sweep's kernel tiles too, so that a
  // recorded step and a direct one run the same arithmetic (the sweep matches the loop bit for bit)
  const bool fused = p->ax[0].method == 0 && sweep_tiled(nx) && !c.ports;
  // stage values alternate between two buffer pairs; stages 2 and 3 project the previous
  // stage's value themselves while staging it (P.psi), so only the last stage runs
  // correct2d_kernel, into the caller's u, v
  T *ub[2] = {uh, upb}, *vb[2] = {vh, vpb};
  for (int st = 0; st < 3; ++st) {
    StageParams<T> P = S;
    P.up = st == 0 ? u0 : ub[(st + 1) % 2];
    P.vp = st == 0 ? v0 : vb[(st + 1) % 2];
    P.psi = st == 0 ? nullptr : pa;
    P.uh = ub[st % 2];
    P.vh = vb[st % 2];
    P.a = T(RK[st][0]);
    P.b = T(RK[st][1]);
    P.w = T(RK[st][2]);
    P.partials = partials + (size_t)st * p->nblocks * std::max(p->nq, 1);
    P.dt_here = st == 0 && !control;
    P.paint_part = c.paint ? reinterpret_cast<double *>(ws + p->off_ppart) + (size_t)st * p->nblocks * 2 : nullptr;
    const T *th_in = st == 0 ? static_cast<const T *>(f->theta0) : tb[(st - 1) % 2];
    if (thermal) {
      P.thp = th_in;
      // the previous theta stage reads this stage's outputs of the last one (nu_t, face velocities)
      if (st > 0) AERO_CUDA_TRY(cudaStreamWaitEvent(s, p->ev_join[st - 1], 0));
    }
    if (rec) {
      if constexpr (std::is_same<T, float>::value) {
        Op o = new_tiled_op(sw::STAGE, p->gx, p->gy, rec->tiles);
        o.a.st = P;
        rec->ops.push_back(o);
      }
    } else {
      if (placed)
        (void)(thermal ? aero::launch_k(stage2d_kernel<T, false, true, true>, grid, block, 0, s, P)
                       : aero::launch_k(stage2d_kernel<T, false, false, true>, grid, block, 0, s, P));
      else if (thermal)
        (void)aero::launch_k(stage2d_kernel<T, false, true>, grid, block, 0, s, P);
      else
        (void)aero::launch_k(stage2d_kernel<T, false, false>, grid, block, 0, s, P);
      AERO_CUDA_TRY(cudaGetLastError());
    }
    if (thermal) {  // theta of this stage on the side stream, beside the pressure solve
      ThetaParams<T> Q = TP;
      Q.thp = th_in;
      Q.th = st == 2 ? static_cast<T *>(f->theta) : tb[st % 2];
      Q.upf = S.up_out;
      Q.vpf = S.vp_out;
      Q.a = P.a;
      Q.b = P.b;
      Q.heat_part = reinterpret_cast<double *>(ws + p->off_hpart) + (size_t)st * p->nblocks * std::max(c.n_temp, 1);
      Q.rep_part = st == 2 ? reinterpret_cast<double *>(ws + p->off_rpart) : nullptr;
      Q.heat = c.heaters ? static_cast<const T *>(g->heat) : nullptr;
      Q.paint_u = c.paint ? static_cast<const T *>(g->paint_u) : nullptr;
      Q.paint_v = c.paint ? static_cast<const T *>(g->paint_v) : nullptr;
      Q.src_neg = c.ports ? static_cast<const T *>(g->src_neg) : nullptr;
      Q.pt_chi = c.ports ? static_cast<const T *>(g->pt_chi) : nullptr;
      Q.pt_a = c.ports ? static_cast<const T *>(g->pt_a) : nullptr;
      Q.jet_part = Q.pt_chi ? reinterpret_cast<double *>(ws + p->off_jpart) + (size_t)st * p->nblocks : nullptr;
      AERO_CUDA_TRY(cudaEventRecord(p->ev_fork[st], s));
      AERO_CUDA_TRY(cudaStreamWaitEvent(p->side, p->ev_fork[st], 0));
      (void)aero::launch_k(theta2d_kernel<T>, grid, block, 0, p->side, Q);
      AERO_CUDA_TRY(cudaGetLastError());
      AERO_CUDA_TRY(cudaEventRecord(p->ev_join[st], p->side));
    }
    const int acc_mode = st == 0 ? 0 : (st == 1 ? 1 : 2);
    if (fused) {
      aero::TransformParams<T> F{};
      F.fuse_div = 2;
      F.uh = ub[st % 2];
      F.vh = vb[st % 2];
      F.inv_h = T(1.0 / c.h);
      F.p_acc = p_out;
      F.wgt = T(RK[st][2]);
      F.acc_mode = acc_mode;
      F.dt = small;
      const int rc = poisson2d_passes<T>(p, nullptr, pa, ws, s, &F, rec);
      if (rc) return rc;
    } else if (rec) {
      if constexpr (std::is_same<T, float>::value) {
        Op d = new_op(sw::DIV, (nx + sw::NTHR * sw::EW - 1) / (sw::NTHR * sw::EW), ny);
        d.a.dv = {nx, ny, T(1.0 / c.h), ub[st % 2], vb[st % 2], pa};
        rec->ops.push_back(d);
        const int rc = poisson2d_passes<T>(p, pa, pa, ws, s, nullptr, rec);
        if (rc) return rc;
        Op a = new_op(sw::PSIACC, ((long long)p->nc + sw::NTHR * sw::EW - 1) / (sw::NTHR * sw::EW), 1);
        a.a.pa = {pa, p_out, (long long)p->nc, T(RK[st][2]), acc_mode, small};
        rec->ops.push_back(a);
      }
    } else {
      (void)aero::launch_k(divergence2d_kernel<T>, dim3((nx + 127) / 128, ny), 128, 0, s, nx, ny, T(1.0 / c.h),
                           ub[st % 2], vb[st % 2], pa);
      AERO_CUDA_TRY(cudaGetLastError());
      if (c.ports) {
        (void)aero::launch_k(port_source2d_kernel<T>, (int)std::min<size_t>((p->nc + 255) / 256, 148 * 8), 256, 0, s,
                             pa, static_cast<const T *>(g->src), p->nc);
        AERO_CUDA_TRY(cudaGetLastError());
      }
      const int rc = poisson2d_passes<T>(p, pa, pa, ws, s);
      if (rc) return rc;
      AERO_CUDA_TRY(aero::launch_psi_accumulate<T>(pa, p_out, p->nc, T(RK[st][2]), acc_mode, small, s));
    }
    if (st == 2 && rec) {
      if constexpr (std::is_same<T, float>::value) {
        Op o = new_op(sw::CORRECT, (nx + sw::NTHR * sw::EW - 1) / (sw::NTHR * sw::EW), ny);
        o.a.co = {nx, ny, c.periodic, T(1.0 / c.h), ub[st % 2], vb[st % 2], pa, static_cast<T *>(f->u),
                  static_cast<T *>(f->v)};
        rec->ops.push_back(o);
      }
    } else if (st == 2) {
      (void)aero::launch_k(correct2d_kernel<T>, dim3((nx + 127) / 128, ny), 128, 0, s, nx, ny, c.periodic,
                           T(1.0 / c.h), ub[st % 2], vb[st % 2], pa, static_cast<T *>(f->u), static_cast<T *>(f->v));
      AERO_CUDA_TRY(cudaGetLastError());
    }
  }
  if (thermal) {
    AERO_CUDA_TRY(cudaStreamWaitEvent(s, p->ev_join[2], 0));
    ReportParams<T> R{};
    R.nx = nx;
    R.ny = ny;
    R.periodic = c.periodic;
    R.closed = c.closed;
    R.nblocks = p->nblocks;
    R.n_temp = TP.n_temp;
    R.n_flux = TP.n_flux;
    R.h = T(c.h);
    R.hd = c.h;
    R.h2 = T(c.h * c.h);
    R.kappa = T(c.kappa);
    R.live_kappa = static_cast<const T *>(g->kappa);
    R.theta_in = T(c.theta_in);
    for (int q = 0; q < 4; ++q) {
      R.mode[q] = c.wall_mode[q];
      R.wval[q] = T(c.wall_value[q]);
    }
    for (int q = 0; q < 3; ++q) R.wgt[q] = T(RK[q][2]);
    R.heat_part = reinterpret_cast<const double *>(ws + p->off_hpart);
    R.rep_part = reinterpret_cast<const double *>(ws + p->off_rpart);
    R.theta = static_cast<const T *>(f->theta);
    R.u = static_cast<const T *>(f->u);
    R.dt = small;
    R.heat = static_cast<double *>(f->heat);
    R.theta_wall = static_cast<double *>(f->theta_wall);
    R.wall_heat = static_cast<double *>(f->wall_heat);
    R.heat_storage = static_cast<double *>(f->heat_storage);
    R.flow_heat = static_cast<double *>(f->flow_heat);
    R.ports = c.ports;
    R.jet_part = c.ports && g->pt_chi ? reinterpret_cast<const double *>(ws + p->off_jpart) : nullptr;
    R.jet_heat = static_cast<double *>(f->jet_heat);
    R.vent_heat = static_cast<double *>(f->vent_heat);
    (void)aero::launch_k(heat_report2d_kernel<T>, 1, 256, 0, s, R);
    AERO_CUDA_TRY(cudaGetLastError());
  }
  // ---- dye with the step's final velocity
  if (c.dye && c.dye_channels > 0) {   // smoke channels with emitter groups and smoking jets
    DyeChannelsParams<T> D{};
    D.nx = nx;
    D.ny = ny;
    D.periodic = c.periodic;
    D.closed = c.closed;
    D.nch = c.dye_channels;
    D.ngroup = c.n_groups;
    D.inv_h = T(1.0 / c.h);
    for (int ch = 0; ch < c.dye_channels; ++ch) {
      D.c0[ch] = ch == 0 ? static_cast<const T *>(f->dye0) : static_cast<const T *>(f->dye_extra0) + (size_t)(ch - 1) * p->nc;
      D.c[ch] = ch == 0 ? static_cast<T *>(f->dye) : static_cast<T *>(f->dye_extra) + (size_t)(ch - 1) * p->nc;
      D.port_w[ch] = static_cast<const T *>(g->port_dye[ch]);
    }
    D.u = static_cast<const T *>(f->u);
    D.v = static_cast<const T *>(f->v);
    D.dt = small;
    D.t0 = static_cast<const T *>(f->t0);
    D.inflow = static_cast<const T *>(g->dye_inflow);
    D.src_neg = c.ports ? static_cast<const T *>(g->src_neg) : nullptr;
    for (int q = 0; q < c.n_groups; ++q) {
      D.gch[q] = c.group_channel[q];
      D.gw[q] = static_cast<const T *>(g->group_w[q]);
      D.gtarget[q] = static_cast<const T *>(g->group_target[q]);
      D.gtiming[q] = static_cast<const T *>(g->group_timing[q]);
    }
    D.has_win = has_win;
    for (int q = 0; q < 4; ++q) D.win[q] = c.window[q];
    D.chi_c = static_cast<const T *>(g->chi_c);
    D.paint_c = c.paint ? static_cast<const T *>(g->paint_c) : nullptr;
    (void)aero::launch_k(dye_channels2d_kernel<T>, dim3((nx + 127) / 128, ny), 128, 0, s, D);
    AERO_CUDA_TRY(cudaGetLastError());
  } else if (c.dye) {
    DyeParams<T> D{};
    D.nx = nx;
    D.ny = ny;
    D.periodic = c.periodic;
    D.inv_h = T(1.0 / c.h);
    D.c0 = static_cast<const T *>(f->dye0);
    D.u = static_cast<const T *>(f->u);
    D.v = static_cast<const T *>(f->v);
    D.dt = small;
    D.inlet = static_cast<const T *>(g->dye_inlet);
    D.c = static_cast<T *>(f->dye);
    D.has_win = has_win;
    for (int q = 0; q < 4; ++q) D.win[q] = c.window[q];
    D.chi_c = static_cast<const T *>(g->chi_c);
    D.paint_c = c.paint ? static_cast<const T *>(g->paint_c) : nullptr;
    (void)aero::launch_k(dye2d_kernel<T>, dim3((nx + 127) / 128, ny), 128, 0, s, D);
    AERO_CUDA_TRY(cudaGetLastError());
  }
  if (rec) {
    if constexpr (std::is_same<T, float>::value) {
      Op o = new_op(sw::FINAL, 1, 1);
      o.a.fi = {partials, p->nblocks, S.nbody, c.h, c.force_ref, small, static_cast<const T *>(f->t0),
                static_cast<T *>(f->t), static_cast<T *>(f->dt), static_cast<T *>(f->coeffs)};
      rec->ops.push_back(o);
    }
    return AERO_OK;
  }
  if (c.paint && f->paint_force) {
    (void)aero::launch_k(paint_force2d_kernel<T>, 1, 64, 0, s, (const double *)(ws + p->off_ppart), p->nblocks,
                         c.h * c.h, c.force_ref, (const T *)small, static_cast<T *>(f->paint_force));
    AERO_CUDA_TRY(cudaGetLastError());
  }
  (void)aero::launch_k(finalize2d_kernel<T>, 1, 256, 0, s, partials, p->nblocks, S.nbody, c.h, c.force_ref, small,
                                         static_cast<const T *>(f->t0), static_cast<T *>(f->t),
                                         static_cast<T *>(f->dt), static_cast<T *>(f->coeffs));
  AERO_CUDA_TRY(cudaGetLastError());
  return AERO_OK;
}

}  // namespace

extern "C" {

int aero_ns2d_plan_create(const AeroNs2dConfig *cfg, AeroNs2dPlan **plan) {
  if (!cfg || !plan) return set_error(AERO_EINVAL, "null argument");
  *plan = nullptr;
  const AeroNs2dConfig &c = *cfg;
  if (c.abi_version != AERO_ABI_VERSION) return set_error(AERO_EINVAL, "ABI version mismatch");
  if (c.dtype != AERO_F32 && c.dtype != AERO_F64) return set_error(AERO_EINVAL, "dtype must be float32 or float64");
  if (c.nx < 4 || c.ny < 4) return set_error(AERO_EINVAL, "the grid needs at least 4 x 4 cells");
  if (!(c.h > 0) || !std::isfinite(c.h)) return set_error(AERO_EINVAL, "cell size h must be positive");
  if (c.periodic && c.closed) return set_error(AERO_EINVAL, "a periodic domain cannot also be closed");
  if (c.advection != AERO_ADV_UPWIND3 && c.advection != AERO_ADV_CENTRAL) return set_error(AERO_EINVAL, "unknown advection");
  if (c.les < AERO_LES_NONE || c.les > AERO_LES_VREMAN) return set_error(AERO_EINVAL, "unknown turbulence model");
  if (c.nbody < 0 || c.nbody > AERO_MAX_BODIES)
    return set_error(AERO_EUNSUPPORTED, "at most " + std::to_string(AERO_MAX_BODIES) + " bodies");
  for (int q = 0; q < 2; ++q)
    for (int a = 0; a < 2; ++a)
      for (int s = 0; s < 2; ++s)
        if (c.ghost_kind[q][a][s] < AERO_GHOST_EDGE || c.ghost_kind[q][a][s] > AERO_GHOST_PERIODIC_FACE)
          return set_error(AERO_EINVAL, "unknown ghost rule");
  const bool has_win = c.window[1] > c.window[0] && c.window[3] > c.window[2];
  if (has_win && (c.window[0] < 0 || c.window[1] > c.ny || c.window[2] < 0 || c.window[3] > c.nx))
    return set_error(AERO_EINVAL, "body window outside the domain");
  if (!(c.eta > 0)) return set_error(AERO_EINVAL, "eta must be positive");
  if (c.thermal) {
    if (c.n_temp < 0 || c.n_temp > AERO_MAX_BODIES || c.n_flux < 0 || c.n_flux > AERO_MAX_BODIES)
      return set_error(AERO_EUNSUPPORTED, "at most " + std::to_string(AERO_MAX_BODIES) + " temperature / heat-flux bodies");
    if ((c.n_temp || c.n_flux || c.has_ins || c.has_vol) && !has_win)
      return set_error(AERO_EINVAL, "thermal body masks need a body window");
    for (int q = 0; q < 4; ++q)
      if (c.wall_mode[q] < AERO_TH2_ADIABATIC || c.wall_mode[q] > AERO_TH2_PERIODIC)
        return set_error(AERO_EINVAL, "unknown temperature boundary mode");
    if (c.periodic != (c.wall_mode[0] == AERO_TH2_PERIODIC))
      return set_error(AERO_EINVAL, "temperature boundary modes disagree with the periodicity of the domain");
    if (!(c.prt > 0)) return set_error(AERO_EINVAL, "turbulent Prandtl number must be positive");
    if (c.n_temp && !(c.eta_t > 0)) return set_error(AERO_EINVAL, "eta_t must be positive");
  }
  if (c.nfan < 0 || c.nfan > AERO_MAX_FANS)
    return set_error(AERO_EUNSUPPORTED, "at most " + std::to_string(AERO_MAX_FANS) + " fans");
  if (c.heaters && !c.thermal) return set_error(AERO_EINVAL, "heaters need heat transfer");
  if (c.dye_channels < 0 || c.dye_channels > AERO_MAX_DYE_CHANNELS || c.n_groups < 0 ||
      c.n_groups > AERO_MAX_DYE_GROUPS || (c.dye_channels > 0 && !c.dye))
    return set_error(AERO_EINVAL, "smoke channels: 1..4 with dye on, at most 8 emitter groups");
  for (int q = 0; q < c.n_groups; ++q)
    if (c.group_channel[q] < 0 || c.group_channel[q] >= c.dye_channels)
      return set_error(AERO_EINVAL, "an emitter group's channel is out of range");
  auto *p = new AeroNs2dPlan();
  p->cfg = c;
  const size_t e = c.dtype == AERO_F64 ? 8 : 4;
  p->esz = e;
  const size_t nx = c.nx, ny = c.ny;
  p->nu = ny * (nx + 1);
  p->nv = (ny + 1) * nx;
  p->nc = ny * nx;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t at = off;
    off += aero_host::align_up(bytes);
    return at;
  };
  p->off_uh = take(p->nu * e);
  p->off_vh = take(p->nv * e);
  p->off_up = take(p->nu * e);
  p->off_vp = take(p->nv * e);
  p->off_pa = take(p->nc * e);
  p->off_small = take(8 * e);
  p->off_scalars = take(sizeof(double) * aero::SC_COUNT);
  p->off_zero = take(sizeof(double));
  p->gx = (int)((nx + aero::ns2d::TX - 1) / aero::ns2d::TX);
  p->gy = (int)((ny + aero::ns2d::TY - 1) / aero::ns2d::TY);
  p->nblocks = p->gx * p->gy;
  p->nq = has_win ? 4 * c.nbody : 0;
  p->off_partials = take(sizeof(double) * 3 * (size_t)p->nblocks * std::max(p->nq, 1));
  if (c.nfan) p->off_thrust = take((size_t)c.nfan * e);
  if (c.paint) p->off_ppart = take(sizeof(double) * 3 * (size_t)p->nblocks * 2);
  if (c.ports && c.thermal) p->off_jpart = take(sizeof(double) * 3 * (size_t)p->nblocks);
  if (c.thermal) {
    p->off_nut = take(p->nc * e);
    p->off_tb0 = take(p->nc * e);
    p->off_tb1 = take(p->nc * e);
    p->off_hpart = take(sizeof(double) * 3 * (size_t)p->nblocks * std::max(c.n_temp, 1));
    p->off_rpart = take(sizeof(double) * (size_t)p->nblocks * (3 + c.n_flux));
    p->off_upf = take(p->nu * e);
    p->off_vpf = take(p->nv * e);
    bool ok = cudaStreamCreateWithFlags(&p->side, cudaStreamNonBlocking) == cudaSuccess;
    for (int q = 0; q < 3 && ok; ++q)
      ok = cudaEventCreateWithFlags(&p->ev_fork[q], cudaEventDisableTiming) == cudaSuccess &&
           cudaEventCreateWithFlags(&p->ev_join[q], cudaEventDisableTiming) == cudaSuccess;
    if (!ok) {
      (void)cudaGetLastError();
      aero_ns2d_plan_destroy(p);
      return set_error(AERO_ECUDA, "cannot create the heat-transfer side stream");
    }
  }
  aero_host::axis_setup(p->ax[0], c.nx, c.periodic != 0, e);
  aero_host::axis_setup(p->ax[1], c.ny, c.periodic != 0, e);
  for (int a = 0; a < 2; ++a) aero_host::axis_place(p->ax[a], e, take);
  p->total = off;
  *plan = p;
  return AERO_OK;
}

void aero_ns2d_plan_destroy(AeroNs2dPlan *plan) {
  if (!plan) return;
  for (int q = 0; q < 3; ++q) {
    if (plan->ev_fork[q]) cudaEventDestroy(plan->ev_fork[q]);
    if (plan->ev_join[q]) cudaEventDestroy(plan->ev_join[q]);
  }
  if (plan->side) cudaStreamDestroy(plan->side);
  delete plan;
}

size_t aero_ns2d_workspace_bytes(const AeroNs2dPlan *plan) { return plan ? plan->total : 0; }

int aero_ns2d_workspace_init(const AeroNs2dPlan *plan, void *workspace, void *stream) {
  if (!plan || !workspace) return set_error(AERO_EINVAL, "null argument");
  if (reinterpret_cast<uintptr_t>(workspace) % aero_host::ALIGN)
    return set_error(AERO_EINVAL, "workspace must be 256-byte aligned");
  auto s = static_cast<cudaStream_t>(stream);
  auto ws = static_cast<unsigned char *>(workspace);
  return plan->cfg.dtype == AERO_F64 ? init2d_impl<double>(plan, ws, s) : init2d_impl<float>(plan, ws, s);
}

int aero_ns2d_step(const AeroNs2dPlan *plan, const AeroNs2dFields *f, const AeroNs2dGeom *g, const void *dt_in,
                   void *workspace, void *stream) {
  if (!plan || !f || !g || !workspace) return set_error(AERO_EINVAL, "null argument");
  if (reinterpret_cast<uintptr_t>(workspace) % aero_host::ALIGN)
    return set_error(AERO_EINVAL, "workspace must be 256-byte aligned");
  const AeroNs2dConfig &c = plan->cfg;
  if (!f->u0 || !f->v0 || !f->t0 || !f->u || !f->v || !f->p || !f->t || !f->dt)
    return set_error(AERO_EINVAL, "missing state pointer");
  if (c.dye && (!f->dye0 || !f->dye)) return set_error(AERO_EINVAL, "dye needs dye pointers");
  if (c.dye && f->dye0 == f->dye) return set_error(AERO_EINVAL, "dye output must not alias dye input");
  if (!c.periodic && !c.closed && !g->u_inlet) return set_error(AERO_EINVAL, "missing inlet profile");
  const bool has_win = c.nbody > 0 && c.window[1] > c.window[0] && c.window[3] > c.window[2];
  if (has_win && (!g->chi_u || !g->chi_v || !g->chi_c || !g->a_u || !g->a_v || !g->k_u || !g->k_v || !f->coeffs))
    return set_error(AERO_EINVAL, "missing body masks");
  if (c.thermal) {
    if (!f->theta0 || !f->theta || !f->wall_heat || !f->heat_storage || !f->flow_heat)
      return set_error(AERO_EINVAL, "heat transfer needs theta and report pointers");
    if ((c.n_temp && (!f->heat || !g->chi_t || !g->a_t || !g->w_t)) || (c.n_flux && (!f->theta_wall || !g->q_skin || !g->w_f)) ||
        (c.has_ins && (!g->ins_u || !g->ins_v)) || (c.has_vol && (!g->vol_u || !g->vol_v)))
      return set_error(AERO_EINVAL, "missing thermal body masks or report pointers");
  }
  auto s = static_cast<cudaStream_t>(stream);
  auto ws = static_cast<unsigned char *>(workspace);
  return c.dtype == AERO_F64 ? step2d_impl<double>(plan, f, g, dt_in, ws, s)
                             : step2d_impl<float>(plan, f, g, dt_in, ws, s);
}

int aero_ns2d_poisson_solve(const AeroNs2dPlan *plan, const void *f, void *psi, void *workspace, void *stream) {
  if (!plan || !f || !psi || !workspace) return set_error(AERO_EINVAL, "null argument");
  auto s = static_cast<cudaStream_t>(stream);
  auto ws = static_cast<unsigned char *>(workspace);
  return plan->cfg.dtype == AERO_F64
             ? poisson2d_passes<double>(plan, static_cast<const double *>(f), static_cast<double *>(psi), ws, s)
             : poisson2d_passes<float>(plan, static_cast<const float *>(f), static_cast<float *>(psi), ws, s);
}

}  // extern "C"


// ---------------------------------------------------------------------------------------
// the batched sweep (C ABI)
// ---------------------------------------------------------------------------------------

struct AeroNs2dSweep {
  std::vector<Op> ops;                          // phase by phase
  std::vector<int> item_op;                     // operation of every work item
  std::vector<long long> op_first, phase_base, phase_items;
  long long items = 0;
  int n = 0, nphase = 0, lcap = 2, ctas_per_sm = 1, order = 0, sched = 0, grid = 0;
  size_t smem = 0;
  // workspace: [0, 4) status, [16, 24) barrier words, [24, 32) queue, [32, 32 + 4 n) finished
  // items per instance (all but the status reset before every step), then the tables
  size_t sync_bytes = 0, off_ops = 0, off_io = 0, off_of = 0, off_pb = 0, off_pi = 0, total = 0;
  int spin_limit = 1 << 26, extra = 0;
  bool has_line = false;  // any transform pass on run-time stage tables
};

namespace {

using SweepKernel = void (*)(const aero::ns2d::sweep::Tables);

template <int LCAP, int MINB>
SweepKernel sweep_kernel_line(bool line) {
  namespace sw = aero::ns2d::sweep;
  return line ? sw::sweep2d_kernel<LCAP, MINB, true> : sw::sweep2d_kernel<LCAP, MINB, false>;
}

// the kernel of a tuning: widest transform tile 2^lcap, registers capped for 2, 3 or 4 CTAs per
// SM, with or without the run-time-table transform body
SweepKernel sweep_kernel(int lcap, int cps, bool line) {
  if (cps >= 4) return lcap == 2 ? sweep_kernel_line<2, 4>(line) : sweep_kernel_line<3, 4>(line);
  if (cps == 3) return lcap == 2 ? sweep_kernel_line<2, 3>(line) : sweep_kernel_line<3, 3>(line);
  return lcap == 2 ? sweep_kernel_line<2, 2>(line) : sweep_kernel_line<3, 2>(line);
}

size_t op_smem(const Op &o, int lcap) {
  namespace sw = aero::ns2d::sweep;
  if (o.kind == sw::POW2) {
    const int l2 = sw::tile_l2(o.n, lcap), L = 1 << l2;
    const size_t e = sizeof(float);
    return (size_t)o.n * 2 * e + ((((size_t)o.n * (L + 1) * e) + 15) & ~size_t(15)) + 2 * (size_t)o.n * (L / 2) * 2 * e;
  }
  if (o.kind == sw::LINE) return aero::transform_smem_bytes<float>(o.n, o.a.tr.L);
  return 0;
}

}  // namespace

extern "C" {

int aero_ns2d_sweep_create(int32_t n, const AeroNs2dPlan *const *plans, const AeroNs2dFields *fields,
                           const AeroNs2dGeom *geoms, void *const *workspaces, const AeroSweepTuning *tuning,
                           AeroNs2dSweep **sweep) {
  if (!plans || !fields || !geoms || !workspaces || !sweep || n < 1) return set_error(AERO_EINVAL, "null argument");
  *sweep = nullptr;
  const int lcap = tuning ? tuning->lcap : 2, cps = tuning ? tuning->ctas_per_sm : 1, order = tuning ? tuning->order : 1;
  const int sched = tuning ? tuning->schedule : 1, tiles = tuning ? tuning->tiles : 1;
  if (lcap < 2 || lcap > 3 || cps < 1 || cps > 4 || order < 0 || order > 1 || sched < 0 || sched > 2 || tiles < 1 ||
      tiles > 16)
    return set_error(AERO_EINVAL, "tuning: lcap 2..3, ctas_per_sm 1..4, order 0..1, schedule 0..2, tiles 1..16");
  std::vector<std::vector<Op>> per(n);
  std::vector<long long> size(n);
  for (int k = 0; k < n; ++k) {
    if (!plans[k] || !workspaces[k]) return set_error(AERO_EINVAL, "null plan or workspace");
    if (plans[k]->cfg.dtype != AERO_F32) return set_error(AERO_EUNSUPPORTED, "the persistent sweep runs FP32 plans");
    Recorder rec;
    rec.lcap = lcap;
    rec.tiles = tiles;
    const int rc = step2d_impl<float>(plans[k], &fields[k], &geoms[k], nullptr,
                                      static_cast<unsigned char *>(workspaces[k]), nullptr, &rec);
    if (rc) return rc;
    per[k] = std::move(rec.ops);
    size[k] = (long long)plans[k]->cfg.nx * plans[k]->cfg.ny;
  }
  std::vector<int> inst(n);
  for (int k = 0; k < n; ++k) inst[k] = k;
  if (order == 1)   // largest instances first: their work items start first in every phase
    std::stable_sort(inst.begin(), inst.end(), [&](int a, int b) { return size[a] > size[b]; });
  auto *S = new AeroNs2dSweep();
  S->n = n;
  S->lcap = lcap;
  S->ctas_per_sm = cps;
  S->order = order;
  S->sched = sched;
  size_t longest = 0;
  for (auto &v : per) longest = std::max(longest, v.size());
  S->nphase = (int)longest;
  std::vector<long long> seen(n, 0);   // work items of each instance's operations so far
  for (int ph = 0; ph < S->nphase; ++ph) {
    S->phase_base.push_back(S->items);
    for (int k : inst) {
      if ((size_t)ph >= per[k].size()) continue;
      Op o = per[k][ph];
      const long long cnt = (long long)o.gx * o.gy;
      o.inst = k;
      o.need = (int)seen[k];
      seen[k] += cnt;
      S->op_first.push_back(S->items);
      S->item_op.insert(S->item_op.end(), (size_t)cnt, (int)S->ops.size());
      S->ops.push_back(o);
      S->smem = std::max(S->smem, op_smem(o, lcap));
      S->items += cnt;
    }
    S->phase_items.push_back(S->items - S->phase_base.back());
  }
  for (long long x : seen)
    if (x >= (1ll << 31)) {
      delete S;
      return set_error(AERO_EUNSUPPORTED, "an instance has more than 2^31 work items per step");
    }
  S->sync_bytes = aero_host::align_up(32 + 4 * (size_t)n);
  size_t off = S->sync_bytes;
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off = aero_host::align_up(off + bytes);
    return o;
  };
  S->off_ops = take(S->ops.size() * sizeof(Op));
  S->off_io = take(S->item_op.size() * sizeof(int));
  S->off_of = take(S->op_first.size() * sizeof(long long));
  S->off_pb = take(S->phase_base.size() * sizeof(long long));
  S->off_pi = take(S->phase_items.size() * sizeof(long long));
  S->total = off;
  // co-resident CTAs: every CTA waits at the grid barriers
  int dev = 0, nsm = 0, occ = 0;
  for (const Op &o : S->ops) S->has_line = S->has_line || o.kind == aero::ns2d::sweep::LINE;
  const SweepKernel kern = sweep_kernel(lcap, cps, S->has_line);
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)std::max<size_t>(S->smem, 1));
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, aero::ns2d::sweep::NTHR, S->smem);
  if (e != cudaSuccess || occ < 1) {
    delete S;
    return set_error(AERO_ECUDA, std::string("persistent sweep kernel does not fit an SM: ") +
                                     (e != cudaSuccess ? cudaGetErrorString(e) : "no resident block"));
  }
  S->grid = nsm * std::min(occ, cps);
  *sweep = S;
  return AERO_OK;
}

void aero_ns2d_sweep_destroy(AeroNs2dSweep *sweep) { delete sweep; }

size_t aero_ns2d_sweep_workspace_bytes(const AeroNs2dSweep *sweep) { return sweep ? sweep->total : 0; }

int aero_ns2d_sweep_init(const AeroNs2dSweep *sweep, void *workspace, void *stream) {
  if (!sweep || !workspace) return set_error(AERO_EINVAL, "null argument");
  if (reinterpret_cast<uintptr_t>(workspace) % aero_host::ALIGN)
    return set_error(AERO_EINVAL, "workspace must be 256-byte aligned");
  auto *ws = static_cast<unsigned char *>(workspace);
  auto s = static_cast<cudaStream_t>(stream);
  const AeroNs2dSweep &S = *sweep;
  AERO_CUDA_TRY(cudaMemsetAsync(ws, 0, S.sync_bytes, s));
  AERO_CUDA_TRY(cudaMemcpyAsync(ws + S.off_ops, S.ops.data(), S.ops.size() * sizeof(Op), cudaMemcpyHostToDevice, s));
  AERO_CUDA_TRY(cudaMemcpyAsync(ws + S.off_io, S.item_op.data(), S.item_op.size() * sizeof(int),
                                cudaMemcpyHostToDevice, s));
  AERO_CUDA_TRY(cudaMemcpyAsync(ws + S.off_of, S.op_first.data(), S.op_first.size() * sizeof(long long),
                                cudaMemcpyHostToDevice, s));
  AERO_CUDA_TRY(cudaMemcpyAsync(ws + S.off_pb, S.phase_base.data(), S.phase_base.size() * sizeof(long long),
                                cudaMemcpyHostToDevice, s));
  AERO_CUDA_TRY(cudaMemcpyAsync(ws + S.off_pi, S.phase_items.data(), S.phase_items.size() * sizeof(long long),
                                cudaMemcpyHostToDevice, s));
  AERO_CUDA_TRY(cudaStreamSynchronize(s));   // the host tables are pageable: finish before returning
  return AERO_OK;
}

int aero_ns2d_sweep_step(const AeroNs2dSweep *sweep, void *workspace, void *stream) {
  if (!sweep || !workspace) return set_error(AERO_EINVAL, "null argument");
  namespace sw = aero::ns2d::sweep;
  auto *ws = static_cast<unsigned char *>(workspace);
  auto s = static_cast<cudaStream_t>(stream);
  const AeroNs2dSweep &S = *sweep;
  sw::Tables T{};
  T.ops = reinterpret_cast<const Op *>(ws + S.off_ops);
  T.item_op = reinterpret_cast<const int *>(ws + S.off_io);
  T.op_first = reinterpret_cast<const long long *>(ws + S.off_of);
  T.phase_base = reinterpret_cast<const long long *>(ws + S.off_pb);
  T.phase_items = reinterpret_cast<const long long *>(ws + S.off_pi);
  T.total = S.items;
  T.nphase = S.nphase;
  T.sched = S.sched;
  T.status = reinterpret_cast<int *>(ws);
  T.bar = reinterpret_cast<unsigned int *>(ws + 16);
  T.queue = reinterpret_cast<unsigned long long *>(ws + 24);
  T.done = reinterpret_cast<unsigned int *>(ws + 32);
  T.spin_limit = S.spin_limit;
  T.extra = S.extra;
  // barrier words, queue and finished-item counters start at zero (the status word is kept)
  AERO_CUDA_TRY(cudaMemsetAsync(ws + 16, 0, 16 + 4 * (size_t)S.n, s));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(S.grid);
  cfg.blockDim = dim3(sw::NTHR);
  cfg.dynamicSmemBytes = S.smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;   // all CTAs resident together (they meet at barriers)
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  AERO_CUDA_TRY(cudaLaunchKernelEx(&cfg, sweep_kernel(S.lcap, S.ctas_per_sm, S.has_line), T));
  return AERO_OK;
}

int aero_ns2d_sweep_read_status(const AeroNs2dSweep *sweep, void *workspace, int32_t *status, void *stream) {
  if (!sweep || !workspace || !status) return set_error(AERO_EINVAL, "null argument");
  auto s = static_cast<cudaStream_t>(stream);
  AERO_CUDA_TRY(cudaMemcpyAsync(status, workspace, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  AERO_CUDA_TRY(cudaStreamSynchronize(s));
  AERO_CUDA_TRY(cudaMemsetAsync(workspace, 0, sizeof(int32_t), s));
  return AERO_OK;
}

int aero_ns2d_sweep_set_barrier(AeroNs2dSweep *sweep, int32_t spin_limit, int32_t extra) {
  if (!sweep || spin_limit < 1 || extra < 0) return set_error(AERO_EINVAL, "bad barrier settings");
  sweep->spin_limit = spin_limit;
  sweep->extra = extra;
  return AERO_OK;
}

int aero_ns2d_sweep_info(const AeroNs2dSweep *sweep, int64_t out[6]) {
  if (!sweep || !out) return set_error(AERO_EINVAL, "null argument");
  out[0] = sweep->nphase;
  out[1] = (int64_t)sweep->ops.size();
  out[2] = sweep->items;
  out[3] = sweep->grid;
  out[4] = (int64_t)sweep->smem;
  out[5] = sweep->lcap;
  return AERO_OK;
}

}  // extern "C"
