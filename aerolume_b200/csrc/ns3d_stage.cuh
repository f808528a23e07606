// The eddy-viscosity kernel and the SSP-RK3 stage kernel of the 3D step (templates; each
// precision is instantiated in its own translation unit, ns3d_stage_f32.cu / ns3d_stage_f64.cu).
//
// Arithmetic follows the reference's plain-torch step (Aerolume ns3d/core.py:765-883)
// operation by operation, so float64 runs agree with it to round-off:
//   advection   core.py:331-390      diffusion  core.py:393-397, 557-560
//   LES         core.py:400-524      RK update  core.py:819-827
//   boundaries  core.py:281-297, 527-543
//   penalty     core.py:615-634      buoyancy   physics.py:744-790
//   theta       physics.py:609-708
//
// Layout: C-contiguous (z, y, x) arrays with the staggered shapes of core.py:11-14; the
// stage-start u is read from a copy with a 16-byte row pitch (the reference's u rows hold
// nx + 1 values).  Both kernels tile x-y in 32 x 8 columns and march along z through a ring
// of plane slots in shared memory.  One thread streams each new z-plane of every field into
// its slot with TMA (cp.async.bulk.tensor, completion on the slot's mbarrier) one plane
// ahead of the computation, so the copies overlap the arithmetic; tiles on the domain
// boundary then overwrite their out-of-range entries with the ghost-cell rules.  Shapes
// whose rows are not 16-byte multiples use a synchronous loader into the same slots.
// What the z direction needs on both sides of a plane -- the z fluxes of the momentum
// components and of theta, the x-z / y-z shear stresses and tau_33 -- is evaluated once
// per interface and carried to the next plane in registers.
#pragma once

#include "ns3d.cuh"
#include "stencil.cuh"
#include "tma.cuh"

namespace aero {

constexpr int TX = 32, TY = 8;
// stage tile: x from i0 - 4 (a 16-byte aligned TMA start) to i0 + TX + 3, y from j0 - 2
constexpr int PX = TX + 8, PY = TY + 4, PPL = PX * PY;
// eddy-viscosity tile of the stage kernel: nu array columns i0 .. i0 + TX + 3, rows j0 .. j0 + TY + 1
constexpr int NUX = TX + 4, NUY = TY + 2, NUPL = 384;  // 360 used, slots padded to 128 bytes
constexpr int NSLOT = 6;
// nu kernel tile: x from i0 - 4, y from j0 - 2, 36 x 10; a ring of QSLOT planes per velocity
// component, which lets the TMA copies run QSLOT - 3 planes ahead of the computation
constexpr int QX = TX + 4, QY = TY + 2, QPL = 384;
template <typename T>
struct NuRing {
  static constexpr int QSLOT = sizeof(T) == 4 ? 8 : 4;  // 36 KB (FP32) / 36 KB (FP64) of planes
  static constexpr int AHEAD = QSLOT - 3;
};

// --------------------------------------------------------------------------------------
// eddy viscosity nu_t on cells -1..n of every axis (core.py:400-482, 498-504), written to
// nu[k + 1][j + 1][i + 1] of an (nz+2, ny+2, nx+2) array, plus its maximum
// --------------------------------------------------------------------------------------

template <typename T>
struct NuSmem {
  alignas(128) T vel[3][NuRing<T>::QSLOT][QPL];
  uint64_t bar[NuRing<T>::QSLOT];
};

template <typename T, int MODEL>
__global__ void __launch_bounds__(TX *TY) nu_kernel(const __grid_constant__ NuParams<T> P) {
  aero::pdl_wait();
  __shared__ NuSmem<T> S;
  constexpr int QSLOT = NuRing<T>::QSLOT, AHEAD = NuRing<T>::AHEAD;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;  // cells of the tile: (j0-1+ty, i0-1+tx)
  const int qb = blockIdx.z * P.zc, qe = min(qb + P.zc, P.nz + 2);
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  const T inv = P.inv_h;
  // tile entry (ly, lx) <-> x index i0 - 4 + lx (face for u, cell for v / w), y index j0 - 2 + ly
  const bool interior_xy = i0 - 2 >= 0 && i0 + TX <= nx && j0 - 2 >= 0 && j0 + TY <= ny;
  const uint32_t bytes = 3u * QX * QY * sizeof(T) + (uint32_t)P.wait_extra_tx;
  const int limit = P.wait_limit > 0 ? P.wait_limit : (1 << 24);
  auto SL = [&](int kp) { return (kp - qb + 2) & (QSLOT - 1); };
  auto issue = [&](int kp) {
    const int s = SL(kp);
    fence_proxy_async();
    mbar_arrive_expect_tx(&S.bar[s], bytes);
    tma_load_3d(S.vel[0][s], &P.map_u, i0 - 4, j0 - 2, kp, &S.bar[s]);
    tma_load_3d(S.vel[1][s], &P.map_v, i0 - 4, j0 - 2, kp, &S.bar[s]);
    tma_load_3d(S.vel[2][s], &P.map_w, i0 - 4, j0 - 2, kp, &S.bar[s]);
  };
  // entries outside an array get the ghost rule's value (all entries on the slow path)
  auto fill = [&](int kp, bool all) {
    const int s = SL(kp);
    if (!all && interior_xy && kp >= 0 && kp < nz) return;
    for (int e = tid; e < QX * QY; e += TX * TY) {
      const int ly = e / QX, lx = e - ly * QX;
      if (lx < 2) continue;
      const int gj = j0 - 2 + ly, gi = i0 - 4 + lx;
      if (all || gi < 0 || gi > nx || gj < 0 || gj >= ny || kp < 0 || kp >= nz)
        S.vel[0][s][e] = padded<T>(P.up, P.ru, kp, gj, gi);
      if (all || gi < 0 || gi >= nx || gj < 0 || gj > ny || kp < 0 || kp >= nz)
        S.vel[1][s][e] = padded<T>(P.vp, P.rv, kp, gj, gi);
      if (all || gi < 0 || gi >= nx || gj < 0 || gj >= ny || kp < 0 || kp > nz)
        S.vel[2][s][e] = padded<T>(P.wp, P.rw, kp, gj, gi);
    }
  };
  auto await_plane = [&](int kp) -> bool {
    const int m = kp - qb + 2;
    return mbar_wait_bounded(&S.bar[SL(kp)], (uint32_t)((m / QSLOT) & 1), P.status, limit);
  };
  // after a wait ran out (the CTA agrees on that at its next barrier): let the copies it issued,
  // planes up to `last`, land (bounded again) and return without writing further cells
  auto drain = [&](int last) {
    if (tid == 0)
      for (int kp = max(qb - 2, last - QSLOT + 1); kp <= last; ++kp)
        mbar_wait_bounded(&S.bar[SL(kp)], (uint32_t)(((kp - qb + 2) / QSLOT) & 1), nullptr, limit);
  };
  if (tid == 0) {
    for (int q = 0; q < QSLOT; ++q) mbar_init(&S.bar[q], 1);
    mbar_fence_init();
  }
  __syncthreads();
  // nu plane q holds cells k = q - 1, which need velocity planes q - 2 .. q; the last plane
  // any iteration needs is qe - 1.  Iteration q issues plane q + AHEAD, so the ring holds
  // planes q - 2 .. q + AHEAD (QSLOT of them) and the slot it refills (plane q - 3) was last
  // read in iteration q - 1, which ended with a barrier.
  bool ok = true;
  if (P.use_tma) {
    if (tid == 0)
      for (int kp = qb - 2; kp <= min(qb + AHEAD - 1, qe - 1); ++kp) issue(kp);
    for (int kp = qb - 2; kp <= qb && ok; ++kp) {
      ok = await_plane(kp);
      if (ok) fill(kp, false);
    }
  } else {
    for (int kp = qb - 2; kp <= qb; ++kp) fill(kp, true);
  }
  if (__syncthreads_or(!ok)) {
    drain(min(qb + AHEAD - 1, qe - 1));
    return;
  }
#define V3(c, dz, yy, xx) S.vel[c][SL(kn + (dz))][(yy) * QX + (xx)]
  T mx = T(0);
  for (int q = qb; q < qe; ++q) {
    const bool pre = q + 1 < qe;
    if (P.use_tma && tid == 0 && q + AHEAD <= qe - 1) issue(q + AHEAD);
    const int kn = q - 1;
    const int cj = j0 - 1 + ty, ci = i0 - 1 + tx;  // this thread's cell
    if (cj <= ny && ci <= nx) {
      const int y = ty + 1, x = tx + 3;
      const T qq = T(0.25);
      T g[3][3];
      g[0][0] = (V3(0, 0, y, x + 1) - V3(0, 0, y, x)) * inv;
      g[1][1] = (V3(1, 0, y + 1, x) - V3(1, 0, y, x)) * inv;
      g[0][1] = ((((V3(0, 0, y, x) - V3(0, 0, y - 1, x)) * inv + (V3(0, 0, y + 1, x) - V3(0, 0, y, x)) * inv) +
                  (V3(0, 0, y, x + 1) - V3(0, 0, y - 1, x + 1)) * inv) +
                 (V3(0, 0, y + 1, x + 1) - V3(0, 0, y, x + 1)) * inv) *
                qq;
      g[0][2] = ((((V3(0, 0, y, x) - V3(0, -1, y, x)) * inv + (V3(0, 1, y, x) - V3(0, 0, y, x)) * inv) +
                  (V3(0, 0, y, x + 1) - V3(0, -1, y, x + 1)) * inv) +
                 (V3(0, 1, y, x + 1) - V3(0, 0, y, x + 1)) * inv) *
                qq;
      g[1][0] = ((((V3(1, 0, y, x) - V3(1, 0, y, x - 1)) * inv + (V3(1, 0, y + 1, x) - V3(1, 0, y + 1, x - 1)) * inv) +
                  (V3(1, 0, y, x + 1) - V3(1, 0, y, x)) * inv) +
                 (V3(1, 0, y + 1, x + 1) - V3(1, 0, y + 1, x)) * inv) *
                qq;
      g[1][2] = ((((V3(1, 0, y, x) - V3(1, -1, y, x)) * inv + (V3(1, 1, y, x) - V3(1, 0, y, x)) * inv) +
                  (V3(1, 0, y + 1, x) - V3(1, -1, y + 1, x)) * inv) +
                 (V3(1, 1, y + 1, x) - V3(1, 0, y + 1, x)) * inv) *
                qq;
      g[2][0] = ((((V3(2, 0, y, x) - V3(2, 0, y, x - 1)) * inv + (V3(2, 1, y, x) - V3(2, 1, y, x - 1)) * inv) +
                  (V3(2, 0, y, x + 1) - V3(2, 0, y, x)) * inv) +
                 (V3(2, 1, y, x + 1) - V3(2, 1, y, x)) * inv) *
                qq;
      g[2][1] = ((((V3(2, 0, y, x) - V3(2, 0, y - 1, x)) * inv + (V3(2, 1, y, x) - V3(2, 1, y - 1, x)) * inv) +
                  (V3(2, 0, y + 1, x) - V3(2, 0, y, x)) * inv) +
                 (V3(2, 1, y + 1, x) - V3(2, 1, y, x)) * inv) *
                qq;
      g[2][2] = -(g[0][0] + g[1][1]);
      T nu = eddy_viscosity<T>(g, MODEL, P.cd2);
      T fac = T(1);
      if (P.has_win && kn >= P.win[0] && kn < P.win[1] && cj >= P.win[2] && cj < P.win[3] && ci >= P.win[4] &&
          ci < P.win[5]) {
        const T chi = P.chi_c[((size_t)(kn - P.win[0]) * P.wny + (cj - P.win[2])) * P.wnx + (ci - P.win[4])];
        fac = T(1) - chi;
        nu = nu * fac;
      }
      const size_t at = ((size_t)q * (ny + 2) + (cj + 1)) * P.nu_pitch + (ci + 1);
      P.nu[at] = nu;
      if (P.grad) {  // the learned closure's inputs
        const T gg[9] = {g[0][0], g[0][1], g[0][2], g[1][0], g[1][1], g[1][2], g[2][0], g[2][1], fac};
#pragma unroll
        for (int c = 0; c < 9; ++c) P.grad[c * P.grad_plane + at] = (float)gg[c];
      }
      mx = (nu > mx || nu != nu) ? nu : mx;
    }
    if (pre) {
      if (P.use_tma) {
        ok = await_plane(q + 1);
        if (ok) fill(q + 1, false);
      } else {
        fill(q + 1, true);
      }
    }
    if (__syncthreads_or(!ok)) {
      drain(min(q + AHEAD, qe - 1));
      return;
    }
  }
#undef V3
  if (P.nut_max) block_max_atomic<T>(mx, P.nut_max);
}

// --------------------------------------------------------------------------------------
// the stage kernel
// --------------------------------------------------------------------------------------

template <typename T>
struct StageSmem {
  alignas(128) T vel[3][NSLOT][PPL];
  alignas(128) T th[NSLOT][PPL];
  alignas(128) T nu[NSLOT][NUPL];
  double acc[8][AERO_MAX_BODIES * 10];  // per-warp force / heat sums
  uint64_t bar[NSLOT];
};

// UPWIND, LES and THERMAL are the plan's advection scheme, LES switch and heat switch, fixed at
// compile time so that each configuration's body is straight-line code; PLACED adds the placed
// physics that acts inside a stage (fans, jets and vents, painted solids, volumetric heaters),
// which the other instantiations leave out entirely.
template <typename T, bool UPWIND, bool LES, bool THERMAL, bool PLACED>
__global__ void __launch_bounds__(TX *TY, sizeof(T) == 4 ? 3 : 2) stage_kernel(const __grid_constant__ StageParams<T> P) {
  aero::pdl_wait();
  extern __shared__ __align__(128) unsigned char smem_raw[];
  StageSmem<T> &S = *reinterpret_cast<StageSmem<T> *>(smem_raw);
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int lane = tid & 31, warp = tid >> 5;
  const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
  const int kb = blockIdx.z * P.zc, ke = min(kb + P.zc, P.nz);
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  const int i = i0 + tx, j = j0 + ty;
  constexpr bool les = LES, upwind = UPWIND, thermal = THERMAL;
  const T inv = P.inv_h;
  const int nq = P.nq;

  for (int q = tid; q < 8 * AERO_MAX_BODIES * 10; q += TX * TY) (&S.acc[0][0])[q] = 0.0;

  // ---- plane slots: plane kp of every field (and nu cell plane kp - 1) lives in slot SL(kp)
  // tile entry (ly, lx) <-> x index i0 - 4 + lx, y index j0 - 2 + ly
  const bool interior_xy = i0 - 2 >= 0 && i0 + TX + 2 <= nx && j0 - 2 >= 0 && j0 + TY + 2 <= ny;
  const uint32_t bytes = (uint32_t)sizeof(T) * ((3u + (thermal ? 1u : 0u)) * PPL + (les ? (uint32_t)(NUX * NUY) : 0u)) +
                         (uint32_t)P.wait_extra_tx;
  const int limit = P.wait_limit > 0 ? P.wait_limit : (1 << 24);
  auto SL = [&](int kp) { return (kp - kb + 2) % NSLOT; };
  auto issue = [&](int kp) {
    const int s = SL(kp);
    fence_proxy_async();
    mbar_arrive_expect_tx(&S.bar[s], bytes);
    tma_load_3d(S.vel[0][s], &P.map_u, i0 - 4, j0 - 2, kp, &S.bar[s]);
    tma_load_3d(S.vel[1][s], &P.map_v, i0 - 4, j0 - 2, kp, &S.bar[s]);
    tma_load_3d(S.vel[2][s], &P.map_w, i0 - 4, j0 - 2, kp, &S.bar[s]);
    if (thermal) tma_load_3d(S.th[s], &P.map_th, i0 - 4, j0 - 2, kp, &S.bar[s]);
    if (les) tma_load_3d(S.nu[s], &P.map_nu, i0, j0, kp, &S.bar[s]);
  };
  // entries outside an array get the ghost rule's value (every entry on the slow path)
  auto fill = [&](int kp, bool all) {
    const int s = SL(kp);
    if (!all && interior_xy && kp >= 0 && kp < nz) return;
    for (int e = tid; e < PPL; e += TX * TY) {
      const int ly = e / PX, lx = e - ly * PX;
      if (lx < 2) continue;
      const int gj = j0 - 2 + ly, gi = i0 - 4 + lx;
      const bool oc = gi < 0 || gi >= nx || gj < 0 || gj >= ny || kp < 0 || kp >= nz;
      if (all || oc || gi == nx) S.vel[0][s][e] = padded<T>(P.up, P.ru, kp, gj, gi);
      if (all || oc || gj == ny) S.vel[1][s][e] = padded<T>(P.vp, P.rv, kp, gj, gi);
      if (all || oc || kp == nz) S.vel[2][s][e] = padded<T>(P.wp, P.rw, kp, gj, gi);
      if (thermal && (all || oc)) S.th[s][e] = theta_padded<T>(P.thp, nz, ny, nx, P.sides, P.h, kp, gj, gi);
    }
    if (all && les) {
      const int q = min(max(kp, 0), nz + 1);
      for (int e = tid; e < NUX * NUY; e += TX * TY) {
        const int ly = e / NUX, lx = e - ly * NUX;
        const int r = min(j0 + ly, ny + 1), c = min(i0 + lx, nx + 1);
        S.nu[s][e] = __ldg(P.nu + ((size_t)q * (ny + 2) + r) * P.nu_pitch + c);
      }
    }
  };
  auto await_plane = [&](int kp) -> bool {
    const int m = kp - kb + 2;
    return mbar_wait_bounded(&S.bar[SL(kp)], (uint32_t)((m / NSLOT) & 1), P.status, limit);
  };
  // after a wait ran out: let the copies issued so far (planes up to `last`) land, then return
  // with the rest of the chunk unwritten (the status word tells the host)
  auto drain = [&](int last) {
    if (tid == 0)
      for (int kp = max(kb - 2, last - NSLOT + 1); kp <= last; ++kp)
        mbar_wait_bounded(&S.bar[SL(kp)], (uint32_t)(((kp - kb + 2) / NSLOT) & 1), nullptr, limit);
  };
#define VEL(c, dz, yy, xx) S.vel[c][SL(kc + (dz))][(yy) * PX + (xx)]
#define TH(dz, yy, xx) S.th[SL(kc + (dz))][(yy) * PX + (xx)]
#define NU(dz, yy, xx) S.nu[SL(kc + (dz) + 1)][(yy) * NUX + (xx)]

  const int y = ty + 2, x = tx + 4;      // this thread's cell / faces in the plane tile
  const int ny2 = ty + 1, nx2 = tx + 1;  // ... in the eddy-viscosity tile
  const bool valid = (i < nx) && (j < ny);
  const int wk0 = P.win[0], wk1 = P.win[1], wj0 = P.win[2], wj1 = P.win[3], wi0 = P.win[4], wi1 = P.win[5];
  const int wzn = wk1 - wk0, wyn = wj1 - wj0, wxn = wi1 - wi0;
  // which of the window's face / cell columns this thread's (j, i) lies in, evaluated once:
  // bit 0 u faces (i), 1 v faces (j), 2 cells and w faces, 3 u face i + 1, 4 v face j + 1
  int wcol = 0;
  if (P.has_win && valid) {
    const bool jc = j >= wj0 && j < wj1, ic = i >= wi0 && i < wi1;
    wcol = ((jc && i >= wi0 && i <= wi1) ? 1 : 0) | ((ic && j >= wj0 && j <= wj1) ? 2 : 0) | ((jc && ic) ? 4 : 0) |
           ((jc && i + 1 >= wi0 && i + 1 <= wi1) ? 8 : 0) | ((ic && j + 1 >= wj0 && j + 1 <= wj1) ? 16 : 0);
  }
  const bool warp_win = __any_sync(0xffffffffu, wcol != 0);  // warp-uniform
  const T two = T(2), qq = T(0.25);
  const T kh = P.kh;
  auto kface = [&](T n1, T n2, bool boundary) -> T {
    if (!les || boundary) return kh;
    return kh + P.kprt * (n1 + n2);
  };

  // ---- the z interface above plane kc (between kc and kc + 1), evaluated once and carried
  T zu = T(0), zv = T(0), zw = T(0), z13 = T(0), z23 = T(0), z33 = T(0), zth = T(0);
  auto z_interface = [&](const int kc) {
    // u: z flux on the x-z edge (kc+1, i); v: on the y-z edge (kc+1, j); w: at the cell centre kc
    zu = face_flux<T>(VEL(2, 1, y, x - 1) + VEL(2, 1, y, x), VEL(0, -1, y, x), VEL(0, 0, y, x), VEL(0, 1, y, x),
                      VEL(0, 2, y, x), upwind);
    zv = face_flux<T>(VEL(2, 1, y - 1, x) + VEL(2, 1, y, x), VEL(1, -1, y, x), VEL(1, 0, y, x), VEL(1, 1, y, x),
                      VEL(1, 2, y, x), upwind);
    zw = face_flux<T>(VEL(2, 0, y, x) + VEL(2, 1, y, x), VEL(2, -1, y, x), VEL(2, 0, y, x), VEL(2, 1, y, x),
                      VEL(2, 2, y, x), upwind);
    if (les) {  // tau_13, tau_23 on those edges; tau_33 at the cell centre kc
      const T n13 = (((NU(0, ny2, nx2 - 1) + NU(1, ny2, nx2 - 1)) + NU(0, ny2, nx2)) + NU(1, ny2, nx2)) * qq;
      const T s13 = (VEL(0, 1, y, x) - VEL(0, 0, y, x)) * inv + (VEL(2, 1, y, x) - VEL(2, 1, y, x - 1)) * inv;
      z13 = n13 * s13;
      const T n23 = (((NU(0, ny2 - 1, nx2) + NU(1, ny2 - 1, nx2)) + NU(0, ny2, nx2)) + NU(1, ny2, nx2)) * qq;
      const T s23 = (VEL(1, 1, y, x) - VEL(1, 0, y, x)) * inv + (VEL(2, 1, y, x) - VEL(2, 1, y - 1, x)) * inv;
      z23 = n23 * s23;
      z33 = two * NU(0, ny2, nx2) * ((VEL(2, 1, y, x) - VEL(2, 0, y, x)) * inv);
    }
    if (thermal) {  // theta flux through the z face kc + 1 (between cells kc and kc + 1)
      const T kz = kface(NU(0, ny2, nx2), NU(1, ny2, nx2), !P.pz && (kc + 1 == nz || kc + 1 == 0));
      const T cb = TH(0, y, x), cc = TH(1, y, x);
      T f = muscl_flux<T>(TH(-1, y, x), cb, cc, TH(2, y, x), VEL(2, 1, y, x)) - kz * (cc - cb);
      if ((wcol & 4) && P.has_adia && kc + 1 >= wk0 && kc + 1 <= wk1)
        f += kz * P.adia_w[((size_t)(kc + 1 - wk0) * wyn + (j - wj0)) * wxn + (i - wi0)] * (cc - cb);
      zth = f;
    }
  };

  // ---- prologue: planes kb-2 .. kb+2 (nu cell planes kb-3 .. kb+1); the interface below kb
  if (tid == 0) {
    for (int q = 0; q < NSLOT; ++q) mbar_init(&S.bar[q], 1);
    mbar_fence_init();
  }
  __syncthreads();
  bool ok = true;
  if (P.use_tma) {
    if (tid == 0)
      for (int kp = kb - 2; kp <= kb + 2; ++kp) issue(kp);
    for (int kp = kb - 2; kp <= kb + 2 && ok; ++kp) {
      ok = await_plane(kp);
      if (ok) fill(kp, false);
    }
  } else {
    for (int kp = kb - 2; kp <= kb + 2; ++kp) fill(kp, true);
  }
  if (__syncthreads_or(!ok)) {
    drain(kb + 2);
    return;
  }
  {
    const int kc = kb - 1;
    if (valid) z_interface(kc);
  }

  for (int k = kb; k < ke; ++k) {
    // stream plane k + 3 into the slot plane k - 3 used while this plane is computed
    const bool pre = k + 3 <= ke + 1;
    if (P.use_tma && pre && tid == 0) issue(k + 3);
    const int kc = k;
    const T bdt = P.bdt_scale * *P.dt;
    const T a = P.a;

    double cu = 0.0, cv = 0.0, cw = 0.0, ct = 0.0;  // weighted window increments
    int fu_in = 0, fv_in = 0, fw_in = 0, ft_in = 0;
    size_t wu = 0, wv = 0, ww = 0, wt = 0;

    if (valid) {
      // step-start values of this cell's faces for the RK blend, requested before the
      // tendencies so that their DRAM latency hides behind the arithmetic
      const size_t iu = ((size_t)k * ny + j) * (nx + 1) + i;
      const size_t iv = ((size_t)k * (ny + 1) + j) * nx + i;
      const size_t iw = ((size_t)k * ny + j) * nx + i;
      const bool blend = a != T(0);
      const T u0v = blend ? __ldg(P.u0 + iu) : T(0);
      const T v0v = blend ? __ldg(P.v0 + iv) : T(0);
      const T w0v = blend ? __ldg(P.w0 + iw) : T(0);
      const T t0v = (blend && thermal) ? __ldg(P.th0 + iw) : T(0);
      // the interface below this plane, carried from the previous plane
      const T zu_l = zu, zv_l = zv, zw_l = zw, z13_l = z13, z23_l = z23, z33_l = z33, zth_l = zth;
      z_interface(kc);
      const T kadv = P.kadv, nuh2 = P.nu_h2;
      // ================= momentum tendencies (core.py:353-397, 485-524) ===============
      T lu, lv, lw;
      {  // ---- u face (k, j, i)
        T au = face_flux<T>(VEL(0, 0, y, x - 1) + VEL(0, 0, y, x), VEL(0, 0, y, x - 2), VEL(0, 0, y, x - 1),
                            VEL(0, 0, y, x), VEL(0, 0, y, x + 1), upwind) -
               face_flux<T>(VEL(0, 0, y, x) + VEL(0, 0, y, x + 1), VEL(0, 0, y, x - 1), VEL(0, 0, y, x),
                            VEL(0, 0, y, x + 1), VEL(0, 0, y, x + 2), upwind);
        const T gyl = face_flux<T>(VEL(1, 0, y, x - 1) + VEL(1, 0, y, x), VEL(0, 0, y - 2, x), VEL(0, 0, y - 1, x),
                                   VEL(0, 0, y, x), VEL(0, 0, y + 1, x), upwind);
        const T gyr = face_flux<T>(VEL(1, 0, y + 1, x - 1) + VEL(1, 0, y + 1, x), VEL(0, 0, y - 1, x), VEL(0, 0, y, x),
                                   VEL(0, 0, y + 1, x), VEL(0, 0, y + 2, x), upwind);
        au = au + (gyl - gyr);
        au = (au + (zu_l - zu)) * kadv;
        const T lap = ((VEL(0, 0, y, x + 1) + VEL(0, 0, y, x - 1)) + (VEL(0, 0, y + 1, x) + VEL(0, 0, y - 1, x)) +
                       (VEL(0, 1, y, x) + VEL(0, -1, y, x))) -
                      T(6) * VEL(0, 0, y, x);
        lu = au + nuh2 * lap;
        if (les) {
          const T t11r = two * NU(0, ny2, nx2) * ((VEL(0, 0, y, x + 1) - VEL(0, 0, y, x)) * inv);
          const T t11l = two * NU(0, ny2, nx2 - 1) * ((VEL(0, 0, y, x) - VEL(0, 0, y, x - 1)) * inv);
          const T n12l = (((NU(0, ny2 - 1, nx2 - 1) + NU(0, ny2, nx2 - 1)) + NU(0, ny2 - 1, nx2)) + NU(0, ny2, nx2)) * qq;
          const T s12l = (VEL(0, 0, y, x) - VEL(0, 0, y - 1, x)) * inv + (VEL(1, 0, y, x) - VEL(1, 0, y, x - 1)) * inv;
          const T n12r = (((NU(0, ny2, nx2 - 1) + NU(0, ny2 + 1, nx2 - 1)) + NU(0, ny2, nx2)) + NU(0, ny2 + 1, nx2)) * qq;
          const T s12r =
              (VEL(0, 0, y + 1, x) - VEL(0, 0, y, x)) * inv + (VEL(1, 0, y + 1, x) - VEL(1, 0, y + 1, x - 1)) * inv;
          lu = lu + (((((t11r - t11l) + n12r * s12r) - n12l * s12l) + z13) - z13_l) * inv;
        }
      }
      {  // ---- v face (k, j, i)
        T av = face_flux<T>(VEL(0, 0, y - 1, x) + VEL(0, 0, y, x), VEL(1, 0, y, x - 2), VEL(1, 0, y, x - 1),
                            VEL(1, 0, y, x), VEL(1, 0, y, x + 1), upwind) -
               face_flux<T>(VEL(0, 0, y - 1, x + 1) + VEL(0, 0, y, x + 1), VEL(1, 0, y, x - 1), VEL(1, 0, y, x),
                            VEL(1, 0, y, x + 1), VEL(1, 0, y, x + 2), upwind);
        const T gyl = face_flux<T>(VEL(1, 0, y - 1, x) + VEL(1, 0, y, x), VEL(1, 0, y - 2, x), VEL(1, 0, y - 1, x),
                                   VEL(1, 0, y, x), VEL(1, 0, y + 1, x), upwind);
        const T gyr = face_flux<T>(VEL(1, 0, y, x) + VEL(1, 0, y + 1, x), VEL(1, 0, y - 1, x), VEL(1, 0, y, x),
                                   VEL(1, 0, y + 1, x), VEL(1, 0, y + 2, x), upwind);
        av = av + (gyl - gyr);
        av = (av + (zv_l - zv)) * kadv;
        const T lap = ((VEL(1, 0, y, x + 1) + VEL(1, 0, y, x - 1)) + (VEL(1, 0, y + 1, x) + VEL(1, 0, y - 1, x)) +
                       (VEL(1, 1, y, x) + VEL(1, -1, y, x))) -
                      T(6) * VEL(1, 0, y, x);
        lv = av + nuh2 * lap;
        if (les) {
          const T n12l = (((NU(0, ny2 - 1, nx2 - 1) + NU(0, ny2, nx2 - 1)) + NU(0, ny2 - 1, nx2)) + NU(0, ny2, nx2)) * qq;
          const T s12l = (VEL(0, 0, y, x) - VEL(0, 0, y - 1, x)) * inv + (VEL(1, 0, y, x) - VEL(1, 0, y, x - 1)) * inv;
          const T n12r = (((NU(0, ny2 - 1, nx2) + NU(0, ny2, nx2)) + NU(0, ny2 - 1, nx2 + 1)) + NU(0, ny2, nx2 + 1)) * qq;
          const T s12r =
              (VEL(0, 0, y, x + 1) - VEL(0, 0, y - 1, x + 1)) * inv + (VEL(1, 0, y, x + 1) - VEL(1, 0, y, x)) * inv;
          const T t22r = two * NU(0, ny2, nx2) * ((VEL(1, 0, y + 1, x) - VEL(1, 0, y, x)) * inv);
          const T t22l = two * NU(0, ny2 - 1, nx2) * ((VEL(1, 0, y, x) - VEL(1, 0, y - 1, x)) * inv);
          lv = lv + (((((n12r * s12r - n12l * s12l) + t22r) - t22l) + z23) - z23_l) * inv;
        }
      }
      {  // ---- w face (k, j, i)
        T aw = face_flux<T>(VEL(0, -1, y, x) + VEL(0, 0, y, x), VEL(2, 0, y, x - 2), VEL(2, 0, y, x - 1),
                            VEL(2, 0, y, x), VEL(2, 0, y, x + 1), upwind) -
               face_flux<T>(VEL(0, -1, y, x + 1) + VEL(0, 0, y, x + 1), VEL(2, 0, y, x - 1), VEL(2, 0, y, x),
                            VEL(2, 0, y, x + 1), VEL(2, 0, y, x + 2), upwind);
        const T gyl = face_flux<T>(VEL(1, -1, y, x) + VEL(1, 0, y, x), VEL(2, 0, y - 2, x), VEL(2, 0, y - 1, x),
                                   VEL(2, 0, y, x), VEL(2, 0, y + 1, x), upwind);
        const T gyr = face_flux<T>(VEL(1, -1, y + 1, x) + VEL(1, 0, y + 1, x), VEL(2, 0, y - 1, x), VEL(2, 0, y, x),
                                   VEL(2, 0, y + 1, x), VEL(2, 0, y + 2, x), upwind);
        aw = aw + (gyl - gyr);
        aw = (aw + (zw_l - zw)) * kadv;
        const T lap = ((VEL(2, 0, y, x + 1) + VEL(2, 0, y, x - 1)) + (VEL(2, 0, y + 1, x) + VEL(2, 0, y - 1, x)) +
                       (VEL(2, 1, y, x) + VEL(2, -1, y, x))) -
                      T(6) * VEL(2, 0, y, x);
        lw = aw + nuh2 * lap;
        if (les) {
          // tau_13 on the x-z edges (k, i) and (k, i+1), tau_23 on the y-z edges (k, j) and (k, j+1):
          // the (k, i) and (k, j) ones are this thread's carried u / v interface values
          const T n13r = (((NU(-1, ny2, nx2) + NU(0, ny2, nx2)) + NU(-1, ny2, nx2 + 1)) + NU(0, ny2, nx2 + 1)) * qq;
          const T s13r =
              (VEL(0, 0, y, x + 1) - VEL(0, -1, y, x + 1)) * inv + (VEL(2, 0, y, x + 1) - VEL(2, 0, y, x)) * inv;
          const T n23r = (((NU(-1, ny2, nx2) + NU(0, ny2, nx2)) + NU(-1, ny2 + 1, nx2)) + NU(0, ny2 + 1, nx2)) * qq;
          const T s23r =
              (VEL(1, 0, y + 1, x) - VEL(1, -1, y + 1, x)) * inv + (VEL(2, 0, y + 1, x) - VEL(2, 0, y, x)) * inv;
          lw = lw + (((((n13r * s13r - z13_l) + n23r * s23r) - z23_l) + z33) - z33_l) * inv;
        }
      }
      if (PLACED && P.forcing) {   // + the uniform body force, after the subgrid stress
        lu = lu + P.force[0];
        lv = lv + P.force[1];
        lw = lw + P.force[2];
      }

      // ================= actuator discs (physics.py:944-952): + f T (+ s amp), fan by fan
      for (int q = 0; q < (PLACED ? P.nfan : 0); ++q) {
        const FanForce<T> &F = P.fan[q];
        // this cell's u / v / w faces inside the fan's window (faces i..i1 / j..j1 / k..k1)
        const bool jc = j >= F.win[2] && j < F.win[3], ic = i >= F.win[4] && i < F.win[5];
        const bool kin = k >= F.win[0] && k < F.win[1];
        const bool in_u = kin && jc && i >= F.win[4] && i <= F.win[5];
        const bool in_v = kin && ic && j >= F.win[2] && j <= F.win[3];
        const bool in_w = jc && ic && k >= F.win[0] && k <= F.win[1];
        if (in_u || in_v || in_w) {
          const int fwy = F.win[3] - F.win[2], fwx = F.win[5] - F.win[4];
          const T thrust = *F.thrust, amp = P.fan_swirl ? *F.swirl_amp : T(0);
          if (in_u) {
            const size_t e = ((size_t)(k - F.win[0]) * fwy + (j - F.win[2])) * (fwx + 1) + (i - F.win[4]);
            lu = lu + F.f[0][e] * thrust;
            if (P.fan_swirl) lu = lu + F.s[0][e] * amp;
          }
          if (in_v) {
            const size_t e = ((size_t)(k - F.win[0]) * (fwy + 1) + (j - F.win[2])) * fwx + (i - F.win[4]);
            lv = lv + F.f[1][e] * thrust;
            if (P.fan_swirl) lv = lv + F.s[1][e] * amp;
          }
          if (in_w) {
            const size_t e = ((size_t)(k - F.win[0]) * fwy + (j - F.win[2])) * fwx + (i - F.win[4]);
            lw = lw + F.f[2][e] * thrust;
            if (P.fan_swirl) lw = lw + F.s[2][e] * amp;
          }
        }
      }

      // ================= jets and vents (physics.py:1033-1041): + f, or + f u for a vent =====
      for (int q = 0; q < (PLACED ? P.nport : 0); ++q) {
        const PortSource<T> &Q = P.port[q];
        const bool jc = j >= Q.win[2] && j < Q.win[3], ic = i >= Q.win[4] && i < Q.win[5];
        const bool kin = k >= Q.win[0] && k < Q.win[1];  // (kc names the plane)
        const int fwy = Q.win[3] - Q.win[2], fwx = Q.win[5] - Q.win[4];
        if (kin && jc && i >= Q.win[4] && i <= Q.win[5]) {
          const T f = Q.f[0][((size_t)(k - Q.win[0]) * fwy + (j - Q.win[2])) * (fwx + 1) + (i - Q.win[4])];
          lu = lu + (Q.vent ? f * VEL(0, 0, y, x) : f);
        }
        if (kin && ic && j >= Q.win[2] && j <= Q.win[3]) {
          const T f = Q.f[1][((size_t)(k - Q.win[0]) * (fwy + 1) + (j - Q.win[2])) * fwx + (i - Q.win[4])];
          lv = lv + (Q.vent ? f * VEL(1, 0, y, x) : f);
        }
        if (jc && ic && k >= Q.win[0] && k <= Q.win[1]) {
          const T f = Q.f[2][((size_t)(k - Q.win[0]) * fwy + (j - Q.win[2])) * fwx + (i - Q.win[4])];
          lw = lw + (Q.vent ? f * VEL(2, 0, y, x) : f);
        }
      }

      // ================= boundary tendencies and RK update (core.py:527-543, 819-827) =
      const T up0 = VEL(0, 0, y, x), vp0 = VEL(1, 0, y, x), wp0 = VEL(2, 0, y, x);
      T uh, vh, wh;
      if (a == T(0)) {
        uh = up0 + lu * bdt;
        vh = vp0 + lv * bdt;
        wh = wp0 + lw * bdt;
      } else {
        uh = lerp_t<T>(up0, u0v, a) + lu * bdt;
        vh = lerp_t<T>(vp0, v0v, a) + lv * bdt;
        wh = lerp_t<T>(wp0, w0v, a) + lw * bdt;
      }
      if (!P.px && i == 0) uh = P.closed ? T(0) : P.u_inlet[(size_t)k * ny + j];
      if (!P.py && j == 0) vh = T(0);
      if (!P.pz && k == 0) wh = T(0);

      // ================= window penalisation (core.py:615-634) =========================
      const T wg = P.wgt;
      if (wcol) {
        const T kpen = bdt / P.eta;
        if ((wcol & 1) && k >= wk0 && k < wk1) {
          wu = ((size_t)(k - wk0) * wyn + (j - wj0)) * (wxn + 1) + (i - wi0);
          const T un = (uh + kpen * P.a_u[wu]) / (T(1) + kpen * P.chi_u[wu]);
          cu = (double)((un - uh) * wg);
          uh = un;
          fu_in = 1;
        }
        if ((wcol & 2) && k >= wk0 && k < wk1) {
          wv = ((size_t)(k - wk0) * (wyn + 1) + (j - wj0)) * wxn + (i - wi0);
          const T vn = (vh + kpen * P.a_v[wv]) / (T(1) + kpen * P.chi_v[wv]);
          cv = (double)((vn - vh) * wg);
          vh = vn;
          fv_in = 1;
        }
        if ((wcol & 4) && k >= wk0 && k <= wk1) {
          ww = ((size_t)(k - wk0) * wyn + (j - wj0)) * wxn + (i - wi0);
          const T wn = (wh + kpen * P.a_w[ww]) / (T(1) + kpen * P.chi_w[ww]);
          cw = (double)((wn - wh) * wg);
          wh = wn;
          fw_in = 1;
        }
      }

      // ================= painted solids, after the bodies (physics.py:1132-1137) =========
      if (PLACED && P.paint_u) {
        const T kpen = bdt / P.eta;
        uh = uh / (T(1) + kpen * P.paint_u[iu]);
        vh = vh / (T(1) + kpen * P.paint_v[iv]);
        wh = wh / (T(1) + kpen * P.paint_w[iw]);
      }

      // ================= buoyancy after the penalisation (physics.py:744-790) =========
      if (thermal && P.ri != T(0)) {
        if (k > 0) {
          const T tf = T(0.5) * (TH(0, y, x) + TH(-1, y, x));
          wh = wh + tf * (bdt * P.ri);
        } else if (P.pz) {
          const T edge = (TH(0, y, x) + TH(-1, y, x)) * (T(0.5) * P.ri) * bdt;
          wh = wh + edge;
        }
        if (fw_in && P.vol_w) {
          // theta on the w-face from the two cells around it (clamped / wrapped at the ends)
          const T tl = (k == 0 && !P.pz) ? TH(0, y, x) : TH(-1, y, x);
          const T tw = T(0.5) * (TH(0, y, x) + tl);
          const T share = (tw * P.vol_w[ww]) * (bdt * (P.ri * wg));
          cw += (double)share;
        }
      }

      // ================= outputs ==========================================================
      P.uh[iu] = uh;
      P.vh[iv] = vh;
      P.wh[iw] = wh;
      if (i == nx - 1 && !P.px) {  // the outlet face (or the closed domain's wall)
        const size_t io = iu + 1;
        T uo;
        if (P.closed) {
          uo = T(0);
        } else {
          const T upo = VEL(0, 0, y, x + 1), upi = VEL(0, 0, y, x);
          const T lo = (upi - upo) * inv;
          uo = (a == T(0) ? upo : lerp_t<T>(upo, __ldg(P.u0 + io), a)) + lo * bdt;
          uo = uo + *P.outlet_corr;
          if (PLACED && P.paint_u) uo = uo / (T(1) + (bdt / P.eta) * P.paint_u[io]);
        }
        P.uh[io] = uo;
      }
      if (j == ny - 1 && !P.py) P.vh[iv + nx] = T(0);
      // the top w face is a boundary face (chi_w = vol_w = 0 there): zero normal velocity
      if (k == nz - 1 && !P.pz) P.wh[iw + (size_t)ny * nx] = T(0);

      // ================= theta stage (physics.py:647-708) ================================
      if (thermal) {
        const T c = TH(0, y, x);
        const T kxl = kface(NU(0, ny2, nx2 - 1), NU(0, ny2, nx2), !P.px && i == 0);
        const T kxr = kface(NU(0, ny2, nx2), NU(0, ny2, nx2 + 1), !P.px && i == nx - 1);
        T fxl = muscl_flux<T>(TH(0, y, x - 2), TH(0, y, x - 1), c, TH(0, y, x + 1), VEL(0, 0, y, x)) -
                kxl * (c - TH(0, y, x - 1));
        T fxr = muscl_flux<T>(TH(0, y, x - 1), c, TH(0, y, x + 1), TH(0, y, x + 2), VEL(0, 0, y, x + 1)) -
                kxr * (TH(0, y, x + 1) - c);
        const T kyl = kface(NU(0, ny2 - 1, nx2), NU(0, ny2, nx2), !P.py && j == 0);
        const T kyr = kface(NU(0, ny2, nx2), NU(0, ny2 + 1, nx2), !P.py && j == ny - 1);
        T fyl = muscl_flux<T>(TH(0, y - 2, x), TH(0, y - 1, x), c, TH(0, y + 1, x), VEL(1, 0, y, x)) -
                kyl * (c - TH(0, y - 1, x));
        T fyr = muscl_flux<T>(TH(0, y - 1, x), c, TH(0, y + 1, x), TH(0, y + 2, x), VEL(1, 0, y + 1, x)) -
                kyr * (TH(0, y + 1, x) - c);
        if ((wcol & 27) && P.has_adia && k >= wk0 && k < wk1) {  // adiabatic bodies block conduction (physics.py:666-675)
          {
            if (wcol & 1)
              fxl += kxl * P.adia_u[((size_t)(k - wk0) * wyn + (j - wj0)) * (wxn + 1) + (i - wi0)] * (c - TH(0, y, x - 1));
            if (wcol & 8)
              fxr += kxr * P.adia_u[((size_t)(k - wk0) * wyn + (j - wj0)) * (wxn + 1) + (i + 1 - wi0)] *
                     (TH(0, y, x + 1) - c);
          }
          {
            if (wcol & 2)
              fyl += kyl * P.adia_v[((size_t)(k - wk0) * (wyn + 1) + (j - wj0)) * wxn + (i - wi0)] * (c - TH(0, y - 1, x));
            if (wcol & 16)
              fyr += kyr * P.adia_v[((size_t)(k - wk0) * (wyn + 1) + (j + 1 - wj0)) * wxn + (i - wi0)] *
                     (TH(0, y + 1, x) - c);
          }
        }
        const T D = ((fxr - fxl) + (fyr - fyl) + (zth - zth_l)) * inv;
        const size_t ic = ((size_t)k * ny + j) * nx + i;
        T ch = (a == T(0) ? c : lerp_t<T>(c, t0v, a)) - bdt * D;
        const bool in_body = (wcol & 4) && k >= wk0 && k < wk1;
        // volumetric heaters, then the heat-flux skins (physics.py:692-697)
        for (int q = 0; q < (PLACED ? P.nheat : 0); ++q) {
          const auto &Hq = P.heat[q];
          if (k >= Hq.win[0] && k < Hq.win[1] && j >= Hq.win[2] && j < Hq.win[3] && i >= Hq.win[4] && i < Hq.win[5])
            ch = ch + (bdt * P.kappa) * Hq.q[((size_t)(k - Hq.win[0]) * (Hq.win[3] - Hq.win[2]) + (j - Hq.win[2])) *
                                                 (Hq.win[5] - Hq.win[4]) +
                                             (i - Hq.win[4])];
        }
        if (in_body) {
          wt = ((size_t)(k - wk0) * wyn + (j - wj0)) * wxn + (i - wi0);
          if (P.skin) ch = ch + (bdt * P.kappa) * P.skin[wt];
        }
        if (PLACED) {
          // jets and vents (physics.py:1049-1072): a vent takes the local value out with its
          // fluid, a jet brings its own; then an unbalanced closed box's uniform leak
          for (int q = 0; q < P.nport; ++q) {
            const PortSource<T> &Q = P.port[q];
            if (k >= Q.win[0] && k < Q.win[1] && j >= Q.win[2] && j < Q.win[3] && i >= Q.win[4] && i < Q.win[5]) {
              const T m = Q.m[((size_t)(k - Q.win[0]) * (Q.win[3] - Q.win[2]) + (j - Q.win[2])) *
                                  (Q.win[5] - Q.win[4]) +
                              (i - Q.win[4])];
              if (Q.vent)
                ch = ch + (bdt * m) * c;
              else if (Q.theta != T(0))
                ch = ch + (bdt * Q.theta) * m;
            }
          }
          if (P.port_leak != T(0)) ch = ch - c * (bdt * P.port_leak);
        }
        if (in_body) {
          if (P.chi_t) {
            const T kt = bdt / P.eta_t;
            const T nw = (ch + kt * P.a_t[wt]) / (T(1) + kt * P.chi_t[wt]);
            ct = (double)((nw - ch) * wg);
            ch = nw;
            ft_in = 1;
          }
        }
        P.thh[ic] = ch;
      }
    }

    // ================= force / heat sums: per-warp, fixed order (deterministic) ===========
    if (warp_win) {
      const unsigned any = __ballot_sync(0xffffffffu, fu_in | fv_in | fw_in | ft_in);
      if (any) {
        const size_t wsz_u = (size_t)wzn * wyn * (wxn + 1);
        const size_t wsz_v = (size_t)wzn * (wyn + 1) * wxn;
        const size_t wsz_w = (size_t)(wzn + 1) * wyn * wxn;
        const size_t wsz_c = (size_t)wzn * wyn * wxn;
        for (int b = 0; b < P.nbody; ++b) {
          for (int c3 = 0; c3 < 3; ++c3) {
            double xu = fu_in ? cu * (double)P.k_u[((size_t)b * 3 + c3) * wsz_u + wu] : 0.0;
            double xv = fv_in ? cv * (double)P.k_v[((size_t)b * 3 + c3) * wsz_v + wv] : 0.0;
            double xw = fw_in ? cw * (double)P.k_w[((size_t)b * 3 + c3) * wsz_w + ww] : 0.0;
            xu = warp_sum(xu);
            xv = warp_sum(xv);
            xw = warp_sum(xw);
            if (lane == 0) {
              S.acc[warp][b * 9 + c3] += xu;
              S.acc[warp][b * 9 + 3 + c3] += xv;
              S.acc[warp][b * 9 + 6 + c3] += xw;
            }
          }
        }
        for (int t = 0; t < P.n_tbody; ++t) {
          double xt = ft_in ? ct * (double)P.w_t[(size_t)t * wsz_c + wt] : 0.0;
          xt = warp_sum(xt);
          if (lane == 0) S.acc[warp][P.nbody * 9 + t] += xt;
        }
      }
    }
    if (pre) {
      if (P.use_tma) {
        ok = await_plane(k + 3);
        if (ok) fill(k + 3, false);
      } else {
        fill(k + 3, true);
      }
    }
    if (__syncthreads_or(!ok)) {
      drain(min(k + 3, ke + 1));
      return;
    }
  }

  if (P.has_win && P.partials) {
    __syncthreads();
    const size_t blk = ((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
    for (int q = tid; q < nq; q += TX * TY) {
      double s = 0.0;
      for (int w = 0; w < TX * TY / 32; ++w) s += S.acc[w][q];
      P.partials[blk * nq + q] = s;
    }
  }
#undef VEL
#undef TH
#undef NU
}

// --------------------------------------------------------------------------------------
// launchers
// --------------------------------------------------------------------------------------

template <typename T>
size_t stage_smem_bytes() {
  return sizeof(StageSmem<T>);
}

template <typename T, bool UPWIND, bool LES, bool THERMAL, bool PLACED>
cudaError_t launch_stage_cfg(const StageParams<T> &P, cudaStream_t s) {
  const size_t smem = sizeof(StageSmem<T>);
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(stage_kernel<T, UPWIND, LES, THERMAL, PLACED>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  dim3 grid((P.nx + TX - 1) / TX, (P.ny + TY - 1) / TY, (P.nz + P.zc - 1) / P.zc);
  (void)aero::launch_k(stage_kernel<T, UPWIND, LES, THERMAL, PLACED>, grid, dim3(TX, TY), smem, s, P);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_stage(const StageParams<T> &P, cudaStream_t s) {
  using Launch = cudaError_t (*)(const StageParams<T> &, cudaStream_t);
  // index: placed x 8 + upwind x 4 + les x 2 + thermal
  static const Launch table[16] = {
      launch_stage_cfg<T, false, false, false, false>, launch_stage_cfg<T, false, false, true, false>,
      launch_stage_cfg<T, false, true, false, false>,  launch_stage_cfg<T, false, true, true, false>,
      launch_stage_cfg<T, true, false, false, false>,  launch_stage_cfg<T, true, false, true, false>,
      launch_stage_cfg<T, true, true, false, false>,   launch_stage_cfg<T, true, true, true, false>,
      launch_stage_cfg<T, false, false, false, true>,  launch_stage_cfg<T, false, false, true, true>,
      launch_stage_cfg<T, false, true, false, true>,   launch_stage_cfg<T, false, true, true, true>,
      launch_stage_cfg<T, true, false, false, true>,   launch_stage_cfg<T, true, false, true, true>,
      launch_stage_cfg<T, true, true, false, true>,    launch_stage_cfg<T, true, true, true, true>};
  const bool placed = P.paint_u != nullptr || P.nfan > 0 || P.nport > 0 || P.nheat > 0 || P.forcing;
  const int idx = (placed ? 8 : 0) + (P.upwind ? 4 : 0) + (P.les != AERO_LES_NONE ? 2 : 0) + (P.thermal ? 1 : 0);
  return table[idx](P, s);
}

template <typename T>
cudaError_t launch_nu(const NuParams<T> &P, cudaStream_t s) {
  dim3 grid((P.nx + 2 + TX - 1) / TX, (P.ny + 2 + TY - 1) / TY, (P.nz + 2 + P.zc - 1) / P.zc);
  switch (P.les) {
    case AERO_LES_SMAGORINSKY: (void)aero::launch_k(nu_kernel<T, AERO_LES_SMAGORINSKY>, grid, dim3(TX, TY), 0, s, P); break;
    case AERO_LES_WALE: (void)aero::launch_k(nu_kernel<T, AERO_LES_WALE>, grid, dim3(TX, TY), 0, s, P); break;
    case AERO_LES_VREMAN: (void)aero::launch_k(nu_kernel<T, AERO_LES_VREMAN>, grid, dim3(TX, TY), 0, s, P); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}


}  // namespace aero
