// The 3D SSP-RK3 stage kernel and its helpers (pre-pass, time step, outlet sums,
// correction, smoke, end of step).
//
// Arithmetic follows the reference's plain-torch step (Aerolume ns3d/core.py:765-883)
// operation by operation, so float64 runs agree with it to round-off:
//   advection   core.py:331-390      diffusion  core.py:393-397, 557-560
//   LES         core.py:400-524      RK update  core.py:819-827
//   boundaries  core.py:281-297, 527-543
//   penalty     core.py:615-634      buoyancy   physics.py:744-790
//   theta       physics.py:609-708   dt rule    core.py:637-646, physics.py:723-742,1230-1262
//   smoke       dye.py:232-312
//
// Layout: every field is a C-contiguous (z, y, x) array with the staggered shapes of
// core.py:11-14.  The stage kernel tiles x-y in 32 x 8 columns and marches along z,
// keeping five planes of each velocity component and of theta (two ghost layers) and
// three planes of the eddy viscosity in shared memory.
#include "ns3d.cuh"

namespace aero {

// --------------------------------------------------------------------------------------
// small device helpers
// --------------------------------------------------------------------------------------

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
template <typename T>
__device__ __forceinline__ T van_leer(T p, T q) {
  const T pq = p * q;
  return pq > T(0) ? T(2) * pq / (p + q) : T(0);
}

template <typename T>
__device__ __forceinline__ T muscl_flux(T a, T b, T c, T d, T vel) {
  const T up = b + T(0.5) * van_leer(b - a, c - b);
  const T dn = c - T(0.5) * van_leer(c - b, d - c);
  return vel * (vel > T(0) ? up : dn);
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
  if (model == AERO_LES_SMAGORINSKY) return cd2 * sqrt(T(2) * ss + T(1e-30));
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
    const T num = pow(sdp, T(1.5));
    const T den = pow(ssp, T(2.5)) + pow(sdp, T(1.25)) + T(1e-30);
    return cd2 * num / den;
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
  return cd2 * sqrt(bb / (aa + T(1e-30)) + T(1e-30));
}

// --------------------------------------------------------------------------------------
// the stage kernel
// --------------------------------------------------------------------------------------

constexpr int TX = 32, TY = 8, HX = TX + 4, HY = TY + 4, NPL = HX * HY;  // velocity / theta planes
constexpr int NX2 = TX + 2, NY2 = TY + 2, NNU = NX2 * NY2;               // eddy-viscosity planes

template <typename T>
struct StageSmem {
  T vel[3][5][NPL];
  T th[5][NPL];
  T nu[3][NNU];
  double acc[8][AERO_MAX_BODIES * 10];  // per-warp force / heat sums
};

template <typename T>
__global__ void __launch_bounds__(TX *TY) stage_kernel(const StageParams<T> P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  StageSmem<T> &S = *reinterpret_cast<StageSmem<T> *>(smem_raw);
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int lane = tid & 31, warp = tid >> 5;
  const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
  const int kb = blockIdx.z * P.zc, ke = min(kb + P.zc, P.nz);
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  const int i = i0 + tx, j = j0 + ty;
  const bool les = P.les != AERO_LES_NONE;
  const bool upwind = P.upwind != 0;
  const T inv = P.inv_h;
  const int nq = P.nq;
  const bool nut_only = P.mode == MODE_NUT_ONLY;

  if (!nut_only)
    for (int q = tid; q < 8 * AERO_MAX_BODIES * 10; q += TX * TY) (&S.acc[0][0])[q] = 0.0;

  // ---- loaders -------------------------------------------------------------------
  auto load_plane = [&](int kp) {
    const int slot = ((kp % 5) + 5) % 5;
    for (int e = tid; e < NPL; e += TX * TY) {
      const int ly = e / HX, lx = e - ly * HX;
      const int gj = j0 - 2 + ly, gi = i0 - 2 + lx;
      S.vel[0][slot][e] = padded<T>(P.up, P.ru, kp, gj, gi);
      S.vel[1][slot][e] = padded<T>(P.vp, P.rv, kp, gj, gi);
      S.vel[2][slot][e] = padded<T>(P.wp, P.rw, kp, gj, gi);
      if (P.thermal) S.th[slot][e] = theta_padded<T>(P.thp, nz, ny, nx, P.sides, P.h, kp, gj, gi);
    }
  };
  // velocity at plane (kc + dz), local cell (ly, lx) of the halo-2 tile
#define VEL(c, dz, ly, lx) S.vel[c][(((kc + (dz)) % 5) + 5) % 5][(ly) * HX + (lx)]
#define TH(dz, ly, lx) S.th[(((kc + (dz)) % 5) + 5) % 5][(ly) * HX + (lx)]
#define NU(dz, ly, lx) S.nu[(((kc + (dz)) % 3) + 3) % 3][(ly) * NX2 + (lx)]

  // eddy viscosity of plane kn for the (TY+2) x (TX+2) cells of the tile and its ring
  T nut_local_max = T(0);
  auto compute_nu = [&](int kn) {
    const int kc = kn;  // velocity offsets are relative to plane kn
    const int slot = ((kn % 3) + 3) % 3;
    for (int e = tid; e < NNU; e += TX * TY) {
      const int ly = e / NX2, lx = e - ly * NX2;
      const int cj = j0 - 1 + ly, ci = i0 - 1 + lx;
      T nu = T(0);
      if (cj >= -1 && cj <= ny && ci >= -1 && ci <= nx && kn >= -1 && kn <= nz) {
        const int y = ly + 1, x = lx + 1;  // this cell in the halo-2 tile
        T g[3][3];
        g[0][0] = (VEL(0, 0, y, x + 1) - VEL(0, 0, y, x)) * inv;
        g[1][1] = (VEL(1, 0, y + 1, x) - VEL(1, 0, y, x)) * inv;
        const T q = T(0.25);
        g[0][1] = ((((VEL(0, 0, y, x) - VEL(0, 0, y - 1, x)) * inv + (VEL(0, 0, y + 1, x) - VEL(0, 0, y, x)) * inv) +
                    (VEL(0, 0, y, x + 1) - VEL(0, 0, y - 1, x + 1)) * inv) +
                   (VEL(0, 0, y + 1, x + 1) - VEL(0, 0, y, x + 1)) * inv) *
                  q;
        g[0][2] = ((((VEL(0, 0, y, x) - VEL(0, -1, y, x)) * inv + (VEL(0, 1, y, x) - VEL(0, 0, y, x)) * inv) +
                    (VEL(0, 0, y, x + 1) - VEL(0, -1, y, x + 1)) * inv) +
                   (VEL(0, 1, y, x + 1) - VEL(0, 0, y, x + 1)) * inv) *
                  q;
        g[1][0] = ((((VEL(1, 0, y, x) - VEL(1, 0, y, x - 1)) * inv + (VEL(1, 0, y + 1, x) - VEL(1, 0, y + 1, x - 1)) * inv) +
                    (VEL(1, 0, y, x + 1) - VEL(1, 0, y, x)) * inv) +
                   (VEL(1, 0, y + 1, x + 1) - VEL(1, 0, y + 1, x)) * inv) *
                  q;
        g[1][2] = ((((VEL(1, 0, y, x) - VEL(1, -1, y, x)) * inv + (VEL(1, 1, y, x) - VEL(1, 0, y, x)) * inv) +
                    (VEL(1, 0, y + 1, x) - VEL(1, -1, y + 1, x)) * inv) +
                   (VEL(1, 1, y + 1, x) - VEL(1, 0, y + 1, x)) * inv) *
                  q;
        g[2][0] = ((((VEL(2, 0, y, x) - VEL(2, 0, y, x - 1)) * inv + (VEL(2, 1, y, x) - VEL(2, 1, y, x - 1)) * inv) +
                    (VEL(2, 0, y, x + 1) - VEL(2, 0, y, x)) * inv) +
                   (VEL(2, 1, y, x + 1) - VEL(2, 1, y, x)) * inv) *
                  q;
        g[2][1] = ((((VEL(2, 0, y, x) - VEL(2, 0, y - 1, x)) * inv + (VEL(2, 1, y, x) - VEL(2, 1, y - 1, x)) * inv) +
                    (VEL(2, 0, y + 1, x) - VEL(2, 0, y, x)) * inv) +
                   (VEL(2, 1, y + 1, x) - VEL(2, 1, y, x)) * inv) *
                  q;
        g[2][2] = -(g[0][0] + g[1][1]);
        nu = eddy_viscosity<T>(g, P.les, P.les_cd2);
        if (kn >= P.win[0] && kn < P.win[1] && cj >= P.win[2] && cj < P.win[3] && ci >= P.win[4] && ci < P.win[5]) {
          const T chi = P.chi_c[((size_t)(kn - P.win[0]) * P.wny + (cj - P.win[2])) * P.wnx + (ci - P.win[4])];
          nu = nu * (T(1) - chi);
        }
        nut_local_max = fmax(nut_local_max, nu);
      }
      S.nu[slot][e] = nu;
    }
  };

  // ---- preload -----------------------------------------------------------------------
  for (int kp = kb - 2; kp <= kb + 1; ++kp) load_plane(kp);
  __syncthreads();
  if (les) {
    compute_nu(kb - 1);
    compute_nu(kb);
  }

  // per-thread register carry of theta / force sums
  for (int k = kb; k < ke; ++k) {
    __syncthreads();
    load_plane(k + 2);
    __syncthreads();
    if (les) {
      compute_nu(k + 1);
      __syncthreads();
    }
    if (nut_only) continue;
    const int kc = k;
    const int y = ty + 2, x = tx + 2;  // this thread's cell / faces in the halo-2 tile
    const int ny2 = ty + 1, nx2 = tx + 1;  // ... in the eddy-viscosity tile
    const bool valid = (i < nx) && (j < ny);
    const T bdt = P.bdt_scale * *P.dt;
    const T a = P.a;

    double cu = 0.0, cv = 0.0, cw = 0.0, ct = 0.0;  // weighted window increments
    int fu_in = 0, fv_in = 0, fw_in = 0, ft_in = 0;  // which faces lie in the window
    size_t wu = 0, wv = 0, ww = 0, wt = 0;

    if (valid) {
      // ================= momentum tendencies (core.py:353-397, 485-524) ===============
      const T kadv = P.kadv, nuh2 = P.nu_h2;
      // ---- u face (k, j, i)
      T lu;
      {
        T au = face_flux<T>(VEL(0, 0, y, x - 1) + VEL(0, 0, y, x), VEL(0, 0, y, x - 2), VEL(0, 0, y, x - 1),
                            VEL(0, 0, y, x), VEL(0, 0, y, x + 1), upwind) -
               face_flux<T>(VEL(0, 0, y, x) + VEL(0, 0, y, x + 1), VEL(0, 0, y, x - 1), VEL(0, 0, y, x),
                            VEL(0, 0, y, x + 1), VEL(0, 0, y, x + 2), upwind);
        const T gyl = face_flux<T>(VEL(1, 0, y, x - 1) + VEL(1, 0, y, x), VEL(0, 0, y - 2, x), VEL(0, 0, y - 1, x),
                                   VEL(0, 0, y, x), VEL(0, 0, y + 1, x), upwind);
        const T gyr = face_flux<T>(VEL(1, 0, y + 1, x - 1) + VEL(1, 0, y + 1, x), VEL(0, 0, y - 1, x), VEL(0, 0, y, x),
                                   VEL(0, 0, y + 1, x), VEL(0, 0, y + 2, x), upwind);
        au = au + (gyl - gyr);
        const T gzl = face_flux<T>(VEL(2, 0, y, x - 1) + VEL(2, 0, y, x), VEL(0, -2, y, x), VEL(0, -1, y, x),
                                   VEL(0, 0, y, x), VEL(0, 1, y, x), upwind);
        const T gzr = face_flux<T>(VEL(2, 1, y, x - 1) + VEL(2, 1, y, x), VEL(0, -1, y, x), VEL(0, 0, y, x),
                                   VEL(0, 1, y, x), VEL(0, 2, y, x), upwind);
        au = (au + (gzl - gzr)) * kadv;
        const T lap = ((VEL(0, 0, y, x + 1) + VEL(0, 0, y, x - 1)) + (VEL(0, 0, y + 1, x) + VEL(0, 0, y - 1, x)) +
                       (VEL(0, 1, y, x) + VEL(0, -1, y, x))) -
                      T(6) * VEL(0, 0, y, x);
        lu = au + nuh2 * lap;
        if (les) {
          const T two = T(2), q = T(0.25);
          const T t11r = two * NU(0, ny2, nx2) * ((VEL(0, 0, y, x + 1) - VEL(0, 0, y, x)) * inv);
          const T t11l = two * NU(0, ny2, nx2 - 1) * ((VEL(0, 0, y, x) - VEL(0, 0, y, x - 1)) * inv);
          const T n12l = (((NU(0, ny2 - 1, nx2 - 1) + NU(0, ny2, nx2 - 1)) + NU(0, ny2 - 1, nx2)) + NU(0, ny2, nx2)) * q;
          const T s12l = (VEL(0, 0, y, x) - VEL(0, 0, y - 1, x)) * inv + (VEL(1, 0, y, x) - VEL(1, 0, y, x - 1)) * inv;
          const T n12r = (((NU(0, ny2, nx2 - 1) + NU(0, ny2 + 1, nx2 - 1)) + NU(0, ny2, nx2)) + NU(0, ny2 + 1, nx2)) * q;
          const T s12r =
              (VEL(0, 0, y + 1, x) - VEL(0, 0, y, x)) * inv + (VEL(1, 0, y + 1, x) - VEL(1, 0, y + 1, x - 1)) * inv;
          const T n13l = (((NU(-1, ny2, nx2 - 1) + NU(0, ny2, nx2 - 1)) + NU(-1, ny2, nx2)) + NU(0, ny2, nx2)) * q;
          const T s13l = (VEL(0, 0, y, x) - VEL(0, -1, y, x)) * inv + (VEL(2, 0, y, x) - VEL(2, 0, y, x - 1)) * inv;
          const T n13r = (((NU(0, ny2, nx2 - 1) + NU(1, ny2, nx2 - 1)) + NU(0, ny2, nx2)) + NU(1, ny2, nx2)) * q;
          const T s13r = (VEL(0, 1, y, x) - VEL(0, 0, y, x)) * inv + (VEL(2, 1, y, x) - VEL(2, 1, y, x - 1)) * inv;
          const T fu = (((((t11r - t11l) + n12r * s12r) - n12l * s12l) + n13r * s13r) - n13l * s13l) * inv;
          lu = lu + fu;
        }
      }
      // ---- v face (k, j, i)
      T lv;
      {
        T av = face_flux<T>(VEL(0, 0, y - 1, x) + VEL(0, 0, y, x), VEL(1, 0, y, x - 2), VEL(1, 0, y, x - 1),
                            VEL(1, 0, y, x), VEL(1, 0, y, x + 1), upwind) -
               face_flux<T>(VEL(0, 0, y - 1, x + 1) + VEL(0, 0, y, x + 1), VEL(1, 0, y, x - 1), VEL(1, 0, y, x),
                            VEL(1, 0, y, x + 1), VEL(1, 0, y, x + 2), upwind);
        const T gyl = face_flux<T>(VEL(1, 0, y - 1, x) + VEL(1, 0, y, x), VEL(1, 0, y - 2, x), VEL(1, 0, y - 1, x),
                                   VEL(1, 0, y, x), VEL(1, 0, y + 1, x), upwind);
        const T gyr = face_flux<T>(VEL(1, 0, y, x) + VEL(1, 0, y + 1, x), VEL(1, 0, y - 1, x), VEL(1, 0, y, x),
                                   VEL(1, 0, y + 1, x), VEL(1, 0, y + 2, x), upwind);
        av = av + (gyl - gyr);
        const T gzl = face_flux<T>(VEL(2, 0, y - 1, x) + VEL(2, 0, y, x), VEL(1, -2, y, x), VEL(1, -1, y, x),
                                   VEL(1, 0, y, x), VEL(1, 1, y, x), upwind);
        const T gzr = face_flux<T>(VEL(2, 1, y - 1, x) + VEL(2, 1, y, x), VEL(1, -1, y, x), VEL(1, 0, y, x),
                                   VEL(1, 1, y, x), VEL(1, 2, y, x), upwind);
        av = (av + (gzl - gzr)) * kadv;
        const T lap = ((VEL(1, 0, y, x + 1) + VEL(1, 0, y, x - 1)) + (VEL(1, 0, y + 1, x) + VEL(1, 0, y - 1, x)) +
                       (VEL(1, 1, y, x) + VEL(1, -1, y, x))) -
                      T(6) * VEL(1, 0, y, x);
        lv = av + nuh2 * lap;
        if (les) {
          const T two = T(2), q = T(0.25);
          const T n12l = (((NU(0, ny2 - 1, nx2 - 1) + NU(0, ny2, nx2 - 1)) + NU(0, ny2 - 1, nx2)) + NU(0, ny2, nx2)) * q;
          const T s12l = (VEL(0, 0, y, x) - VEL(0, 0, y - 1, x)) * inv + (VEL(1, 0, y, x) - VEL(1, 0, y, x - 1)) * inv;
          const T n12r = (((NU(0, ny2 - 1, nx2) + NU(0, ny2, nx2)) + NU(0, ny2 - 1, nx2 + 1)) + NU(0, ny2, nx2 + 1)) * q;
          const T s12r =
              (VEL(0, 0, y, x + 1) - VEL(0, 0, y - 1, x + 1)) * inv + (VEL(1, 0, y, x + 1) - VEL(1, 0, y, x)) * inv;
          const T t22r = two * NU(0, ny2, nx2) * ((VEL(1, 0, y + 1, x) - VEL(1, 0, y, x)) * inv);
          const T t22l = two * NU(0, ny2 - 1, nx2) * ((VEL(1, 0, y, x) - VEL(1, 0, y - 1, x)) * inv);
          const T n23l = (((NU(-1, ny2 - 1, nx2) + NU(0, ny2 - 1, nx2)) + NU(-1, ny2, nx2)) + NU(0, ny2, nx2)) * q;
          const T s23l = (VEL(1, 0, y, x) - VEL(1, -1, y, x)) * inv + (VEL(2, 0, y, x) - VEL(2, 0, y - 1, x)) * inv;
          const T n23r = (((NU(0, ny2 - 1, nx2) + NU(1, ny2 - 1, nx2)) + NU(0, ny2, nx2)) + NU(1, ny2, nx2)) * q;
          const T s23r = (VEL(1, 1, y, x) - VEL(1, 0, y, x)) * inv + (VEL(2, 1, y, x) - VEL(2, 1, y - 1, x)) * inv;
          const T fv = (((((n12r * s12r - n12l * s12l) + t22r) - t22l) + n23r * s23r) - n23l * s23l) * inv;
          lv = lv + fv;
        }
      }
      // ---- w face (k, j, i)
      T lw;
      {
        T aw = face_flux<T>(VEL(0, -1, y, x) + VEL(0, 0, y, x), VEL(2, 0, y, x - 2), VEL(2, 0, y, x - 1),
                            VEL(2, 0, y, x), VEL(2, 0, y, x + 1), upwind) -
               face_flux<T>(VEL(0, -1, y, x + 1) + VEL(0, 0, y, x + 1), VEL(2, 0, y, x - 1), VEL(2, 0, y, x),
                            VEL(2, 0, y, x + 1), VEL(2, 0, y, x + 2), upwind);
        const T gyl = face_flux<T>(VEL(1, -1, y, x) + VEL(1, 0, y, x), VEL(2, 0, y - 2, x), VEL(2, 0, y - 1, x),
                                   VEL(2, 0, y, x), VEL(2, 0, y + 1, x), upwind);
        const T gyr = face_flux<T>(VEL(1, -1, y + 1, x) + VEL(1, 0, y + 1, x), VEL(2, 0, y - 1, x), VEL(2, 0, y, x),
                                   VEL(2, 0, y + 1, x), VEL(2, 0, y + 2, x), upwind);
        aw = aw + (gyl - gyr);
        const T gzl = face_flux<T>(VEL(2, -1, y, x) + VEL(2, 0, y, x), VEL(2, -2, y, x), VEL(2, -1, y, x),
                                   VEL(2, 0, y, x), VEL(2, 1, y, x), upwind);
        const T gzr = face_flux<T>(VEL(2, 0, y, x) + VEL(2, 1, y, x), VEL(2, -1, y, x), VEL(2, 0, y, x),
                                   VEL(2, 1, y, x), VEL(2, 2, y, x), upwind);
        aw = (aw + (gzl - gzr)) * kadv;
        const T lap = ((VEL(2, 0, y, x + 1) + VEL(2, 0, y, x - 1)) + (VEL(2, 0, y + 1, x) + VEL(2, 0, y - 1, x)) +
                       (VEL(2, 1, y, x) + VEL(2, -1, y, x))) -
                      T(6) * VEL(2, 0, y, x);
        lw = aw + nuh2 * lap;
        if (les) {
          const T two = T(2), q = T(0.25);
          const T n13l = (((NU(-1, ny2, nx2 - 1) + NU(0, ny2, nx2 - 1)) + NU(-1, ny2, nx2)) + NU(0, ny2, nx2)) * q;
          const T s13l = (VEL(0, 0, y, x) - VEL(0, -1, y, x)) * inv + (VEL(2, 0, y, x) - VEL(2, 0, y, x - 1)) * inv;
          const T n13r = (((NU(-1, ny2, nx2) + NU(0, ny2, nx2)) + NU(-1, ny2, nx2 + 1)) + NU(0, ny2, nx2 + 1)) * q;
          const T s13r =
              (VEL(0, 0, y, x + 1) - VEL(0, -1, y, x + 1)) * inv + (VEL(2, 0, y, x + 1) - VEL(2, 0, y, x)) * inv;
          const T n23l = (((NU(-1, ny2 - 1, nx2) + NU(0, ny2 - 1, nx2)) + NU(-1, ny2, nx2)) + NU(0, ny2, nx2)) * q;
          const T s23l = (VEL(1, 0, y, x) - VEL(1, -1, y, x)) * inv + (VEL(2, 0, y, x) - VEL(2, 0, y - 1, x)) * inv;
          const T n23r = (((NU(-1, ny2, nx2) + NU(0, ny2, nx2)) + NU(-1, ny2 + 1, nx2)) + NU(0, ny2 + 1, nx2)) * q;
          const T s23r =
              (VEL(1, 0, y + 1, x) - VEL(1, -1, y + 1, x)) * inv + (VEL(2, 0, y + 1, x) - VEL(2, 0, y, x)) * inv;
          const T t33r = two * NU(0, ny2, nx2) * ((VEL(2, 1, y, x) - VEL(2, 0, y, x)) * inv);
          const T t33l = two * NU(-1, ny2, nx2) * ((VEL(2, 0, y, x) - VEL(2, -1, y, x)) * inv);
          const T fw = (((((n13r * s13r - n13l * s13l) + n23r * s23r) - n23l * s23l) + t33r) - t33l) * inv;
          lw = lw + fw;
        }
      }

      // ================= boundary tendencies and RK update (core.py:527-543, 819-827) =
      const size_t iu = ((size_t)k * ny + j) * (nx + 1) + i;
      const size_t iv = ((size_t)k * (ny + 1) + j) * nx + i;
      const size_t iw = ((size_t)k * ny + j) * nx + i;
      const T up0 = VEL(0, 0, y, x), vp0 = VEL(1, 0, y, x), wp0 = VEL(2, 0, y, x);
      T uh, vh, wh;
      if (a == T(0)) {
        uh = up0 + lu * bdt;
        vh = vp0 + lv * bdt;
        wh = wp0 + lw * bdt;
      } else {
        uh = lerp_t<T>(up0, P.u0[iu], a) + lu * bdt;
        vh = lerp_t<T>(vp0, P.v0[iv], a) + lv * bdt;
        wh = lerp_t<T>(wp0, P.w0[iw], a) + lw * bdt;
      }
      if (!P.px && i == 0) uh = P.closed ? T(0) : P.u_inlet[(size_t)k * ny + j];
      if (!P.py && j == 0) vh = T(0);
      if (!P.pz && k == 0) wh = T(0);

      // ================= window penalisation (core.py:615-634) =========================
      const T kpen = bdt / P.eta;
      const T wg = P.wgt;
      if (P.has_win) {
        const int k0 = P.win[0], k1 = P.win[1], wj0 = P.win[2], wj1 = P.win[3], wi0 = P.win[4], wi1 = P.win[5];
        if (k >= k0 && k < k1 && j >= wj0 && j < wj1 && i >= wi0 && i <= wi1) {
          wu = ((size_t)(k - k0) * (wj1 - wj0) + (j - wj0)) * (wi1 - wi0 + 1) + (i - wi0);
          const T un = (uh + kpen * P.a_u[wu]) / (T(1) + kpen * P.chi_u[wu]);
          cu = (double)((un - uh) * wg);
          uh = un;
          fu_in = 1;
        }
        if (k >= k0 && k < k1 && j >= wj0 && j <= wj1 && i >= wi0 && i < wi1) {
          wv = ((size_t)(k - k0) * (wj1 - wj0 + 1) + (j - wj0)) * (wi1 - wi0) + (i - wi0);
          const T vn = (vh + kpen * P.a_v[wv]) / (T(1) + kpen * P.chi_v[wv]);
          cv = (double)((vn - vh) * wg);
          vh = vn;
          fv_in = 1;
        }
        if (k >= k0 && k <= k1 && j >= wj0 && j < wj1 && i >= wi0 && i < wi1) {
          ww = ((size_t)(k - k0) * (wj1 - wj0) + (j - wj0)) * (wi1 - wi0) + (i - wi0);
          const T wn = (wh + kpen * P.a_w[ww]) / (T(1) + kpen * P.chi_w[ww]);
          cw = (double)((wn - wh) * wg);
          wh = wn;
          fw_in = 1;
        }
      }

      // ================= buoyancy after the penalisation (physics.py:744-790) =========
      if (P.thermal && P.ri != T(0)) {
        if (k > 0 || P.pz) {
          if (k > 0) {
            const T tf = T(0.5) * (TH(0, y, x) + TH(-1, y, x));
            wh = wh + tf * (bdt * P.ri);
          } else {
            const T edge = (TH(0, y, x) + TH(-1, y, x)) * (T(0.5) * P.ri) * bdt;
            wh = wh + edge;
          }
        }
        if (fw_in && P.vol_w) {
          // theta on the w-face from the two cells around it (clamped / wrapped at the ends)
          const int kl = (k == 0) ? (P.pz ? nz - 1 : 0) : k - 1;
          const int kr = (k == nz) ? (P.pz ? 0 : nz - 1) : k;
          const T tl = P.thp[((size_t)kl * ny + j) * nx + i], tr = P.thp[((size_t)kr * ny + j) * nx + i];
          const T tw = T(0.5) * (tr + tl);
          const T share = (tw * P.vol_w[ww]) * (bdt * (P.ri * wg));
          cw += (double)share;
        }
      }

      // ================= outputs ==========================================================
      P.uh[iu] = uh;
      P.vh[iv] = vh;
      P.wh[iw] = wh;
      // the high boundary faces
      if (i == nx - 1 && !P.px) {
        const size_t io = iu + 1;
        T uo;
        if (P.closed) {
          uo = T(0);
        } else {
          const T upo = VEL(0, 0, y, x + 1), upi = VEL(0, 0, y, x);
          const T lo = (upi - upo) * inv;
          uo = (a == T(0) ? upo : lerp_t<T>(upo, P.u0[io], a)) + lo * bdt;
          uo = uo + P.outlet_corr[0];
        }
        P.uh[io] = uo;
      }
      if (j == ny - 1 && !P.py) P.vh[iv + nx] = T(0);
      if (k == nz - 1 && !P.pz) P.wh[iw + (size_t)ny * nx] = T(0);

      // ================= theta stage (physics.py:647-708) ================================
      if (P.thermal) {
        const T kh = P.kh;
        auto kface = [&](T n1, T n2, bool boundary) -> T {
          if (!les || boundary) return kh;
          return kh + P.kprt * (n1 + n2);
        };
        const T c = TH(0, y, x);
        // x faces i and i+1
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
        const T kzl = kface(NU(-1, ny2, nx2), NU(0, ny2, nx2), !P.pz && k == 0);
        const T kzr = kface(NU(0, ny2, nx2), NU(1, ny2, nx2), !P.pz && k == nz - 1);
        T fzl = muscl_flux<T>(TH(-2, y, x), TH(-1, y, x), c, TH(1, y, x), VEL(2, 0, y, x)) - kzl * (c - TH(-1, y, x));
        T fzr = muscl_flux<T>(TH(-1, y, x), c, TH(1, y, x), TH(2, y, x), VEL(2, 1, y, x)) - kzr * (TH(1, y, x) - c);
        if (P.has_adia) {  // adiabatic bodies block conduction (physics.py:666-675)
          const int k0 = P.win[0], k1 = P.win[1], wj0 = P.win[2], wj1 = P.win[3], wi0 = P.win[4], wi1 = P.win[5];
          const int wzn = k1 - k0, wyn = wj1 - wj0, wxn = wi1 - wi0;
          if (k >= k0 && k < k1 && j >= wj0 && j < wj1) {
            if (i >= wi0 && i <= wi1)
              fxl += kxl * P.adia_u[((size_t)(k - k0) * wyn + (j - wj0)) * (wxn + 1) + (i - wi0)] * (c - TH(0, y, x - 1));
            if (i + 1 >= wi0 && i + 1 <= wi1)
              fxr += kxr * P.adia_u[((size_t)(k - k0) * wyn + (j - wj0)) * (wxn + 1) + (i + 1 - wi0)] *
                     (TH(0, y, x + 1) - c);
          }
          if (k >= k0 && k < k1 && i >= wi0 && i < wi1) {
            if (j >= wj0 && j <= wj1)
              fyl += kyl * P.adia_v[((size_t)(k - k0) * (wyn + 1) + (j - wj0)) * wxn + (i - wi0)] * (c - TH(0, y - 1, x));
            if (j + 1 >= wj0 && j + 1 <= wj1)
              fyr += kyr * P.adia_v[((size_t)(k - k0) * (wyn + 1) + (j + 1 - wj0)) * wxn + (i - wi0)] *
                     (TH(0, y + 1, x) - c);
          }
          if (j >= wj0 && j < wj1 && i >= wi0 && i < wi1) {
            if (k >= k0 && k <= k1)
              fzl += kzl * P.adia_w[((size_t)(k - k0) * wyn + (j - wj0)) * wxn + (i - wi0)] * (c - TH(-1, y, x));
            if (k + 1 >= k0 && k + 1 <= k1)
              fzr += kzr * P.adia_w[((size_t)(k + 1 - k0) * wyn + (j - wj0)) * wxn + (i - wi0)] * (TH(1, y, x) - c);
          }
          (void)wzn;
        }
        const T D = ((fxr - fxl) + (fyr - fyl) + (fzr - fzl)) * inv;
        const size_t ic = ((size_t)k * ny + j) * nx + i;
        T ch = (a == T(0) ? c : lerp_t<T>(c, P.th0[ic], a)) - bdt * D;
        const int k0 = P.win[0], k1 = P.win[1], wj0 = P.win[2], wj1 = P.win[3], wi0 = P.win[4], wi1 = P.win[5];
        if (P.has_win && k >= k0 && k < k1 && j >= wj0 && j < wj1 && i >= wi0 && i < wi1) {
          wt = ((size_t)(k - k0) * (wj1 - wj0) + (j - wj0)) * (wi1 - wi0) + (i - wi0);
          if (P.skin) ch = ch + (bdt * P.kappa) * P.skin[wt];
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
    if (P.has_win) {
      const unsigned any = __ballot_sync(0xffffffffu, fu_in | fv_in | fw_in | ft_in);
      if (any) {
        const size_t wsz_u = (size_t)(P.win[1] - P.win[0]) * (P.win[3] - P.win[2]) * (P.win[5] - P.win[4] + 1);
        const size_t wsz_v = (size_t)(P.win[1] - P.win[0]) * (P.win[3] - P.win[2] + 1) * (P.win[5] - P.win[4]);
        const size_t wsz_w = (size_t)(P.win[1] - P.win[0] + 1) * (P.win[3] - P.win[2]) * (P.win[5] - P.win[4]);
        const size_t wsz_c = (size_t)(P.win[1] - P.win[0]) * (P.win[3] - P.win[2]) * (P.win[5] - P.win[4]);
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
  }

  if (les) {
    // block max of nu_t, then one atomic per block
    T m = nut_local_max;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    __syncthreads();
    __shared__ double wmax[TX * TY / 32];
    if (lane == 0) wmax[warp] = (double)m;
    __syncthreads();
    if (tid == 0 && P.nut_max) {
      double mm = 0.0;
      for (int w = 0; w < TX * TY / 32; ++w) mm = fmax(mm, wmax[w]);
      atomic_max_nonneg(P.nut_max, mm);
    }
  }
  if (!nut_only && P.has_win && P.partials) {
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
// pre-pass maxima, time step, outlet sums
// --------------------------------------------------------------------------------------

template <typename T>
__global__ void absmax_kernel(const T *__restrict__ a, size_t n, unsigned long long *out) {
  T m = T(0);
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const T v = fabs(a[e]);
    m = (v > m || v != v) ? v : m;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const T other = __shfl_xor_sync(0xffffffffu, m, o);
    m = (other > m || other != other) ? other : m;
  }
  if ((threadIdx.x & 31) == 0) atomic_max_nonneg(out, (double)m);
}

// One thread: the step's dt from the maxima (core.py:637-646, physics.py:723-742, 1230-1262),
// rounded through the field type as the reference computes it.
template <typename T>
__global__ void dt_kernel(const DtParams P) {
  const double *sc = P.scalars;
  const unsigned long long *bits = reinterpret_cast<const unsigned long long *>(sc);
  T dt;
  if (P.dt_in) {
    dt = *reinterpret_cast<const T *>(P.dt_in);
  } else if (P.has_dt_fixed) {
    dt = T(P.dt_fixed);
  } else {
    const T mu = T(as_double(bits[SC_MAXU])), mv = T(as_double(bits[SC_MAXV])), mw = T(as_double(bits[SC_MAXW]));
    T umax = (mu + mv) + mw;
    umax = umax > T(1e-6) ? umax : T(1e-6);
    if (umax != umax) umax = mu + mv + mw;  // keep NaN
    dt = T(P.cfl * P.h) / umax;
    const bool les = P.les != 0;
    const T nut_max = T(as_double(bits[SC_NUTMAX]));
    const T nu = les ? T(P.nu) + nut_max : T(P.nu);
    const T dv = T(P.viscous_dt * P.h * P.h) / nu;
    dt = dv < dt ? dv : dt;
    if (P.thermal) {
      const T kap = les ? T(P.kappa) + nut_max / T(P.prt) : T(P.kappa);
      const T diff_rate = kap / T(P.viscous_dt * P.h * P.h);
      const T lim = T(1) / (umax * T(1.0 / (0.5 * P.h)) + diff_rate);
      dt = lim < dt ? lim : dt;
      if (P.ri != 0.0) {
        T acc = T(fabs(P.ri)) * T(as_double(bits[SC_MAXT]));
        acc = acc > T(1e-12) ? acc : T(1e-12);
        const T f = T(P.cfl) * sqrt(T(P.h) / acc);
        dt = f < dt ? f : dt;
      }
      if (P.has_heat_max) {
        T s = T(P.heat_max);
        s = s > T(1e-12) ? s : T(1e-12);
        const T l1 = T(1) / s;
        dt = l1 < dt ? l1 : dt;
        if (P.ri != 0.0) {
          const T l2 = pow(T(6.0 * P.cfl * P.h) / (T(fabs(P.ri)) * s), T(1.0 / 3.0));
          dt = l2 < dt ? l2 : dt;
        }
      }
    }
  }
  *reinterpret_cast<T *>(P.dt_out) = dt;
  P.scalars[SC_DT] = (double)dt;
  if (!(dt == dt) || !(dt > T(0)) || isinf((double)dt)) atomicOr(P.status, 1);
}

// Outlet-plane sums in a fixed order (deterministic): one block of 1024 threads.
// sums[0] = sum u[..., nx], sums[1] = sum u[..., nx-1] (and sums[2] = sum u0[..., nx] when
// u0 is given).  The stage blends them into the outlet correction by linearity.
template <typename T>
__global__ void outlet_sum_kernel(const T *__restrict__ u, const T *__restrict__ u0, int nx, int rows,
                                  double *sums) {
  __shared__ double red[3][32];
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  for (int r = threadIdx.x; r < rows; r += blockDim.x) {
    const size_t base = (size_t)r * (nx + 1);
    s0 += (double)u[base + nx];
    s1 += (double)u[base + nx - 1];
    if (u0) s2 += (double)u0[base + nx];
  }
  s0 = warp_sum(s0);
  s1 = warp_sum(s1);
  s2 = warp_sum(s2);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) {
    red[0][w] = s0;
    red[1][w] = s1;
    red[2][w] = s2;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0, c = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) {
      a += red[0][q];
      b += red[1][q];
      c += red[2][q];
    }
    sums[0] = a;
    sums[1] = b;
    if (u0) sums[2] = c;
  }
}

// corr = (sum u_inlet - sum uh[..., nx]) / (ny nz) with sum uh[..., nx] blended from the
// stage-start sums: sum lerp(up, u0, a) + b dt / h (sum up[nx-1] - sum up[nx]).
template <typename T>
__global__ void outlet_corr_kernel(const double *sums_p, const double *sum_u0, const double *sum_inlet, const T *dt,
                                   double a, double bscale, double inv_h, double inv_rows, T *corr) {
  const double bdt = (double)(T(bscale) * *dt);
  const double so = sums_p[0], si = sums_p[1], s0 = *sum_u0;
  const double out = (1.0 - a) * so + a * s0 + bdt * inv_h * (si - so);
  *corr = T((*sum_inlet - out) * inv_rows);
}

// --------------------------------------------------------------------------------------
// projection: divergence and gradient correction (core.py:577-601)
// --------------------------------------------------------------------------------------

template <typename T>
__global__ void divergence_kernel(const T *__restrict__ u, const T *__restrict__ v, const T *__restrict__ w, int nx,
                                  int ny, int nz, int px, int py, int pz, T inv_h, T *__restrict__ div) {
  const size_t n = (size_t)nx * ny * nz;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(e % nx);
    const size_t r = e / nx;
    const int j = (int)(r % ny), k = (int)(r / ny);
    const T ur = (px && i == nx - 1) ? u[((size_t)k * ny + j) * (nx + 1)] : u[((size_t)k * ny + j) * (nx + 1) + i + 1];
    const T ul = u[((size_t)k * ny + j) * (nx + 1) + i];
    const T vr = (py && j == ny - 1) ? v[((size_t)k * (ny + 1)) * nx + i] : v[((size_t)k * (ny + 1) + j + 1) * nx + i];
    const T vl = v[((size_t)k * (ny + 1) + j) * nx + i];
    const T wr = (pz && k == nz - 1) ? w[(size_t)j * nx + i] : w[((size_t)(k + 1) * ny + j) * nx + i];
    const T wl = w[((size_t)k * ny + j) * nx + i];
    div[e] = ((ur - ul) + (vr - vl) + (wr - wl)) * inv_h;
  }
}

// u <- uh - grad psi on every face; boundary-normal faces keep uh (non-periodic), periodic
// duplicate faces equal face 0.
template <typename T>
__global__ void correct_kernel(const CorrectParams<T> P) {
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  const size_t nu = (size_t)nz * ny * (nx + 1), nv = (size_t)nz * (ny + 1) * nx, nw = (size_t)(nz + 1) * ny * nx;
  const T inv = P.inv_h;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < nu + nv + nw; e += (size_t)gridDim.x * blockDim.x) {
    if (e < nu) {
      int i = (int)(e % (nx + 1));
      const size_t r = e / (nx + 1);
      const int j = (int)(r % ny), k = (int)(r / ny);
      T val;
      if (P.px) {
        const int ii = (i == nx) ? 0 : i;
        const int il = (ii == 0) ? nx - 1 : ii - 1;
        const size_t c = ((size_t)k * ny + j) * nx;
        val = P.uh[((size_t)k * ny + j) * (nx + 1) + ii] - (P.psi[c + ii] - P.psi[c + il]) * inv;
      } else if (i == 0 || i == nx) {
        val = P.uh[e];
      } else {
        const size_t c = ((size_t)k * ny + j) * nx + i;
        val = P.uh[e] - (P.psi[c] - P.psi[c - 1]) * inv;
      }
      P.u[e] = val;
    } else if (e < nu + nv) {
      const size_t f = e - nu;
      const int i = (int)(f % nx);
      const size_t r = f / nx;
      int j = (int)(r % (ny + 1));
      const int k = (int)(r / (ny + 1));
      T val;
      if (P.py) {
        const int jj = (j == ny) ? 0 : j;
        const int jl = (jj == 0) ? ny - 1 : jj - 1;
        val = P.vh[((size_t)k * (ny + 1) + jj) * nx + i] -
              (P.psi[((size_t)k * ny + jj) * nx + i] - P.psi[((size_t)k * ny + jl) * nx + i]) * inv;
      } else if (j == 0 || j == ny) {
        val = P.vh[f];
      } else {
        val = P.vh[f] - (P.psi[((size_t)k * ny + j) * nx + i] - P.psi[((size_t)k * ny + j - 1) * nx + i]) * inv;
      }
      P.v[f] = val;
    } else {
      const size_t f = e - nu - nv;
      const int i = (int)(f % nx);
      const size_t r = f / nx;
      const int j = (int)(r % ny);
      int k = (int)(r / ny);
      T val;
      if (P.pz) {
        const int kk = (k == nz) ? 0 : k;
        const int kl = (kk == 0) ? nz - 1 : kk - 1;
        val = P.wh[((size_t)kk * ny + j) * nx + i] -
              (P.psi[((size_t)kk * ny + j) * nx + i] - P.psi[((size_t)kl * ny + j) * nx + i]) * inv;
      } else if (k == 0 || k == nz) {
        val = P.wh[f];
      } else {
        val = P.wh[f] - (P.psi[((size_t)k * ny + j) * nx + i] - P.psi[((size_t)(k - 1) * ny + j) * nx + i]) * inv;
      }
      P.w[f] = val;
    }
  }
}

// --------------------------------------------------------------------------------------
// smoke: MUSCL forward Euler, clip and floor, solids and nozzles (dye.py:232-312)
// --------------------------------------------------------------------------------------

template <typename T>
__device__ __forceinline__ T dye_at(const T *__restrict__ c, int nz, int ny, int nx, int px, int py, int pz, int k,
                                    int j, int i) {
  // pad_dye ghosts (dye.py:232-263): inlet zeros, outlet zero-gradient, mirrored y / z
  if (i < 0) {
    if (!px) return T(0);
    i += nx;
  } else if (i >= nx) {
    i = px ? i - nx : nx - 1;
  }
  if (j < 0) j = py ? j + ny : -1 - j;
  else if (j >= ny) j = py ? j - ny : 2 * ny - 1 - j;
  if (k < 0) k = pz ? k + nz : -1 - k;
  else if (k >= nz) k = pz ? k - nz : 2 * nz - 1 - k;
  return __ldg(c + ((size_t)k * ny + j) * nx + i);
}

template <typename T>
__global__ void smoke_kernel(const SmokeParams<T> P) {
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  const size_t n = (size_t)nx * ny * nz;
  const T dt = *P.dt;
  const T kk = dt * P.inv_h;
  const T t = P.t_new ? *P.t_new : *P.t0 + dt;
  const T on = (fmod(t, T(P.pulse_period)) < T(P.pulse_on)) ? T(1) : T(0);
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(e % nx);
    const size_t r = e / nx;
    const int j = (int)(r % ny), k = (int)(r / ny);
    auto C = [&](int dk, int dj, int di) { return dye_at<T>(P.c0, nz, ny, nx, P.px, P.py, P.pz, k + dk, j + dj, i + di); };
    const T c = C(0, 0, 0);
    const T fx0 = muscl_flux<T>(C(0, 0, -2), C(0, 0, -1), c, C(0, 0, 1), P.u[((size_t)k * ny + j) * (nx + 1) + i]);
    const T fx1 = muscl_flux<T>(C(0, 0, -1), c, C(0, 0, 1), C(0, 0, 2), P.u[((size_t)k * ny + j) * (nx + 1) + i + 1]);
    const T fy0 = muscl_flux<T>(C(0, -2, 0), C(0, -1, 0), c, C(0, 1, 0), P.v[((size_t)k * (ny + 1) + j) * nx + i]);
    const T fy1 = muscl_flux<T>(C(0, -1, 0), c, C(0, 1, 0), C(0, 2, 0), P.v[((size_t)k * (ny + 1) + j + 1) * nx + i]);
    const T fz0 = muscl_flux<T>(C(-2, 0, 0), C(-1, 0, 0), c, C(1, 0, 0), P.w[((size_t)k * ny + j) * nx + i]);
    const T fz1 = muscl_flux<T>(C(-1, 0, 0), c, C(1, 0, 0), C(2, 0, 0), P.w[((size_t)(k + 1) * ny + j) * nx + i]);
    T v = c - kk * (((fx1 - fx0) + (fy1 - fy0)) + (fz1 - fz0));
    v = v > T(1) ? T(1) : v;
    v = v < T(1e-8) ? T(0) : v;
    if (P.chi_c && k >= P.win[0] && k < P.win[1] && j >= P.win[2] && j < P.win[3] && i >= P.win[4] && i < P.win[5]) {
      const T chi = P.chi_c[((size_t)(k - P.win[0]) * (P.win[3] - P.win[2]) + (j - P.win[2])) * (P.win[5] - P.win[4]) +
                            (i - P.win[4])];
      if (chi > T(0.5)) v = T(0);
    }
    if (P.weight && k >= P.dwin[0] && k < P.dwin[1] && j >= P.dwin[2] && j < P.dwin[3] && i >= P.dwin[4] &&
        i < P.dwin[5]) {
      const T wgt = P.weight[((size_t)(k - P.dwin[0]) * (P.dwin[3] - P.dwin[2]) + (j - P.dwin[2])) * (P.dwin[5] - P.dwin[4]) +
                             (i - P.dwin[4])];
      v = v + wgt * on * (T(1) - v);
    }
    P.c[e] = v;
  }
}

// --------------------------------------------------------------------------------------
// end of step: p, coefficients, heat rates, t and dt (core.py:653-678, 875-883,
// physics.py:713-721)
// --------------------------------------------------------------------------------------

template <typename T>
__global__ void finalize_kernel(const FinalizeParams<T> P) {
  __shared__ double tot[AERO_MAX_BODIES * 10];
  const T dt = *P.dt;
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    *P.t_out = *P.t0 + dt;
    *P.dt_out = dt;
  }
  if (blockIdx.x == 0) {
    for (int q = threadIdx.x; q < P.nq; q += blockDim.x) {
      double s = 0.0;
      for (int st = 0; st < 3; ++st)
        for (int b = 0; b < P.nblocks; ++b) s += P.partials[((size_t)st * P.nblocks + b) * P.nq + q];
      tot[q] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      const double ddt = (double)dt;
      int bad = 0;
      for (int b = 0; b < P.nbody; ++b) {
        const double scale = -(P.h * P.h * P.h) / ddt;
        const double *r = tot + b * 9;
        double fx = r[0] * scale, fy = r[3] * scale, fz = r[6] * scale;
        double mx = r[4] * scale + r[7] * scale, my = r[1] * scale + r[8] * scale, mz = r[2] * scale + r[5] * scale;
        if (P.symmetry) {
          const double dy = P.moment_ref_y - P.y0;
          fx *= 2.0;
          fz *= 2.0;
          my *= 2.0;
          fy = 0.0;
          mx = -dy * fz;
          mz = dy * fx;
        }
        const double qa = 0.5 * P.ref_area;
        const double c6[6] = {fx / qa, fy / qa, fz / qa, mx / (qa * P.span_ref), my / (qa * P.length_ref),
                              mz / (qa * P.span_ref)};
        for (int c = 0; c < 6; ++c) {
          P.coeffs[b * 6 + c] = T(c6[c]);
          if (!(c6[c] == c6[c])) bad = 1;
        }
      }
      if (P.heat_rate) {
        const double sym = P.symmetry ? 2.0 : 1.0;
        const double scale = sym * P.h * P.h * P.h * P.pe / (double)dt;
        for (int b = 0; b < P.nbody; ++b) {
          double q = 0.0;
          for (int t = 0; t < P.n_tbody; ++t)
            if (P.t_index[t] == b) q += tot[P.nbody * 9 + t];
          q = q * scale + P.flux_rate[b] * sym;
          P.heat_rate[b] = T(q);
          if (!(q == q)) bad = 1;
        }
      }
      if (bad) atomicOr(P.status, 1);
    }
  }
  // p = psi_w / dt over the whole field
  const size_t n = P.ncell;
  const T rdt = T(1) / dt;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
    P.p[e] = P.p[e] * rdt;
}

// psi_w (in p) <- psi * wgt (first stage) or psi_w + wgt * psi
template <typename T>
__global__ void psi_accumulate_kernel(const T *__restrict__ psi, T *__restrict__ pw, size_t n, T wgt, int first) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
    pw[e] = first ? psi[e] * wgt : pw[e] + wgt * psi[e];
}

// --------------------------------------------------------------------------------------
// launchers
// --------------------------------------------------------------------------------------

template <typename T>
size_t stage_smem_bytes() {
  return sizeof(StageSmem<T>);
}

template <typename T>
cudaError_t launch_stage(const StageParams<T> &P, cudaStream_t s) {
  const size_t smem = sizeof(StageSmem<T>);
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(stage_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  dim3 grid((P.nx + TX - 1) / TX, (P.ny + TY - 1) / TY, (P.nz + P.zc - 1) / P.zc);
  stage_kernel<T><<<grid, dim3(TX, TY), smem, s>>>(P);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_absmax(const T *a, size_t n, unsigned long long *out, cudaStream_t s) {
  int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 8);
  absmax_kernel<T><<<blocks, 256, 0, s>>>(a, n, out);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_dt(const DtParams &P, cudaStream_t s) {
  dt_kernel<T><<<1, 1, 0, s>>>(P);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_outlet_sum(const T *u, const T *u0, int nx, int rows, double *sums, cudaStream_t s) {
  outlet_sum_kernel<T><<<1, 1024, 0, s>>>(u, u0, nx, rows, sums);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_outlet_corr(const double *sums_p, const double *sum_u0, const double *sum_inlet, const T *dt,
                               double a, double b, double inv_h, double inv_rows, T *corr, cudaStream_t s) {
  outlet_corr_kernel<T><<<1, 1, 0, s>>>(sums_p, sum_u0, sum_inlet, dt, a, b, inv_h, inv_rows, corr);
  return cudaGetLastError();
}

static inline int grid_for(size_t n) { return (int)std::max<size_t>(1, std::min<size_t>((n + 255) / 256, 148 * 16)); }

template <typename T>
cudaError_t launch_divergence(const T *u, const T *v, const T *w, int nx, int ny, int nz, int px, int py, int pz,
                              T inv_h, T *div, cudaStream_t s) {
  divergence_kernel<T><<<grid_for((size_t)nx * ny * nz), 256, 0, s>>>(u, v, w, nx, ny, nz, px, py, pz, inv_h, div);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_correct(const CorrectParams<T> &P, cudaStream_t s) {
  const size_t n = (size_t)P.nz * P.ny * (P.nx + 1) * 3 + (size_t)P.nx * P.ny;
  correct_kernel<T><<<grid_for(n), 256, 0, s>>>(P);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_smoke(const SmokeParams<T> &P, cudaStream_t s) {
  smoke_kernel<T><<<grid_for((size_t)P.nx * P.ny * P.nz), 256, 0, s>>>(P);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_finalize(const FinalizeParams<T> &P, cudaStream_t s) {
  finalize_kernel<T><<<grid_for(P.ncell), 256, 0, s>>>(P);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_psi_accumulate(const T *psi, T *pw, size_t n, T wgt, int first, cudaStream_t s) {
  psi_accumulate_kernel<T><<<grid_for(n), 256, 0, s>>>(psi, pw, n, wgt, first);
  return cudaGetLastError();
}

#define INSTANTIATE(T)                                                                                               \
  template size_t stage_smem_bytes<T>();                                                                             \
  template cudaError_t launch_stage<T>(const StageParams<T> &, cudaStream_t);                                       \
  template cudaError_t launch_absmax<T>(const T *, size_t, unsigned long long *, cudaStream_t);                     \
  template cudaError_t launch_dt<T>(const DtParams &, cudaStream_t);                                                \
  template cudaError_t launch_outlet_sum<T>(const T *, const T *, int, int, double *, cudaStream_t);                 \
  template cudaError_t launch_outlet_corr<T>(const double *, const double *, const double *, const T *, double,      \
                                             double, double, double, T *, cudaStream_t);                             \
  template cudaError_t launch_divergence<T>(const T *, const T *, const T *, int, int, int, int, int, int, T, T *,    \
                                            cudaStream_t);                                                           \
  template cudaError_t launch_correct<T>(const CorrectParams<T> &, cudaStream_t);                                   \
  template cudaError_t launch_smoke<T>(const SmokeParams<T> &, cudaStream_t);                                       \
  template cudaError_t launch_finalize<T>(const FinalizeParams<T> &, cudaStream_t);                                 \
  template cudaError_t launch_psi_accumulate<T>(const T *, T *, size_t, T, int, cudaStream_t);

INSTANTIATE(float)
INSTANTIATE(double)

}  // namespace aero
