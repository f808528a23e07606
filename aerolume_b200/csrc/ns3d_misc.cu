// Small kernels of the 3D step: maxima, time step, outlet sums, divergence, gradient
// correction, smoke, partial-sum reduction and the end of the step.
//
// Arithmetic follows Aerolume ns3d/core.py:577-678, 875-883, physics.py:713-742, 1230-1262
// and dye.py:232-312 operation by operation.
#include "ns3d.cuh"
#include "stencil.cuh"

namespace aero {

// --------------------------------------------------------------------------------------
// pre-pass maxima, time step, outlet sums
// --------------------------------------------------------------------------------------

// max |a| over an array: warp shuffles, then one atomic per block
template <typename T>
__global__ void absmax_kernel(const T *__restrict__ a, size_t n, unsigned long long *out) {
  aero::pdl_wait();
  T m = T(0);
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const T v = fabs(a[e]);
    m = (v > m || v != v) ? v : m;
  }
  block_max_atomic<T>(m, out);
}

// max |a| of up to three arrays in one launch (blockIdx.y selects the array), 16-byte vector
// loads when every array starts on a 16-byte boundary
template <typename T>
__global__ void __launch_bounds__(512) absmax_multi_kernel(const MaxJobs<T> J) {
  aero::pdl_wait();
  const MaxJob<T> &q = J.job[blockIdx.y];
  const size_t stride = (size_t)gridDim.x * blockDim.x, start = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  T m = T(0);
  auto take = [&](T x) {
    const T v = fabs(x);
    m = (v > m || v != v) ? v : m;
  };
  size_t done = 0;
  if (J.vec) {
    if constexpr (sizeof(T) == 4) {
      const float4 *a4 = reinterpret_cast<const float4 *>(q.a);
      const size_t nv = q.n / 4;
      for (size_t e = start; e < nv; e += stride) {
        const float4 x = __ldg(a4 + e);
        take(x.x), take(x.y), take(x.z), take(x.w);
      }
      done = nv * 4;
    } else {
      const double2 *a2 = reinterpret_cast<const double2 *>(q.a);
      const size_t nv = q.n / 2;
      for (size_t e = start; e < nv; e += stride) {
        const double2 x = __ldg(a2 + e);
        take(x.x), take(x.y);
      }
      done = nv * 2;
    }
  }
  for (size_t e = done + start; e < q.n; e += stride) take(__ldg(q.a + e));
  block_max_atomic<T>(m, q.out);
}

// u0 (rows of nx + 1) into the stage-start buffer with a 16-byte row pitch, with max |u0|.
// A fixed grid strides over the rows (one max atomic per block, not per row); the thread of
// x = nx - 1 also copies the last face, x = nx.
template <typename T>
__global__ void copy_u_kernel(const T *__restrict__ u, T *__restrict__ out, int nx, int ny, int nz, int pitch,
                              unsigned long long *mx) {
  aero::pdl_wait();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int rows = ny * nz;
  T m = T(0);
  if (i < nx) {
    for (int r = blockIdx.y * blockDim.y + threadIdx.y; r < rows; r += gridDim.y * blockDim.y) {
      const T *src = u + (size_t)r * (nx + 1);
      T *dst = out + (size_t)r * pitch;
      const T a = src[i];
      if (AERO_IN((size_t)r * pitch + i, (long long)rows * pitch, 201)) dst[i] = a;
      T ma = fabs(a);
      if (i == nx - 1) {
        const T b = src[nx];
        if (AERO_IN((size_t)r * pitch + nx, (long long)rows * pitch, 202)) dst[nx] = b;
        const T fb = fabs(b);
        ma = (fb > ma || fb != fb) ? fb : ma;
      }
      m = (ma > m || ma != ma) ? ma : m;
    }
  }
  if (mx) block_max_atomic<T>(m, mx);
}

// One block per fan (physics.py:922-942): the disc-averaged axial velocity of the step-start
// state, sum(m_u u) + sum(m_v v) + sum(m_w w) over the fan's faces (each sum in FP64 in a
// fixed order, rounded to the field type), then the PI update of a velocity-mode fan's thrust
// T <- clamp(T + kP (e - e_prev) + kI dt e, -tmax, tmax) with e = target - ud, and the swirl
// amplitude swirl ud |ud|.
template <typename T>
__global__ void __launch_bounds__(1024) fan_begin_kernel(const __grid_constant__ FanBeginParams<T> P) {
  aero::pdl_wait();
  __shared__ double red[3][32];
  const auto &F = P.fan[blockIdx.x];
  const int nx = P.nx, ny = P.ny;
  const int k0 = F.win[0], j0 = F.win[2], i0 = F.win[4];
  const int wz = F.win[1] - k0, wy = F.win[3] - j0, wx = F.win[5] - i0;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int c = 0; c < 3; ++c) {
    // face window of component c: (wz + [c == 2]) x (wy + [c == 1]) x (wx + [c == 0]); the
    // faces spread over all threads with 32-bit index arithmetic, four loads in flight each
    const int ez = wz + (c == 2), ey = wy + (c == 1), ex = wx + (c == 0);
    const T *vel = c == 0 ? P.u0 : (c == 1 ? P.v0 : P.w0);
    const int rowlen = c == 0 ? nx + 1 : nx, rows = c == 1 ? ny + 1 : ny;
    const int n = ez * ey * ex;
    double acc = 0.0;
#pragma unroll 4
    for (int e = tid; e < n; e += blockDim.x) {
      const int x = e % ex, r = e / ex;
      const int y = r % ey, z = r / ey;
      acc += (double)F.m[c][e] * (double)vel[((size_t)(k0 + z) * rows + (j0 + y)) * rowlen + (i0 + x)];
    }
    acc = warp_sum(acc);
    if (lane == 0) red[c][warp] = acc;
  }
  __syncthreads();
  if (tid == 0) {
    T part[3];
    for (int c = 0; c < 3; ++c) {
      double t = 0.0;
      for (int w = 0; w < (int)(blockDim.x / 32); ++w) t += red[c][w];
      part[c] = T(t);
    }
    const T ud = (part[0] + part[1]) + part[2];
    *F.ud = ud;
    const T e = T(F.target) - ud;
    if (F.velocity_mode) {
      T nw = (*F.thrust + T(F.kp) * (e - *F.e_prev)) + (T(F.ki) * *P.dt) * e;
      const T tm = T(F.tmax);
      nw = nw > tm ? tm : nw;  // NaN passes through, as torch.minimum / maximum
      nw = nw < -tm ? -tm : nw;
      *F.thrust = nw;
      *F.e_prev = e;
    }
    if (P.any_swirl) *F.swirl_amp = (T(F.swirl) * ud) * fabs(ud);
  }
}

// One thread: the step's dt from the maxima (core.py:637-646, physics.py:723-742, 1230-1262),
// rounded through the field type as the reference computes it.
template <typename T>
__global__ void dt_kernel(const DtParams P) {
  aero::pdl_wait();
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
    if (P.u_floor > 0.0) {  // the sources' speed scale bounds dt from rest (physics.py:1239-1241)
      const T cap = T(P.cfl * P.h / P.u_floor);
      dt = dt > cap ? cap : dt;
      umax = umax < T(P.u_floor) ? T(P.u_floor) : umax;
    }
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
    if (P.pid) {
      // PID control towards pid_target x the limit on e = log(want / dt_prev)
      // (physics.py:1161-1173): gains (kI, kP, kD) = (0.3, 0.4, 0.05), the growth factor
      // within [0.5, 1.2], never above the limit; the first step takes the target itself
      T *dprev = static_cast<T *>(P.pid_dt_prev), *e1p = static_cast<T *>(P.pid_e1), *e2p = static_cast<T *>(P.pid_e2);
      const T want = dt * T(P.pid_target);
      const bool first = *dprev <= T(0);
      const T prev = first ? want : *dprev;
      const T e = log(want / prev);
      const T e1 = *e1p, e2 = *e2p;
      T fac = exp((T(0.3) * e + T(0.4) * (e - e1)) + T(0.05) * ((e - T(2) * e1) + e2));
      fac = fac < T(0.5) ? T(0.5) : (fac > T(1.2) ? T(1.2) : fac);
      const T d = first ? want : prev * fac;
      dt = (d < dt || d != d) ? d : dt;
      *e2p = e1;
      *e1p = first ? T(0) : e;
      *dprev = dt;
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
  aero::pdl_wait();
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
// Outlet correction of a stage by linearity (core.py:281-297): the stage value's outlet sum is
// (1 - a) sum up[nx] + a sum u0[nx] + b dt / h (sum up[nx-1] - sum up[nx]); every sum is the
// in-order total of the plane-sum kernel's per-block partials.
template <typename T>
__global__ void outlet_corr_kernel(const double *p_out, const double *p_in, const double *p_u0, const double *p_inlet,
                                   int parts, const T *dt, double a, double bscale, double inv_h, double inv_rows,
                                   double source, T *corr) {
  aero::pdl_wait();
  double so = 0.0, si = 0.0, s0 = 0.0, sn = 0.0;
  for (int q = 0; q < parts; ++q) {
    so += p_out[q];
    si += p_in[q];
    s0 += p_u0[q];
    sn += p_inlet[q];
  }
  const double bdt = (double)(T(bscale) * *dt);
  const double out = (1.0 - a) * so + a * s0 + bdt * inv_h * (si - so);
  T c = T((sn - out) * inv_rows);
  // the ports' net mass flux leaves through the outlet too (core.py:294-296)
  if (source != 0.0) c = c + T(source) * T(inv_rows);
  *corr = c;
}

// div -= m on the cells of each port's window, one port after the other as the reference
// applies them (physics.py:1043-1047); one block, the windows are small
template <typename T>
__global__ void port_continuity_kernel(T *div, int nx, int ny, int nport, PortParamsBlock<T> P) {
  aero::pdl_wait();
  for (int q = 0; q < nport; ++q) {
    const PortSource<T> &Q = P.port[q];
    const int wz = Q.win[1] - Q.win[0], wy = Q.win[3] - Q.win[2], wx = Q.win[5] - Q.win[4];
    const size_t n = (size_t)wz * wy * wx;
    for (size_t e = threadIdx.x; e < n; e += blockDim.x) {
      const int x = (int)(e % wx), y = (int)((e / wx) % wy), z = (int)(e / ((size_t)wx * wy));
      T &d = div[((size_t)(Q.win[0] + z) * ny + (Q.win[2] + y)) * nx + (Q.win[4] + x)];
      d = d - Q.m[e];
    }
    __syncthreads();
  }
}

// --------------------------------------------------------------------------------------
// projection: divergence and gradient correction (core.py:577-601)
// --------------------------------------------------------------------------------------

template <typename T>
__global__ void divergence_kernel(const T *__restrict__ u, const T *__restrict__ v, const T *__restrict__ w, int nx,
                                  int ny, int nz, int px, int py, int pz, T inv_h, T *__restrict__ div) {
  aero::pdl_wait();
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
  if (i >= nx) return;
  const size_t ru = ((size_t)k * ny + j) * (nx + 1);
  const T ur = (px && i == nx - 1) ? u[ru] : u[ru + i + 1];
  const T ul = u[ru + i];
  const size_t rv = (size_t)k * (ny + 1) * nx;
  const T vr = (py && j == ny - 1) ? v[rv + i] : v[rv + (size_t)(j + 1) * nx + i];
  const T vl = v[rv + (size_t)j * nx + i];
  const T wr = (pz && k == nz - 1) ? w[(size_t)j * nx + i] : w[((size_t)(k + 1) * ny + j) * nx + i];
  const T wl = w[((size_t)k * ny + j) * nx + i];
  div[((size_t)k * ny + j) * nx + i] = ((ur - ul) + (vr - vl) + (wr - wl)) * inv_h;
}

// u <- uh - grad psi on every face; boundary-normal faces keep uh (non-periodic), periodic
// duplicate faces equal face 0.
template <typename T>
__global__ void correct_kernel(const CorrectParams<T> P) {
  aero::pdl_wait();
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  const int i0 = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
  const T inv = P.inv_h;
  // u faces (k, j, i): x = 0 .. nx; the thread of x = nx - 1 also does x = nx
  const int ilast = (i0 < nx && j < ny && k < nz) ? (i0 == nx - 1 ? nx : i0) : i0 - 1;
  for (int i = i0; i <= ilast; ++i) {
    const size_t e = ((size_t)k * ny + j) * (nx + 1) + i;
    const size_t c = ((size_t)k * ny + j) * nx;
    T val;
    if (P.px) {
      const int ii = (i == nx) ? 0 : i;
      const int il = (ii == 0) ? nx - 1 : ii - 1;
      val = P.uh[e - i + ii] - (P.psi[c + ii] - P.psi[c + il]) * inv;
    } else if (i == 0 || i == nx) {
      val = P.uh[e];
    } else {
      val = P.uh[e] - (P.psi[c + i] - P.psi[c + i - 1]) * inv;
    }
    P.u[((size_t)k * ny + j) * P.pu_out + i] = val;
  }
  const int i = i0;
  if (i < nx && j <= ny && k < nz) {  // v face (k, j, i)
    const size_t e = ((size_t)k * (ny + 1) + j) * nx + i;
    T val;
    if (P.py) {
      const int jj = (j == ny) ? 0 : j;
      const int jl = (jj == 0) ? ny - 1 : jj - 1;
      val = P.vh[((size_t)k * (ny + 1) + jj) * nx + i] -
            (P.psi[((size_t)k * ny + jj) * nx + i] - P.psi[((size_t)k * ny + jl) * nx + i]) * inv;
    } else if (j == 0 || j == ny) {
      val = P.vh[e];
    } else {
      val = P.vh[e] - (P.psi[((size_t)k * ny + j) * nx + i] - P.psi[((size_t)k * ny + j - 1) * nx + i]) * inv;
    }
    P.v[e] = val;
  }
  if (i < nx && j < ny && k <= nz) {  // w face (k, j, i)
    const size_t e = ((size_t)k * ny + j) * nx + i;
    T val;
    if (P.pz) {
      const int kk = (k == nz) ? 0 : k;
      const int kl = (kk == 0) ? nz - 1 : kk - 1;
      val = P.wh[((size_t)kk * ny + j) * nx + i] -
            (P.psi[((size_t)kk * ny + j) * nx + i] - P.psi[((size_t)kl * ny + j) * nx + i]) * inv;
    } else if (k == 0 || k == nz) {
      val = P.wh[e];
    } else {
      val = P.wh[e] - (P.psi[e] - P.psi[e - (size_t)ny * nx]) * inv;
    }
    P.w[e] = val;
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

// Smoke update (dye.py:265-312 advect_dye3d, solver.py:646-684): a 32 x 8 column of cells
// marches up SMOKE_ZC planes.  Each plane of dye, with two ghost / halo cells on each side in
// x and y, is loaded once into a 6-plane ring in shared memory (the plane three ahead is
// fetched into registers while the current plane is computed), so every cell reads its
// x / y / z stencil from shared memory and one barrier separates the planes.
constexpr int SMOKE_TX = 32, SMOKE_TY = 8, SMOKE_ZC = 16;
constexpr int SMOKE_PX = SMOKE_TX + 4, SMOKE_PY = SMOKE_TY + 4, SMOKE_PPL = SMOKE_PX * SMOKE_PY;  // 432
constexpr int SMOKE_NSLOT = 6;
constexpr int SMOKE_LOADS = (SMOKE_PPL + SMOKE_TX * SMOKE_TY - 1) / (SMOKE_TX * SMOKE_TY);      // 2

template <typename T>
__global__ void __launch_bounds__(SMOKE_TX *SMOKE_TY, sizeof(T) == 4 ? 4 : 1) smoke_kernel(const __grid_constant__ SmokeParams<T> P) {
  aero::pdl_wait();
  __shared__ T ring[SMOKE_NSLOT][SMOKE_PPL];
  const int nx = P.nx, ny = P.ny, nz = P.nz;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * SMOKE_TX + tx;
  const int i0 = blockIdx.x * SMOKE_TX, j0 = blockIdx.y * SMOKE_TY;
  const int kb = blockIdx.z * SMOKE_ZC, ke = min(kb + SMOKE_ZC, nz);
  const T dt = *P.dt;
  const T kk = dt * P.inv_h;
  const T t = P.t_new ? *P.t_new : *P.t0 + dt;
  const T on = (fmod(t, T(P.pulse_period)) < T(P.pulse_on)) ? T(1) : T(0);
  auto slot = [&](int k) { return (k - kb + 2 + 2 * SMOKE_NSLOT) % SMOKE_NSLOT; };  // k >= kb - 2
  // this thread's share of plane k (tile entry e = tid + q * 256 <-> (j0 - 2 + e / 36, i0 - 2 + e % 36))
  auto fetch = [&](int k, T *r) {
#pragma unroll
    for (int q = 0; q < SMOKE_LOADS; ++q) {
      const int e = tid + q * SMOKE_TX * SMOKE_TY;
      if (e < SMOKE_PPL) {
        // entries beyond the second ghost layer (x > nx + 1, y > ny + 1) feed no cell
        const int ly = e / SMOKE_PX, lx = e - ly * SMOKE_PX;
        const int gj = j0 - 2 + ly, gi = i0 - 2 + lx;
        r[q] = (gi <= nx + 1 && gj <= ny + 1) ? dye_at<T>(P.c0, nz, ny, nx, P.px, P.py, P.pz, k, gj, gi) : T(0);
      }
    }
  };
  auto store = [&](int k, const T *r) {
    T *dst = ring[slot(k)];
#pragma unroll
    for (int q = 0; q < SMOKE_LOADS; ++q) {
      const int e = tid + q * SMOKE_TX * SMOKE_TY;
      if (e < SMOKE_PPL) dst[e] = r[q];
    }
  };
  T r[SMOKE_LOADS];
  for (int k = kb - 2; k <= min(kb + 2, ke + 1); ++k) {
    fetch(k, r);
    store(k, r);
  }
  __syncthreads();
  const int i = i0 + tx, j = j0 + ty;
  const bool mine = i < nx && j < ny;
  const int cx = tx + 2, cy = ty + 2, ce = cy * SMOKE_PX + cx;
  T wlo = (mine && kb < nz) ? __ldg(P.w + ((size_t)kb * ny + j) * nx + i) : T(0);
  for (int k = kb; k < ke; ++k) {
    const bool more = k + 3 <= ke + 1;  // plane k + 3 is needed by the plane k + 1 stencil
    if (more) fetch(k + 3, r);
    if (mine) {
      const T *S0 = ring[slot(k)];
      const T c = S0[ce];
      const T ul = __ldg(P.u + ((size_t)k * ny + j) * (nx + 1) + i);
      const T ur = __ldg(P.u + ((size_t)k * ny + j) * (nx + 1) + i + 1);
      const T vl = __ldg(P.v + ((size_t)k * (ny + 1) + j) * nx + i);
      const T vr = __ldg(P.v + ((size_t)k * (ny + 1) + j + 1) * nx + i);
      const T whi = __ldg(P.w + ((size_t)(k + 1) * ny + j) * nx + i);
      const T fx0 = muscl_flux<T>(S0[ce - 2], S0[ce - 1], c, S0[ce + 1], ul);
      const T fx1 = muscl_flux<T>(S0[ce - 1], c, S0[ce + 1], S0[ce + 2], ur);
      const T fy0 = muscl_flux<T>(S0[ce - 2 * SMOKE_PX], S0[ce - SMOKE_PX], c, S0[ce + SMOKE_PX], vl);
      const T fy1 = muscl_flux<T>(S0[ce - SMOKE_PX], c, S0[ce + SMOKE_PX], S0[ce + 2 * SMOKE_PX], vr);
      const T zm2 = ring[slot(k - 2)][ce], zm1 = ring[slot(k - 1)][ce];
      const T zp1 = ring[slot(k + 1)][ce], zp2 = ring[slot(k + 2)][ce];
      const T fz0 = muscl_flux<T>(zm2, zm1, c, zp1, wlo);
      const T fz1 = muscl_flux<T>(zm1, c, zp1, zp2, whi);
      wlo = whi;
      T v = c - kk * (((fx1 - fx0) + (fy1 - fy0)) + (fz1 - fz0));
      v = v > T(1) ? T(1) : v;
      v = v < T(1e-8) ? T(0) : v;
      if (P.chi_c && k >= P.win[0] && k < P.win[1] && j >= P.win[2] && j < P.win[3] && i >= P.win[4] &&
          i < P.win[5]) {
        const T chi = P.chi_c[((size_t)(k - P.win[0]) * (P.win[3] - P.win[2]) + (j - P.win[2])) *
                                  (P.win[5] - P.win[4]) +
                              (i - P.win[4])];
        if (chi > T(0.5)) v = T(0);
      }
      if (P.weight && k >= P.dwin[0] && k < P.dwin[1] && j >= P.dwin[2] && j < P.dwin[3] && i >= P.dwin[4] &&
          i < P.dwin[5]) {
        const T wgt = P.weight[((size_t)(k - P.dwin[0]) * (P.dwin[3] - P.dwin[2]) + (j - P.dwin[2])) *
                                   (P.dwin[5] - P.dwin[4]) +
                               (i - P.dwin[4])];
        v = v + wgt * on * (T(1) - v);
      }
      // painted solids hold no smoke, after the sources (ns3d/solver.py:642-644)
      if (P.paint_c && P.paint_c[((size_t)k * ny + j) * nx + i] > T(0.5)) v = T(0);
      P.c[((size_t)k * ny + j) * nx + i] = v;
    }
    // plane k + 3 goes into the slot of plane k - 3, which no thread reads from here on
    if (more) store(k + 3, r);
    __syncthreads();
  }
}

// --------------------------------------------------------------------------------------
// end of step: p, coefficients, heat rates, t and dt (core.py:653-678, 875-883,
// physics.py:713-721)
// --------------------------------------------------------------------------------------

// tot[q] = sum over stages and blocks of partials[stage][block][q]: one block per q, a
// fixed thread-to-term mapping and tree, so the sum is the same on every run.
__global__ void partials_reduce_kernel(const double *__restrict__ partials, int nblocks, int nq, double *tot) {
  aero::pdl_wait();
  const int q = blockIdx.x;
  double s = 0.0;
  for (int e = threadIdx.x; e < 3 * nblocks; e += blockDim.x) s += partials[(size_t)e * nq + q];
  s = warp_sum(s);
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    tot[q] = t;
  }
}

// Diagnostics: sum of squares of an array (physics.py:1303-1305 (div * div).sum()), in FP64 with
// a fixed block count and thread-to-element mapping, then one block adding the block sums in
// order: the same value on every run.
template <typename T>
__global__ void sumsq_partial_kernel(const T *__restrict__ a, size_t n, double *__restrict__ part) {
  aero::pdl_wait();
  double acc = 0.0;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const double x = (double)a[e];
    acc += x * x;
  }
  acc = warp_sum(acc);
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    part[blockIdx.x] = t;
  }
}

template <typename T>
__global__ void sumsq_final_kernel(const double *__restrict__ part, int nparts, T *out) {
  aero::pdl_wait();
  double acc = 0.0;
  for (int q = threadIdx.x; q < nparts; q += blockDim.x) acc += part[q];
  acc = warp_sum(acc);
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    *out = T(t);
  }
}

template <typename T>
__global__ void finalize_kernel(const FinalizeParams<T> P) {
  aero::pdl_wait();
  const T dt = *P.dt;
  *P.t_out = *P.t0 + dt;
  *P.dt_out = dt;
  const double *tot = P.tot;
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
    const double scale = sym * P.h * P.h * P.h * P.pe / ddt;
    for (int b = 0; b < P.nbody; ++b) {
      double q = 0.0;
      for (int t = 0; t < P.n_tbody; ++t)
        if (P.t_index[t] == b) q += tot[P.nbody * 9 + t];
      q = q * scale + P.flux_rate[b] * sym;
      P.heat_rate[b] = T(q);
      if (!(q == q)) bad = 1;
    }
  }
  if (bad || !(dt == dt)) atomicOr(P.status, 1);
}

// psi_w (in p) <- psi * wgt (mode 0), psi_w + wgt * psi (mode 1), or, at the last stage,
// (psi_w + wgt * psi) * (1 / dt): the step-averaged pressure (core.py:874-875, mode 2)
template <typename T>
__global__ void psi_accumulate_kernel(const T *__restrict__ psi, T *__restrict__ pw, size_t n, T wgt, int mode,
                                      const T *__restrict__ dt) {
  aero::pdl_wait();
  const T rdt = mode == 2 ? T(1) / *dt : T(1);
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    if (mode == 0) {
      pw[e] = psi[e] * wgt;
    } else {
      const T s = pw[e] + wgt * psi[e];
      pw[e] = mode == 2 ? s * rdt : s;
    }
  }
}

// --------------------------------------------------------------------------------------
// launchers
// --------------------------------------------------------------------------------------

template <typename T>
cudaError_t launch_absmax(const T *a, size_t n, unsigned long long *out, cudaStream_t s) {
  int blocks = (int)std::min<size_t>((n + 1023) / 1024, 148 * 2);
  (void)aero::launch_k(absmax_kernel<T>, blocks, 1024, 0, s, a, n, out);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_absmax_multi(const MaxJobs<T> &J, int njobs, cudaStream_t s) {
  if (njobs <= 0) return cudaSuccess;
  size_t n = 0;
  MaxJobs<T> K = J;
  K.vec = 1;
  for (int q = 0; q < njobs; ++q) {
    n = std::max(n, J.job[q].n);
    if (reinterpret_cast<uintptr_t>(J.job[q].a) % 16) K.vec = 0;
  }
  const size_t per = K.vec ? 512 * (16 / sizeof(T)) : 512;
  const int blocks = (int)std::max<size_t>(1, std::min<size_t>((n + per - 1) / per, 148 * 4 / (size_t)njobs));
  (void)aero::launch_k(absmax_multi_kernel<T>, dim3(blocks, njobs), 512, 0, s, K);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_copy_u(const T *u, T *out, int nx, int ny, int nz, int pitch, unsigned long long *mx,
                          cudaStream_t s) {
  const unsigned gx = (unsigned)((nx + 127) / 128);
  const unsigned rows = (unsigned)ny * (unsigned)nz;
  const unsigned gy = std::max(1u, std::min((rows + 1) / 2, 2368u / gx));
  (void)aero::launch_k(copy_u_kernel<T>, dim3(gx, gy), dim3(128, 2), 0, s, u, out, nx, ny, nz, pitch, mx);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_fan_begin(const FanBeginParams<T> &P, cudaStream_t s) {
  if (P.nfan <= 0) return cudaSuccess;
  (void)aero::launch_k(fan_begin_kernel<T>, P.nfan, 1024, 0, s, P);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_dt(const DtParams &P, cudaStream_t s) {
  (void)aero::launch_k(dt_kernel<T>, 1, 1, 0, s, P);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_outlet_sum(const T *u, const T *u0, int nx, int rows, double *sums, cudaStream_t s) {
  (void)aero::launch_k(outlet_sum_kernel<T>, 1, 1024, 0, s, u, u0, nx, rows, sums);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_outlet_corr(const double *p_out, const double *p_in, const double *p_u0, const double *p_inlet,
                               int parts, const T *dt, double a, double b, double inv_h, double inv_rows,
                               double source, T *corr, cudaStream_t s) {
  (void)aero::launch_k(outlet_corr_kernel<T>, 1, 1, 0, s, p_out, p_in, p_u0, p_inlet, parts, dt, a, b, inv_h, inv_rows, source, corr);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_port_continuity(T *div, int nx, int ny, int nport, const PortSource<T> *ports, cudaStream_t s) {
  if (nport <= 0) return cudaSuccess;
  PortParamsBlock<T> P{};
  for (int q = 0; q < nport; ++q) P.port[q] = ports[q];
  (void)aero::launch_k(port_continuity_kernel<T>, 1, 1024, 0, s, div, nx, ny, nport, P);
  return cudaGetLastError();
}

static inline int grid_for(size_t n) { return (int)std::max<size_t>(1, std::min<size_t>((n + 255) / 256, 148 * 16)); }

template <typename T>
cudaError_t launch_divergence(const T *u, const T *v, const T *w, int nx, int ny, int nz, int px, int py, int pz,
                              T inv_h, T *div, cudaStream_t s) {
  (void)aero::launch_k(divergence_kernel<T>, dim3((nx + 127) / 128, ny, nz), 128, 0, s, u, v, w, nx, ny, nz, px, py, pz, inv_h, div);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_sumsq(const T *a, size_t n, double *part, T *out, cudaStream_t s) {
  (void)aero::launch_k(sumsq_partial_kernel<T>, SUMSQ_PARTS, 256, 0, s, a, n, part);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  (void)aero::launch_k(sumsq_final_kernel<T>, 1, 256, 0, s, (const double *)part, SUMSQ_PARTS, out);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_correct(const CorrectParams<T> &P, cudaStream_t s) {
  (void)aero::launch_k(correct_kernel<T>, dim3((P.nx + 127) / 128, P.ny + 1, P.nz + 1), 128, 0, s, P);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_smoke(const SmokeParams<T> &P, cudaStream_t s) {
  const dim3 grid((P.nx + SMOKE_TX - 1) / SMOKE_TX, (P.ny + SMOKE_TY - 1) / SMOKE_TY, (P.nz + SMOKE_ZC - 1) / SMOKE_ZC);
  (void)aero::launch_k(smoke_kernel<T>, grid, dim3(SMOKE_TX, SMOKE_TY), 0, s, P);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_finalize(const FinalizeParams<T> &P, cudaStream_t s) {
  if (P.nq > 0) {
    (void)aero::launch_k(partials_reduce_kernel, P.nq, 256, 0, s, P.partials, P.nblocks, P.nq, P.tot);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  (void)aero::launch_k(finalize_kernel<T>, 1, 1, 0, s, P);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_psi_accumulate(const T *psi, T *pw, size_t n, T wgt, int mode, const T *dt, cudaStream_t s) {
  (void)aero::launch_k(psi_accumulate_kernel<T>, grid_for(n), 256, 0, s, psi, pw, n, wgt, mode, dt);
  return cudaGetLastError();
}

#define INSTANTIATE(T)                                                                                               \
  template cudaError_t launch_absmax<T>(const T *, size_t, unsigned long long *, cudaStream_t);                     \
  template cudaError_t launch_absmax_multi<T>(const MaxJobs<T> &, int, cudaStream_t);                              \
  template cudaError_t launch_dt<T>(const DtParams &, cudaStream_t);                                                \
  template cudaError_t launch_fan_begin<T>(const FanBeginParams<T> &, cudaStream_t);                                \
  template cudaError_t launch_copy_u<T>(const T *, T *, int, int, int, int, unsigned long long *, cudaStream_t);                                                \
  template cudaError_t launch_outlet_sum<T>(const T *, const T *, int, int, double *, cudaStream_t);                 \
  template cudaError_t launch_outlet_corr<T>(const double *, const double *, const double *, const double *, int,  \
                                             const T *, double, double, double, double, double, T *, cudaStream_t); \
  template cudaError_t launch_port_continuity<T>(T *, int, int, int, const PortSource<T> *, cudaStream_t);           \
  template cudaError_t launch_divergence<T>(const T *, const T *, const T *, int, int, int, int, int, int, T, T *,    \
                                            cudaStream_t);                                                           \
  template cudaError_t launch_correct<T>(const CorrectParams<T> &, cudaStream_t);                                   \
  template cudaError_t launch_sumsq<T>(const T *, size_t, double *, T *, cudaStream_t);                              \
  template cudaError_t launch_smoke<T>(const SmokeParams<T> &, cudaStream_t);                                       \
  template cudaError_t launch_finalize<T>(const FinalizeParams<T> &, cudaStream_t);                                 \
  template cudaError_t launch_psi_accumulate<T>(const T *, T *, size_t, T, int, const T *, cudaStream_t);

INSTANTIATE(float)
INSTANTIATE(double)

}  // namespace aero
