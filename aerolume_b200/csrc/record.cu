// Per-step bookkeeping of the 3D solver on the device: Aerolume ns3d/solver.py:706-744
// (FlowSolver3D._record and _welford).
//
// record_kernel (one warp): the history ring row [t, the bodies' coefficients summed over
// the bodies] at slot hist_n mod capacity, the body coefficients kept for the caller, the
// physics-history row [t, extra...], the ring counter, and the averaging clock's pending time
// (+ dt, FP64).  welford_kernel: the time-weighted Welford update of up to five fields in one
// launch (blockIdx.y selects the field), 16-byte vector loads when every array of a field
// starts on a 16-byte boundary; each element is read once and its mean and second moment
// written once (the reference makes four passes per field).  welford_clock_kernel then moves
// the pending time into the total (the field kernel reads both before).
#include <cstdint>

#include "host_common.cuh"

namespace aero {
namespace rec {

constexpr int MAXF = 5;

template <typename T>
struct RecordParams {
  const T *t, *dt, *coeffs;  // coeffs (nbody, 6)
  int nbody;
  T *body_c;                 // (nbody, 6) or NULL
  T *hist;                   // (capacity, 7)
  long long capacity;
  long long *hist_n;
  const T *extra;            // (n_extra) or NULL
  int n_extra;
  T *phist;                  // (capacity, 1 + n_extra) or NULL
  double *pending;           // NULL: no averaging
};

template <typename T>
__global__ void record_kernel(const __grid_constant__ RecordParams<T> P) {
  aero::pdl_wait();
  const int lane = threadIdx.x;
  const long long n = *P.hist_n;
  const long long slot = ((n % P.capacity) + P.capacity) % P.capacity;  // as torch.remainder
  const T t = *P.t;
  if (lane < 7) {
    T v = t;
    if (lane > 0) {
      v = T(0);
      for (int b = 0; b < P.nbody; ++b) v = b == 0 ? P.coeffs[lane - 1] : v + P.coeffs[6 * b + lane - 1];
    }
    P.hist[slot * 7 + lane] = v;
  }
  if (P.body_c)
    for (int e = lane; e < 6 * P.nbody; e += 32) P.body_c[e] = P.coeffs[e];
  if (P.phist)
    for (int e = lane; e <= P.n_extra; e += 32) P.phist[slot * (1 + P.n_extra) + e] = e == 0 ? t : P.extra[e - 1];
  __syncwarp();
  if (lane == 0) {
    *P.hist_n = n + 1;
    if (P.pending) *P.pending += (double)*P.dt;
  }
}

template <typename T>
struct WelfordParams {
  const T *x[MAXF];
  T *mean[MAXF], *m2[MAXF];
  long long n[MAXF];
  int vec[MAXF];
  const double *pending, *time;
};

template <typename T>
__device__ __forceinline__ void welford_one(T x, T &m, T &s, T r, T wf) {
  const T d = x - m;
  m = m + d * r;
  s = s + (d * (x - m)) * wf;
}

template <typename T>
__global__ void __launch_bounds__(256) welford_kernel(const __grid_constant__ WelfordParams<T> P) {
  aero::pdl_wait();
  const int f = blockIdx.y;
  const double w = *P.pending;
  const T r = T(w / (*P.time + w));  // solver.py:736-737: the weight over the new total time
  const T wf = T(w);
  const T *x = P.x[f];
  T *mean = P.mean[f], *m2 = P.m2[f];
  const long long n = P.n[f];
  const long long stride = (long long)gridDim.x * blockDim.x, start = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long done = 0;
  if (P.vec[f]) {
    if constexpr (sizeof(T) == 4) {
      const long long nv = n / 4;
      for (long long e = start; e < nv; e += stride) {
        const float4 a = __ldg(reinterpret_cast<const float4 *>(x) + e);
        float4 m = reinterpret_cast<float4 *>(mean)[e], s = reinterpret_cast<float4 *>(m2)[e];
        welford_one<T>(a.x, m.x, s.x, r, wf);
        welford_one<T>(a.y, m.y, s.y, r, wf);
        welford_one<T>(a.z, m.z, s.z, r, wf);
        welford_one<T>(a.w, m.w, s.w, r, wf);
        reinterpret_cast<float4 *>(mean)[e] = m;
        reinterpret_cast<float4 *>(m2)[e] = s;
      }
      done = nv * 4;
    } else {
      const long long nv = n / 2;
      for (long long e = start; e < nv; e += stride) {
        const double2 a = __ldg(reinterpret_cast<const double2 *>(x) + e);
        double2 m = reinterpret_cast<double2 *>(mean)[e], s = reinterpret_cast<double2 *>(m2)[e];
        welford_one<T>(a.x, m.x, s.x, r, wf);
        welford_one<T>(a.y, m.y, s.y, r, wf);
        reinterpret_cast<double2 *>(mean)[e] = m;
        reinterpret_cast<double2 *>(m2)[e] = s;
      }
      done = nv * 2;
    }
  }
  for (long long e = done + start; e < n; e += stride) {
    T m = mean[e], s = m2[e];
    welford_one<T>(__ldg(x + e), m, s, r, wf);
    mean[e] = m;
    m2[e] = s;
  }
}

// time += pending; pending = 0 (solver.py:736, 744), after the field update has read both
__global__ void welford_clock_kernel(double *pending, double *time) {
  aero::pdl_wait();
  *time += *pending;
  *pending = 0.0;
}

}  // namespace rec
}  // namespace aero

namespace {

using aero_host::set_error;

bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

template <typename T>
int record_impl(const void *t, const void *dt, const void *coeffs, int nbody, void *body_c, void *hist,
                long long capacity, long long *hist_n, const void *extra, int n_extra, void *phist, double *pending,
                cudaStream_t s) {
  aero::rec::RecordParams<T> P{};
  P.t = static_cast<const T *>(t);
  P.dt = static_cast<const T *>(dt);
  P.coeffs = static_cast<const T *>(coeffs);
  P.nbody = nbody;
  P.body_c = static_cast<T *>(body_c);
  P.hist = static_cast<T *>(hist);
  P.capacity = capacity;
  P.hist_n = hist_n;
  P.extra = static_cast<const T *>(extra);
  P.n_extra = n_extra;
  P.phist = static_cast<T *>(phist);
  P.pending = pending;
  (void)aero::launch_k(aero::rec::record_kernel<T>, 1, 32, 0, s, P);
  AERO_CUDA_TRY(cudaGetLastError());
  return AERO_OK;
}

template <typename T>
int welford_impl(int nfield, const void *const *x, void *const *mean, void *const *m2, const int64_t *count,
                 double *pending, double *time, cudaStream_t s) {
  aero::rec::WelfordParams<T> P{};
  long long most = 0;
  for (int f = 0; f < nfield; ++f) {
    P.x[f] = static_cast<const T *>(x[f]);
    P.mean[f] = static_cast<T *>(mean[f]);
    P.m2[f] = static_cast<T *>(m2[f]);
    P.n[f] = count[f];
    P.vec[f] = aligned16(x[f]) && aligned16(mean[f]) && aligned16(m2[f]);
    most = std::max(most, (long long)count[f]);
  }
  P.pending = pending;
  P.time = time;
  // two 256-thread blocks per SM per field, each thread a few 16-byte words
  const long long per = 256LL * (16 / sizeof(T));
  const unsigned gx = (unsigned)std::max(1LL, std::min((most + per - 1) / per, 296LL));
  (void)aero::launch_k(aero::rec::welford_kernel<T>, dim3(gx, nfield), 256, 0, s, P);
  AERO_CUDA_TRY(cudaGetLastError());
  (void)aero::launch_k(aero::rec::welford_clock_kernel, 1, 1, 0, s, pending, time);
  AERO_CUDA_TRY(cudaGetLastError());
  return AERO_OK;
}

}  // namespace

extern "C" {

int aero_record_history(int32_t dtype, const void *t, const void *dt, const void *coeffs, int32_t nbody,
                        void *body_c, void *hist, int64_t capacity, int64_t *hist_n, const void *extra,
                        int32_t n_extra, void *phist, double *pending, void *stream) {
  if (dtype != AERO_F32 && dtype != AERO_F64) return set_error(AERO_EINVAL, "dtype must be float32 or float64");
  if (!t || !hist || !hist_n || capacity < 1) return set_error(AERO_EINVAL, "missing history ring");
  if (nbody < 0 || (nbody > 0 && !coeffs)) return set_error(AERO_EINVAL, "missing body coefficients");
  if (n_extra < 0 || (phist && n_extra > 0 && !extra)) return set_error(AERO_EINVAL, "missing physics-history row");
  if (pending && !dt) return set_error(AERO_EINVAL, "the averaging clock needs dt");
  auto s = static_cast<cudaStream_t>(stream);
  return dtype == AERO_F64 ? record_impl<double>(t, dt, coeffs, nbody, body_c, hist, capacity, (long long *)hist_n,
                                                 extra, n_extra, phist, pending, s)
                           : record_impl<float>(t, dt, coeffs, nbody, body_c, hist, capacity, (long long *)hist_n,
                                                extra, n_extra, phist, pending, s);
}

int aero_welford(int32_t dtype, int32_t nfield, const void *const *x, void *const *mean, void *const *m2,
                 const int64_t *count, double *pending, double *time, void *stream) {
  if (dtype != AERO_F32 && dtype != AERO_F64) return set_error(AERO_EINVAL, "dtype must be float32 or float64");
  if (nfield < 1 || nfield > aero::rec::MAXF) return set_error(AERO_EINVAL, "1 to 5 fields");
  if (!x || !mean || !m2 || !count || !pending || !time) return set_error(AERO_EINVAL, "null argument");
  for (int f = 0; f < nfield; ++f)
    if (count[f] < 0 || (count[f] > 0 && (!x[f] || !mean[f] || !m2[f])))
      return set_error(AERO_EINVAL, "missing field buffers");
  auto s = static_cast<cudaStream_t>(stream);
  return dtype == AERO_F64 ? welford_impl<double>(nfield, x, mean, m2, count, pending, time, s)
                           : welford_impl<float>(nfield, x, mean, m2, count, pending, time, s);
}

}  // extern "C"
