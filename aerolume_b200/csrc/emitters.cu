// Smoke emitters on the device: Aerolume ns3d/emitters.py:83-87 (release_switch) and 200-210
// (apply_smoke_sources).  One launch per emitter, in order (windows of one channel may
// overlap): every thread of the window evaluates the release switch from the device
// parameters [rate, start, stop, period, t_on] and the device time, and relaxes its cell
// towards the rate, c += w on (rate - c).  The float remainder is torch's, exact through fmod.
#include <cstdint>

#include "host_common.cuh"

namespace aero {
namespace emit {

template <typename T>
struct EmitParams {
  T *c;                      // the channel (nz, ny, nx)
  int ny, nx;
  int win[6];
  const T *w;                // weights on the window (wz, wy, wx)
  const T *p;                // [rate, start, stop, period, t_on]
  const T *t;
};

template <typename T>
__global__ void __launch_bounds__(256) emit_kernel(const __grid_constant__ EmitParams<T> P) {
  aero::pdl_wait();
  const int wx = P.win[5] - P.win[4], wy = P.win[3] - P.win[2], wz = P.win[1] - P.win[0];
  const long long n = (long long)wx * wy * wz;
  const T t = *P.t;
  const T since = t - P.p[1];
  T rem = fmod(since, P.p[3]);
  if (rem != T(0) && ((P.p[3] < T(0)) != (rem < T(0)))) rem = rem + P.p[3];
  const T on = (since >= T(0) && t < P.p[2] && rem < P.p[4]) ? T(1) : T(0);
  const T rate = P.p[0];
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(e % wx);
    const long long r = e / wx;
    const int y = (int)(r % wy), z = (int)(r / wy);
    T *cell = P.c + ((size_t)(P.win[0] + z) * P.ny + (P.win[2] + y)) * P.nx + (P.win[4] + x);
    const T c = *cell;
    *cell = c + (P.w[e] * on) * (rate - c);
  }
}

}  // namespace emit
}  // namespace aero

namespace {

using aero_host::set_error;

template <typename T>
int emit_impl(int nz, int ny, int nx, void *const *channels, int nchannel, const AeroSmokeEmitter *em, int nemit,
              const void *t, cudaStream_t s) {
  for (int q = 0; q < nemit; ++q) {
    const AeroSmokeEmitter &E = em[q];
    aero::emit::EmitParams<T> P{};
    P.c = static_cast<T *>(channels[E.channel]);
    P.ny = ny;
    P.nx = nx;
    for (int e = 0; e < 6; ++e) P.win[e] = E.window[e];
    P.w = static_cast<const T *>(E.weight);
    P.p = static_cast<const T *>(E.params);
    P.t = static_cast<const T *>(t);
    const long long n = (long long)(E.window[1] - E.window[0]) * (E.window[3] - E.window[2]) * (E.window[5] - E.window[4]);
    const unsigned blocks = (unsigned)std::max(1LL, std::min((n + 255) / 256, 1184LL));
    (void)aero::launch_k(aero::emit::emit_kernel<T>, blocks, 256, 0, s, P);
    AERO_CUDA_TRY(cudaGetLastError());
  }
  (void)nz;
  (void)nchannel;
  return AERO_OK;
}

}  // namespace

extern "C" {

int aero_smoke_emitters(int32_t dtype, int32_t nz, int32_t ny, int32_t nx, void *const *channels, int32_t nchannel,
                        const AeroSmokeEmitter *emitters, int32_t nemit, const void *t, void *stream) {
  if (dtype != AERO_F32 && dtype != AERO_F64) return set_error(AERO_EINVAL, "dtype must be float32 or float64");
  if (nz < 1 || ny < 1 || nx < 1 || nchannel < 1 || nemit < 0) return set_error(AERO_EINVAL, "bad sizes");
  if (!channels || (nemit > 0 && (!emitters || !t))) return set_error(AERO_EINVAL, "null argument");
  for (int q = 0; q < nemit; ++q) {
    const AeroSmokeEmitter &E = emitters[q];
    const int *w = E.window;
    if (E.channel < 0 || E.channel >= nchannel || !channels[E.channel])
      return set_error(AERO_EINVAL, "emitter channel out of range");
    if (w[1] <= w[0] || w[3] <= w[2] || w[5] <= w[4] || w[0] < 0 || w[1] > nz || w[2] < 0 || w[3] > ny || w[4] < 0 ||
        w[5] > nx)
      return set_error(AERO_EINVAL, "emitter window empty or outside the grid");
    if (!E.weight || !E.params) return set_error(AERO_EINVAL, "missing emitter weights or parameters");
  }
  auto s = static_cast<cudaStream_t>(stream);
  return dtype == AERO_F64 ? emit_impl<double>(nz, ny, nx, channels, nchannel, emitters, nemit, t, s)
                           : emit_impl<float>(nz, ny, nx, channels, nchannel, emitters, nemit, t, s);
}

}  // extern "C"
