// Host harness for aerolume_b200/csrc/fft_tile.cuh: runs the tile transform's phases thread
// by thread (256 "threads", one phase after another) so the tests can compare the exact
// device code path with scipy's orthonormal DCT / Hartley transforms on the CPU.
//
//   fft_tile_host <f32|f64> <N = 2^a or 3 * 2^a> <kind 0 DCT|1 DHT> <inverse 0|1> [narrow 0|1]
//   stdin: N * L doubles, row m of the tile then the next (L = the tile width for N, or 2 with
//   narrow = 1), stdout the transformed tile in the same layout.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "fft_tile.cuh"

using namespace aero::fft;

struct SerialExec {
  int nthr;
  template <class F>
  void operator()(F &&f) {
    for (int t = 0; t < nthr; ++t) f(t, nthr);
  }
};

template <typename T, int N, int LOG2L>
int run_tile(int kind, int inverse) {
  constexpr int L = 1 << LOG2L, LD = L + 1;
  std::vector<double> in((size_t)N * L);
  if (fread(in.data(), sizeof(double), in.size(), stdin) != in.size()) return 2;
  std::vector<Cx<T>> tw(N), post(N), cs(N);
  const double pi = 3.14159265358979323846264338327950288;
  for (int m = 0; m < N; ++m) {
    tw[m] = {T(std::cos(2.0 * pi * m / N)), T(-std::sin(2.0 * pi * m / N))};
    const double a = 0.5 * pi * m / N, sk = m == 0 ? std::sqrt(1.0 / N) : std::sqrt(2.0 / N);
    post[m] = {T(sk * std::cos(a)), T(-sk * std::sin(a))};
    cs[m] = {T(std::cos(a)), T(std::sin(a))};
  }
  AxisView<T> A{tw.data(), post.data(), cs.data(), T(std::sqrt(1.0 / N)), T(std::sqrt(2.0 / N)),
                T(1.0 / std::sqrt((double)N)), kind};
  std::vector<T> R((size_t)N * LD);
  std::vector<Cx<T>> C0((size_t)N * L / 2), C1((size_t)N * L / 2);
  for (int m = 0; m < N; ++m)
    for (int l = 0; l < L; ++l) R[(size_t)m * LD + l] = T(in[(size_t)m * L + l]);
  SerialExec ex{256};
  transform_tile<T, N, LOG2L>(R.data(), C0.data(), C1.data(), tw.data(), A, inverse != 0, ex);
  std::vector<double> out((size_t)N * L);
  for (int m = 0; m < N; ++m)
    for (int l = 0; l < L; ++l) out[(size_t)m * L + l] = (double)R[(size_t)m * LD + l];
  fwrite(out.data(), sizeof(double), out.size(), stdout);
  return 0;
}

template <typename T, int N>
int run(int kind, int inverse, int narrow) {
  if (narrow) return run_tile<T, N, 1>(kind, inverse);
  return run_tile<T, N, tile_log2L(N, (int)sizeof(T))>(kind, inverse);
}

template <typename T>
int dispatch(int n, int kind, int inverse, int narrow) {
  switch (n) {
    case 8: return run<T, 8>(kind, inverse, narrow);
    case 16: return run<T, 16>(kind, inverse, narrow);
    case 32: return run<T, 32>(kind, inverse, narrow);
    case 64: return run<T, 64>(kind, inverse, narrow);
    case 128: return run<T, 128>(kind, inverse, narrow);
    case 256: return run<T, 256>(kind, inverse, narrow);
    case 512: return run<T, 512>(kind, inverse, narrow);
    case 1024: return run<T, 1024>(kind, inverse, narrow);
    case 2048: return run<T, 2048>(kind, inverse, narrow);
    case 12: return run<T, 12>(kind, inverse, narrow);
    case 24: return run<T, 24>(kind, inverse, narrow);
    case 48: return run<T, 48>(kind, inverse, narrow);
    case 96: return run<T, 96>(kind, inverse, narrow);
    case 192: return run<T, 192>(kind, inverse, narrow);
    case 384: return run<T, 384>(kind, inverse, narrow);
    case 768: return run<T, 768>(kind, inverse, narrow);
    case 1536: return run<T, 1536>(kind, inverse, narrow);
  }
  return 3;
}

int main(int argc, char **argv) {
  if (argc != 5 && argc != 6) return 1;
  const bool f64 = std::strcmp(argv[1], "f64") == 0;
  const int n = std::atoi(argv[2]), kind = std::atoi(argv[3]), inverse = std::atoi(argv[4]);
  const int narrow = argc == 6 ? std::atoi(argv[5]) : 0;
  return f64 ? dispatch<double>(n, kind, inverse, narrow) : dispatch<float>(n, kind, inverse, narrow);
}
