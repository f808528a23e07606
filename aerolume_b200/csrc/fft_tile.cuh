// Orthonormal DCT-II / DCT-III / Hartley transforms of a tile of L = 2^LOG2L real lines of
// length N = 2^a or 3 * 2^a (8 <= N <= 2048), with every length, stride and stage constant at
// compile time: the Stockham FFT's index arithmetic is shifts, masks and multiplications by
// constants, its loops unroll, and no stage table is read at run time.  Used by the Poisson
// solve (Aerolume ns3d/poisson.py:74-90 defines the bases: DCT-II for homogeneous Neumann
// axes, Hartley for periodic ones).
//
//   DCT-II   Makhoul's even/odd reordering, a length-N complex FFT carrying two real lines
//            at once (real and imaginary parts), then X_k = s_k Re(e^{-i pi k/2N} V_k)
//   DCT-III  V_k = e^{i pi k/2N} (Y_k - i Y_{N-k}) / 2 (V_0 = Y_0), inverse FFT, un-reordering
//   DHT      H_k = (Re F_k - Im F_k) / sqrt(N)  (its own inverse)
//
// The work is written as phases, each a function of (thread, thread count) whose threads
// read one buffer and write another; an executor runs a phase on every thread and then
// synchronises.  On the GPU the executor is the thread block and __syncthreads(); the
// host test harness runs the same phases thread by thread, so it executes this exact code.
#pragma once

#ifdef __CUDACC__
#define AERO_HD __host__ __device__ __forceinline__
#else
#define AERO_HD inline
#endif

namespace aero {
namespace fft {

template <typename T>
struct Cx {
  T x, y;
};

template <typename T>
AERO_HD Cx<T> cmul(Cx<T> a, Cx<T> b) {
  return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}

constexpr int ilog2(int n) { return n <= 1 ? 0 : 1 + ilog2(n / 2); }

// Stockham plan of N = 2^a or 3 * 2^a: floor(a / 2) radix-4 stages, one radix-2 stage when a
// is odd, then one radix-3 stage when 3 divides N.  Before stage s the span of the finished
// sub-transforms is ns(s), a power of two in every stage (the radix-3 stage comes last).
constexpr bool pow2_len(int n) { return n >= 1 && (n & (n - 1)) == 0; }
constexpr bool tile_len(int n) { return n >= 8 && n <= 2048 && (pow2_len(n) || (n % 3 == 0 && pow2_len(n / 3) && n / 3 >= 4)); }

template <int N>
struct Pow2 {
  static_assert(tile_len(N), "lengths 2^a or 3 * 2^a, 8..2048");
  static constexpr bool THREE = N % 3 == 0;
  static constexpr int LOG2P2 = ilog2(THREE ? N / 3 : N);  // log2 of the power-of-two part
  static constexpr int N4 = LOG2P2 / 2, N2 = LOG2P2 & 1;
  static constexpr int NST = N4 + N2 + (THREE ? 1 : 0);
  static constexpr int radix(int s) { return s < N4 ? 4 : (s < N4 + N2 ? 2 : 3); }
  static constexpr int ns(int s) { return s == 0 ? 1 : ns(s - 1) * radix(s - 1); }
};

// One Stockham stage over P = 2^LOG2P interleaved complex lines (element m of line p at
// m * P + p): in -> out.
template <typename T, int N, int LOG2P, int S, bool INV>
AERO_HD void stockham_stage(const Cx<T> *in, Cx<T> *out, const Cx<T> *tw, int tid, int nthr) {
  constexpr int R = Pow2<N>::radix(S), M = N / R, NS = Pow2<N>::ns(S), STRIDE = N / (NS * R);
  constexpr int P = 1 << LOG2P, ITEMS = M * P;
  const T sgn = INV ? T(1) : T(-1);
  for (int item = tid; item < ITEMS; item += nthr) {
    const int p = item & (P - 1), jj = item >> LOG2P;
    const int k = jj & (NS - 1), g = jj / NS;  // NS is a power of two
    Cx<T> v[R];
#pragma unroll
    for (int t = 0; t < R; ++t) v[t] = in[((jj + t * M) << LOG2P) + p];
#pragma unroll
    for (int t = 1; t < R; ++t) {
      Cx<T> w = tw[t * k * STRIDE];
      if (INV) w.y = -w.y;
      v[t] = cmul(v[t], w);
    }
    Cx<T> V[R];
    if constexpr (R == 4) {
      const Cx<T> a0 = {v[0].x + v[2].x, v[0].y + v[2].y}, a1 = {v[0].x - v[2].x, v[0].y - v[2].y};
      const Cx<T> a2 = {v[1].x + v[3].x, v[1].y + v[3].y};
      const Cx<T> d = {v[1].x - v[3].x, v[1].y - v[3].y};
      const Cx<T> a3 = {-sgn * d.y, sgn * d.x};  // sgn * i * d
      V[0] = {a0.x + a2.x, a0.y + a2.y};
      V[2] = {a0.x - a2.x, a0.y - a2.y};
      V[1] = {a1.x + a3.x, a1.y + a3.y};
      V[3] = {a1.x - a3.x, a1.y - a3.y};
    } else if constexpr (R == 2) {
      V[0] = {v[0].x + v[1].x, v[0].y + v[1].y};
      V[1] = {v[0].x - v[1].x, v[0].y - v[1].y};
    } else {  // R == 3: X_1,2 = v0 - (v1 + v2) / 2 -+ sgn i (sqrt 3 / 2) (v1 - v2)
      const T h3 = T(0.866025403784438646763723170752936183);
      const Cx<T> t1 = {v[1].x + v[2].x, v[1].y + v[2].y};
      const Cx<T> t2 = {v[0].x - T(0.5) * t1.x, v[0].y - T(0.5) * t1.y};
      const Cx<T> d = {v[1].x - v[2].x, v[1].y - v[2].y};
      const Cx<T> t3 = {-sgn * h3 * d.y, sgn * h3 * d.x};  // sgn * i * (sqrt3/2) * d
      V[0] = {v[0].x + t1.x, v[0].y + t1.y};
      V[1] = {t2.x + t3.x, t2.y + t3.y};
      V[2] = {t2.x - t3.x, t2.y - t3.y};
    }
    const int base = g * NS * R + k;
#pragma unroll
    for (int t = 0; t < R; ++t) out[((base + t * NS) << LOG2P) + p] = V[t];
  }
}

// All stages, ping-ponging between a and b; returns the buffer holding the result.
template <typename T, int N, int LOG2P, bool INV, int S = 0, class Exec>
AERO_HD Cx<T> *stockham(Cx<T> *a, Cx<T> *b, const Cx<T> *tw, Exec &ex) {
  if constexpr (S == Pow2<N>::NST) {
    return a;
  } else {
    ex([&](int tid, int nthr) { stockham_stage<T, N, LOG2P, S, INV>(a, b, tw, tid, nthr); });
    return stockham<T, N, LOG2P, INV, S + 1>(b, a, tw, ex);
  }
}

// Makhoul reordering: v[m] = x[perm(m)]
AERO_HD int makhoul(int m, int n) { return (2 * m < n) ? 2 * m : 2 * (n - 1 - m) + 1; }

// Tables of one axis (device or host memory): tw[m] = e^{-2 pi i m / N}, post[k] =
// s_k e^{-i pi k / 2N}, cs[k] = (cos, sin)(pi k / 2N); s0 = sqrt(1/N), s1 = sqrt(2/N).
template <typename T>
struct AxisView {
  const Cx<T> *tw, *post, *cs;
  T s0, s1, rsqrt_n;
  int kind;  // 0 DCT (Neumann), 1 Hartley (periodic)
};

// In place on the real tile R[m * (L + 1) + l] (N rows, L columns): the orthonormal forward
// (DCT-II / DHT) or inverse (DCT-III / DHT) transform of each column.  C0 and C1 hold
// N * L / 2 complex values each; tw is the twiddle table (any memory the threads can read).
template <typename T, int N, int LOG2L, class Exec>
AERO_HD void transform_tile(T *R, Cx<T> *C0, Cx<T> *C1, const Cx<T> *tw, const AxisView<T> &A, bool inverse,
                            Exec &ex) {
  constexpr int L = 1 << LOG2L, LD = L + 1, LOG2P = LOG2L - 1, P = L / 2;
  constexpr int ITEMS = N * P;
  const bool dct3 = A.kind == 0 && inverse;
  // ---- pack two real columns per complex line
  ex([&](int tid, int nthr) {
    for (int item = tid; item < ITEMS; item += nthr) {
      const int p = item & (P - 1), m = item >> LOG2P;
      Cx<T> z;
      if (A.kind == 1) {  // Hartley: natural order
        z = {R[m * LD + 2 * p], R[m * LD + 2 * p + 1]};
      } else if (!inverse) {  // DCT-II: reorder
        const int src = makhoul(m, N);
        z = {R[src * LD + 2 * p], R[src * LD + 2 * p + 1]};
      } else {  // DCT-III
        const int k = m;
        const Cx<T> e = A.cs[k];
        Cx<T> va, vb;
        if (k == 0) {
          va = {A.s0 * R[2 * p], T(0)};
          vb = {A.s0 * R[2 * p + 1], T(0)};
        } else {
          const T ya = A.s1 * R[k * LD + 2 * p], yra = A.s1 * R[(N - k) * LD + 2 * p];
          const T yb = A.s1 * R[k * LD + 2 * p + 1], yrb = A.s1 * R[(N - k) * LD + 2 * p + 1];
          va = cmul(e, Cx<T>{T(0.5) * ya, -T(0.5) * yra});
          vb = cmul(e, Cx<T>{T(0.5) * yb, -T(0.5) * yrb});
        }
        z = {va.x - vb.y, va.y + vb.x};  // va + i vb
      }
      C0[(m << LOG2P) + p] = z;
    }
  });
  Cx<T> *Z = dct3 ? stockham<T, N, LOG2P, true>(C0, C1, tw, ex) : stockham<T, N, LOG2P, false>(C0, C1, tw, ex);
  // ---- unpack into R (R is free: its content went into C0 and nothing reads it here)
  ex([&](int tid, int nthr) {
    for (int item = tid; item < ITEMS; item += nthr) {
      const int p = item & (P - 1), k = item >> LOG2P;
      const Cx<T> z = Z[(k << LOG2P) + p];
      if (dct3) {  // z = v_a[k] + i v_b[k]
        const int dst = makhoul(k, N);
        R[dst * LD + 2 * p] = z.x;
        R[dst * LD + 2 * p + 1] = z.y;
      } else {
        const Cx<T> zr = Z[((k == 0 ? 0 : N - k) << LOG2P) + p];
        const T ar = T(0.5) * (z.x + zr.x), ai = T(0.5) * (z.y - zr.y);   // F_a = (Z_k + conj Z_{N-k}) / 2
        const T br = T(0.5) * (z.y + zr.y), bi = -T(0.5) * (z.x - zr.x);  // F_b = (Z_k - conj Z_{N-k}) / 2i
        T xa, xb;
        if (A.kind == 1) {
          xa = (ar - ai) * A.rsqrt_n;
          xb = (br - bi) * A.rsqrt_n;
        } else {
          const Cx<T> w = A.post[k];
          xa = w.x * ar - w.y * ai;
          xb = w.x * br - w.y * bi;
        }
        R[k * LD + 2 * p] = xa;
        R[k * LD + 2 * p + 1] = xb;
      }
    }
  });
}

// Lines per tile for length N and element size E: a power of two, 2..64, keeping the tile
// (real tile + two complex buffers, 3 N L elements) within about 48 KiB.
constexpr int tile_log2L(int n, int e) {
  int l = (48 * 1024) / (3 * e * n);
  l = l > 64 ? 64 : (l < 2 ? 2 : l);
  return ilog2(l);
}

}  // namespace fft
}  // namespace aero
