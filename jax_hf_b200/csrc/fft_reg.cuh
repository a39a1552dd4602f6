// Register-resident DFTs of compile-time size and the two-level line FFT used
// by the fast Fock passes.
//
// rdft<N>: an N-point DFT on a register array (all indices compile-time after
// unrolling).  Composite N = A*B is split Cooley-Tukey style: A-point DFTs over
// x[n2 + B n1], the twiddle W_N^{n2 k1}, B-point DFTs, output X[k1 + A k2].
// Radices 2/3/4/5/8 are the butterflies of fft_engine.cuh; other primes use a
// direct DFT.  Inner twiddles are compile-time constants (CtTwiddle).
//
// Line FFT of length N = N1*N2 over TPL threads per line (TPL | N1, TPL | N2):
//   pattern A: thread t holds x[n2 + N2 n1] for n2 = t + TPL i (i < N2/TPL), all n1
//   pattern B: thread t holds X[k1 + N1 k2] for k1 = t + TPL j (j < N1/TPL), all k2
// fwd_AB: step 1 (N1-point DFTs, twiddle W_N^{n2 k1}) -> shared-memory
// exchange -> step 2 (N2-point DFTs).  inv_BA is the decimation-in-frequency
// inverse that starts from pattern B (N2-point IDFTs, twiddle, exchange,
// N1-point IDFTs), so the spectrum never needs reordering between a forward
// and an inverse transform.  Each call has one exchange; buf is [N][16] slots.
// The runtime twiddles of a thread (they depend on t) come from its own row of
// a shared-memory table (build_line_twiddles), indexed by compile-time offsets.
#pragma once

#include <utility>

#include "fft_engine.cuh"

namespace hf {

__host__ __device__ constexpr bool ct_is_prime(int n) {
  if (n < 2) return false;
  for (int d = 2; d * d <= n; ++d)
    if (n % d == 0) return false;
  return true;
}

__host__ __device__ constexpr int ct_first_factor(int n) {
  return (n % 8 == 0 && n > 8) ? 8 : (n % 4 == 0 && n > 4) ? 4 : (n % 2 == 0 && n > 2) ? 2
       : (n % 3 == 0 && n > 3) ? 3 : (n % 5 == 0 && n > 5) ? 5 : n;
}

template <bool INV, typename C>
__device__ __forceinline__ C twmul(C v, C w) {
  return INV ? cmulc(v, w) : cmul(v, w);
}

// Compile-time W_n^e = exp(-2 pi i e / n): exact octant reduction in integers,
// then Taylor series on [0, pi/4] (terms to x^29, error below 1e-17).
__host__ __device__ constexpr double ct_sin_series(double x) {
  double x2 = x * x, term = x, sum = x;
  for (int k = 1; k < 15; ++k) {
    term *= -x2 / (double)((2 * k) * (2 * k + 1));
    sum += term;
  }
  return sum;
}
__host__ __device__ constexpr double ct_cos_series(double x) {
  double x2 = x * x, term = 1.0, sum = 1.0;
  for (int k = 1; k < 15; ++k) {
    term *= -x2 / (double)((2 * k - 1) * (2 * k));
    sum += term;
  }
  return sum;
}
// cos / sin of 2 pi e / n
__host__ __device__ constexpr double ct_cos2pi(int e, int n, bool want_sin) {
  e %= n;
  if (e < 0) e += n;
  // angle = (pi/2) (q + r/n), q = quadrant
  const int q = (4 * e) / n;
  int r = 4 * e - q * n;  // 0 <= r < n, angle within quadrant = (pi/2) r / n
  const double hp = 1.5707963267948966192313216916397514;
  bool swap = false;
  if (2 * r > n) { r = n - r; swap = true; }  // use the complementary angle
  const double x = hp * (double)r / (double)n;
  double c = ct_cos_series(x), s = ct_sin_series(x);
  if (swap) { const double t = c; c = s; s = t; }
  // rotate by q quadrants: (c, s) -> (-s, c)
  for (int k = 0; k < q; ++k) { const double t = c; c = -s; s = t; }
  return want_sin ? s : c;
}
template <int E, int N>
struct CtTwiddle {
  static constexpr double re = ct_cos2pi(E, N, false);
  static constexpr double im = -ct_cos2pi(E, N, true);
};
template <int E, int N, bool INV, typename C>
__device__ __forceinline__ C ct_twmul(C v) {
  using T = decltype(v.x);
  constexpr double wr = CtTwiddle<E % N, N>::re, wi = CtTwiddle<E % N, N>::im;
  const T r = (T)wr, i = INV ? (T)(-wi) : (T)wi;
  return make_c<C>(v.x * r - v.y * i, v.x * i + v.y * r);
}

template <int N, int TWN, bool INV, typename C>
__device__ __forceinline__ void rdft(C* x, const C* __restrict__ tw);

template <int N, bool INV, int K, typename C, int... Ns>
__device__ __forceinline__ C prime_row(const C* x, std::integer_sequence<int, Ns...>) {
  C acc = x[0];
  ((acc = cadd(acc, ct_twmul<(Ns + 1) * K, N, INV>(x[Ns + 1]))), ...);
  return acc;
}
template <int N, bool INV, typename C, int... Ks>
__device__ __forceinline__ void prime_all(const C* x, C* y, std::integer_sequence<int, Ks...>) {
  ((y[Ks] = prime_row<N, INV, Ks>(x, std::make_integer_sequence<int, N - 1>{})), ...);
}
template <int N, bool INV, typename C>
__device__ __forceinline__ void rdft_prime(const C* x, C* y) {
  prime_all<N, INV>(x, y, std::make_integer_sequence<int, N>{});
}

// step 1 of the split for one n2: A-point DFT over x[n2 + B n1], twiddle W_N^{n2 k1}
template <int N, int A, int B, int N2, int TWN, bool INV, typename C, int... K1s>
__device__ __forceinline__ void split_tw(const C* t, C* y, std::integer_sequence<int, K1s...>) {
  ((y[K1s * B + N2] = ct_twmul<N2 * K1s, N, INV>(t[K1s])), ...);
}
template <int N, int A, int B, int TWN, bool INV, typename C, int... N2s>
__device__ __forceinline__ void rdft_split(const C* x, C* y, const C* tw, std::integer_sequence<int, N2s...>) {
  (
      [&] {
        constexpr int n2 = N2s;
        C t[A];
#pragma unroll
        for (int n1 = 0; n1 < A; ++n1) t[n1] = x[n2 + B * n1];
        rdft<A, TWN, INV>(t, tw);
        split_tw<N, A, B, n2, TWN, INV>(t, y, std::make_integer_sequence<int, A>{});
      }(),
      ...);
}
template <int N, int A, int B, int TWN, bool INV, typename C>
__device__ __forceinline__ void rdft_second(C* x, const C* y, const C* tw) {
#pragma unroll
  for (int k1 = 0; k1 < A; ++k1) {
    C t[B];
#pragma unroll
    for (int n2 = 0; n2 < B; ++n2) t[n2] = y[k1 * B + n2];
    rdft<B, TWN, INV>(t, tw);
#pragma unroll
    for (int k2 = 0; k2 < B; ++k2) x[k1 + A * k2] = t[k2];
  }
}

template <int N, int TWN, bool INV, typename C>
__device__ __forceinline__ void rdft(C* x, const C* __restrict__ tw) {
  static_assert(TWN % N == 0, "twiddle table must be a multiple of the DFT size");
  if constexpr (N == 1) {
    return;
  } else if constexpr (N == 2) {
    bfly2<INV>(x[0], x[1]);
  } else if constexpr (N == 3) {
    bfly3<INV>(x);
  } else if constexpr (N == 4) {
    bfly4<INV>(x);
  } else if constexpr (N == 5) {
    bfly5<INV>(x);
  } else if constexpr (N == 8) {
    bfly8<INV>(x);
  } else if constexpr (ct_is_prime(N)) {
    C y[N];
    rdft_prime<N, INV>(x, y);
#pragma unroll
    for (int k = 0; k < N; ++k) x[k] = y[k];
  } else {
    constexpr int A = ct_first_factor(N);
    constexpr int B = N / A;
    C y[N];
    rdft_split<N, A, B, TWN, INV>(x, y, tw, std::make_integer_sequence<int, B>{});
    rdft_second<N, A, B, TWN, INV>(x, y, tw);
  }
}

template <int N_, int N1_, int N2_, int TPL_>
struct LineShape {
  static constexpr int N = N_, N1 = N1_, N2 = N2_, TPL = TPL_;
  static constexpr int E1 = N2 / TPL;  // step-1 DFTs per thread
  static constexpr int E2 = N1 / TPL;  // step-2 DFTs per thread
  static constexpr int E = N / TPL;    // elements per thread
  static constexpr int TS = E + 1;     // twiddle-row stride (odd in 16-byte units: no bank conflicts)
  static_assert(N1 * N2 == N && N2 % TPL == 0 && N1 % TPL == 0, "bad line shape");
  // index of element (i, n1) of pattern A and (j, k2) of pattern B
  __device__ static __forceinline__ int idxA(int t, int i, int n1) { return t + TPL * i + N2 * n1; }
  __device__ static __forceinline__ int idxB(int t, int j, int k2) { return t + TPL * j + N1 * k2; }
};

// Per-thread twiddle rows of a line shape: the step-1 twiddles W_N^{n2 k1} of
// part t (n2 = t + TPL i) at twf[t TS + i N1 + k1], and the inverse-step
// twiddles W_N^{k1 m2} (k1 = t + TPL j) at twi[t TS + j N2 + m2].  Each table
// holds TPL * TS entries; values are exp(-2 pi i e / N) from the compile-time
// series (ct_cos2pi), so a pass copies its rows from a constant table in global
// memory instead of evaluating 2 N FP64 sines in its prologue.
template <class S>
struct LineTwTable {
  double v[2][S::TPL * S::E][2];  // [forward / inverse step][t E + r][re, im]
};
template <class S>
constexpr LineTwTable<S> make_line_twiddles() {
  LineTwTable<S> T{};
  for (int q = 0; q < S::TPL * S::E; ++q) {
    const int t = q / S::E, r = q - t * S::E;
    const int ef = ((t + S::TPL * (r / S::N1)) * (r % S::N1)) % S::N;
    const int ei = ((t + S::TPL * (r / S::N2)) * (r % S::N2)) % S::N;
    T.v[0][q][0] = ct_cos2pi(ef, S::N, false);
    T.v[0][q][1] = -ct_cos2pi(ef, S::N, true);
    T.v[1][q][0] = ct_cos2pi(ei, S::N, false);
    T.v[1][q][1] = -ct_cos2pi(ei, S::N, true);
  }
  return T;
}
template <class S>
__device__ constexpr LineTwTable<S> kLineTwiddles = make_line_twiddles<S>();

template <class S, typename T>
__device__ __forceinline__ void build_line_twiddles(cpx_t<T>* twf, cpx_t<T>* twi) {
  const LineTwTable<S>& tab = kLineTwiddles<S>;
  for (int q = threadIdx.x; q < S::TPL * S::E; q += blockDim.x) {
    const int t = q / S::E, r = q - t * S::E;
    twf[t * S::TS + r] = mk<cpx_t<T>>(tab.v[0][q][0], tab.v[0][q][1]);
    twi[t * S::TS + r] = mk<cpx_t<T>>(tab.v[1][q][0], tab.v[1][q][1]);
  }
}

// pattern A -> pattern B (forward).  tw = this thread's row of twf.  x[i*N1 + n1] in, x[j*N2 + k2] out.
template <class S, typename C>
__device__ __forceinline__ void fwd_AB(C* x, C* __restrict__ buf, const C* __restrict__ tw, int t, int s) {
#pragma unroll
  for (int i = 0; i < S::E1; ++i) {
    rdft<S::N1, S::N, false>(x + i * S::N1, tw);
    const int n2 = t + S::TPL * i;
#pragma unroll
    for (int k1 = 0; k1 < S::N1; ++k1) {
      C v = x[i * S::N1 + k1];
      if (k1 != 0) v = cmul(v, tw[i * S::N1 + k1]);
      buf[(k1 * S::N2 + n2) * 16 + s] = v;
    }
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < S::E2; ++j) {
    const int k1 = t + S::TPL * j;
#pragma unroll
    for (int n2 = 0; n2 < S::N2; ++n2) x[j * S::N2 + n2] = buf[(k1 * S::N2 + n2) * 16 + s];
    rdft<S::N2, S::N, false>(x + j * S::N2, tw);
  }
}

// pattern B -> pattern A (inverse, unnormalised).  x[j*N2 + k2] in, x[i*N1 + m1] out.
// tw = this thread's row of twi (applied conjugated; the k1 = 0 row is all ones).
// pre() runs after the N2-point IDFTs (registers only) and before the first
// write to buf, e.g. a wait until buf may be overwritten.
template <class S, typename C, typename Pre>
__device__ __forceinline__ void inv_BA(C* x, C* __restrict__ buf, const C* __restrict__ tw, int t, int s, Pre pre) {
#pragma unroll
  for (int j = 0; j < S::E2; ++j) {
    rdft<S::N2, S::N, true>(x + j * S::N2, tw);
#pragma unroll
    for (int m2 = 1; m2 < S::N2; ++m2) x[j * S::N2 + m2] = cmulc(x[j * S::N2 + m2], tw[j * S::N2 + m2]);
  }
  pre();
#pragma unroll
  for (int j = 0; j < S::E2; ++j) {
    const int k1 = t + S::TPL * j;
#pragma unroll
    for (int m2 = 0; m2 < S::N2; ++m2) buf[(k1 * S::N2 + m2) * 16 + s] = x[j * S::N2 + m2];
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < S::E1; ++i) {
    const int m2 = t + S::TPL * i;
#pragma unroll
    for (int k1 = 0; k1 < S::N1; ++k1) x[i * S::N1 + k1] = buf[(k1 * S::N2 + m2) * 16 + s];
    rdft<S::N1, S::N, true>(x + i * S::N1, tw);
  }
}
template <class S, typename C>
__device__ __forceinline__ void inv_BA(C* x, C* __restrict__ buf, const C* __restrict__ tw, int t, int s) {
  inv_BA<S>(x, buf, tw, t, s, [] {});
}

}  // namespace hf
