// Batched line FFTs in shared memory for the exchange convolution.
//
// A CTA owns `LS` independent lines (band-pair channels, "slots") of length N,
// stored slot-minor as buf[i * LS + s].  This matches the HBM layout of the
// (nk1, nk2, nb, nb) arrays, whose channel index is innermost, so that global
// loads/stores of one k-point row are contiguous and coalesced, and every lane
// of a warp walks the same FFT index pattern (warp-uniform twiddle reads).
//
// The transform is a mixed-radix Stockham auto-sort FFT (no bit reversal):
// each stage reads R elements with stride N/R, applies the inter-stage twiddle
// W_{Ns R}^{(j mod Ns) r}, does an R-point DFT in registers and writes the
// outputs at stride Ns.  Radices 2, 3, 4, 5, 8 are hand-written; any other
// prime radix uses a direct O(R^2) DFT.  Twiddles come from a per-CTA table
// tw[e] = exp(-2 pi i e / N) built with CUDA's sincospi in double precision.
#pragma once

#include "common.cuh"

namespace hf {

constexpr int kMaxStages = 24;

struct FftPlan1D {
  int n;
  int nstages;
  int radix[kMaxStages];
};

// Builds the twiddle table exp(-2 pi i e / n), e in [0, n), cooperatively.
template <typename T>
__device__ __forceinline__ void build_twiddles(cpx_t<T>* tw, int n) {
  for (int e = threadIdx.x; e < n; e += blockDim.x) {
    // reduce to the nearest symmetric angle for accuracy: angle = -2 e / n (in units of pi)
    double s, c;
    sincospi(-2.0 * (double)e / (double)n, &s, &c);
    tw[e] = mk<cpx_t<T>>(c, s);
  }
}

// --- fixed-radix butterflies (forward: kernel exp(-2 pi i jk/R); inverse: conj) ---
template <bool INV, typename C>
__device__ __forceinline__ void bfly2(C& a, C& b) {
  C t = csub(a, b);
  a = cadd(a, b);
  b = t;
}

template <bool INV, typename C>
__device__ __forceinline__ void bfly4(C* v) {
  C t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
  C t2 = cadd(v[1], v[3]), t3 = csub(v[1], v[3]);
  t3 = INV ? mul_pi(t3) : mul_mi(t3);
  v[0] = cadd(t0, t2);
  v[2] = csub(t0, t2);
  v[1] = cadd(t1, t3);
  v[3] = csub(t1, t3);
}

template <bool INV, typename C>
__device__ __forceinline__ void bfly3(C* v) {
  using T = decltype(v[0].x);
  const T s3 = (T)0.86602540378443864676372317075294;  // sin(pi/3)
  C t1 = cadd(v[1], v[2]);
  C t2 = make_c<C>(v[0].x - (T)0.5 * t1.x, v[0].y - (T)0.5 * t1.y);
  C d = csub(v[1], v[2]);
  // forward: y1 = t2 - i s3 d ; y2 = t2 + i s3 d
  C r = INV ? mul_pi(d) : mul_mi(d);
  r = make_c<C>(r.x * s3, r.y * s3);
  v[0] = cadd(v[0], t1);
  v[1] = cadd(t2, r);
  v[2] = csub(t2, r);
}

template <bool INV, typename C>
__device__ __forceinline__ void bfly5(C* v) {
  using T = decltype(v[0].x);
  // cos/sin of 2 pi/5 and 4 pi/5 in closed form
  const T c1 = (T)0.30901699437494742410229341718282;   // (sqrt5 - 1)/4
  const T c2 = (T)-0.80901699437494742410229341718282;  // -(sqrt5 + 1)/4
  const T s1 = (T)0.95105651629515357211643933337938;   // sqrt(10 + 2 sqrt5)/4
  const T s2 = (T)0.58778525229247312916870595463907;   // sqrt(10 - 2 sqrt5)/4
  C a1 = cadd(v[1], v[4]), b1 = csub(v[1], v[4]);
  C a2 = cadd(v[2], v[3]), b2 = csub(v[2], v[3]);
  C x0 = v[0];
  C r1 = make_c<C>(x0.x + c1 * a1.x + c2 * a2.x, x0.y + c1 * a1.y + c2 * a2.y);
  C r2 = make_c<C>(x0.x + c2 * a1.x + c1 * a2.x, x0.y + c2 * a1.y + c1 * a2.y);
  // forward: y1 = r1 - i (s1 b1 + s2 b2); y4 = r1 + i (...)
  //          y2 = r2 - i (s2 b1 - s1 b2); y3 = r2 + i (...)
  C i1 = make_c<C>(s1 * b1.x + s2 * b2.x, s1 * b1.y + s2 * b2.y);
  C i2 = make_c<C>(s2 * b1.x - s1 * b2.x, s2 * b1.y - s1 * b2.y);
  i1 = INV ? mul_pi(i1) : mul_mi(i1);
  i2 = INV ? mul_pi(i2) : mul_mi(i2);
  v[0] = make_c<C>(x0.x + a1.x + a2.x, x0.y + a1.y + a2.y);
  v[1] = cadd(r1, i1);
  v[4] = csub(r1, i1);
  v[2] = cadd(r2, i2);
  v[3] = csub(r2, i2);
}

template <bool INV, typename C>
__device__ __forceinline__ void bfly8(C* v) {
  using T = decltype(v[0].x);
  const T h = (T)0.70710678118654752440084436210485;  // sqrt(1/2)
  // radix-2 first stage over stride 4, then twiddle W8^k, then two radix-4
  C a[4], b[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) { a[k] = cadd(v[k], v[k + 4]); b[k] = csub(v[k], v[k + 4]); }
  // b[k] *= W8^k  (forward W8 = (1 - i)/sqrt2)
  b[1] = INV ? make_c<C>(h * (b[1].x - b[1].y), h * (b[1].x + b[1].y))
             : make_c<C>(h * (b[1].x + b[1].y), h * (b[1].y - b[1].x));
  b[2] = INV ? mul_pi(b[2]) : mul_mi(b[2]);
  b[3] = INV ? make_c<C>(-h * (b[3].x + b[3].y), h * (b[3].x - b[3].y))
             : make_c<C>(h * (b[3].y - b[3].x), -h * (b[3].x + b[3].y));
  bfly4<INV>(a);
  bfly4<INV>(b);
  // outputs: even from a, odd from b
  v[0] = a[0]; v[2] = a[1]; v[4] = a[2]; v[6] = a[3];
  v[1] = b[0]; v[3] = b[1]; v[5] = b[2]; v[7] = b[3];
}

// One Stockham stage with compile-time radix R over LS slots.
template <int R, bool INV, typename C>
__device__ __forceinline__ void stockham_stage(const C* __restrict__ src, C* __restrict__ dst,
                                               const C* __restrict__ tw, int n, int ns, int LS) {
  const int nr = n / R;
  const int items = nr * LS;
  const int tstride = n / (ns * R);  // W_{ns R}^{m} = tw[m * tstride]
  for (int it = threadIdx.x; it < items; it += blockDim.x) {
    const int j = it / LS, s = it - j * LS;
    const int jm = j % ns;
    C v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = src[(j + r * nr) * LS + s];
    if (ns > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) {
        C w = tw[(jm * r * tstride) % n];
        v[r] = INV ? cmulc(v[r], w) : cmul(v[r], w);
      }
    }
    if constexpr (R == 2) bfly2<INV>(v[0], v[1]);
    else if constexpr (R == 3) bfly3<INV>(v);
    else if constexpr (R == 4) bfly4<INV>(v);
    else if constexpr (R == 5) bfly5<INV>(v);
    else if constexpr (R == 8) bfly8<INV>(v);
    const int d = (j / ns) * ns * R + jm;
#pragma unroll
    for (int r = 0; r < R; ++r) dst[(d + r * ns) * LS + s] = v[r];
  }
}

// Generic prime radix: direct R-point DFT using the N-point table.
template <bool INV, typename C>
__device__ void stockham_stage_generic(const C* __restrict__ src, C* __restrict__ dst,
                                       const C* __restrict__ tw, int n, int ns, int R, int LS) {
  const int nr = n / R;
  const int items = nr * LS;
  const int tstride = n / (ns * R);
  const int rstride = n / R;  // W_R^m = tw[m * rstride]
  for (int it = threadIdx.x; it < items; it += blockDim.x) {
    const int j = it / LS, s = it - j * LS;
    const int jm = j % ns;
    const int d = (j / ns) * ns * R + jm;
    for (int k = 0; k < R; ++k) {
      C acc = mk<C>(0.0, 0.0);
      for (int r = 0; r < R; ++r) {
        C x = src[(j + r * nr) * LS + s];
        if (ns > 1 && r > 0) {
          C w = tw[(jm * r * tstride) % n];
          x = INV ? cmulc(x, w) : cmul(x, w);
        }
        C w2 = tw[((r * k) % R) * rstride];
        x = INV ? cmulc(x, w2) : cmul(x, w2);
        acc = cadd(acc, x);
      }
      dst[(d + k * ns) * LS + s] = acc;
    }
  }
}

// Runs all stages; data starts in `a`, returns the buffer holding the result.
template <bool INV, typename C>
__device__ C* fft_lines(const FftPlan1D& plan, C* a, C* b, const C* tw, int LS) {
  int ns = 1;
  C* src = a;
  C* dst = b;
  for (int st = 0; st < plan.nstages; ++st) {
    const int R = plan.radix[st];
    switch (R) {
      case 2: stockham_stage<2, INV>(src, dst, tw, plan.n, ns, LS); break;
      case 3: stockham_stage<3, INV>(src, dst, tw, plan.n, ns, LS); break;
      case 4: stockham_stage<4, INV>(src, dst, tw, plan.n, ns, LS); break;
      case 5: stockham_stage<5, INV>(src, dst, tw, plan.n, ns, LS); break;
      case 8: stockham_stage<8, INV>(src, dst, tw, plan.n, ns, LS); break;
      default: stockham_stage_generic<INV>(src, dst, tw, plan.n, ns, R, LS); break;
    }
    __syncthreads();
    ns *= R;
    C* t = src; src = dst; dst = t;
  }
  return src;
}

}  // namespace hf
