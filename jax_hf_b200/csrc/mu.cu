// Chemical potential: mu such that sum_k w_k sum_j f(eps_kj - mu) = N.
//
// One thread-block cluster (up to 16 CTAs) runs the whole root find: every
// iteration each CTA reduces its slice, publishes the partial in its shared
// memory, one cluster barrier, and warp 0 of every CTA then reads all partials
// through distributed shared memory and reduces them with a fixed shuffle tree.
// All CTAs therefore hold bit-identical (mu, lo, hi) and take identical
// branches; no global-memory round trip and no second launch per iteration.
// The bisection evaluates two levels per pass (the 3 midpoints of the next two
// levels in one reduction, then the two decisions in order).  Each pass costs a
// chain of block and cluster reductions whose latency grows with the number of
// sums: on 2304 eigenvalues (9 CTAs) the 54 steps take 52 us at two levels per
// pass (27 passes), 59 us at three, 65 us at one and 91 us at four; storing the
// warp partials into every CTA's shared memory behind a single cluster barrier
// instead of the two-stage reduction measured slower (63 us at two levels).
//
// Methods (reference):
//   0  _find_mu_bisection  utils.py:353-382 (maxiter 54 f64 / 30 f32)
//   1  _find_mu_newton     utils.py:385-442 (maxiter 25 f64 / 15 f32)
//   2  _solve_mu           solver.py:62-101 (maxiter 25, warm start mu0)
// The iterations replay the reference update rules.  Bisection stops early
// only at an exact fixed point of (lo, hi); the Newton variants stop once the
// accepted Newton step is below 4 ulp of mu (the reference keeps iterating
// there, moving mu by at most a few ulp).
#include <cooperative_groups.h>

#include <climits>
#include <map>
#include <mutex>
#include <utility>

#include "common.cuh"

namespace cg = cooperative_groups;

namespace hf {

constexpr int kMuThreads = 1024;
constexpr int kMuMaxCluster = 16;  // non-portable size, used when the device schedules it
constexpr int kBisLevels = 2;  // bisection levels per pass of the 256-thread variant
constexpr int kMuCertPasses = 6;  // Newton passes of a hinted bisection (certified bracket)

struct MuArgs {
  const void* eps;
  const void* w;
  int n, nb, method, maxiter;
  double target, T;
  const double* mu0;
  double* out;
  const int* active;  // optional device flag: return at once when *active == 0
  int cache;          // elements per thread kept in shared memory as (eps, w); 0: read from L2
};
// loads in flight per thread when the elements are read from L2
constexpr int kMuCacheU = 4;
// the shared-memory cache holds up to this many (eps, w) entries per thread (layout
// [u][thread]; 192 KB for 1024 threads): a 144 x 144 x 8 spectrum on 16 CTAs needs 11
constexpr int kMuCacheMax = 12;

template <typename RT>
__device__ __forceinline__ double load_eps(const MuArgs& a, int e) {
  return (double)static_cast<const RT*>(a.eps)[e];
}
template <typename RT>
__device__ __forceinline__ double load_w(const MuArgs& a, int e) {
  return (double)static_cast<const RT*>(a.w)[e / a.nb];
}

// Visits the elements e = gt, gt + gs, ... < n in batches of U with all U loads of
// a batch issued before any use, so each thread keeps U L2 requests in flight
// instead of one (the passes are load-latency bound, not exp bound).
template <typename RT, int U, class F>
__device__ __forceinline__ void for_each_eps(const MuArgs& a, int gt, int gs, F&& f) {
  for (int base = gt; base < a.n; base += U * gs) {
    double ev[U], wv[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int e = base + u * gs;
      ev[u] = e < a.n ? load_eps<RT>(a, e) : 0.0;
      wv[u] = e < a.n ? load_w<RT>(a, e) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < U; ++u)
      if (base + u * gs < a.n) f(ev[u], wv[u]);
  }
}

// Cluster-wide sum of (x, y); every thread of every CTA receives the total.
// Each CTA publishes its block sum in its `slots`; after the cluster barrier,
// lane r of warp 0 reads CTA r's slot (one distributed-shared-memory read per
// lane, all in flight together) and warp 0 reduces them with a fixed shuffle
// tree, so every CTA obtains bit-identical totals.  slots is double-buffered by
// `parity`: a CTA may publish the next pass while a slower one still reads this.
__device__ __forceinline__ void cluster_sum2(cg::cluster_group& cl, double& x, double& y,
                                             double (*slots)[2], double* wsm, int parity) {
  x = warp_sum(x);
  y = warp_sum(y);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (lane == 0) { wsm[2 * wid] = x; wsm[2 * wid + 1] = y; }
  __syncthreads();
  if (wid == 0) {  // the warp partials, reduced by one warp
    double sx = lane < nw ? wsm[2 * lane] : 0.0, sy = lane < nw ? wsm[2 * lane + 1] : 0.0;
    sx = warp_sum(sx);
    sy = warp_sum(sy);
    if (lane == 0) {
      slots[parity][0] = sx;
      slots[parity][1] = sy;
    }
  }
  cl.sync();
  if (wid == 0) {
    double tx = 0.0, ty = 0.0;
    if (lane < (int)cl.num_blocks()) {
      double(*rs)[2] = cl.map_shared_rank(slots, lane);
      tx = rs[parity][0];
      ty = rs[parity][1];
    }
    tx = warp_sum(tx);
    ty = warp_sum(ty);
    if (lane == 0) { wsm[64] = tx; wsm[65] = ty; }
  }
  __syncthreads();
  x = wsm[64];
  y = wsm[65];
}

// Cluster-wide sums of K values (as cluster_sum2); v[] holds this thread's terms
// on entry and the totals on return.  bsm: 32 * K + K doubles, slots: [2][K].
template <int K>
__device__ __forceinline__ void cluster_sum_n(cg::cluster_group& cl, double (&v)[K], double (*slots)[K], double* bsm,
                                              int parity) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int j = 0; j < K; ++j) {
    v[j] = warp_sum(v[j]);
    if (lane == 0) bsm[wid * K + j] = v[j];
  }
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int j = 0; j < K; ++j) {
      double t = lane < nw ? bsm[lane * K + j] : 0.0;
      t = warp_sum(t);
      if (lane == 0) slots[parity][j] = t;
    }
  }
  cl.sync();
  if (wid == 0) {
    double(*rs)[K] = lane < (int)cl.num_blocks() ? cl.map_shared_rank(slots, lane) : nullptr;
    double t[K];
#pragma unroll
    for (int j = 0; j < K; ++j) t[j] = rs ? rs[parity][j] : 0.0;
#pragma unroll
    for (int j = 0; j < K; ++j) {
      t[j] = warp_sum(t[j]);
      if (lane == 0) bsm[32 * K + j] = t[j];
    }
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < K; ++j) v[j] = bsm[32 * K + j];
}

__device__ __forceinline__ void cluster_minmax(cg::cluster_group& cl, double& mn, double& mx,
                                               double (*slots)[2], double* wsm) {
  for (int off = 16; off > 0; off >>= 1) {
    mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, off));
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (lane == 0) { wsm[2 * wid] = mn; wsm[2 * wid + 1] = mx; }
  __syncthreads();
  if (wid == 0) {
    double a = lane < nw ? wsm[2 * lane] : INFINITY, b = lane < nw ? wsm[2 * lane + 1] : -INFINITY;
    for (int off = 16; off > 0; off >>= 1) {
      a = fmin(a, __shfl_xor_sync(0xffffffffu, a, off));
      b = fmax(b, __shfl_xor_sync(0xffffffffu, b, off));
    }
    if (lane == 0) {
      slots[2][0] = a;
      slots[2][1] = b;
    }
  }
  cl.sync();
  if (wid == 0) {
    double a = INFINITY, b = -INFINITY;
    if (lane < (int)cl.num_blocks()) {
      double(*rs)[2] = cl.map_shared_rank(slots, lane);
      a = rs[2][0];
      b = rs[2][1];
    }
    for (int off = 16; off > 0; off >>= 1) {
      a = fmin(a, __shfl_xor_sync(0xffffffffu, a, off));
      b = fmax(b, __shfl_xor_sync(0xffffffffu, b, off));
    }
    if (lane == 0) { wsm[64] = a; wsm[65] = b; }
  }
  __syncthreads();
  mn = wsm[64];
  mx = wsm[65];
}

__device__ __forceinline__ double expit(double x) { return 1.0 / (1.0 + exp(-x)); }

// x / b, correctly rounded, for a divisor b fixed over a pass with rb = 1 / b (correctly
// rounded).  q0 = x rb is within 1.5 ulp of x / b; one fma remainder step x - q0 b and
// correction makes it faithful, and by Markstein's theorem (P. Markstein, IBM J. Res.
// Dev. 34 (1990) 111-119: with y the correctly rounded 1/b and q faithful, r = x - q b is
// exact under an fma and q + r y rounds to the correctly rounded x / b) a second step
// gives the correctly rounded quotient, the bits of x / b.  The remainder must not
// underflow nor the products overflow, so numerators outside [2^-900, 2^900] in
// magnitude (and NaN and infinities) take the division, and so does every x when
// rb = 0 (recip_of: divisors outside [2^-64, 2^64]).  Five fp64 operations in place
// of a division routine per element, at the same bits.
__device__ __forceinline__ double recip_of(double b) {
  return (fabs(b) >= 0x1p-64 && fabs(b) <= 0x1p+64) ? 1.0 / b : 0.0;
}
__device__ __forceinline__ double div_by(double x, double b, double rb) {
  const double ax = fabs(x);
  if (!(ax >= 0x1p-900 && ax <= 0x1p+900) || rb == 0.0) return x / b;
  double q = x * rb;
  double r = fma(-q, b, x);
  q = fma(r, rb, q);
  r = fma(-q, b, x);
  return fma(r, rb, q);
}

// BT threads per CTA; the bisection evaluates L levels per pass (L = 2 for the
// 256-thread variant, 1 for the 1024-thread variant, whose register budget is 64).
// NEWTON: methods 1 and 2 only (1024 threads); otherwise the bisection only, so that
// neither variant carries the other's registers (1024-thread CTAs have 64 per thread).
template <typename RT, int BT, bool NEWTON>
__global__ void __launch_bounds__(BT) k_find_mu(const MuArgs a) {
  constexpr int L = BT <= 256 ? kBisLevels : 1, NODES = (1 << L) - 1;
  if (a.active && !*a.active) return;  // uniform across the cluster: no barrier is skipped by a subset
  cg::cluster_group cl = cg::this_cluster();
  __shared__ double slots[3][2];
  __shared__ double wsm[66];
  __shared__ double bslots[2][NODES];
  __shared__ double bsm[33 * NODES];
  __shared__ double cslots[2][5];  // the certifying Newton passes of a hinted bisection
  __shared__ double csm[33 * 5];
  extern __shared__ double2 mu_cache[];  // a.cache: (eps, w) of this thread's elements, [u][thread]
  const int gt = cl.block_rank() * blockDim.x + threadIdx.x;
  const int gs = cl.num_blocks() * blockDim.x;
  // every pass visits this thread's elements in the same order, from shared memory when
  // they fit (each thread reads back only what it stored: no barrier), else from L2
  if (a.cache) {
    for (int u = 0; u < a.cache; ++u) {
      const int e = gt + u * gs;
      mu_cache[u * blockDim.x + threadIdx.x] =
          e < a.n ? make_double2(load_eps<RT>(a, e), load_w<RT>(a, e)) : make_double2(0.0, 0.0);
    }
  }
  auto visit = [&](auto&& f) {
    if (a.cache) {  // the same elements in the same order as the L2 path
      for (int u = 0; u < a.cache; ++u)
        if (gt + u * gs < a.n) {
          const double2 c = mu_cache[u * blockDim.x + threadIdx.x];
          f(c.x, c.y);
        }
    } else {
      for_each_eps<RT, kMuCacheU>(a, gt, gs, f);
    }
  };

  // method 0 with a hint (the caller's previous mu): read before any CTA can write a.out
  const double hint = (!NEWTON && a.mu0 != nullptr) ? a.mu0[0] : 0.0;
  const bool has_hint = !NEWTON && a.mu0 != nullptr && isfinite(hint);
  // Method 2 with a warm start: the min/max pass also forms N and Z at mu0, which
  // are the first Newton evaluation whenever mu0 lies inside the bracket.
  const bool fuse_first = NEWTON && a.method == 2 && a.mu0 != nullptr;
  const double mu0v = fuse_first ? a.mu0[0] : 0.0;
  const double Tf = fmax(a.T, 1e-12), rTf = recip_of(Tf);
  double mn = INFINITY, mx = -INFINITY, N0 = 0.0, Z0 = 0.0;
  if (fuse_first) {
    visit([&](double v, double w) {
      mn = fmin(mn, v);
      mx = fmax(mx, v);
      const double p = expit(div_by(mu0v - v, Tf, rTf));
      N0 += w * p;
      Z0 += div_by(w * (p * (1.0 - p)), Tf, rTf);
    });
  } else {
    visit([&](double v, double) {
      mn = fmin(mn, v);
      mx = fmax(mx, v);
    });
  }
  cluster_minmax(cl, mn, mx, slots, wsm);
  int parity = 0;
  if (fuse_first) {
    cluster_sum2(cl, N0, Z0, slots, wsm, parity);
    parity ^= 1;
  }

  double result;
  if constexpr (!NEWTON) {
    // L levels of the bisection per pass: the counts at all 2^L - 1
    // midpoints of the next L levels (a binary tree of intervals, each midpoint
    // formed exactly as the one-level loop would form it) come from one cluster
    // reduction, then the L decisions are replayed in order; same decisions and
    // result as one level per pass, with L times fewer dependent reductions.
    const double T = a.T;
    const double span = mx - mn + 10.0 * fmax(T, 1e-6);
    double lo = mn - span, hi = mx + span;
    const double Td = T + 1e-12, iTd = 1.0 / Td;
    int it = 0;
    bool fixed = false;
    if (has_hint) {
      // Certified bracket from the hint.  N(x) = sum w / (1 + exp((e - x) / Td)) is
      // increasing in x; an evaluation N~(x) differs from it by at most E = (kpt + 24) u W
      // (kpt terms summed per thread, a reduction tree of depth <= 14, about 6 u per term
      // and u W for the rounding of the exponent's argument; W = sum w).  So once
      // N~(A) > target + margin with margin = 8 (kpt + 24) u W >= 2E, every x >= A has
      // N~(x) > target: the bisection's decision at a midpoint m >= A is "above" without
      // an evaluation, and likewise "below" for m <= B once N~(B) < target - margin.
      // Newton passes from the hint put A and B within a few margin / N' of the root,
      // each evaluating N and N' at the iterate and N at two probes around it; then the
      // levels whose midpoints lie outside (B, A) are replayed without evaluations and
      // only the last few levels are evaluated.  The decisions, and so the result, are
      // those of evaluating every level.
      const int kpt = (a.n + gs - 1) / gs;
      double A = INFINITY, B = -INFINITY;
      double m = fmin(fmax(hint, lo), hi), d = 0.0;
      for (int t = 0; t < kMuCertPasses; ++t) {
        const double pl = m - d, ph = m + d;
        double v[5] = {0.0, 0.0, 0.0, 0.0, 0.0};  // N(m), N'(m) Td, N(pl), N(ph), W
        visit([&](double ev, double w) {
          const double f = 1.0 / (1.0 + exp((ev - m) * iTd));
          v[0] += w * f;
          v[1] += w * (f * (1.0 - f));
          v[2] += w / (1.0 + exp((ev - pl) * iTd));
          v[3] += w / (1.0 + exp((ev - ph) * iTd));
          v[4] += w;
        });
        cluster_sum_n<5>(cl, v, cslots, csm, parity);
        parity ^= 1;
        const double margin = 8.0 * (kpt + 24) * 1.1102230246251565e-16 * v[4];
        const double xs[3] = {m, pl, ph}, ns[3] = {v[0], v[2], v[3]};
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          if (ns[q] > a.target + margin) A = fmin(A, xs[q]);
          if (ns[q] < a.target - margin) B = fmax(B, xs[q]);
        }
        const double Z = v[1] * iTd;
        const double bl = fmax(B, lo), bh = fmin(A, hi);
        double r = m - (v[0] - a.target) / Z;
        if (!(Z > 0.0) || !isfinite(r) || r <= bl || r >= bh) r = 0.5 * (bl + bh);
        const double floor_w = Z > 0.0 ? 2.0 * margin / Z : INFINITY;
        if (A - B <= 4.0 * floor_w) break;  // as narrow as the margin allows
        d = fmax(2.0 * fabs(r - m), floor_w);
        m = r;
      }
      while (it < a.maxiter) {  // the levels decided by the certified bracket
        const double mid = 0.5 * (lo + hi);
        double nl, nh;
        if (mid >= A) { nl = lo; nh = mid; }
        else if (mid <= B) { nl = mid; nh = hi; }
        else break;
        if (nl == lo && nh == hi) { fixed = true; break; }
        lo = nl;
        hi = nh;
        ++it;
      }
    }
    while (it < a.maxiter && !fixed) {
      double nlo[NODES + 1], nhi[NODES + 1], mid[NODES + 1];
      nlo[1] = lo;
      nhi[1] = hi;
#pragma unroll
      for (int j = 1; j <= NODES; ++j) {
        mid[j] = 0.5 * (nlo[j] + nhi[j]);
        if (2 * j + 1 <= NODES) {
          nlo[2 * j] = nlo[j];
          nhi[2 * j] = mid[j];
          nlo[2 * j + 1] = mid[j];
          nhi[2 * j + 1] = nhi[j];
        }
      }
      // exp((e - m_j) / Td) = exp((e - m_1) / Td) * exp((m_1 - m_j) / Td) where the
      // second factor is finite and nonzero; direct exp for the other midpoints
      // the factors are the same for every thread: lane j - 1 of each warp evaluates
      // factor j and the warp shares them
      double r[NODES + 1];
      bool fac[NODES + 1];
      {
        const int ln = threadIdx.x & 31;
        double zl = 0.0;
#pragma unroll
        for (int j = 1; j <= NODES; ++j)
          if (ln == j - 1) zl = (mid[1] - mid[j]) * iTd;
        const double rl = fabs(zl) < 700.0 ? exp(zl) : 0.0;
#pragma unroll
        for (int j = 1; j <= NODES; ++j) {
          fac[j] = fabs((mid[1] - mid[j]) * iTd) < 700.0;
          r[j] = __shfl_sync(0xffffffffu, rl, j - 1);
        }
      }
      double cnt[NODES];
#pragma unroll
      for (int j = 0; j < NODES; ++j) cnt[j] = 0.0;
      visit([&](double ev, double w) {
        const double g = exp((ev - mid[1]) * iTd);
#pragma unroll
        for (int j = 1; j <= NODES; ++j) {
          const double x = fac[j] ? g * r[j] : exp((ev - mid[j]) * iTd);
          cnt[j - 1] += w / (1.0 + x);
        }
      });
      cluster_sum_n<NODES>(cl, cnt, bslots, bsm, parity);
      parity ^= 1;
      int node = 1;
#pragma unroll
      for (int l = 0; l < L; ++l) {
        if (fixed || it >= a.maxiter) break;
        // node's count and midpoint by select chains (no dynamically indexed arrays)
        double cn = 0.0, mn_ = 0.0;
#pragma unroll
        for (int j = 1; j <= NODES; ++j)
          if (j == node) { cn = cnt[j - 1]; mn_ = mid[j]; }
        const bool above = cn > a.target;
        const double nl = above ? lo : mn_;
        const double nh = above ? mn_ : hi;
        if (nl == lo && nh == hi) {  // exact fixed point
          fixed = true;
          break;
        }
        lo = nl;
        hi = nh;
        node = 2 * node + (above ? 0 : 1);
        ++it;
      }
    }
    result = 0.5 * (lo + hi);
  } else {
    const double Tj = fmax(a.T, 1e-12), rTj = recip_of(Tj);
    double lo, hi, mu;
    if (a.method == 1) {
      const double span = mx - mn + 10.0 * fmax(Tj, 1e-6);
      lo = mn - span;
      hi = mx + span;
      mu = 0.5 * (lo + hi);
    } else {
      lo = mn - 50.0 * Tj;
      hi = mx + 50.0 * Tj;
      const double m0 = a.mu0 ? a.mu0[0] : 0.0;
      mu = fmin(fmax(m0, lo), hi);
    }
    const bool have_first = fuse_first && mu == mu0v;
    for (int it = 0; it < a.maxiter; ++it) {
      double N = 0.0, Z = 0.0;
      if (it == 0 && have_first) {
        N = N0;
        Z = Z0;
      } else {
        visit([&](double ev, double w) {
          const double p = expit(div_by(mu - ev, Tj, rTj));
          N += w * p;
          Z += div_by(w * (p * (1.0 - p)), Tj, rTj);
        });
        cluster_sum2(cl, N, Z, slots, wsm, parity);
        parity ^= 1;
      }
      const double g = N - a.target;
      if (g < 0) lo = mu;
      if (g > 0) hi = mu;
      double mn2 = mu - g / fmax(Z, 1e-18);
      const double mb = 0.5 * (lo + hi);
      bool newton = true;
      if (mn2 <= lo || mn2 >= hi) { mn2 = mb; newton = false; }
      mn2 = fmin(fmax(mn2, lo), hi);
      if (!isfinite(mn2)) { mn2 = mb; newton = false; }
      const double step = fabs(mn2 - mu);
      mu = mn2;
      if (newton && step <= 4.0 * 2.220446049250313e-16 * fmax(1.0, fabs(mu))) break;
    }
    if (a.method == 1) {
      double N = 0.0, dummy = 0.0;
      visit([&](double ev, double w) { N += w * expit(div_by(mu - ev, Tj, rTj)); });
      cluster_sum2(cl, N, dummy, slots, wsm, parity);
      parity ^= 1;
      if (fabs(N - a.target) > 1e-12) mu = 0.5 * (lo + hi);
    }
    result = mu;
  }
  if (cl.block_rank() == 0 && threadIdx.x == 0) a.out[0] = result;
  cl.sync();  // keep every CTA's shared memory alive until all remote reads are done
}

}  // namespace hf

using namespace hf;

namespace hf {
int find_mu_internal(void* stream, int dtype, int method, int nk1, int nk2, int nb, const void* eps,
                     const void* weights, double n_electrons, double T, int maxiter, const double* mu0,
                     double* mu_out, const int* active);
}

extern "C" int hf_find_mu(void* stream, int dtype, int method, int nk1, int nk2, int nb,
                          const void* eps, const void* weights, double n_electrons, double T,
                          int maxiter, const double* mu0, double* mu_out) {
  return hf::find_mu_internal(stream, dtype, method, nk1, nk2, nb, eps, weights, n_electrons, T, maxiter, mu0,
                              mu_out, nullptr);
}

int hf::find_mu_internal(void* stream, int dtype, int method, int nk1, int nk2, int nb, const void* eps,
                         const void* weights, double n_electrons, double T, int maxiter, const double* mu0,
                         double* mu_out, const int* active) {
  if (dtype != HF_C128 && dtype != HF_C64) return fail(HF_ERR_INVALID, "bad dtype");
  if (method < 0 || method > 2) return fail(HF_ERR_INVALID, "method must be 0, 1 or 2");
  if (nk1 < 1 || nk2 < 1 || nb < 1) return fail(HF_ERR_INVALID, "bad shape");
  if (!eps || !weights || !mu_out) return fail(HF_ERR_INVALID, "NULL argument");
  const bool single = dtype == HF_C64;
  if (maxiter <= 0) {
    if (method == 0) maxiter = single ? 30 : 54;
    else if (method == 1) maxiter = single ? 15 : 25;
    else maxiter = 25;
  }
  const size_t n_all = (size_t)nk1 * (size_t)nk2 * (size_t)nb;
  if (n_all > (size_t)INT_MAX) return fail(HF_ERR_UNSUPPORTED, "more than 2^31 - 1 eigenvalues");
  MuArgs a;
  a.eps = eps; a.w = weights;
  a.n = (int)n_all; a.nb = nb; a.method = method; a.maxiter = maxiter;
  a.target = n_electrons; a.T = T; a.mu0 = mu0; a.out = mu_out; a.active = active;
  // bisection: every pass evaluates 3 midpoints per eigenvalue, so small
  // meshes use 256-thread CTAs with one eigenvalue per thread, spread over up to 16
  // SMs; the Newton variants (one evaluation per pass, bound by the cluster barrier
  // of each pass): up to four per thread of 1024-thread CTAs
  const int threads = (method == 0 && a.n <= kMuMaxCluster * 256) ? 256 : kMuThreads;
  const int per_cta = method == 0 ? threads : kMuCacheU * kMuThreads;
  int csize = (a.n + per_cta - 1) / per_cta;
  if (csize < 1) csize = 1;
  if (csize > kMuMaxCluster) csize = kMuMaxCluster;
  const void* fn = method != 0 ? (single ? (const void*)k_find_mu<float, kMuThreads, true>
                                         : (const void*)k_find_mu<double, kMuThreads, true>)
                   : threads == 256 ? (single ? (const void*)k_find_mu<float, 256, false>
                                              : (const void*)k_find_mu<double, 256, false>)
                                    : (single ? (const void*)k_find_mu<float, kMuThreads, false>
                                              : (const void*)k_find_mu<double, kMuThreads, false>);
  unsigned long long ctx = 0;
  if (int cst = context_id(&ctx)) return cst;
  // per (kernel, context), set up once under a lock: the largest schedulable cluster
  // size (beyond the portable 8 only as large as the device can co-schedule) and the
  // opt-in for the shared-memory cache of the largest block
  static std::mutex mu_setup;
  static std::map<std::pair<const void*, unsigned long long>, int> max_cluster;
  {
    std::lock_guard<std::mutex> lk(mu_setup);
    auto key = std::make_pair(fn, ctx);
    auto it = max_cluster.find(key);
    if (it == max_cluster.end()) {
      int mc = 8;
      if (cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess) {
        cudaLaunchConfig_t q = {};
        q.gridDim = dim3(kMuMaxCluster, 1, 1);
        q.blockDim = dim3(threads, 1, 1);
        cudaLaunchAttribute qa[1];
        qa[0].id = cudaLaunchAttributeClusterDimension;
        qa[0].val.clusterDim.x = kMuMaxCluster;
        qa[0].val.clusterDim.y = 1;
        qa[0].val.clusterDim.z = 1;
        q.attrs = qa;
        q.numAttrs = 1;
        int c = 0;
        if (cudaOccupancyMaxPotentialClusterSize(&c, fn, &q) == cudaSuccess && c >= 8) mc = c < kMuMaxCluster ? c : kMuMaxCluster;
      }
      cudaGetLastError();  // a refused query leaves the portable size
      HF_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)((size_t)kMuCacheMax * kMuThreads * sizeof(double2))));
      it = max_cluster.emplace(key, mc).first;
    }
    if (csize > it->second) csize = it->second;
  }
  {
    const long long per = ((long long)a.n + (long long)csize * threads - 1) / ((long long)csize * threads);
    a.cache = per <= kMuCacheMax ? (int)per : 0;
  }
  const size_t cache_bytes = (size_t)a.cache * threads * sizeof(double2);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(csize, 1, 1);
  cfg.blockDim = dim3(threads, 1, 1);
  cfg.dynamicSmemBytes = a.cache ? cache_bytes : 0;
  cfg.stream = static_cast<cudaStream_t>(stream);
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = csize;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (method != 0) {
    if (single) HF_CUDA(cudaLaunchKernelEx(&cfg, k_find_mu<float, kMuThreads, true>, a));
    else HF_CUDA(cudaLaunchKernelEx(&cfg, k_find_mu<double, kMuThreads, true>, a));
  } else if (threads == 256) {
    if (single) HF_CUDA(cudaLaunchKernelEx(&cfg, k_find_mu<float, 256, false>, a));
    else HF_CUDA(cudaLaunchKernelEx(&cfg, k_find_mu<double, 256, false>, a));
  } else {
    if (single) HF_CUDA(cudaLaunchKernelEx(&cfg, k_find_mu<float, kMuThreads, false>, a));
    else HF_CUDA(cudaLaunchKernelEx(&cfg, k_find_mu<double, kMuThreads, false>, a));
  }
  return HF_OK;
}
