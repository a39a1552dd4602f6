// Device operations used by the SCF (reference_scf.py) and trust-region Newton
// (solver.py:686-1078) loops: occupations, residuals and commutators, the DIIS
// Gram matrix, linear combinations, joint (X, p) inner products, the Newton
// preconditioner and the two halves of the Hessian-vector product.
//
// All arrays are complex128 / float64 (the loops run in FP64).  Reductions are
// deterministic: per-CTA Neumaier partials, then one CTA sums them in order.
#include "common.cuh"
#include "perk.cuh"

namespace hf {

constexpr int kOpsThreads = 256;
constexpr int kOpsBlocks = 148 * 4;
constexpr int kOpsMaxSums = 32;

__device__ __forceinline__ double sigm(double x) { return 1.0 / (1.0 + exp(-x)); }

template <int NS>
__device__ __forceinline__ void write_partials(KSum (&acc)[NS], double* part, double* sm) {
  for (int q = 0; q < NS; ++q) {
    KSum r = block_reduce(acc[q], sm);
    if (threadIdx.x == 0) {
      part[((size_t)blockIdx.x * NS + q) * 2] = r.s;
      part[((size_t)blockIdx.x * NS + q) * 2 + 1] = r.c;
    }
  }
}

// Finish of the device reductions: sum q of ns gets one CTA, whose threads take the
// block partials (Neumaier pairs) b = t, t + blockDim, ... and merge them with the
// fixed-shape block reduction, so the result is deterministic for a launch shape.
// (One warp walking every partial in one dependent chain took ~150 us at 592 blocks.)
constexpr int kSumThreads = 128;
__global__ void __launch_bounds__(kSumThreads) k_sum_partials(const double* __restrict__ part, int nblk, int ns,
                                                              double* __restrict__ out) {
  __shared__ double sm[2 * 32];
  const int q = blockIdx.x;
  KSum t;
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) {
    t.add(part[((size_t)b * ns + q) * 2]);
    t.add(part[((size_t)b * ns + q) * 2 + 1]);
  }
  t = block_reduce(t, sm);
  if (threadIdx.x == 0) out[q] = t.value();
}

static int nblocks(size_t n) {
  size_t b = (n + kOpsThreads - 1) / kOpsThreads;
  if (b < 1) b = 1;
  if (b > (size_t)kOpsBlocks) b = kOpsBlocks;
  return (int)b;
}

// ------------------------------------------------------------ occupations --
// mode 0: fermidirac(eps - mu, T) = expit(-(eps - mu)/(T + 1e-12))  (utils.py:51-53)
// mode 1: sigmoid((mu - eps)/max(T, 1e-12))                        (solver.py:394)
// mode 2: eps + level_shift (1 - fermidirac(eps - mu, T))           (reference_scf.py:92)
__global__ void k_fermi(size_t n, const double* __restrict__ eps, const double* __restrict__ mu, double T,
                        int mode, double shift, double* __restrict__ out) {
  const double m = mu[0];
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const double x = eps[e];
    if (mode == 0) out[e] = sigm(-(x - m) / (T + 1e-12));
    else if (mode == 1) out[e] = sigm((m - x) / fmax(T, 1e-12));
    else out[e] = x + shift * (1.0 - sigm(-(x - m) / (T + 1e-12)));
  }
}

// --------------------------------------------------------- SCF residuals --
// delta = Pn - P, comm = F P - P F (stored), sums: w|delta|^2, w|comm|^2, w Re tr(F delta)
// comm_slot (may be NULL): comm is the history slot *comm_slot of comm_stride elements each
__global__ void k_scf_residuals(int nk, int nb, const double2* __restrict__ F, const double2* __restrict__ P,
                                const double2* __restrict__ Pn, const double* __restrict__ w,
                                double2* __restrict__ comm, double2* __restrict__ delta, double* part,
                                const int* __restrict__ comm_slot, size_t comm_stride) {
  if (comm && comm_slot) comm += (size_t)(*comm_slot) * comm_stride;
  extern __shared__ double2 smd[];
  __shared__ double red[64];
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const int nb2 = nb * nb;
  double2* f = smd + (size_t)wi * 3 * nb2;
  double2* pp = f + nb2;
  double2* dd = pp + nb2;
  KSum acc[3];
  for (int k = blockIdx.x * wpb + wi; k < nk; k += gridDim.x * wpb) {
    const size_t base = (size_t)k * nb2;
    const double wk = w[k];
    for (int e = lane; e < nb2; e += 32) {
      f[e] = F[base + e];
      pp[e] = P[base + e];
      const double2 d = csub(Pn[base + e], pp[e]);
      dd[e] = d;
      if (delta) delta[base + e] = d;
      acc[0].add(wk * (d.x * d.x + d.y * d.y));
    }
    __syncwarp();
    for (int e = lane; e < nb2; e += 32) {
      const int i = e / nb, j = e - i * nb;
      double2 c = make_double2(0.0, 0.0);
      double2 tr = make_double2(0.0, 0.0);
      for (int m = 0; m < nb; ++m) {
        c = cadd(c, csub(cmul(f[i * nb + m], pp[m * nb + j]), cmul(pp[i * nb + m], f[m * nb + j])));
      }
      if (comm) comm[base + e] = c;
      acc[1].add(wk * (c.x * c.x + c.y * c.y));
      tr = cmul(f[e], dd[j * nb + i]);  // F_ij delta_ji
      acc[2].add(wk * tr.x);
    }
    __syncwarp();
  }
  write_partials<3>(acc, part, red);
}

// ------------------------------------------------------- DIIS Gram matrix --
// B[i][j] = sum_k w_k Re tr(R_i^H R_j) for i, j < n (R_i at R + i*stride)
// N (history slots) is a template parameter so that every loop has a compile-time
// trip count and the N (N + 1) / 2 accumulators stay in registers.
template <int N>
__global__ void k_gram(size_t stride, size_t len, int nb2, const double2* __restrict__ R,
                       const double* __restrict__ w, double* part) {
  __shared__ double red[64];
  constexpr int np = N * (N + 1) / 2;
  // a thread sums its few elements in plain FP64; the thread, block and grid partials
  // are then merged with compensated (Neumaier) sums
  double acc[np];
#pragma unroll
  for (int q = 0; q < np; ++q) acc[q] = 0.0;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < len; e += (size_t)gridDim.x * blockDim.x) {
    const double wk = w[e / nb2];
    double2 r[N];
#pragma unroll
    for (int i = 0; i < N; ++i) r[i] = R[i * stride + e];
    int q = 0;
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
      for (int j = i; j < N; ++j, ++q) acc[q] = fma(wk, fma(r[i].x, r[j].x, r[i].y * r[j].y), acc[q]);
  }
#pragma unroll
  for (int q = 0; q < np; ++q) {
    KSum t;
    t.add(acc[q]);
    KSum rr = block_reduce(t, red);
    if (threadIdx.x == 0) {
      part[((size_t)blockIdx.x * np + q) * 2] = rr.s;
      part[((size_t)blockIdx.x * np + q) * 2 + 1] = rr.c;
    }
  }
}

// One row of the DIIS Gram matrix: b[j] = sum_k w_k Re tr(R_i^H R_j) for j < N and a
// fixed i.  A DIIS step replaces one history slot, so only that slot's row changes;
// the SCF driver keeps the rest of B and refreshes the row with one launch.  Every
// entry is formed exactly as in k_gram (fma(x_i, x_j, y_i y_j) is symmetric in i, j).
template <int N>
__global__ void k_gram_row(size_t stride, size_t len, int nb2, const double2* __restrict__ R, int inew,
                           const double* __restrict__ w, double* part, const int* __restrict__ inew_dev = nullptr) {
  if (inew_dev) inew = *inew_dev;
  __shared__ double red[64];
  double acc[N];
#pragma unroll
  for (int q = 0; q < N; ++q) acc[q] = 0.0;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < len; e += (size_t)gridDim.x * blockDim.x) {
    const double wk = w[e / nb2];
    const double2 a = R[inew * stride + e];
#pragma unroll
    for (int j = 0; j < N; ++j) {
      const double2 b = R[j * stride + e];
      acc[j] = fma(wk, fma(a.x, b.x, a.y * b.y), acc[j]);
    }
  }
#pragma unroll
  for (int q = 0; q < N; ++q) {
    KSum t;
    t.add(acc[q]);
    KSum rr = block_reduce(t, red);
    if (threadIdx.x == 0) {
      part[((size_t)blockIdx.x * N + q) * 2] = rr.s;
      part[((size_t)blockIdx.x * N + q) * 2 + 1] = rr.c;
    }
  }
}

// out = sum_i c_i X_i (+ optional herm)
__global__ void k_lincomb(int n, size_t stride, size_t len, int nb, const double2* __restrict__ X,
                          const double* __restrict__ c, double2* __restrict__ out) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < len; e += (size_t)gridDim.x * blockDim.x) {
    double2 acc = make_double2(0.0, 0.0);
    for (int i = 0; i < n; ++i) acc = cadd(acc, cscale(X[i * stride + e], c[i]));
    out[e] = acc;
  }
}

// out = a x + b y, hermitised when herm != 0 (complex arrays, nb x nb per k)
__global__ void k_axpby(size_t nk, int nb, double a, const double2* __restrict__ x, double b,
                        const double2* __restrict__ y, int herm, double2* __restrict__ out) {
  const int nb2 = nb * nb;
  const size_t n = nk * nb2;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const double2 v = cadd(cscale(x[e], a), y ? cscale(y[e], b) : make_double2(0.0, 0.0));
    if (!herm) { out[e] = v; continue; }
    const size_t k = e / nb2;
    const int r = (int)(e - k * nb2), i = r / nb, j = r - (r / nb) * nb;
    const size_t t = k * nb2 + (size_t)j * nb + i;
    const double2 u = cadd(cscale(x[t], a), y ? cscale(y[t], b) : make_double2(0.0, 0.0));
    out[e] = make_double2(0.5 * (v.x + u.x), 0.5 * (v.y - u.y));
  }
}

__global__ void k_axpby_real(size_t n, double a, const double* __restrict__ x, double b,
                             const double* __restrict__ y, double* __restrict__ out) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
    out[e] = a * x[e] + (y ? b * y[e] : 0.0);
}

// joint inner product sum_k wX_k sum Re(conj(aX) bX) + sum_k wp_k sum ap bp  (solver.py:205-233, 783-787)
__global__ void k_jdot(size_t nk, int nb, const double2* __restrict__ aX, const double2* __restrict__ bX,
                       const double* __restrict__ wX, const double* __restrict__ ap, const double* __restrict__ bp,
                       const double* __restrict__ wp, double* part) {
  __shared__ double red[64];
  KSum acc[1];
  const int nb2 = nb * nb;
  if (aX) {
    const size_t n = nk * nb2;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
      const double wk = wX ? wX[e / nb2] : 1.0;
      acc[0].add(wk * (aX[e].x * bX[e].x + aX[e].y * bX[e].y));
    }
  }
  if (ap) {
    const size_t n = nk * nb;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
      const double wk = wp ? wp[e / nb] : 1.0;
      acc[0].add(wk * ap[e] * bp[e]);
    }
  }
  write_partials<1>(acc, part, red);
}

// Up to four joint inner products in one pass: product q is accumulated by every thread
// exactly as k_jdot accumulates it (same grid, same elements, same order) and finished
// with the same reductions, so each value equals the separate hf_jdot's bit for bit.
struct JdotSpec {
  const double2 *aX, *bX;
  const double *wX, *ap, *bp, *wp;
};
struct JdotMulti {
  JdotSpec d[4];
  int n;
};

__global__ void k_jdot_multi(size_t nk, int nb, const __grid_constant__ JdotMulti m, double* part) {
  __shared__ double red[64];
  KSum acc[4];
  const int nb2 = nb * nb;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    if (q >= m.n) break;
    const JdotSpec& d = m.d[q];
    if (d.aX) {
      const size_t n = nk * nb2;
      for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const double wk = d.wX ? d.wX[e / nb2] : 1.0;
        acc[q].add(wk * (d.aX[e].x * d.bX[e].x + d.aX[e].y * d.bX[e].y));
      }
    }
    if (d.ap) {
      const size_t n = nk * nb;
      for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const double wk = d.wp ? d.wp[e / nb] : 1.0;
        acc[q].add(wk * d.ap[e] * d.bp[e]);
      }
    }
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    if (q >= m.n) break;
    KSum r = block_reduce(acc[q], red);
    if (threadIdx.x == 0) {
      part[((size_t)blockIdx.x * m.n + q) * 2] = r.s;
      part[((size_t)blockIdx.x * m.n + q) * 2 + 1] = r.c;
    }
  }
}

// ---------------------------------------------------------------- Newton --
// G = skew((p_j - p_i) Ft) offdiag, eps = Re diag(Ft)                 (solver.py:898-900)
__global__ void k_orbital_grad(size_t nk, int nb, const double2* __restrict__ Ft, const double* __restrict__ p,
                               double2* __restrict__ G, double* __restrict__ eps) {
  const int nb2 = nb * nb;
  const size_t n = nk * nb2;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const size_t k = e / nb2;
    const int r = (int)(e - k * nb2), i = r / nb, j = r - (r / nb) * nb;
    const double2 f = Ft[e];
    if (i == j) {
      G[e] = make_double2(0.0, 0.0);
      if (eps) eps[k * nb + i] = f.x;
      continue;
    }
    const double2 ft = Ft[k * nb2 + (size_t)j * nb + i];
    const double d = p[k * nb + j] - p[k * nb + i];
    G[e] = make_double2(0.5 * d * (f.x + ft.x), 0.5 * d * (f.y - ft.y));
  }
}

// z = (rX / sqrt(gap^2 + lam^2), rp p(1-p)/T) with p clipped to [occ_clip, 1-occ_clip]; sum w2d zp
__global__ void k_newton_prec(size_t nk, int nb, const double2* __restrict__ rX, const double* __restrict__ rp,
                              const double* __restrict__ eps, const double* __restrict__ p, double lam, double T,
                              double clipv, const double* __restrict__ w2d, double2* __restrict__ zX,
                              double* __restrict__ zp, double* part) {
  __shared__ double red[64];
  KSum acc[1];
  const int nb2 = nb * nb;
  const size_t n = nk * nb2;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const size_t k = e / nb2;
    const int r = (int)(e - k * nb2), i = r / nb, j = r - (r / nb) * nb;
    const double gap = eps[k * nb + i] - eps[k * nb + j];
    const double d = sqrt(gap * gap + lam * lam);
    zX[e] = make_double2(rX[e].x / d, rX[e].y / d);
  }
  const size_t nv = nk * nb;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < nv; e += (size_t)gridDim.x * blockDim.x) {
    const double pc = fmin(fmax(p[e], clipv), 1.0 - clipv);
    const double z = rp[e] * (pc * (1.0 - pc) / T);
    zp[e] = z;
    acc[0].add(w2d[e / nb] * z);
  }
  write_partials<1>(acc, part, red);
}

__global__ void k_sub_scalar(size_t n, double* __restrict__ x, const double* __restrict__ c, double scale) {
  const double v = c[0] * scale;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) x[e] -= v;
}

// dP = herm(Q M Q^H), M = X o (p_j - p_i) + diag(dp)                 (solver.py:916-919)
__global__ void k_newton_dP(int nk, int nb, const double2* __restrict__ Q, const double2* __restrict__ X,
                            const double* __restrict__ dp, const double* __restrict__ p, double2* __restrict__ dP) {
  extern __shared__ double2 smd[];
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const int nb2 = nb * nb;
  double2* q = smd + (size_t)wi * 3 * nb2;
  double2* m = q + nb2;
  double2* t = m + nb2;
  for (int k = blockIdx.x * wpb + wi; k < nk; k += gridDim.x * wpb) {
    const size_t base = (size_t)k * nb2;
    for (int e = lane; e < nb2; e += 32) {
      const int i = e / nb, j = e - i * nb;
      q[e] = Q[base + e];
      const double2 x = X[base + e];
      const double d = p[(size_t)k * nb + j] - p[(size_t)k * nb + i];
      double2 v = make_double2(x.x * d, x.y * d);
      if (i == j) v.x += dp[(size_t)k * nb + i];
      m[e] = v;
    }
    __syncwarp();
    for (int e = lane; e < nb2; e += 32) {  // t = Q M
      const int i = e / nb, j = e - i * nb;
      double2 acc = make_double2(0.0, 0.0);
      for (int n = 0; n < nb; ++n) acc = cadd(acc, cmul(q[i * nb + n], m[n * nb + j]));
      t[e] = acc;
    }
    __syncwarp();
    for (int e = lane; e < nb2; e += 32) {  // m = t Q^H
      const int i = e / nb, j = e - i * nb;
      double2 acc = make_double2(0.0, 0.0);
      for (int n = 0; n < nb; ++n) acc = cadd(acc, cmulc(t[i * nb + n], q[j * nb + n]));
      m[e] = acc;
    }
    __syncwarp();
    for (int e = lane; e < nb2; e += 32) {
      const int i = e / nb, j = e - i * nb;
      const double2 x = m[e], y = m[j * nb + i];
      dP[base + e] = make_double2(0.5 * (x.x + y.x), 0.5 * (x.y - y.y));
    }
    __syncwarp();
  }
}

// St = Q^H (Fr - h) Q; A = Ft X - X Ft + St; C = dpij Ft + pij A;
// HX = skew(C) offdiag; Hp = Re diag(A) + T/(pc(1-pc)) dp            (solver.py:920-929)
__global__ void k_newton_hvp(int nk, int nb, const double2* __restrict__ Q, const double2* __restrict__ Ft,
                             const double2* __restrict__ X, const double* __restrict__ dp,
                             const double* __restrict__ p, const double2* __restrict__ Fr,
                             const double2* __restrict__ h, double T, double clipv, double pen,
                             const double2* __restrict__ dPpen, double2* __restrict__ HX, double* __restrict__ Hp,
                             const double* __restrict__ w2d, double* part) {
  extern __shared__ double2 smd[];
  __shared__ double red[64];
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const int nb2 = nb * nb;
  double2* q = smd + (size_t)wi * 5 * nb2;
  double2* s = q + nb2;
  double2* t = s + nb2;
  double2* f = t + nb2;
  double2* x = f + nb2;
  KSum acc[1];
  for (int k = blockIdx.x * wpb + wi; k < nk; k += gridDim.x * wpb) {
    const size_t base = (size_t)k * nb2, vb = (size_t)k * nb;
    for (int e = lane; e < nb2; e += 32) {
      q[e] = Q[base + e];
      double2 r = csub(Fr[base + e], h[base + e]);
      if (dPpen) r = cadd(r, cscale(dPpen[base + e], pen));
      s[e] = r;
      f[e] = Ft[base + e];
      x[e] = X[base + e];
    }
    __syncwarp();
    warp_qhaq(q, s, t, nb, lane);  // s <- Q^H resp Q
    __syncwarp();
    for (int e = lane; e < nb2; e += 32) {  // t = A
      const int i = e / nb, j = e - i * nb;
      double2 acc2 = s[e];
      for (int n = 0; n < nb; ++n)
        acc2 = cadd(acc2, csub(cmul(f[i * nb + n], x[n * nb + j]), cmul(x[i * nb + n], f[n * nb + j])));
      t[e] = acc2;
    }
    __syncwarp();
    for (int e = lane; e < nb2; e += 32) {  // C into s
      const int i = e / nb, j = e - i * nb;
      const double ddp = dp[vb + j] - dp[vb + i];
      const double dpp = p[vb + j] - p[vb + i];
      s[e] = cadd(cscale(f[e], ddp), cscale(t[e], dpp));
    }
    __syncwarp();
    for (int e = lane; e < nb2; e += 32) {
      const int i = e / nb, j = e - i * nb;
      if (i == j) { HX[base + e] = make_double2(0.0, 0.0); continue; }
      const double2 c = s[e], ct = s[j * nb + i];
      HX[base + e] = make_double2(0.5 * (c.x - ct.x), 0.5 * (c.y + ct.y));
    }
    for (int i = lane; i < nb; i += 32) {
      const double pc = fmin(fmax(p[vb + i], clipv), 1.0 - clipv);
      const double v = t[i * nb + i].x + (T / (pc * (1.0 - pc))) * dp[vb + i];
      Hp[vb + i] = v;
      acc[0].add(w2d[k] * v);
    }
    __syncwarp();
  }
  write_partials<1>(acc, part, red);
}

// C = A B per k
__global__ void k_matmul(int nk, int nb, const double2* __restrict__ A, const double2* __restrict__ B,
                         double2* __restrict__ Cm) {
  extern __shared__ double2 smd[];
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const int nb2 = nb * nb;
  double2* a = smd + (size_t)wi * 2 * nb2;
  double2* b = a + nb2;
  for (int k = blockIdx.x * wpb + wi; k < nk; k += gridDim.x * wpb) {
    const size_t base = (size_t)k * nb2;
    for (int e = lane; e < nb2; e += 32) { a[e] = A[base + e]; b[e] = B[base + e]; }
    __syncwarp();
    for (int e = lane; e < nb2; e += 32) {
      const int i = e / nb, j = e - i * nb;
      double2 acc = make_double2(0.0, 0.0);
      for (int n = 0; n < nb; ++n) acc = cadd(acc, cmul(a[i * nb + n], b[n * nb + j]));
      Cm[base + e] = acc;
    }
    __syncwarp();
  }
}

__global__ void k_real_diag(size_t nk, int nb, const double2* __restrict__ A, double* __restrict__ d) {
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < nk * nb; e += (size_t)gridDim.x * blockDim.x) {
    const size_t k = e / nb;
    const int i = (int)(e - k * nb);
    d[e] = A[k * (size_t)nb * nb + (size_t)i * nb + i].x;
  }
}

static int perk_grid(int nk) {
  int b = (nk + 3) / 4;
  if (b > 148 * 16) b = 148 * 16;
  return b < 1 ? 1 : b;
}

static int finish(cudaStream_t s, double* part, int nblk, int ns, double* out) {
  HF_LAUNCH_CHECK("reduction kernel");
  k_sum_partials<<<ns, kSumThreads, 0, s>>>(part, nblk, ns, out);
  HF_LAUNCH_CHECK("k_sum_partials");
  return HF_OK;
}

}  // namespace hf

using namespace hf;

#define HF_S static_cast<cudaStream_t>(stream)

extern "C" int hf_ops_workspace_size(size_t* bytes) {
  if (!bytes) return fail(HF_ERR_INVALID, "bytes is NULL");
  *bytes = (size_t)kOpsBlocks * 2 * kOpsMaxSums * 2 * sizeof(double);
  return HF_OK;
}

extern "C" int hf_fermi(void* stream, size_t n, const double* eps, const double* mu, double T, int mode,
                        double shift, double* out) {
  if (!eps || !mu || !out || mode < 0 || mode > 2) return fail(HF_ERR_INVALID, "hf_fermi: bad argument");
  if (n == 0) return HF_OK;
  k_fermi<<<nblocks(n), kOpsThreads, 0, HF_S>>>(n, eps, mu, T, mode, shift, out);
  HF_LAUNCH_CHECK("k_fermi");
  return HF_OK;
}

extern "C" int hf_scf_residuals(void* stream, int nk, int nb, const void* F, const void* P, const void* Pn,
                                const double* w, void* comm, void* delta, double* sums3, void* ws) {
  if (!F || !P || !Pn || !w || !sums3 || !ws || nb > 32) return fail(HF_ERR_INVALID, "hf_scf_residuals: bad argument");
  const int g = perk_grid(nk);
  const size_t sm = (size_t)3 * nb * nb * sizeof(double2) * 4;
  HF_SMEM_CAP(k_scf_residuals);
  k_scf_residuals<<<g, 128, sm, HF_S>>>(nk, nb, (const double2*)F, (const double2*)P, (const double2*)Pn, w,
                                        (double2*)comm, (double2*)delta, (double*)ws, nullptr, 0);
  return finish(HF_S, (double*)ws, g, 3, sums3);
}

// The SCF steps of a DIIS history whose current slot is a device int (the device-resident
// SCF loop): residuals with the commutator into slot *slot of R, F copied into slot *slot
// of Fhist, and row *slot of the Gram matrix.
int hf::scf_residuals_slot(void* stream, int nk, int nb, const void* F, const void* P, const void* Pn,
                           const double* w, void* R, size_t stride, const int* slot, void* delta, double* sums3,
                           void* ws) {
  const int g = perk_grid(nk);
  const size_t sm = (size_t)3 * nb * nb * sizeof(double2) * 4;
  HF_SMEM_CAP(k_scf_residuals);
  k_scf_residuals<<<g, 128, sm, HF_S>>>(nk, nb, (const double2*)F, (const double2*)P, (const double2*)Pn, w,
                                        (double2*)R, (double2*)delta, (double*)ws, slot, stride);
  return finish(HF_S, (double*)ws, g, 3, sums3);
}

__global__ void k_copy_to_slot(size_t n, const double2* __restrict__ x, double2* __restrict__ hist,
                               const int* __restrict__ slot) {
  double2* dst = hist + (size_t)(*slot) * n;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
    dst[e] = x[e];
}

int hf::copy_to_slot(void* stream, size_t n, const void* x, void* hist, const int* slot) {
  k_copy_to_slot<<<nblocks(n), kOpsThreads, 0, HF_S>>>(n, (const double2*)x, (double2*)hist, slot);
  HF_LAUNCH_CHECK("k_copy_to_slot");
  return HF_OK;
}

int hf::gram_row_slot(void* stream, int n, const int* slot, size_t stride, int nk, int nb, const void* R,
                      const double* w, double* b_out, void* ws) {
  if (n < 1 || n > 16) return fail(HF_ERR_INVALID, "gram_row_slot: 1 <= n <= 16");
  const size_t len = (size_t)nk * nb * nb;
  const int g = nblocks(len);
  switch (n) {
#define HF_GRAM_ROW(N)                                                                                      \
  case N:                                                                                                   \
    k_gram_row<N><<<g, kOpsThreads, 0, HF_S>>>(stride, len, nb * nb, (const double2*)R, 0, w, (double*)ws, \
                                                slot);                                                      \
    break;
    HF_GRAM_ROW(1) HF_GRAM_ROW(2) HF_GRAM_ROW(3) HF_GRAM_ROW(4) HF_GRAM_ROW(5) HF_GRAM_ROW(6) HF_GRAM_ROW(7)
    HF_GRAM_ROW(8) HF_GRAM_ROW(9) HF_GRAM_ROW(10) HF_GRAM_ROW(11) HF_GRAM_ROW(12) HF_GRAM_ROW(13)
    HF_GRAM_ROW(14) HF_GRAM_ROW(15) HF_GRAM_ROW(16)
#undef HF_GRAM_ROW
  }
  return finish(HF_S, (double*)ws, g, n, b_out);
}

extern "C" int hf_gram(void* stream, int n, size_t stride, int nk, int nb, const void* R, const double* w,
                       double* B_out, void* ws) {
  if (n < 1 || n > 6 || !R || !w || !B_out || !ws) return fail(HF_ERR_INVALID, "hf_gram: 1 <= n <= 6");
  const size_t len = (size_t)nk * nb * nb;
  const int g = nblocks(len);
  switch (n) {
#define HF_GRAM(N) \
  case N: k_gram<N><<<g, kOpsThreads, 0, HF_S>>>(stride, len, nb * nb, (const double2*)R, w, (double*)ws); break;
    HF_GRAM(1) HF_GRAM(2) HF_GRAM(3) HF_GRAM(4) HF_GRAM(5) HF_GRAM(6)
#undef HF_GRAM
  }
  return finish(HF_S, (double*)ws, g, n * (n + 1) / 2, B_out);
}

extern "C" int hf_gram_row(void* stream, int n, int i, size_t stride, int nk, int nb, const void* R,
                           const double* w, double* b_out, void* ws) {
  if (n < 1 || n > 16 || i < 0 || i >= n || !R || !w || !b_out || !ws)
    return fail(HF_ERR_INVALID, "hf_gram_row: 1 <= n <= 16, 0 <= i < n");
  const size_t len = (size_t)nk * nb * nb;
  const int g = nblocks(len);
  switch (n) {
#define HF_GRAM_ROW(N)                                                                                    \
  case N:                                                                                                 \
    k_gram_row<N><<<g, kOpsThreads, 0, HF_S>>>(stride, len, nb * nb, (const double2*)R, i, w, (double*)ws); \
    break;
    HF_GRAM_ROW(1) HF_GRAM_ROW(2) HF_GRAM_ROW(3) HF_GRAM_ROW(4) HF_GRAM_ROW(5) HF_GRAM_ROW(6) HF_GRAM_ROW(7)
    HF_GRAM_ROW(8) HF_GRAM_ROW(9) HF_GRAM_ROW(10) HF_GRAM_ROW(11) HF_GRAM_ROW(12) HF_GRAM_ROW(13)
    HF_GRAM_ROW(14) HF_GRAM_ROW(15) HF_GRAM_ROW(16)
#undef HF_GRAM_ROW
  }
  return finish(HF_S, (double*)ws, g, n, b_out);
}

extern "C" int hf_lincomb(void* stream, int n, size_t stride, size_t len, const void* X, const double* c, void* out) {
  if (n < 1 || !X || !c || !out) return fail(HF_ERR_INVALID, "hf_lincomb: bad argument");
  k_lincomb<<<nblocks(len), kOpsThreads, 0, HF_S>>>(n, stride, len, 0, (const double2*)X, c, (double2*)out);
  HF_LAUNCH_CHECK("k_lincomb");
  return HF_OK;
}

extern "C" int hf_axpby(void* stream, size_t nk, int nb, double a, const void* x, double b, const void* y,
                        int herm, void* out) {
  if (!x || !out) return fail(HF_ERR_INVALID, "hf_axpby: bad argument");
  if (herm && (out == x || out == y)) return fail(HF_ERR_INVALID, "hf_axpby: herm output may not alias inputs");
  k_axpby<<<nblocks(nk * nb * nb), kOpsThreads, 0, HF_S>>>(nk, nb, a, (const double2*)x, b, (const double2*)y,
                                                         herm, (double2*)out);
  HF_LAUNCH_CHECK("k_axpby");
  return HF_OK;
}

extern "C" int hf_axpby_real(void* stream, size_t n, double a, const double* x, double b, const double* y,
                             double* out) {
  if (!x || !out) return fail(HF_ERR_INVALID, "hf_axpby_real: bad argument");
  k_axpby_real<<<nblocks(n), kOpsThreads, 0, HF_S>>>(n, a, x, b, y, out);
  HF_LAUNCH_CHECK("k_axpby_real");
  return HF_OK;
}

extern "C" int hf_jdot(void* stream, size_t nk, int nb, const void* aX, const void* bX, const double* wX,
                       const double* ap, const double* bp, const double* wp, double* out, void* ws) {
  if (!out || !ws) return fail(HF_ERR_INVALID, "hf_jdot: bad argument");
  const int g = nblocks(nk * nb * nb);
  k_jdot<<<g, kOpsThreads, 0, HF_S>>>(nk, nb, (const double2*)aX, (const double2*)bX, wX, ap, bp, wp, (double*)ws);
  return finish(HF_S, (double*)ws, g, 1, out);
}

// n (1..4) joint inner products of hf_jdot's form into out[0..n) in one pass
int hf::jdot_multi(void* stream, size_t nk, int nb, int n, const void* const* aX, const void* const* bX,
                   const double* const* wX, const double* const* ap, const double* const* bp,
                   const double* const* wp, double* out, void* ws) {
  if (n < 1 || n > 4 || !out || !ws) return fail(HF_ERR_INVALID, "jdot_multi: 1 <= n <= 4");
  JdotMulti m;
  m.n = n;
  for (int q = 0; q < 4; ++q) {
    const bool on = q < n;
    m.d[q].aX = on ? static_cast<const double2*>(aX[q]) : nullptr;
    m.d[q].bX = on ? static_cast<const double2*>(bX[q]) : nullptr;
    m.d[q].wX = on ? wX[q] : nullptr;
    m.d[q].ap = on ? ap[q] : nullptr;
    m.d[q].bp = on ? bp[q] : nullptr;
    m.d[q].wp = on ? wp[q] : nullptr;
  }
  const int g = nblocks(nk * nb * nb);
  k_jdot_multi<<<g, kOpsThreads, 0, HF_S>>>(nk, nb, m, (double*)ws);
  return finish(HF_S, (double*)ws, g, n, out);
}

extern "C" int hf_orbital_grad(void* stream, size_t nk, int nb, const void* Ft, const double* p, void* G, double* eps) {
  if (!Ft || !p || !G) return fail(HF_ERR_INVALID, "hf_orbital_grad: bad argument");
  k_orbital_grad<<<nblocks(nk * nb * nb), kOpsThreads, 0, HF_S>>>(nk, nb, (const double2*)Ft, p, (double2*)G, eps);
  HF_LAUNCH_CHECK("k_orbital_grad");
  return HF_OK;
}

extern "C" int hf_newton_prec(void* stream, size_t nk, int nb, const void* rX, const double* rp, const double* eps,
                              const double* p, double lam, double T, double clipv, const double* w2d, void* zX,
                              double* zp, double* wsum_out, void* ws) {
  if (!rX || !rp || !eps || !p || !w2d || !zX || !zp || !wsum_out || !ws)
    return fail(HF_ERR_INVALID, "hf_newton_prec: bad argument");
  const int g = nblocks(nk * nb * nb);
  k_newton_prec<<<g, kOpsThreads, 0, HF_S>>>(nk, nb, (const double2*)rX, rp, eps, p, lam, T, clipv, w2d,
                                             (double2*)zX, zp, (double*)ws);
  return finish(HF_S, (double*)ws, g, 1, wsum_out);
}

extern "C" int hf_sub_scalar(void* stream, size_t n, double* x, const double* c, double scale) {
  if (!x || !c) return fail(HF_ERR_INVALID, "hf_sub_scalar: bad argument");
  k_sub_scalar<<<nblocks(n), kOpsThreads, 0, HF_S>>>(n, x, c, scale);
  HF_LAUNCH_CHECK("k_sub_scalar");
  return HF_OK;
}

extern "C" int hf_newton_dP(void* stream, int nk, int nb, const void* Q, const void* X, const double* dp,
                            const double* p, void* dP) {
  if (!Q || !X || !dp || !p || !dP || nb > 32) return fail(HF_ERR_INVALID, "hf_newton_dP: bad argument");
  const size_t sm = (size_t)3 * nb * nb * sizeof(double2) * 4;
  HF_SMEM_CAP(k_newton_dP);
  k_newton_dP<<<perk_grid(nk), 128, sm, HF_S>>>(nk, nb, (const double2*)Q, (const double2*)X, dp, p, (double2*)dP);
  HF_LAUNCH_CHECK("k_newton_dP");
  return HF_OK;
}

extern "C" int hf_newton_hvp(void* stream, int nk, int nb, const void* Q, const void* Ft, const void* X,
                             const double* dp, const double* p, const void* Fr, const void* h, double T, double clipv,
                             double pen, const void* dPpen, void* HX, double* Hp, const double* w2d,
                             double* wsum_out, void* ws) {
  if (!Q || !Ft || !X || !dp || !p || !Fr || !h || !HX || !Hp || !w2d || !wsum_out || !ws || nb > 32)
    return fail(HF_ERR_INVALID, "hf_newton_hvp: bad argument");
  const int g = perk_grid(nk);
  const size_t sm = (size_t)5 * nb * nb * sizeof(double2) * 4;
  HF_SMEM_CAP(k_newton_hvp);
  k_newton_hvp<<<g, 128, sm, HF_S>>>(nk, nb, (const double2*)Q, (const double2*)Ft, (const double2*)X, dp, p,
                                     (const double2*)Fr, (const double2*)h, T, clipv, pen, (const double2*)dPpen,
                                     (double2*)HX, Hp, w2d, (double*)ws);
  return finish(HF_S, (double*)ws, g, 1, wsum_out);
}

extern "C" int hf_matmul(void* stream, int nk, int nb, const void* A, const void* B, void* C) {
  if (!A || !B || !C || nb > 32) return fail(HF_ERR_INVALID, "hf_matmul: bad argument");
  const size_t sm = (size_t)2 * nb * nb * sizeof(double2) * 4;
  HF_SMEM_CAP(k_matmul);
  k_matmul<<<perk_grid(nk), 128, sm, HF_S>>>(nk, nb, (const double2*)A, (const double2*)B, (double2*)C);
  HF_LAUNCH_CHECK("k_matmul");
  return HF_OK;
}

extern "C" int hf_real_diag(void* stream, size_t nk, int nb, const void* A, double* d) {
  if (!A || !d) return fail(HF_ERR_INVALID, "hf_real_diag: bad argument");
  k_real_diag<<<nblocks(nk * nb), kOpsThreads, 0, HF_S>>>(nk, nb, (const double2*)A, d);
  HF_LAUNCH_CHECK("k_real_diag");
  return HF_OK;
}
