// Lane-per-row kernels of the device CG loop for nb <= 8.
//
// A group of G lanes (G = 4 for nb <= 4, else 8) owns one k-point and lane r of
// the group holds row r of every nb x nb matrix in registers, so a warp works on
// 32/G k-points at once.  Products read the other operand's rows from a per-group
// shared-memory stage (the G lanes of a group read the same address: broadcast).
// The retraction is the Cayley transform solved directly,
//   U(tau) = (I + tau d / 2)^{-1} (I - tau d / 2) = 2 (I + tau d / 2)^{-1} - I,
// the form of _cayley_retract (solver.py:122-138), by Gauss-Jordan elimination
// with partial pivoting (|re| + |im| pivots, as LAPACK's izamax); it equals the
// spectral form of the reference loop (solver.py:161-197, eigh(i d)) up to
// rounding and costs ~5x fewer FP64 operations per trial than a Jacobi eigh.
#pragma once

#include "common.cuh"
#include "solver_common.cuh"

namespace hf {

template <int NB>
struct RowGroup {
  static constexpr int G = NB <= 4 ? 4 : 8;  // lanes per k-point
  static constexpr int KPW = 32 / G;         // k-points per warp
  static constexpr int LD = NB * NB + 1;     // stage stride (complex); +1 spreads the groups over banks
};
constexpr int kRowWarps = 4;

inline int row_blocks(int nk, int kpw) {
  const int per_block = kRowWarps * kpw;
  int b = (nk + per_block - 1) / per_block;
  if (b > 148 * 16) b = 148 * 16;
  return b < 1 ? 1 : b;
}

// acc + a*b, acc + conj(a)*b, acc + a*conj(b)
__device__ __forceinline__ double2 cfma(double2 a, double2 b, double2 acc) {
  acc.x = fma(a.x, b.x, fma(-a.y, b.y, acc.x));
  acc.y = fma(a.x, b.y, fma(a.y, b.x, acc.y));
  return acc;
}
__device__ __forceinline__ double2 cfma_cj(double2 a, double2 b, double2 acc) {
  acc.x = fma(a.x, b.x, fma(a.y, b.y, acc.x));
  acc.y = fma(a.x, b.y, fma(-a.y, b.x, acc.y));
  return acc;
}
__device__ __forceinline__ double2 cfma_c(double2 a, double2 b, double2 acc) {
  acc.x = fma(a.x, b.x, fma(a.y, b.y, acc.x));
  acc.y = fma(a.y, b.x, fma(-a.x, b.y, acc.y));
  return acc;
}
__device__ __forceinline__ double2 crecip(double2 z) {
  const double s = 1.0 / fma(z.x, z.x, z.y * z.y);
  return make_double2(z.x * s, -z.y * s);
}

// Row r of U(tau) into u[] and every row j of U into SU[j * NB + .] (natural order),
// from row r of d (skew-Hermitian).  `on`: this lane holds a real row of a live
// k-point.  SP: 2*NB complex per group for the pivot row.  Warp-uniform control flow.
template <int NB, int G>
__device__ __forceinline__ void cayley_rows(const double2 (&d)[NB], double tau, int r, bool on, double2* SP,
                                            double2* SU, double2 (&u)[NB]) {
  double2 m[NB], x[NB];
  const double h = 0.5 * tau;
#pragma unroll
  for (int c = 0; c < NB; ++c) {
    m[c] = make_double2((c == r ? 1.0 : 0.0) + h * d[c].x, h * d[c].y);
    x[c] = make_double2(c == r ? 1.0 : 0.0, 0.0);
  }
  bool used = false;
  int mystep = 0;
#pragma unroll
  for (int j = 0; j < NB; ++j) {
    double key = (on && !used) ? fabs(m[j].x) + fabs(m[j].y) : -1.0;
    int who = r;
#pragma unroll
    for (int off = G / 2; off > 0; off >>= 1) {
      const double ok = __shfl_xor_sync(0xffffffffu, key, off);
      const int ow = __shfl_xor_sync(0xffffffffu, who, off);
      if (ok > key || (ok == key && ow < who)) {
        key = ok;
        who = ow;
      }
    }
    if (r == who && on) {
#pragma unroll
      for (int c = 0; c < NB; ++c) {
        SP[c] = m[c];
        SP[NB + c] = x[c];
      }
      used = true;
      mystep = j;
    }
    __syncwarp();
    if (on && r != who) {
      const double2 l = cmul(m[j], crecip(SP[j]));
#pragma unroll
      for (int c = j; c < NB; ++c) m[c] = csub(m[c], cmul(l, SP[c]));
#pragma unroll
      for (int c = 0; c < NB; ++c) x[c] = csub(x[c], cmul(l, SP[NB + c]));
    }
    __syncwarp();
  }
  // the lane that pivoted step s holds row s of the inverse times m[s]
  if (on) {
    double2 piv = m[0];
#pragma unroll
    for (int c = 1; c < NB; ++c)
      if (c == mystep) piv = m[c];
    const double2 ip = crecip(piv);
#pragma unroll
    for (int c = 0; c < NB; ++c) {
      const double2 v = cmul(x[c], ip);
      SU[mystep * NB + c] = make_double2(2.0 * v.x - (c == mystep ? 1.0 : 0.0), 2.0 * v.y);
    }
  }
  __syncwarp();
  if (on) {
#pragma unroll
    for (int c = 0; c < NB; ++c) u[c] = SU[r * NB + c];
  }
}

// eps_t[r] = Re (U^H Ft U)_rr from row r of Ft and the U rows in SU; SW: stage for W = Ft U.
template <int NB>
__device__ __forceinline__ double diag_uhfu_row(const double2 (&ft)[NB], int r, bool on, const double2* SU,
                                                double2* SW) {
  if (on) {
    double2 w[NB];
#pragma unroll
    for (int n = 0; n < NB; ++n) w[n] = make_double2(0.0, 0.0);
#pragma unroll
    for (int j = 0; j < NB; ++j) {
#pragma unroll
      for (int n = 0; n < NB; ++n) w[n] = cfma(ft[j], SU[j * NB + n], w[n]);
    }
#pragma unroll
    for (int n = 0; n < NB; ++n) SW[r * NB + n] = w[n];
  }
  __syncwarp();
  double e = 0.0;
  if (on) {
#pragma unroll
    for (int j = 0; j < NB; ++j) {
      const double2 uj = SU[j * NB + r], wj = SW[j * NB + r];
      e = fma(uj.x, wj.x, fma(uj.y, wj.y, e));
    }
  }
  return e;
}

// ------------------------------------------------ density: p and P = herm(Q p Q^H)
template <int NB>
__global__ void __launch_bounds__(32 * kRowWarps) k_cgr_density(CgArgs a, int force) {
  if (!force && !cg_active(a)) return;
  using RG = RowGroup<NB>;
  constexpr int G = RG::G, KPW = RG::KPW, LD = RG::LD;
  __shared__ double2 st[kRowWarps][KPW][2][LD];
  __shared__ double spv[kRowWarps][KPW][NB];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, g = lane / G, r = lane % G;
  double2* SQ = st[w][g][0];
  double2* SX = st[w][g][1];
  double* SPv = spv[w][g];
  const double mu = a.sc->mu, Tr = a.T_r;
  for (int kb = (blockIdx.x * kRowWarps + w) * KPW; kb < a.nk; kb += gridDim.x * kRowWarps * KPW) {
    const int k = kb + g;
    const bool on = k < a.nk && r < NB;
    const size_t row = ((size_t)k * NB + r) * NB;
    double2 q[NB];
    if (on) {
#pragma unroll
      for (int m = 0; m < NB; ++m) {
        q[m] = a.Q[row + m];
        SQ[r * NB + m] = q[m];
      }
      const double pv = sigmoid((mu - a.eps[(size_t)k * NB + r]) / Tr);
      a.p[(size_t)k * NB + r] = pv;
      SPv[r] = pv;
    }
    __syncwarp();
    double2 x[NB];
    if (on) {
#pragma unroll
      for (int n = 0; n < NB; ++n) q[n] = cscale(q[n], SPv[n]);
#pragma unroll
      for (int c = 0; c < NB; ++c) {
        double2 acc = make_double2(0.0, 0.0);
#pragma unroll
        for (int n = 0; n < NB; ++n) acc = cfma_c(q[n], SQ[c * NB + n], acc);
        x[c] = acc;
        SX[r * NB + c] = acc;
      }
    }
    __syncwarp();
    if (on) {
#pragma unroll
      for (int c = 0; c < NB; ++c) {
        const double2 y = SX[c * NB + r];
        a.P[row + c] = make_double2(0.5 * (x[c].x + y.x), 0.5 * (x[c].y - y.y));
      }
    }
    __syncwarp();
  }
}

// ----------------------------------- grad1: Ft, eps, G, g_p and four norms ---
template <int NB>
__global__ void __launch_bounds__(32 * kRowWarps) k_cgr_grad1(CgArgs a) {
  if (!cg_active(a)) return;
  using RG = RowGroup<NB>;
  constexpr int G = RG::G, KPW = RG::KPW, LD = RG::LD;
  __shared__ double2 st[kRowWarps][KPW][2][LD];
  __shared__ double red[64];
  __shared__ double tot[kMaxSums];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, g = lane / G, r = lane % G;
  double2* SQ = st[w][g][0];
  double2* ST = st[w][g][1];
  const int par = a.sc->k & 1;
  double2* Gc = par ? a.G1 : a.G0;
  const double2* Gp = par ? a.G0 : a.G1;
  double* gp = par ? a.gp1 : a.gp0;
  const double* gpp = par ? a.gp0 : a.gp1;
  const double mu = a.sc->mu;
  KSum acc[4];
  for (int kb = (blockIdx.x * kRowWarps + w) * KPW; kb < a.nk; kb += gridDim.x * kRowWarps * KPW) {
    const int k = kb + g;
    const bool on = k < a.nk && r < NB;
    const size_t row = ((size_t)k * NB + r) * NB;
    double2 f[NB];
    if (on) {
#pragma unroll
      for (int m = 0; m < NB; ++m) {
        SQ[r * NB + m] = a.Q[row + m];
        f[m] = a.F[row + m];
      }
    }
    __syncwarp();
    if (on) {  // T = F Q, row r
#pragma unroll
      for (int n = 0; n < NB; ++n) {
        double2 t = make_double2(0.0, 0.0);
#pragma unroll
        for (int j = 0; j < NB; ++j) t = cfma(f[j], SQ[j * NB + n], t);
        ST[r * NB + n] = t;
      }
    }
    __syncwarp();
    double2 ft[NB];
    if (on) {  // Ft = Q^H T, row r
#pragma unroll
      for (int n = 0; n < NB; ++n) ft[n] = make_double2(0.0, 0.0);
#pragma unroll
      for (int i = 0; i < NB; ++i) {
        const double2 qi = SQ[i * NB + r];
#pragma unroll
        for (int n = 0; n < NB; ++n) ft[n] = cfma_cj(qi, ST[i * NB + n], ft[n]);
      }
    }
    __syncwarp();
    if (on) {
#pragma unroll
      for (int n = 0; n < NB; ++n) {
        SQ[r * NB + n] = ft[n];
        a.Ft[row + n] = ft[n];
      }
    }
    __syncwarp();
    if (on) {
      const double wk = a.w_norm[k];
      const size_t vb = (size_t)k * NB;
      const double pr = a.p[vb + r];
      double ei = ft[0].x;
#pragma unroll
      for (int n = 0; n < NB; ++n) {
        if (n == r) ei = ft[n].x;
        double2 gv = make_double2(0.0, 0.0);
        if (n != r) {
          const double2 fji = SQ[n * NB + r];
          const double dpij = a.p[vb + n] - pr;
          gv = make_double2(0.5 * dpij * (ft[n].x + fji.x), 0.5 * dpij * (ft[n].y - fji.y));
        }
        Gc[row + n] = gv;
        acc[0].add(wk * (gv.x * gv.x + gv.y * gv.y));
        const double2 o = Gp[row + n];
        acc[2].add(wk * (o.x * o.x + o.y * o.y));
      }
      a.epsF[vb + r] = ei;
      const double ps = clip(pr, 1e-6, 1.0 - 1e-6);
      gp[vb + r] = ei + a.T_r * (log(ps) - log1p(-ps)) - mu;
      acc[1].add(ei * ei);
      acc[3].add(wk * gpp[vb + r] * gpp[vb + r]);
    }
    __syncwarp();
  }
  if (publish_partials<4>(acc, a.part, a.counter, red)) {
    gather_partials<4>(a.part, a.counter, tot, red);
    if (threadIdx.x == 0) {
      CgScalars* s = a.sc;
      s->grad_norm = sqrt(fmax(0.0, tot[0]));
      const double eps_scale = sqrt(tot[1] / ((double)a.nk * a.nb) + 1e-30);
      s->lam = fmax(a.T_r, a.denom_scale * eps_scale);
      s->pr_den = tot[2] + tot[3];
    }
  }
}

// -------------------- line-search trials i0 <= i < i1 on the frozen-F free energy
template <int NB, int NT>
__global__ void __launch_bounds__(32 * kRowWarps) k_cgr_trials(CgArgs a, int i0, int i1, int last_chunk) {
  if (!cg_active(a)) return;
  if (a.sc->accepted) return;
  using RG = RowGroup<NB>;
  constexpr int G = RG::G, KPW = RG::KPW, LD = RG::LD;
  __shared__ double2 st[kRowWarps][KPW][2][LD];
  __shared__ double2 spiv[kRowWarps][KPW][2 * NB];
  __shared__ double red[64];
  __shared__ double tot[kMaxSums];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, g = lane / G, r = lane % G;
  double2* SU = st[w][g][0];
  double2* SW = st[w][g][1];
  double2* SP = spiv[w][g];
  const int nt = i1 - i0;
  double taus[NT];
  {
    double tau = a.sc->tau0;
    for (int i = 0; i < i0; ++i) tau = tau * a.bt_shrink;
    for (int i = 0; i < NT; ++i) {
      taus[i] = tau;
      tau = tau * a.bt_shrink;
    }
  }
  KSum acc[2 * NT];
  for (int kb = (blockIdx.x * kRowWarps + w) * KPW; kb < a.nk; kb += gridDim.x * kRowWarps * KPW) {
    const int k = kb + g;
    const bool on = k < a.nk && r < NB;
    const size_t row = ((size_t)k * NB + r) * NB;
    double2 d[NB], ft[NB];
    double pv = 0.0, dpv = 0.0, wk = 0.0;
    if (on) {
#pragma unroll
      for (int m = 0; m < NB; ++m) {
        d[m] = a.dQ[row + m];
        ft[m] = a.Ft[row + m];
      }
      pv = a.p[(size_t)k * NB + r];
      dpv = a.dp[(size_t)k * NB + r];
      wk = a.w_norm[k];
    } else {
#pragma unroll
      for (int m = 0; m < NB; ++m) d[m] = ft[m] = make_double2(0.0, 0.0);
    }
#pragma unroll
    for (int it = 0; it < NT; ++it) {
      if (it < nt) {  // warp-uniform
        double2 u[NB];
        cayley_rows<NB, G>(d, taus[it], r, on, SP, SU, u);
        const double et = diag_uhfu_row<NB>(ft, r, on, SU, SW);
        if (on) {
          const double pt = clip(pv - taus[it] * dpv, 1e-8, 1.0 - 1e-8);
          acc[2 * it].add(wk * pt * et);
          acc[2 * it + 1].add(wk * ent_term(pt));
        }
        __syncwarp();
      }
    }
  }
  if (publish_partials<2 * NT>(acc, a.part, a.counter, red)) {
    gather_partials<2 * NT>(a.part, a.counter, tot, red);
    if (threadIdx.x == 0) {
      CgScalars* s = a.sc;
      const double Tm = fmax(a.T_r, 1e-14);
      for (int it = 0; it < nt; ++it) {
        const double om = tot[2 * it] + Tm * tot[2 * it + 1];
        if (om < s->Omega0) {
          s->accepted = 1;
          s->tau_final = taus[it];
          break;
        }
      }
      if (!s->accepted && last_chunk) s->tau_final = s->tau0 * pow(a.bt_shrink, (double)a.bt_max);
    }
  }
}

// ----------------- retraction: U(tau), Q <- Q U, eps_new = diag(U^H Ft U)
template <int NB>
__global__ void __launch_bounds__(32 * kRowWarps) k_cgr_update(CgArgs a) {
  if (!cg_active(a)) return;
  using RG = RowGroup<NB>;
  constexpr int G = RG::G, KPW = RG::KPW, LD = RG::LD;
  __shared__ double2 st[kRowWarps][KPW][2][LD];
  __shared__ double2 spiv[kRowWarps][KPW][2 * NB];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, g = lane / G, r = lane % G;
  double2* SU = st[w][g][0];
  double2* SW = st[w][g][1];
  double2* SP = spiv[w][g];
  const double tau = a.sc->tau_final;
  for (int kb = (blockIdx.x * kRowWarps + w) * KPW; kb < a.nk; kb += gridDim.x * kRowWarps * KPW) {
    const int k = kb + g;
    const bool on = k < a.nk && r < NB;
    const size_t row = ((size_t)k * NB + r) * NB;
    double2 d[NB], ft[NB];
    if (on) {
#pragma unroll
      for (int m = 0; m < NB; ++m) {
        d[m] = a.dQ[row + m];
        ft[m] = a.Ft[row + m];
      }
    } else {
#pragma unroll
      for (int m = 0; m < NB; ++m) d[m] = ft[m] = make_double2(0.0, 0.0);
    }
    double2 u[NB];
    cayley_rows<NB, G>(d, tau, r, on, SP, SU, u);
    const double et = diag_uhfu_row<NB>(ft, r, on, SU, SW);
    if (on) {
      a.eps[(size_t)k * NB + r] = et;
      double2 q[NB];
#pragma unroll
      for (int m = 0; m < NB; ++m) q[m] = a.Q[row + m];
#pragma unroll
      for (int n = 0; n < NB; ++n) {
        double2 acc = make_double2(0.0, 0.0);
#pragma unroll
        for (int j = 0; j < NB; ++j) acc = cfma(q[j], SU[j * NB + n], acc);
        a.Q[row + n] = acc;
      }
    }
    __syncwarp();
  }
}

}  // namespace hf
