// Lane-per-column kernels of the device CG loop for nb <= 8.
//
// A group of G lanes (G = 4 for nb <= 4, else 8) owns one k-point and lane c of
// the group holds column c of every nb x nb matrix in registers, so a warp works
// on 32/G k-points at once and, for a fixed row, the lanes of a group touch
// consecutive 16-byte elements: global loads and stores are coalesced without
// staging.  A product A B takes B from the lane's own column and A from a
// per-group shared-memory copy read by broadcast (row stride nb + 1, so a lane
// reading along a row of the copy stays clear of bank conflicts).
// The retraction solves the Cayley transform directly,
//   U(tau) = (I + tau d / 2)^{-1} (I - tau d / 2) = 2 (I + tau d / 2)^{-1} - I,
// the form of _cayley_retract (solver.py:122-138), by Gauss-Jordan elimination
// with partial pivoting (|re| + |im| pivots, as LAPACK's izamax); it equals the
// spectral form of the reference loop (solver.py:161-197, eigh(i d)) up to
// rounding and needs ~5x fewer FP64 operations per trial than a Jacobi eigh.
#pragma once

#include "common.cuh"
#include "solver_common.cuh"

namespace hf {

template <int NB>
struct RowGroup {
  static constexpr int G = NB <= 4 ? 4 : 8;  // lanes per k-point
  static constexpr int KPW = 32 / G;         // k-points per warp
  static constexpr int LP = NB + 1;          // row stride of a shared copy (complex)
  static constexpr int MAT = NB * LP;        // one shared copy of an nb x nb matrix
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

// element r of a register column (r runtime): a select chain, no local memory
template <int NB>
__device__ __forceinline__ double2 pick(const double2 (&v)[NB], int r) {
  double2 o = v[0];
#pragma unroll
  for (int i = 1; i < NB; ++i)
    if (i == r) o = v[i];
  return o;
}

// Column c of U(tau) into u[] from column c of d (skew-Hermitian).  `on`: this lane
// holds a real column of a live k-point.  SC: NB complex (pivot column), SX: one
// shared matrix copy.  Warp-uniform control flow.
template <int NB>
__device__ __forceinline__ void cayley_cols(const double2 (&d)[NB], double tau, int c, bool on, double2* SC,
                                            double2* SX, double2 (&u)[NB]) {
  constexpr int LP = RowGroup<NB>::LP;
  double2 m[NB], x[NB];
  const double h = 0.5 * tau;
#pragma unroll
  for (int r = 0; r < NB; ++r) {
    m[r] = make_double2((r == c ? 1.0 : 0.0) + h * d[r].x, h * d[r].y);
    x[r] = make_double2(r == c ? 1.0 : 0.0, 0.0);
  }
  unsigned used = 0;
  int piv[NB];
#pragma unroll
  for (int j = 0; j < NB; ++j) {
    if (on && c == j) {
#pragma unroll
      for (int r = 0; r < NB; ++r) SC[r] = m[r];
    }
    __syncwarp();
    // every lane finds the same pivot from the shared column (first maximum)
    int p = 0;
    double best = -1.0;
#pragma unroll
    for (int r = 0; r < NB; ++r) {
      const double2 v = SC[r];
      const double key = ((used >> r) & 1u) ? -1.0 : fabs(v.x) + fabs(v.y);
      if (key > best) { best = key; p = r; }
    }
    piv[j] = p;
    used |= 1u << p;
    if (on) {
      const double2 ip = crecip(SC[p]);
      const double2 mp = pick<NB>(m, p), xp = pick<NB>(x, p);
#pragma unroll
      for (int r = 0; r < NB; ++r) {
        if (r == p) continue;
        const double2 l = cmul(SC[r], ip);
        m[r] = csub(m[r], cmul(l, mp));
        x[r] = csub(x[r], cmul(l, xp));
      }
    }
    __syncwarp();
  }
  // row piv[j] holds column j's only non-zero: (M^-1)[j][c] = x[piv[j]] / m_j, m_j = M'[piv[j]][j]
  if (on) {
#pragma unroll
    for (int r = 0; r < NB; ++r) SX[r * LP + c] = x[r];
    int pc = piv[0];
#pragma unroll
    for (int i = 1; i < NB; ++i)
      if (i == c) pc = piv[i];
    SC[c] = pick<NB>(m, pc);  // lane c holds column c: its pivot entry M'[piv[c]][c]
  }
  __syncwarp();
  if (on) {
#pragma unroll
    for (int j = 0; j < NB; ++j) {
      const double2 v = cmul(SX[piv[j] * LP + c], crecip(SC[j]));
      u[j] = make_double2(2.0 * v.x - (j == c ? 1.0 : 0.0), 2.0 * v.y);
    }
  }
  __syncwarp();
}

// ------------------------------------------------ density: p and P = herm(Q p Q^H)
template <int NB>
__global__ void __launch_bounds__(32 * kRowWarps) k_cgr_density(CgArgs a, int force) {
  if (!force && !cg_active(a)) return;
  double2* const Qc = q_cur(a);
  using RG = RowGroup<NB>;
  constexpr int G = RG::G, KPW = RG::KPW, LP = RG::LP, MAT = RG::MAT;
  __shared__ double2 st[kRowWarps][KPW][2 * MAT];
  __shared__ double spv[kRowWarps][KPW][NB];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, g = lane / G, c = lane % G;
  double2* SQ = st[w][g];
  double2* SX = SQ + MAT;
  double* SPv = spv[w][g];
  const double mu = a.sc->mu, Tr = a.T_r;
  for (int kb = (blockIdx.x * kRowWarps + w) * KPW; kb < a.nk; kb += gridDim.x * kRowWarps * KPW) {
    const int k = kb + g;
    const bool on = k < a.nk && c < NB;
    const size_t base = (size_t)k * NB * NB + c;
    if (on) {
#pragma unroll
      for (int r = 0; r < NB; ++r) SQ[r * LP + c] = Qc[base + (size_t)r * NB];
      const double pv = sigmoid((mu - a.eps[(size_t)k * NB + c]) / Tr);
      a.p[(size_t)k * NB + c] = pv;
      SPv[c] = pv;
    }
    __syncwarp();
    double2 x[NB];
    if (on) {  // X[r][c] = sum_n Q[r][n] p_n conj(Q[c][n])
      double2 cq[NB];
#pragma unroll
      for (int n = 0; n < NB; ++n) cq[n] = cscale(conj(SQ[c * LP + n]), SPv[n]);
#pragma unroll
      for (int r = 0; r < NB; ++r) {
        double2 acc = make_double2(0.0, 0.0);
#pragma unroll
        for (int n = 0; n < NB; ++n) acc = cfma(SQ[r * LP + n], cq[n], acc);
        x[r] = acc;
        SX[r * LP + c] = acc;
      }
    }
    __syncwarp();
    if (on) {
#pragma unroll
      for (int r = 0; r < NB; ++r) {
        const double2 y = SX[c * LP + r];  // X[c][r]
        a.P[base + (size_t)r * NB] = make_double2(0.5 * (x[r].x + y.x), 0.5 * (x[r].y - y.y));
      }
    }
    __syncwarp();
  }
}

// P = herm(Q diag(p) Q^H) from given occupations (hf_density_from_Qp for complex128,
// nb <= 8): the density step of k_cgr_density without the Fermi function
template <int NB>
__global__ void __launch_bounds__(32 * kRowWarps) k_rows_density(int nk, const double2* __restrict__ Q,
                                                                 const double* __restrict__ p,
                                                                 double2* __restrict__ P) {
  using RG = RowGroup<NB>;
  constexpr int G = RG::G, KPW = RG::KPW, LP = RG::LP, MAT = RG::MAT;
  __shared__ double2 st[kRowWarps][KPW][2 * MAT];
  __shared__ double spv[kRowWarps][KPW][NB];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, g = lane / G, c = lane % G;
  double2* SQ = st[w][g];
  double2* SX = SQ + MAT;
  double* SPv = spv[w][g];
  for (int kb = (blockIdx.x * kRowWarps + w) * KPW; kb < nk; kb += gridDim.x * kRowWarps * KPW) {
    const int k = kb + g;
    const bool on = k < nk && c < NB;
    const size_t base = (size_t)k * NB * NB + c;
    if (on) {
#pragma unroll
      for (int r = 0; r < NB; ++r) SQ[r * LP + c] = Q[base + (size_t)r * NB];
      SPv[c] = p[(size_t)k * NB + c];
    }
    __syncwarp();
    double2 x[NB];
    if (on) {  // X[r][c] = sum_n Q[r][n] p_n conj(Q[c][n])
      double2 cq[NB];
#pragma unroll
      for (int n = 0; n < NB; ++n) cq[n] = cscale(conj(SQ[c * LP + n]), SPv[n]);
#pragma unroll
      for (int r = 0; r < NB; ++r) {
        double2 acc = make_double2(0.0, 0.0);
#pragma unroll
        for (int n = 0; n < NB; ++n) acc = cfma(SQ[r * LP + n], cq[n], acc);
        x[r] = acc;
        SX[r * LP + c] = acc;
      }
    }
    __syncwarp();
    if (on) {
#pragma unroll
      for (int r = 0; r < NB; ++r) {
        const double2 y = SX[c * LP + r];  // X[c][r]
        P[base + (size_t)r * NB] = make_double2(0.5 * (x[r].x + y.x), 0.5 * (x[r].y - y.y));
      }
    }
    __syncwarp();
  }
}

// ----------------------------------- grad1: Ft, eps, G, g_p and four norms ---
// 4 CTAs per SM: 128 registers without spills (16 warps per SM instead of 12)
template <int NB>
__global__ void __launch_bounds__(32 * kRowWarps, 4) k_cgr_grad1(CgArgs a) {
  if (!cg_active(a)) return;
  double2* const Qc = q_cur(a);
  using RG = RowGroup<NB>;
  constexpr int G = RG::G, KPW = RG::KPW, LP = RG::LP, MAT = RG::MAT;
  __shared__ double2 st[kRowWarps][KPW][2 * MAT];
  __shared__ double spv[kRowWarps][KPW][NB];
  __shared__ double red[64];
  __shared__ double tot[kMaxSums];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, g = lane / G, c = lane % G;
  double2* SQ = st[w][g];
  double2* SF = SQ + MAT;  // F, then Ft
  double* SPv = spv[w][g];
  const int par = a.sc->k & 1;
  double2* Gc = par ? a.G1 : a.G0;
  const double2* Gp = par ? a.G0 : a.G1;
  double* gp = par ? a.gp1 : a.gp0;
  const double* gpp = par ? a.gp0 : a.gp1;
  const double mu = a.sc->mu;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
  for (int kb = (blockIdx.x * kRowWarps + w) * KPW; kb < a.nk; kb += gridDim.x * kRowWarps * KPW) {
    const int k = kb + g;
    const bool on = k < a.nk && c < NB;
    const size_t base = (size_t)k * NB * NB + c;
    double2 q[NB];
    if (on) {
#pragma unroll
      for (int r = 0; r < NB; ++r) {
        q[r] = Qc[base + (size_t)r * NB];
        SQ[r * LP + c] = q[r];
        SF[r * LP + c] = a.F[base + (size_t)r * NB];
      }
      SPv[c] = a.p[(size_t)k * NB + c];
    }
    __syncwarp();
    double2 ft[NB];
    if (on) {
      double2 t[NB];  // T = F Q, column c
#pragma unroll
      for (int r = 0; r < NB; ++r) {
        double2 acc = make_double2(0.0, 0.0);
#pragma unroll
        for (int j = 0; j < NB; ++j) acc = cfma(SF[r * LP + j], q[j], acc);
        t[r] = acc;
      }
#pragma unroll
      for (int m = 0; m < NB; ++m) {  // Ft = Q^H T, column c
        double2 acc = make_double2(0.0, 0.0);
#pragma unroll
        for (int i = 0; i < NB; ++i) acc = cfma_cj(SQ[i * LP + m], t[i], acc);
        ft[m] = acc;
      }
    }
    __syncwarp();
    if (on) {
#pragma unroll
      for (int m = 0; m < NB; ++m) {
        SF[m * LP + c] = ft[m];
        a.Ft[base + (size_t)m * NB] = ft[m];
      }
    }
    __syncwarp();
    if (on) {
      const double wk = a.w_norm[k];
      const double pc = SPv[c];
      double ec = ft[0].x;
#pragma unroll
      for (int m = 0; m < NB; ++m) {  // element (i = m, j = c): 0.5 (p_j - p_i)(Ft_ij + conj(Ft_ji))
        if (m == c) ec = ft[m].x;
        double2 gv = make_double2(0.0, 0.0);
        if (m != c) {
          const double2 fji = SF[c * LP + m];
          const double dpij = pc - SPv[m];
          gv = make_double2(0.5 * dpij * (ft[m].x + fji.x), 0.5 * dpij * (ft[m].y - fji.y));
        }
        Gc[base + (size_t)m * NB] = gv;
        s0 += wk * (gv.x * gv.x + gv.y * gv.y);
        const double2 o = Gp[base + (size_t)m * NB];
        s2 += wk * (o.x * o.x + o.y * o.y);
      }
      const size_t vb = (size_t)k * NB + c;
      a.epsF[vb] = ec;
      const double ps = clip(pc, 1e-6, 1.0 - 1e-6);
      gp[vb] = ec + a.T_r * (log(ps) - log1p(-ps)) - mu;
      s1 += ec * ec;
      s3 += wk * gpp[vb] * gpp[vb];
    }
    __syncwarp();
  }
  KSum acc[4];
  acc[0].add(s0);
  acc[1].add(s1);
  acc[2].add(s2);
  acc[3].add(s3);
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

// eps_t[c] = Re (U^H Ft U)_cc from column c of U and the shared copy of Ft
template <int NB>
__device__ __forceinline__ double diag_uhfu_col(const double2 (&u)[NB], const double2* SFt) {
  constexpr int LP = RowGroup<NB>::LP;
  double e = 0.0;
#pragma unroll
  for (int j = 0; j < NB; ++j) {
    double2 wj = make_double2(0.0, 0.0);  // W[j][c] = sum_l Ft[j][l] U[l][c]
#pragma unroll
    for (int l = 0; l < NB; ++l) wj = cfma(SFt[j * LP + l], u[l], wj);
    e = fma(u[j].x, wj.x, fma(u[j].y, wj.y, e));
  }
  return e;
}

// -------------------- line-search trials i0 <= i < i1 on the frozen-F free energy
// The first trial (NT = 1, i0 = 0) also forms, speculatively, what the retraction
// would write if tau0 is accepted: eps = diag(U^H Ft U) into eps and Q U into Vd
// (same arithmetic as k_cgr_update); its last CTA sets first_ok when tau0 is
// accepted, and k_cgr_update then only copies Vd into Q.
// the first trial (NT = 1) and the update at 3 CTAs per SM (at most 168 registers: 12
// warps per SM instead of 8, with at most 24 B of spills at nb = 8); the backtracking
// trials keep the registers they need
template <int NB, int NT>
__global__ void __launch_bounds__(32 * kRowWarps, NT == 1 ? 3 : 1) k_cgr_trials(CgArgs a, int i0, int i1, int last_chunk) {
  if (!cg_active(a)) return;
  if (a.sc->accepted) return;
  using RG = RowGroup<NB>;
  constexpr int G = RG::G, KPW = RG::KPW, LP = RG::LP, MAT = RG::MAT;
  __shared__ double2 st[kRowWarps][KPW][2 * MAT + NB];
  __shared__ double red[64];
  __shared__ double tot[kMaxSums];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, g = lane / G, c = lane % G;
  double2* SFt = st[w][g];
  double2* SX = SFt + MAT;
  double2* SC = SX + MAT;
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
  double se[NT], sh[NT];
#pragma unroll
  for (int i = 0; i < NT; ++i) se[i] = sh[i] = 0.0;
  for (int kb = (blockIdx.x * kRowWarps + w) * KPW; kb < a.nk; kb += gridDim.x * kRowWarps * KPW) {
    const int k = kb + g;
    const bool on = k < a.nk && c < NB;
    const size_t base = (size_t)k * NB * NB + c;
    double2 d[NB];
    double pv = 0.0, dpv = 0.0, wk = 0.0;
    if (on) {
#pragma unroll
      for (int r = 0; r < NB; ++r) {
        d[r] = a.dQ[base + (size_t)r * NB];
        SFt[r * LP + c] = a.Ft[base + (size_t)r * NB];
      }
      pv = a.p[(size_t)k * NB + c];
      dpv = a.dp[(size_t)k * NB + c];
      wk = a.w_norm[k];
    } else {
#pragma unroll
      for (int r = 0; r < NB; ++r) d[r] = make_double2(0.0, 0.0);
    }
    __syncwarp();
#pragma unroll
    for (int it = 0; it < NT; ++it) {
      if (it < nt) {  // warp-uniform
        double2 u[NB];
        cayley_cols<NB>(d, taus[it], c, on, SC, SX, u);  // ends with a warp barrier: SX is free again
        if (on) {
          const double et = diag_uhfu_col<NB>(u, SFt);
          const double pt = clip(pv - taus[it] * dpv, 1e-8, 1.0 - 1e-8);
          se[it] += wk * pt * et;
          sh[it] += wk * ent_term(pt);
          if (NT == 1 && i0 == 0) {
            a.eps[(size_t)k * NB + c] = et;
#pragma unroll
            for (int r = 0; r < NB; ++r) SX[r * LP + c] = q_cur(a)[base + (size_t)r * NB];
          }
        }
        if (NT == 1 && i0 == 0) {
          __syncwarp();
          if (on) {
#pragma unroll
            for (int r = 0; r < NB; ++r) {  // (Q U)[r][c] = sum_j Q[r][j] U[j][c]
              double2 acc = make_double2(0.0, 0.0);
#pragma unroll
              for (int j = 0; j < NB; ++j) acc = cfma(SX[r * LP + j], u[j], acc);
              q_alt(a)[base + (size_t)r * NB] = acc;
            }
          }
          __syncwarp();  // SX is the Cayley stage of the next k-point group
        }
      }
    }
    __syncwarp();
  }
  KSum acc[2 * NT];
#pragma unroll
  for (int i = 0; i < NT; ++i) {
    acc[2 * i].add(se[i]);
    acc[2 * i + 1].add(sh[i]);
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
          if (NT == 1 && i0 == 0 && it == 0) {  // the other buffer holds Q U(tau0): make it current
            s->first_ok = 1;
            s->qsel ^= 1;
          }
          break;
        }
      }
      if (!s->accepted && last_chunk) s->tau_final = s->tau0 * pow(a.bt_shrink, (double)a.bt_max);
    }
  }
}

// ----------------- retraction: U(tau), Q <- Q U, eps_new = diag(U^H Ft U)
template <int NB>
__global__ void __launch_bounds__(32 * kRowWarps, 3) k_cgr_update(CgArgs a) {
  if (!cg_active(a)) return;
  if (a.sc->first_ok) return;  // tau0 accepted: the first trial formed eps and Q U(tau0) already
  double2* const Qc = q_cur(a);
  using RG = RowGroup<NB>;
  constexpr int G = RG::G, KPW = RG::KPW, LP = RG::LP, MAT = RG::MAT;
  __shared__ double2 st[kRowWarps][KPW][2 * MAT + NB];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, g = lane / G, c = lane % G;
  double2* SFt = st[w][g];
  double2* SX = SFt + MAT;  // Cayley stage, then the copy of Q
  double2* SC = SX + MAT;
  const double tau = a.sc->tau_final;
  for (int kb = (blockIdx.x * kRowWarps + w) * KPW; kb < a.nk; kb += gridDim.x * kRowWarps * KPW) {
    const int k = kb + g;
    const bool on = k < a.nk && c < NB;
    const size_t base = (size_t)k * NB * NB + c;
    double2 d[NB];
    if (on) {
#pragma unroll
      for (int r = 0; r < NB; ++r) {
        d[r] = a.dQ[base + (size_t)r * NB];
        SFt[r * LP + c] = a.Ft[base + (size_t)r * NB];
      }
    } else {
#pragma unroll
      for (int r = 0; r < NB; ++r) d[r] = make_double2(0.0, 0.0);
    }
    __syncwarp();
    double2 u[NB];
    cayley_cols<NB>(d, tau, c, on, SC, SX, u);  // ends with a warp barrier: SX is free again
    if (on) {
      a.eps[(size_t)k * NB + c] = diag_uhfu_col<NB>(u, SFt);
#pragma unroll
      for (int r = 0; r < NB; ++r) SX[r * LP + c] = Qc[base + (size_t)r * NB];
    }
    __syncwarp();
    if (on) {
#pragma unroll
      for (int r = 0; r < NB; ++r) {  // (Q U)[r][c] = sum_j Q[r][j] U[j][c]
        double2 acc = make_double2(0.0, 0.0);
#pragma unroll
        for (int j = 0; j < NB; ++j) acc = cfma(SX[r * LP + j], u[j], acc);
        Qc[base + (size_t)r * NB] = acc;
      }
    }
    __syncwarp();
  }
}

// ----------------------------------------------------------- eigensolver ---
// Cyclic Jacobi for Hermitian A (Jacobi 1846; Golub & Van Loan 8.5, complex
// rotations; round-robin pair order as the warp-per-matrix solver in perk.cuh)
// in the lane-per-column layout with A and V kept in shared memory, lane c owning
// column c.  Per round: the lane holding column q of each pair (p, q) computes the
// rotation once; every lane forms its new columns of A G and V G in registers from
// its own and its partner's column, writes them back, then applies the row mix
// G^H A of every pair to its own column in place.  Rounds are a runtime loop, so
// the code stays small.  Sweeps continue while any group of the warp rotated.
template <int NB>
struct JacobiPairs {
  static constexpr int M = NB + (NB & 1);
  __host__ __device__ static int pa(int t, int k) { return k == 0 ? 0 : 1 + ((k - 1 + t) % (M - 1)); }
  __host__ __device__ static int pb(int t, int k) { return 1 + ((M - 1 - k - 1 + t) % (M - 1)); }
};

// The rotation that zeroes a_pq (cosine cc, sine sp; act = 1 when it rotates).  A
// rounding-level change here moves the reference CG's plateau stop on some problems, so
// both Jacobi variants share this one form.
__device__ __forceinline__ void jacobi_rotation(double2 apq, double app, double aqq, double thr, double& cc,
                                                double& act, double2& sp) {
  const double mag = hypot(apq.x, apq.y);
  if (mag > thr) {
    const double tau = (aqq - app) / (2.0 * mag);
    const double tt = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
    cc = 1.0 / sqrt(1.0 + tt * tt);
    const double sn = tt * cc;
    sp = make_double2(sn * apq.x / mag, sn * apq.y / mag);
    act = 1.0;
  }
}

template <int NB>
__device__ __forceinline__ void jacobi_smem_cols(double2* SA, double2* SV, double2* SP, int c, bool on,
                                                 double thr) {
  constexpr int LP = RowGroup<NB>::LP, M = JacobiPairs<NB>::M, NP = M / 2;
  if (NB == 1) return;
  for (int sweep = 0; sweep < 60; ++sweep) {
    bool rotated = false;
    for (int t = 0; t < M - 1; ++t) {
      int partner = -1, kk = -1;
      bool isq = false;
#pragma unroll
      for (int k = 0; k < NP; ++k) {
        const int a0 = JacobiPairs<NB>::pa(t, k), b0 = JacobiPairs<NB>::pb(t, k);
        const int p = a0 < b0 ? a0 : b0, q = a0 < b0 ? b0 : a0;
        if (q < NB) {
          if (c == p) { partner = q; kk = k; }
          if (c == q) { partner = p; kk = k; isq = true; }
        }
      }
      if (on && isq) {
        const int p = partner;
        const double2 apq = SA[p * LP + c];
        double cc = 1.0, act = 0.0;
        double2 sp = make_double2(0.0, 0.0);
        jacobi_rotation(apq, SA[p * LP + p].x, SA[c * LP + c].x, thr, cc, act, sp);
        SP[2 * kk] = make_double2(cc, act);
        SP[2 * kk + 1] = sp;
      }
      __syncwarp();
      // A <- A G, V <- V G on this lane's column: new = cc own + beta partner
      double cc = 1.0, act = 0.0;
      double2 sp = make_double2(0.0, 0.0);
      if (kk >= 0) {
        const double2 h = SP[2 * kk];
        cc = h.x;
        act = h.y;
        sp = SP[2 * kk + 1];
      }
      rotated = rotated || (on && act != 0.0);
      const double2 beta = isq ? sp : make_double2(-sp.x, sp.y);  // q: sp;  p: -conj(sp)
      // the new columns of A, then of V, each read whole before any lane writes (two
      // phases keep half as many values live: at the 128-register cap of nb 5-8 the
      // single phase spilled)
      double2 nc[NB];
      const bool mix = on && act != 0.0;
      if (mix) {
#pragma unroll
        for (int r = 0; r < NB; ++r) nc[r] = cadd(cscale(SA[r * LP + c], cc), cmul(beta, SA[r * LP + partner]));
      }
      __syncwarp();
      if (mix) {
#pragma unroll
        for (int r = 0; r < NB; ++r) SA[r * LP + c] = nc[r];
#pragma unroll
        for (int r = 0; r < NB; ++r) nc[r] = cadd(cscale(SV[r * LP + c], cc), cmul(beta, SV[r * LP + partner]));
      }
      __syncwarp();
      if (mix) {
#pragma unroll
        for (int r = 0; r < NB; ++r) SV[r * LP + c] = nc[r];
      }
      // A <- G^H A: rows p and q of this lane's column, every active pair; then exact zeros
      if (on) {
#pragma unroll
        for (int k = 0; k < NP; ++k) {
          const int a0 = JacobiPairs<NB>::pa(t, k), b0 = JacobiPairs<NB>::pb(t, k);
          const int p = a0 < b0 ? a0 : b0, q = a0 < b0 ? b0 : a0;
          if (q >= NB) continue;
          const double2 hk = SP[2 * k];
          if (hk.y == 0.0) continue;
          const double2 spk = SP[2 * k + 1];
          const double2 x = SA[p * LP + c], y = SA[q * LP + c];
          SA[p * LP + c] = csub(cscale(x, hk.x), cmul(spk, y));
          SA[q * LP + c] = cadd(cmulc(x, spk), cscale(y, hk.x));
        }
        if (act != 0.0) {
          SA[partner * LP + c] = make_double2(0.0, 0.0);
          SA[c * LP + c].y = 0.0;
        }
      }
      __syncwarp();
    }
    if (!__any_sync(0xffffffffu, rotated)) break;
  }
}

// The same cyclic Jacobi with each lane's columns of A and V in registers: the partner's
// column comes by warp shuffles (read before this round's update, consumed row by row),
// the rotation of every pair is broadcast from the pair's q lane, and the rounds are
// unrolled so that every row index is a compile-time constant (register arrays are
// never indexed at run time; the lane's own index selects through compare chains).
// Same rotations, same order and same exact zeros as jacobi_smem_cols.
__device__ __forceinline__ double2 shfl2(double2 v, int src) {
  return make_double2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}

template <int NB>
__device__ __forceinline__ void jacobi_reg_cols(double2 (&a)[NB], double2 (&v)[NB], int c, int gb, bool on,
                                                double thr) {
  constexpr int M = JacobiPairs<NB>::M, NP = M / 2;
  if (NB == 1) return;
  for (int sweep = 0; sweep < 60; ++sweep) {
    bool rotated = false;
#pragma unroll
    for (int t = 0; t < M - 1; ++t) {
      int partner = -1, kk = -1;
      bool isq = false;
#pragma unroll
      for (int k = 0; k < NP; ++k) {
        const int a0 = JacobiPairs<NB>::pa(t, k), b0 = JacobiPairs<NB>::pb(t, k);
        const int p = a0 < b0 ? a0 : b0, q = a0 < b0 ? b0 : a0;
        if (q < NB) {
          if (c == p) { partner = q; kk = k; }
          if (c == q) { partner = p; kk = k; isq = true; }
        }
      }
      const int pl = gb + (partner >= 0 ? partner : (c < NB ? c : 0));
      double2 own = a[0], apq = a[0];  // a[c] and a[partner], by compare chains
#pragma unroll
      for (int r = 1; r < NB; ++r) {
        if (r == c) own = a[r];
        if (r == partner) apq = a[r];
      }
      const double app = __shfl_sync(0xffffffffu, own.x, pl);  // the partner's diagonal
      double cc = 1.0, act = 0.0;
      double2 sp = make_double2(0.0, 0.0);
      if (on && isq) jacobi_rotation(apq, app, own.x, thr, cc, act, sp);
      double hc[NP], ha[NP];
      double2 hs[NP];
#pragma unroll
      for (int k = 0; k < NP; ++k) {
        const int a0 = JacobiPairs<NB>::pa(t, k), b0 = JacobiPairs<NB>::pb(t, k);
        const int q = a0 < b0 ? b0 : a0;
        const int src = gb + (q < NB ? q : 0);
        hc[k] = __shfl_sync(0xffffffffu, cc, src);
        ha[k] = __shfl_sync(0xffffffffu, act, src);
        hs[k] = shfl2(sp, src);
      }
      double mcc = 1.0, mact = 0.0;
      double2 msp = make_double2(0.0, 0.0);
#pragma unroll
      for (int k = 0; k < NP; ++k)
        if (k == kk) {
          mcc = hc[k];
          mact = ha[k];
          msp = hs[k];
        }
      const bool mix = on && mact != 0.0;
      rotated = rotated || mix;
      const double2 beta = isq ? msp : make_double2(-msp.x, msp.y);  // q: sp;  p: -conj(sp)
      // A <- A G, V <- V G on this lane's column: new = cc own + beta partner
#pragma unroll
      for (int r = 0; r < NB; ++r) {
        const double2 xa = shfl2(a[r], pl), xv = shfl2(v[r], pl);
        if (mix) {
          a[r] = cadd(cscale(a[r], mcc), cmul(beta, xa));
          v[r] = cadd(cscale(v[r], mcc), cmul(beta, xv));
        }
      }
      // A <- G^H A: rows p and q of this lane's column, every active pair; then exact zeros
      if (on) {
#pragma unroll
        for (int k = 0; k < NP; ++k) {
          const int a0 = JacobiPairs<NB>::pa(t, k), b0 = JacobiPairs<NB>::pb(t, k);
          const int p = a0 < b0 ? a0 : b0, q = a0 < b0 ? b0 : a0;
          if (q >= NB || ha[k] == 0.0) continue;
          const double2 x = a[p], y = a[q];
          a[p] = csub(cscale(x, hc[k]), cmul(hs[k], y));
          a[q] = cadd(cmulc(x, hs[k]), cscale(y, hc[k]));
        }
        if (mact != 0.0) {
#pragma unroll
          for (int r = 0; r < NB; ++r) {
            if (r == partner) a[r] = make_double2(0.0, 0.0);
            if (r == c) a[r].y = 0.0;
          }
        }
      }
    }
    if (!__any_sync(0xffffffffu, rotated)) break;
  }
}

// eps, Qout <- eigh(A) per k, eigenvalues ascending (solver.py:389, 622-626).  With a
// starting basis Qin (rotate): A is taken in that basis (Qin^H A Qin, nearly diagonal
// when Qin already diagonalises a nearby matrix, so the sweeps converge at once) and
// Qout = Qin V.  Qin may equal Qout: a k-point's rows are read before they are written.
constexpr int kEigWarps = 2;
// mode 1 (no starting basis): the eigensolve of herm(i A), the Cayley spectral setup of
// solver.py:161-166
template <int NB>
__device__ __forceinline__ void eig_cols(int nk, const double2* __restrict__ A, const double2* Qin, double2* Qout,
                                         double* eps, double tol, int mode = 0) {
  const bool rotate = Qin != nullptr;
  using RG = RowGroup<NB>;
  constexpr int G = RG::G, KPW = RG::KPW, LP = RG::LP, MAT = RG::MAT, NP = JacobiPairs<NB>::M / 2;
  __shared__ double2 st[kEigWarps][KPW][3 * MAT + 2 * NP];
  __shared__ double sw[kEigWarps][KPW][NB];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, g = lane / G, c = lane % G;
  double2* SQ = st[w][g];
  double2* SA = SQ + MAT;
  double2* SV = SA + MAT;
  double2* SP = SV + MAT;
  double* SW = sw[w][g];
  for (int kb = (blockIdx.x * kEigWarps + w) * KPW; kb < nk; kb += gridDim.x * kEigWarps * KPW) {
    const int k = kb + g;
    const bool on = k < nk && c < NB;
    const size_t base = (size_t)k * NB * NB + c;
    if (on) {
#pragma unroll
      for (int r = 0; r < NB; ++r) {
        const double2 x = A[base + (size_t)r * NB];
        SA[r * LP + c] = mode ? make_double2(-x.y, x.x) : x;
      }
    }
    if (rotate) {  // SA <- Q^H F Q, column c
      // q_c goes through SQ and t = A q_c through this lane's column of SV (free until V
      // is formed), and Q^H t straight into the lane's column of SA: no nb-vector is held
      // in registers across a barrier (at the 128-register cap of nb 5-8 they spilled)
      if (on) {
#pragma unroll
        for (int r = 0; r < NB; ++r) SQ[r * LP + c] = Qin[base + (size_t)r * NB];
      }
      __syncwarp();
      if (on) {
#pragma unroll
        for (int r = 0; r < NB; ++r) {
          double2 acc = make_double2(0.0, 0.0);
#pragma unroll
          for (int j = 0; j < NB; ++j) acc = cfma(SA[r * LP + j], SQ[j * LP + c], acc);
          SV[r * LP + c] = acc;
        }
      }
      __syncwarp();  // every lane has read A: its column can take (Q^H A q_c) entry by entry
      if (on) {
#pragma unroll
        for (int i = 0; i < NB; ++i) {
          double2 acc = make_double2(0.0, 0.0);
#pragma unroll
          for (int r = 0; r < NB; ++r) acc = cfma_cj(SQ[r * LP + i], SV[r * LP + c], acc);
          SA[i * LP + c] = acc;
        }
      }
    }
    __syncwarp();
    // hermitise (jnp.linalg.eigh symmetrises its input); V = I; Frobenius norm of the group
    double2 hm[NB];
    double fro = 0.0;
    if (on) {
#pragma unroll
      for (int r = 0; r < NB; ++r) {
        const double2 x = SA[r * LP + c], y = SA[c * LP + r];
        hm[r] = r == c ? make_double2(x.x, 0.0) : make_double2(0.5 * (x.x + y.x), 0.5 * (x.y - y.y));
        fro += hm[r].x * hm[r].x + hm[r].y * hm[r].y;
      }
    }
#pragma unroll
    for (int off = G / 2; off > 0; off >>= 1) fro += __shfl_xor_sync(0xffffffffu, fro, off);
    __syncwarp();
    double2 vc[NB];  // this lane's column of V, from the identity
#pragma unroll
    for (int r = 0; r < NB; ++r) vc[r] = make_double2(r == c ? 1.0 : 0.0, 0.0);
    double wc = 0.0;
    const double thr = fmax(tol * sqrt(fro), 1e-300);
    if constexpr (NB <= 4) {
      // columns in registers (measured on a B200: nb = 4 in 0.70 of the shared-memory time;
      // from nb = 8 on, the register version spills and its shuffles cost more)
      jacobi_reg_cols<NB>(hm, vc, c, g * G, on, thr);
#pragma unroll
      for (int r = 0; r < NB; ++r)
        if (r == c) wc = hm[r].x;
    } else {
      if (on) {
#pragma unroll
        for (int r = 0; r < NB; ++r) {
          SA[r * LP + c] = hm[r];
          SV[r * LP + c] = vc[r];
        }
      }
      __syncwarp();
      jacobi_smem_cols<NB>(SA, SV, SP, c, on, thr);
      if (on) {
        wc = SA[c * LP + c].x;
#pragma unroll
        for (int r = 0; r < NB; ++r) vc[r] = SV[r * LP + c];
      }
    }
    // ascending order: lane c's eigenpair goes to column rank(c)
    if (on) SW[c] = wc;
    __syncwarp();
    if (on) {
      int rk = 0;
#pragma unroll
      for (int j = 0; j < NB; ++j) rk += (SW[j] < wc) || (SW[j] == wc && j < c);
      eps[(size_t)k * NB + rk] = wc;
      const size_t out = (size_t)k * NB * NB + rk;
      if (rotate) {  // (Q V)[r][rk] = sum_j Q[r][j] V[j][c]
#pragma unroll
        for (int r = 0; r < NB; ++r) {
          double2 acc = make_double2(0.0, 0.0);
#pragma unroll
          for (int j = 0; j < NB; ++j) acc = cfma(SQ[r * LP + j], vc[j], acc);
          Qout[out + (size_t)r * NB] = acc;
        }
      } else {
#pragma unroll
        for (int r = 0; r < NB; ++r) Qout[out + (size_t)r * NB] = vc[r];
      }
    }
    __syncwarp();
  }
}

template <int NB>
__global__ void __launch_bounds__(32 * kEigWarps, 8) k_cgr_eig(CgArgs a, const double2* __restrict__ A, int rotate,
                                                            double tol) {
  eig_cols<NB>(a.nk, A, rotate ? q_cur(a) : nullptr, a.Q, a.eps, tol);
}
// Standalone eigensolve: eps, Qout <- eigh(A) (Qin == nullptr) or with the starting basis Qin.
template <int NB>
__global__ void __launch_bounds__(32 * kEigWarps, 8) k_eig_cols(int nk, const double2* __restrict__ A,
                                                             const double2* Qin, double2* Qout, double* eps,
                                                             double tol, int mode) {
  eig_cols<NB>(nk, A, Qin, Qout, eps, tol, mode);
}

}  // namespace hf
