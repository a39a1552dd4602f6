// Direct-minimisation solver on the device: preconditioned Riemannian CG on
// Stiefel x capped simplex with the spectral Cayley line search
// (solver.py:307-660).  All state and every scalar of the loop (mu, energy,
// gradient norm, PR beta, step, line-search decision, history, stopping rule)
// live in device memory; the host only enqueues kernels and reads one flag per
// chunk of iterations.
//
// One iteration = density -> Fock build (3 FFT passes) -> energy -> grad1 ->
// grad2 -> direction (+ Jacobi eigh of i d_Q) -> first trial -> remaining
// trials -> retraction -> mu -> step end.  Per-k kernels run one warp per
// k-point; each reduction is finalised by the last CTA to finish (atomic
// ticket), which also performs the scalar update of the reference loop body.
// Every kernel of an iteration returns at once when the device flag `active`
// is clear, so whole chunks can be queued without host round trips.
#include <algorithm>
#include <cmath>
#include <thread>
#include <vector>

#include "common.cuh"
#include "perk.cuh"
#include "solver_common.cuh"

namespace hf {

int fock_build_internal(void* stream, int dtype, unsigned flags, int nk1, int nk2, int nb, const void* P,
                        const void* h, const void* VR, const void* refP, const void* HH, const void* w2d,
                        int n_contact, const void* contact_g, const void* contact_Oi, const void* contact_Oj,
                        void* Sigma, void* H, void* F, void* workspace, size_t workspace_bytes,
                        const int* active);
int energy_internal(void* stream, int dtype, int nk1, int nk2, int nb, const void* P, const void* h,
                    const void* Sigma, const void* H, int H_mode, const void* w2d, double* E_out,
                    void* workspace, size_t workspace_bytes, const int* active);
int find_mu_internal(void* stream, int dtype, int method, int nk1, int nk2, int nb, const void* eps,
                     const void* weights, double n_electrons, double T, int maxiter, const double* mu0,
                     double* mu_out, const int* active);

struct CgScalars {
  int k, active, accepted, converged, k_base;
  int first_ok;  // the first line-search trial was accepted: Q U(tau0) and eps are already formed
  int qsel;      // row path: the current Q is Vd (1) or the caller's Q buffer (0)
  int switched_at;  // whole-batch graph: iteration of the FP32 -> FP64 switch (-1: none)
  double mu, E, E_prev, dE, grad_norm;
  double lam, pr_den, beta, tau0, tau_final, Omega0, E_fin;
};

struct CgArgs {
  int nk, nb, max_iter, cg_restart, bt_max, plateau_window;
  double T_r, tol_E, tol_grad, denom_scale, max_step, bt_shrink, n_target_norm;
  double2 *Q, *P, *F, *Ft, *G0, *G1, *dQ, *Vd, *Fe;  // Vd: eigenvectors of i d (warp path), Q U(tau0) (row path)
  double *p, *eps, *epsF, *gp0, *gp1, *dp, *lamd, *w_norm;
  double* hist_E;
  double* hist_G;
  CgScalars* sc;
  double* part;
  unsigned* counter;
};

__device__ __forceinline__ bool cg_active(const CgArgs& a) { return a.sc->active != 0; }
// Row path (nb <= 8): Q alternates between the caller's buffer and Vd; the first
// line-search trial writes Q U(tau0) into the other one and, when tau0 is
// accepted, flips qsel instead of copying.  Finalize rotates it back into the
// caller's buffer.
__device__ __forceinline__ double2* q_cur(const CgArgs& a) { return a.sc->qsel ? a.Vd : a.Q; }
__device__ __forceinline__ double2* q_alt(const CgArgs& a) { return a.sc->qsel ? a.Q : a.Vd; }
__global__ void k_cg_qsel_reset(CgArgs a) { a.sc->qsel = 0; }

}  // namespace hf

#include "cg_rows.cuh"  // lane-per-row kernels (use CgArgs / cg_active above)

namespace hf {

// ------------------------------------------------------------------ init ---
__global__ void k_cg_init(CgArgs a, const double2* __restrict__ P0, const double* __restrict__ w2d,
                          double weight_sum) {
  const size_t nb2 = (size_t)a.nb * a.nb;
  const size_t nq = (size_t)a.nk * nb2, nv = (size_t)a.nk * a.nb;
  const double ws = fmax(weight_sum, 1e-30);
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < nq; e += (size_t)gridDim.x * blockDim.x) {
    const size_t k = e / nb2;
    const int r = (int)(e - k * nb2), i = r / a.nb, j = r - (r / a.nb) * a.nb;
    const double2 x = P0[e], y = P0[k * nb2 + (size_t)j * a.nb + i];
    a.P[e] = make_double2(0.5 * (x.x + y.x), 0.5 * (x.y - y.y));
    a.G0[e] = a.G1[e] = a.dQ[e] = make_double2(0.0, 0.0);
  }
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < nv; e += (size_t)gridDim.x * blockDim.x)
    a.gp0[e] = a.gp1[e] = a.dp[e] = 0.0;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < (size_t)a.nk; k += (size_t)gridDim.x * blockDim.x)
    a.w_norm[k] = w2d[k] / ws;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    CgScalars* s = a.sc;
    s->k = 0;
    s->k_base = 0;
    s->active = a.max_iter > 0 ? 1 : 0;
    s->accepted = 0;
    s->first_ok = 0;
    s->qsel = 0;
    s->converged = 0;
    s->mu = 0.0;
    s->E = 0.0;
    s->E_prev = INFINITY;
    s->dE = INFINITY;
    s->grad_norm = INFINITY;
    s->lam = s->pr_den = s->beta = s->tau0 = s->tau_final = s->Omega0 = s->E_fin = 0.0;
    *a.counter = 0u;
  }
}

// Rotation threshold of the init / finalize eigensolves, relative to |A|_F: at the
// double-precision rounding level, so converged rotations are not re-made from noise.
constexpr double kEigTol = 1e-15;

// eps, Q <- eigh(A) per k (A = F0 at init, or Ft = Q^H F Q at finalize with Q <- Q V)
__global__ void k_cg_eig(CgArgs a, const double2* __restrict__ A, int rotate) {
  extern __shared__ double2 sm[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const int nb = a.nb, nb2 = nb * nb;
  double2* m = sm + (size_t)w * (jacobi_smem_elems(nb) + 2 * nb2);
  double2* v = m + nb2;
  double2* scr = v + nb2;
  double2* q = scr + nb + 40;
  double2* t = q + nb2;
  double* wv = reinterpret_cast<double*>(scr);
  for (int k = blockIdx.x * wpb + w; k < a.nk; k += gridDim.x * wpb) {
    const size_t base = (size_t)k * nb2;
    if (rotate) {
      for (int e = lane; e < nb2; e += 32) { q[e] = a.Q[base + e]; m[e] = A[base + e]; }
      __syncwarp();
      warp_qhaq(q, m, t, nb, lane);  // m <- Q^H F Q
      __syncwarp();
    } else {
      for (int e = lane; e < nb2; e += 32) m[e] = A[base + e];
      __syncwarp();
    }
    // hermitise (jnp.linalg.eigh symmetrises its input)
    for (int e = lane; e < nb2; e += 32) {
      const int i = e / nb, j = e - i * nb;
      if (i < j) {
        const double2 x = m[e], y = m[j * nb + i];
        const double2 hxy = make_double2(0.5 * (x.x + y.x), 0.5 * (x.y - y.y));
        m[e] = hxy;
        m[j * nb + i] = conj(hxy);
      } else if (i == j) {
        m[e].y = 0.0;
      }
    }
    __syncwarp();
    warp_jacobi_eigh(m, v, scr + nb, nb, lane, kEigTol);
    for (int e = lane; e < nb; e += 32) wv[e] = m[e * nb + e].x;
    __syncwarp();
    for (int i = lane; i < nb; i += 32) {
      const double wi = wv[i];
      int r = 0;
      for (int j = 0; j < nb; ++j) r += (wv[j] < wi) || (wv[j] == wi && j < i);
      a.eps[(size_t)k * nb + r] = wi;
      for (int row = 0; row < nb; ++row) t[row * nb + r] = v[row * nb + i];
    }
    __syncwarp();
    if (rotate) {  // Q <- Q V
      for (int e = lane; e < nb2; e += 32) {
        const int i = e / nb, j = e - i * nb;
        double2 acc = make_double2(0.0, 0.0);
        for (int n = 0; n < nb; ++n) acc = cadd(acc, cmul(q[i * nb + n], t[n * nb + j]));
        a.Q[base + e] = acc;
      }
    } else {
      for (int e = lane; e < nb2; e += 32) a.Q[base + e] = t[e];
    }
    __syncwarp();
  }
}

// ---------------------------------------------- density: p and P = herm(Q p Q^H)
__global__ void k_cg_density(CgArgs a, int force) {
  if (!force && !cg_active(a)) return;
  extern __shared__ double2 sm[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const int nb = a.nb, nb2 = nb * nb;
  double2* q = sm + (size_t)w * (2 * nb2 + nb);
  double2* t = q + nb2;
  double* pp = reinterpret_cast<double*>(t + nb2);
  const double mu = a.sc->mu;
  for (int k = blockIdx.x * wpb + w; k < a.nk; k += gridDim.x * wpb) {
    const size_t base = (size_t)k * nb2;
    for (int e = lane; e < nb2; e += 32) q[e] = a.Q[base + e];
    for (int i = lane; i < nb; i += 32) {
      const double pv = sigmoid((mu - a.eps[(size_t)k * nb + i]) / a.T_r);
      pp[i] = pv;
      a.p[(size_t)k * nb + i] = pv;
    }
    __syncwarp();
    warp_density(q, pp, t, nb, lane);
    __syncwarp();
    for (int e = lane; e < nb2; e += 32) {
      const int i = e / nb, j = e - i * nb;
      const double2 x = t[e], y = t[j * nb + i];
      a.P[base + e] = make_double2(0.5 * (x.x + y.x), 0.5 * (x.y - y.y));
    }
    __syncwarp();
  }
}

// ----------------------------------- grad1: Ft, eps, G, g_p and four norms ---
__global__ void k_cg_grad1(CgArgs a) {
  if (!cg_active(a)) return;
  extern __shared__ double2 sm[];
  __shared__ double red[64];
  __shared__ double tot[kMaxSums];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const int nb = a.nb, nb2 = nb * nb;
  double2* q = sm + (size_t)w * 3 * nb2;
  double2* f = q + nb2;
  double2* t = f + nb2;
  const int par = a.sc->k & 1;
  double2* G = par ? a.G1 : a.G0;
  const double2* Gp = par ? a.G0 : a.G1;
  double* gp = par ? a.gp1 : a.gp0;
  const double* gpp = par ? a.gp0 : a.gp1;
  const double mu = a.sc->mu;
  KSum acc[4];
  for (int k = blockIdx.x * wpb + w; k < a.nk; k += gridDim.x * wpb) {
    const size_t base = (size_t)k * nb2, vb = (size_t)k * nb;
    const double wk = a.w_norm[k];
    for (int e = lane; e < nb2; e += 32) { q[e] = a.Q[base + e]; f[e] = a.F[base + e]; }
    __syncwarp();
    warp_qhaq(q, f, t, nb, lane);
    __syncwarp();
    for (int e = lane; e < nb2; e += 32) {
      const int i = e / nb, j = e - i * nb;
      const double2 ft = f[e];
      a.Ft[base + e] = ft;
      double2 g = make_double2(0.0, 0.0);
      if (i != j) {
        const double2 fji = f[j * nb + i];
        const double dpij = a.p[vb + j] - a.p[vb + i];
        g = make_double2(0.5 * dpij * (ft.x + fji.x), 0.5 * dpij * (ft.y - fji.y));
      }
      G[base + e] = g;
      acc[0].add(wk * (g.x * g.x + g.y * g.y));
      const double2 o = Gp[base + e];
      acc[2].add(wk * (o.x * o.x + o.y * o.y));
    }
    for (int i = lane; i < nb; i += 32) {
      const double ei = f[i * nb + i].x;
      a.epsF[vb + i] = ei;
      const double ps = clip(a.p[vb + i], 1e-6, 1.0 - 1e-6);
      const double g = ei + a.T_r * (log(ps) - log1p(-ps)) - mu;
      gp[vb + i] = g;
      acc[1].add(ei * ei);
      acc[3].add(wk * gpp[vb + i] * gpp[vb + i]);
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

__device__ __forceinline__ double2 precond(double2 g, double ei, double ej, double lam) {
  const double gap = ei - ej;
  const double d = sqrt(gap * gap + lam * lam);
  return make_double2(g.x / d, g.y / d);
}

// Elementwise passes with the band count as a template parameter (index math at
// compile time), one rsqrt per element for the preconditioner, per-thread plain
// double partials and compensated sums across threads and blocks.
template <int NB>
__global__ void __launch_bounds__(256) k_cg_grad2_t(CgArgs a) {
  if (!cg_active(a)) return;
  __shared__ double red[64];
  __shared__ double tot[kMaxSums];
  constexpr unsigned nb2 = NB * NB;
  const int par = a.sc->k & 1;
  const double2* G = par ? a.G1 : a.G0;
  const double2* Gp = par ? a.G0 : a.G1;
  const double* gp = par ? a.gp1 : a.gp0;
  const double* gpp = par ? a.gp0 : a.gp1;
  const double lam2 = a.sc->lam * a.sc->lam;
  const unsigned nq = (unsigned)a.nk * nb2;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
  for (unsigned e = blockIdx.x * blockDim.x + threadIdx.x; e < nq; e += gridDim.x * blockDim.x) {
    const unsigned k = e / nb2, r = e - k * nb2, i = r / NB, j = r - i * NB;
    const double wk = a.w_norm[k];
    const double2 g = G[e], o = Gp[e];
    const double gap = a.epsF[k * NB + i] - a.epsF[k * NB + j];
    const double rs = rsqrt(fma(gap, gap, lam2));
    s0 += wk * rs * (g.x * g.x + g.y * g.y);
    s1 += wk * rs * (o.x * g.x + o.y * g.y);
    if (j == 0) {
      const unsigned vi = k * NB + i;
      const double ps = clip(a.p[vi], 1e-8, 1.0 - 1e-8);
      const double hp = gp[vi] * (ps * (1.0 - ps) / a.T_r);
      s2 += wk * gp[vi] * hp;
      s3 += wk * gpp[vi] * hp;
    }
  }
  KSum acc[4];
  acc[0].add(s0);
  acc[1].add(s1);
  acc[2].add(s2);
  acc[3].add(s3);
  if (publish_partials<4>(acc, a.part, a.counter, red)) {
    gather_partials<4>(a.part, a.counter, tot, red);
    if (threadIdx.x == 0) {
      CgScalars* sc = a.sc;
      const double num = tot[0] - tot[1] + tot[2] - tot[3];
      double beta = sc->pr_den > 1e-30 ? fmax(0.0, num / sc->pr_den) : 0.0;
      beta = fmin(beta, 5.0);
      if (sc->k == 0 || sc->k % a.cg_restart == 0) beta = 0.0;
      sc->beta = beta;
    }
  }
}

template <int NB>
__global__ void __launch_bounds__(256) k_cg_dir_t(CgArgs a) {
  if (!cg_active(a)) return;
  __shared__ double red[64];
  __shared__ double tot[kMaxSums];
  constexpr unsigned nb2 = NB * NB;
  const int par = a.sc->k & 1;
  const double2* G = par ? a.G1 : a.G0;
  const double* gp = par ? a.gp1 : a.gp0;
  const double lam2 = a.sc->lam * a.sc->lam, beta = a.sc->beta;
  const unsigned nq = (unsigned)a.nk * nb2, nv = (unsigned)a.nk * NB;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  for (unsigned e = blockIdx.x * blockDim.x + threadIdx.x; e < nq; e += gridDim.x * blockDim.x) {
    const unsigned k = e / nb2, r = e - k * nb2, i = r / NB, j = r - i * NB;
    const double gap = a.epsF[k * NB + i] - a.epsF[k * NB + j];
    const double rs = rsqrt(fma(gap, gap, lam2));
    const double2 g = G[e], dprev = a.dQ[e];
    const double2 d = make_double2(fma(g.x, rs, beta * dprev.x), fma(g.y, rs, beta * dprev.y));
    a.dQ[e] = d;
    s0 += a.w_norm[k] * (d.x * d.x + d.y * d.y);
  }
  for (unsigned v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
    const unsigned k = v / NB;
    const double wk = a.w_norm[k];
    const double ps = clip(a.p[v], 1e-8, 1.0 - 1e-8);
    const double hp = gp[v] * (ps * (1.0 - ps) / a.T_r);
    a.dp[v] = hp + beta * a.dp[v];
    s1 += wk * ps * a.epsF[v];
    s2 += wk * ent_term(ps);
  }
  KSum acc[3];
  acc[0].add(s0);
  acc[1].add(s1);
  acc[2].add(s2);
  if (publish_partials<3>(acc, a.part, a.counter, red)) {
    gather_partials<3>(a.part, a.counter, tot, red);
    if (threadIdx.x == 0) {
      CgScalars* sc = a.sc;
      const double dn = sqrt(fmax(0.0, tot[0]));
      sc->tau0 = fmin(1.0, a.max_step / fmax(dn, 1e-30));
      sc->Omega0 = tot[1] + fmax(a.T_r, 1e-14) * tot[2];
      sc->accepted = 0;
      sc->first_ok = 0;
      sc->tau_final = sc->tau0;
    }
  }
}

// --------------------------------------------- grad2: PR+ inner products ---
__global__ void k_cg_grad2(CgArgs a) {
  if (!cg_active(a)) return;
  __shared__ double red[64];
  __shared__ double tot[kMaxSums];
  const int par = a.sc->k & 1;
  const double2* G = par ? a.G1 : a.G0;
  const double2* Gp = par ? a.G0 : a.G1;
  const double* gp = par ? a.gp1 : a.gp0;
  const double* gpp = par ? a.gp0 : a.gp1;
  const double lam = a.sc->lam;
  const int nb = a.nb, nb2 = nb * nb;
  const size_t nq = (size_t)a.nk * nb2;
  KSum acc[4];
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < nq; e += (size_t)gridDim.x * blockDim.x) {
    const size_t k = e / nb2;
    const int r = (int)(e - k * nb2), i = r / nb, j = r - (r / nb) * nb;
    const double wk = a.w_norm[k];
    const double2 g = G[e];
    const double2 hq = precond(g, a.epsF[k * nb + i], a.epsF[k * nb + j], lam);
    const double2 o = Gp[e];
    acc[0].add(wk * (g.x * hq.x + g.y * hq.y));
    acc[1].add(wk * (o.x * hq.x + o.y * hq.y));
    if (j == 0) {
      const size_t vi = k * nb + i;
      const double ps = clip(a.p[vi], 1e-8, 1.0 - 1e-8);
      const double hp = gp[vi] * (ps * (1.0 - ps) / a.T_r);
      acc[2].add(wk * gp[vi] * hp);
      acc[3].add(wk * gpp[vi] * hp);
    }
  }
  if (publish_partials<4>(acc, a.part, a.counter, red)) {
    gather_partials<4>(a.part, a.counter, tot, red);
    if (threadIdx.x == 0) {
      CgScalars* s = a.sc;
      const double num = tot[0] - tot[1] + tot[2] - tot[3];
      double beta = s->pr_den > 1e-30 ? fmax(0.0, num / s->pr_den) : 0.0;
      beta = fmin(beta, 5.0);
      if (s->k == 0 || s->k % a.cg_restart == 0) beta = 0.0;
      s->beta = beta;
    }
  }
}

// ---- direction d = H + beta d_prev, eigh(i d) -> (V, lam), Fe = V^H Ft V, tau0, Omega0
__global__ void k_cg_dir(CgArgs a) {
  if (!cg_active(a)) return;
  extern __shared__ double2 sm[];
  __shared__ double red[64];
  __shared__ double tot[kMaxSums];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const int nb = a.nb, nb2 = nb * nb;
  double2* m = sm + (size_t)w * (jacobi_smem_elems(nb) + 2 * nb2);
  double2* v = m + nb2;
  double2* scr = v + nb2;
  double2* ft = scr + nb + 40;
  double2* t = ft + nb2;
  double* wv = reinterpret_cast<double*>(scr);
  const int par = a.sc->k & 1;
  const double2* G = par ? a.G1 : a.G0;
  const double* gp = par ? a.gp1 : a.gp0;
  const double lam = a.sc->lam, beta = a.sc->beta;
  const double Tm = fmax(a.T_r, 1e-14);
  (void)Tm;
  KSum acc[3];
  for (int k = blockIdx.x * wpb + w; k < a.nk; k += gridDim.x * wpb) {
    const size_t base = (size_t)k * nb2, vb = (size_t)k * nb;
    const double wk = a.w_norm[k];
    for (int e = lane; e < nb2; e += 32) {
      const int i = e / nb, j = e - i * nb;
      const double2 hq = precond(G[base + e], a.epsF[vb + i], a.epsF[vb + j], lam);
      const double2 dprev = a.dQ[base + e];
      const double2 d = make_double2(hq.x + beta * dprev.x, hq.y + beta * dprev.y);
      a.dQ[base + e] = d;
      t[e] = d;
      acc[0].add(wk * (d.x * d.x + d.y * d.y));
      ft[e] = a.Ft[base + e];
    }
    for (int i = lane; i < nb; i += 32) {
      const double pv = a.p[vb + i];
      const double ps = clip(pv, 1e-8, 1.0 - 1e-8);
      const double hp = gp[vb + i] * (ps * (1.0 - ps) / a.T_r);
      a.dp[vb + i] = hp + beta * a.dp[vb + i];
      acc[1].add(wk * ps * a.epsF[vb + i]);
      acc[2].add(wk * ent_term(ps));
    }
    __syncwarp();
    // m = herm(i d)
    for (int e = lane; e < nb2; e += 32) {
      const int i = e / nb, j = e - i * nb;
      const double2 x = mul_pi(t[e]), y = mul_pi(t[j * nb + i]);
      m[e] = make_double2(0.5 * (x.x + y.x), 0.5 * (x.y - y.y));
    }
    __syncwarp();
    warp_jacobi_eigh(m, v, scr + nb, nb, lane, 1e-17);
    for (int e = lane; e < nb; e += 32) wv[e] = m[e * nb + e].x;
    __syncwarp();
    for (int i = lane; i < nb; i += 32) {  // ascending order, V columns
      const double wi = wv[i];
      int r = 0;
      for (int j = 0; j < nb; ++j) r += (wv[j] < wi) || (wv[j] == wi && j < i);
      a.lamd[vb + r] = wi;
      for (int row = 0; row < nb; ++row) t[row * nb + r] = v[row * nb + i];
    }
    __syncwarp();
    for (int e = lane; e < nb2; e += 32) a.Vd[base + e] = t[e];
    warp_qhaq(t, ft, m, nb, lane);  // ft <- V^H Ft V
    __syncwarp();
    for (int e = lane; e < nb2; e += 32) a.Fe[base + e] = ft[e];
    __syncwarp();
  }
  if (publish_partials<3>(acc, a.part, a.counter, red)) {
    gather_partials<3>(a.part, a.counter, tot, red);
    if (threadIdx.x == 0) {
      CgScalars* s = a.sc;
      const double dn = sqrt(fmax(0.0, tot[0]));
      s->tau0 = fmin(1.0, a.max_step / fmax(dn, 1e-30));
      s->Omega0 = tot[1] + fmax(a.T_r, 1e-14) * tot[2];
      s->accepted = 0;
      s->first_ok = 0;
      s->tau_final = s->tau0;
    }
  }
}

// ---- direction d = H + beta d_prev (elementwise), tau0 and Omega0: the retraction
// of the lane-per-row path needs no eigendecomposition of d.
__global__ void k_cg_dir_lu(CgArgs a) {
  if (!cg_active(a)) return;
  __shared__ double red[64];
  __shared__ double tot[kMaxSums];
  const int par = a.sc->k & 1;
  const double2* G = par ? a.G1 : a.G0;
  const double* gp = par ? a.gp1 : a.gp0;
  const double lam = a.sc->lam, beta = a.sc->beta;
  const unsigned nb = a.nb, nb2 = nb * nb;
  const unsigned nq = (unsigned)a.nk * nb2, nv = (unsigned)a.nk * nb;
  KSum acc[3];
  for (unsigned e = blockIdx.x * blockDim.x + threadIdx.x; e < nq; e += gridDim.x * blockDim.x) {
    const unsigned k = e / nb2, rr = e - k * nb2, i = rr / nb, j = rr - i * nb;
    const double2 hq = precond(G[e], a.epsF[k * nb + i], a.epsF[k * nb + j], lam);
    const double2 dprev = a.dQ[e];
    const double2 d = make_double2(hq.x + beta * dprev.x, hq.y + beta * dprev.y);
    a.dQ[e] = d;
    acc[0].add(a.w_norm[k] * (d.x * d.x + d.y * d.y));
  }
  for (unsigned v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
    const unsigned k = v / nb;
    const double wk = a.w_norm[k];
    const double ps = clip(a.p[v], 1e-8, 1.0 - 1e-8);
    const double hp = gp[v] * (ps * (1.0 - ps) / a.T_r);
    a.dp[v] = hp + beta * a.dp[v];
    acc[1].add(wk * ps * a.epsF[v]);
    acc[2].add(wk * ent_term(ps));
  }
  if (publish_partials<3>(acc, a.part, a.counter, red)) {
    gather_partials<3>(a.part, a.counter, tot, red);
    if (threadIdx.x == 0) {
      CgScalars* s = a.sc;
      const double dn = sqrt(fmax(0.0, tot[0]));
      s->tau0 = fmin(1.0, a.max_step / fmax(dn, 1e-30));
      s->Omega0 = tot[1] + fmax(a.T_r, 1e-14) * tot[2];
      s->accepted = 0;
      s->first_ok = 0;
      s->tau_final = s->tau0;
    }
  }
}

// -------------------- line-search trials i0 <= i < i1 on the frozen-F free energy
template <int NT>
__global__ void k_cg_trials(CgArgs a, int i0, int i1, int last_chunk) {
  if (!cg_active(a)) return;
  if (a.sc->accepted) return;
  extern __shared__ double2 sm[];
  __shared__ double red[64];
  __shared__ double tot[kMaxSums];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const int nb = a.nb, nb2 = nb * nb;
  double2* v = sm + (size_t)w * (2 * nb2 + nb);
  double2* f = v + nb2;
  double2* c = f + nb2;
  const int nt = i1 - i0;
  double taus[NT];
  {
    double tau = a.sc->tau0;
    for (int i = 0; i < i0; ++i) tau = tau * a.bt_shrink;
    for (int i = 0; i < NT; ++i) { taus[i] = tau; tau = tau * a.bt_shrink; }
  }
  KSum acc[2 * NT];
  for (int k = blockIdx.x * wpb + w; k < a.nk; k += gridDim.x * wpb) {
    const size_t base = (size_t)k * nb2, vb = (size_t)k * nb;
    const double wk = a.w_norm[k];
    for (int e = lane; e < nb2; e += 32) { v[e] = a.Vd[base + e]; f[e] = a.Fe[base + e]; }
    for (int it = 0; it < nt; ++it) {
      __syncwarp();
      for (int i = lane; i < nb; i += 32) c[i] = cayley_factor(taus[it], a.lamd[vb + i]);
      __syncwarp();
      for (int i = lane; i < nb; i += 32) {
        const double et = diag_ufu_row(v, f, c, nb, i);
        const double pt = clip(a.p[vb + i] - taus[it] * a.dp[vb + i], 1e-8, 1.0 - 1e-8);
        acc[2 * it].add(wk * pt * et);
        acc[2 * it + 1].add(wk * ent_term(pt));
      }
    }
    __syncwarp();
  }
  if (publish_partials<2 * NT>(acc, a.part, a.counter, red)) {
    gather_partials<2 * NT>(a.part, a.counter, tot, red);
    if (threadIdx.x == 0) {
      CgScalars* s = a.sc;
      const double Tm = fmax(a.T_r, 1e-14);
      for (int it = 0; it < nt; ++it) {
        const double om = tot[2 * it] + Tm * tot[2 * it + 1];
        if (om < s->Omega0) { s->accepted = 1; s->tau_final = taus[it]; break; }
      }
      if (!s->accepted && last_chunk) s->tau_final = s->tau0 * pow(a.bt_shrink, (double)a.bt_max);
    }
  }
}

// ----------------- retraction: U(tau), Q <- Q U, eps_new = diag(U^H Ft U)
__global__ void k_cg_update(CgArgs a) {
  if (!cg_active(a)) return;
  extern __shared__ double2 sm[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const int nb = a.nb, nb2 = nb * nb;
  double2* v = sm + (size_t)w * (4 * nb2 + nb);
  double2* f = v + nb2;
  double2* u = f + nb2;
  double2* q = u + nb2;
  double2* c = q + nb2;
  const double tau = a.sc->tau_final;
  for (int k = blockIdx.x * wpb + w; k < a.nk; k += gridDim.x * wpb) {
    const size_t base = (size_t)k * nb2, vb = (size_t)k * nb;
    for (int e = lane; e < nb2; e += 32) { v[e] = a.Vd[base + e]; f[e] = a.Fe[base + e]; q[e] = a.Q[base + e]; }
    for (int i = lane; i < nb; i += 32) c[i] = cayley_factor(tau, a.lamd[vb + i]);
    __syncwarp();
    for (int e = lane; e < nb2; e += 32) {
      const int i = e / nb, j = e - i * nb;
      double2 acc = make_double2(0.0, 0.0);
      for (int n = 0; n < nb; ++n) acc = cadd(acc, cmulc(cmul(v[i * nb + n], c[n]), v[j * nb + n]));
      u[e] = acc;
    }
    for (int i = lane; i < nb; i += 32) a.eps[vb + i] = diag_ufu_row(v, f, c, nb, i);
    __syncwarp();
    for (int e = lane; e < nb2; e += 32) {
      const int i = e / nb, j = e - i * nb;
      double2 acc = make_double2(0.0, 0.0);
      for (int n = 0; n < nb; ++n) acc = cadd(acc, cmul(q[i * nb + n], u[n * nb + j]));
      a.Q[base + e] = acc;
    }
    __syncwarp();
  }
}

// ------------------------------- history, |dE| and the stopping rule ---
// solver.py:422-449 and 595-597.  `phase_rel` > 0 only in the FP32-exchange
// phase of the mixed solve: the energy tolerance is raised to the FP32 noise
// floor phase_rel |E|; k_base restarts the plateau window at the FP64 switch
// (k_base = 0 reproduces the reference rule exactly).
__global__ void k_cg_step_end(CgArgs a, double phase_rel) {
  if (!cg_active(a)) return;
  CgScalars* s = a.sc;
  const int k = s->k;
  a.hist_E[k] = s->E;
  a.hist_G[k] = s->grad_norm;
  s->dE = fabs(s->E - s->E_prev);
  s->E_prev = s->E;
  const int kn = k + 1;
  s->k = kn;
  const double tol = phase_rel > 0.0 ? fmax(a.tol_E, phase_rel * fabs(s->E)) : a.tol_E;
  const int kk = kn - s->k_base;
  bool enc;
  if (a.plateau_window > 0) {
    const double e_now = a.hist_E[max(kn - 1, 0)];
    const double e_past = a.hist_E[max(kn - 1 - a.plateau_window, s->k_base)];
    enc = (kk > a.plateau_window) ? (e_past - e_now) > tol : s->dE > tol;
  } else {
    enc = s->dE > tol;
  }
  // FP32 phase: leave it at the energy plateau of the raised tolerance or once the
  // gradient target is met; FP64 (and the plain solver): the reference rule.
  const bool nc = phase_rel > 0.0 ? (enc && !(a.tol_grad > 0.0 && s->grad_norm <= a.tol_grad))
                                  : (a.tol_grad > 0.0 ? s->grad_norm > a.tol_grad : enc);
  s->active = (kn < a.max_iter && nc) ? 1 : 0;
}

// FP32 -> FP64 switch of the mixed solve: continue from the current state.
__global__ void k_cg_rearm(CgArgs a) {
  CgScalars* s = a.sc;
  s->k_base = s->k;
  s->active = s->k < a.max_iter ? 1 : 0;
}

// switched_at == -2: the switch iteration recorded on the device (whole-batch graph)
__global__ void k_cg_converged(CgArgs a, int switched_at, double* __restrict__ out) {
  CgScalars* s = a.sc;
  if (switched_at == -2) switched_at = s->switched_at;
  s->converged = a.tol_grad > 0.0 ? (s->grad_norm <= a.tol_grad) : (s->k < a.max_iter);
  out[0] = s->mu;
  out[1] = s->E_fin;
  out[2] = (double)s->k;
  out[3] = (double)s->converged;
  out[4] = s->grad_norm;
  out[5] = (double)switched_at;
  out[6] = 0.0;
  out[7] = 0.0;
}

// ---- whole-batch graph: device-side loop control (conditional WHILE nodes) ----
__global__ void k_cg_graph_begin(CgArgs a) { a.sc->switched_at = -1; }

// the condition of a loop over iterations: go on while the solve is active, its energy
// finite and its iteration count below the phase's limit (the host loop's tests)
__global__ void k_cg_graph_cond(cudaGraphConditionalHandle h, CgArgs a, int k_limit) {
  const CgScalars* s = a.sc;
  cudaGraphSetConditional(h, (s->active && isfinite(s->E) && s->k < k_limit) ? 1u : 0u);
}

// between the FP32 and the FP64 loops: the host driver's switch (CgSolver::advance)
__global__ void k_cg_graph_switch(CgArgs a) {
  CgScalars* s = a.sc;
  if (isfinite(s->E) && s->k < a.max_iter) {
    s->switched_at = s->k;
    s->k_base = s->k;
    s->active = 1;
  } else {
    s->active = 0;
  }
}

// ============================================================ host driver ===
struct CgLayout {
  size_t off[24];
  size_t total;
};

static size_t cg_layout(const hf_cg_problem& pb, size_t fock_ws, size_t red_ws, CgLayout& L) {
  const size_t nk = (size_t)pb.nk1 * pb.nk2, nb = pb.nb, nq = nk * nb * nb, nv = nk * nb;
  const size_t sizes[] = {
      nq * 16, nq * 16, nq * 16, nq * 16, nq * 16, nq * 16, nq * 16,  // Ft G0 G1 dQ Vd Fe Sigma
      nv * 8, nv * 8, nv * 8, nv * 8, nv * 8, nv * 8,                  // eps epsF gp0 gp1 dp lamd
      nk * 8,                                                          // w_norm
      nb * nb * 16,                                                    // H
      sizeof(CgScalars), 64,                                           // scalars, counter
      (size_t)148 * 16 * kMaxSums * 2 * 8,                             // partials
      fock_ws, red_ws};
  size_t o = 0;
  const int n = sizeof(sizes) / sizeof(sizes[0]);
  for (int i = 0; i < n; ++i) { L.off[i] = o; o += align_up(sizes[i], 256); }
  L.total = o;
  return o;
}

static int fock_ws_size(const hf_cg_problem& pb, unsigned fflags, size_t* out) {
  return hf_fock_workspace_size(HF_C128, fflags, pb.nk1, pb.nk2, pb.nb, out);
}

static unsigned fock_flags(const hf_cg_problem& pb, bool fp32) {
  unsigned f = pb.fock_flags & ~(unsigned)HF_FOCK_FFT_FP32;
  if (fp32) f |= HF_FOCK_FFT_FP32;
  return f;
}

struct CgRun {
  const hf_cg_problem* pb;
  const hf_cg_config* cf;
  CgArgs a;
  void* fock_ws;
  size_t fock_ws_bytes;
  void* red_ws;
  size_t red_ws_bytes;
  double2* Sigma;
  double2* H;
  int nblk;
};

static size_t smem_eig(int nb) { return (jacobi_smem_elems(nb) + 2 * (size_t)nb * nb) * sizeof(double2) * kSolverWarps; }

static int set_smem(const void* fn, size_t) { return allow_max_dynamic_smem(fn); }

static int cg_fock(CgRun& r, cudaStream_t s, bool fp32, const int* active) {
  const hf_cg_problem& pb = *r.pb;
  if (r.cf->fock_cb) {
    const int st = r.cf->fock_cb(r.cf->cb_user, s, r.a.P, r.Sigma, r.H, r.a.F);
    return st == HF_OK ? HF_OK : fail(st, "Fock-build callback failed");
  }
  return fock_build_internal(s, HF_C128, fock_flags(pb, fp32), pb.nk1, pb.nk2, pb.nb, r.a.P, pb.h, pb.VR,
                             pb.refP, pb.HH, pb.w2d, pb.n_contact, pb.contact_g, pb.contact_Oi, pb.contact_Oj,
                             r.Sigma, r.H, r.a.F, r.fock_ws, r.fock_ws_bytes, active);
}

static int cg_project(CgRun& r, cudaStream_t s) {
  if (!r.cf->project_cb) return HF_OK;
  const int st = r.cf->project_cb(r.cf->cb_user, s, r.a.P);
  return st == HF_OK ? HF_OK : fail(st, "projection callback failed");
}

static int cg_energy(CgRun& r, cudaStream_t s, double* out, const int* active) {
  const hf_cg_problem& pb = *r.pb;
  return energy_internal(s, HF_C128, pb.nk1, pb.nk2, pb.nb, r.a.P, pb.h, r.Sigma, r.H, 1, pb.w2d, out, r.red_ws,
                         r.red_ws_bytes, active);
}

static int cg_mu(CgRun& r, cudaStream_t s, int maxiter, const int* active) {
  const hf_cg_problem& pb = *r.pb;
  return find_mu_internal(s, HF_C128, 2, pb.nk1, pb.nk2, pb.nb, r.a.eps, r.a.w_norm, r.a.n_target_norm, r.a.T_r,
                          maxiter, &r.a.sc->mu, &r.a.sc->mu, active);
}

// Grid of an elementwise pass: a few elements per thread, at most 8 CTAs of 256 per SM.
static int elem_blocks(size_t n) {
  size_t b = (n + 4 * 256 - 1) / (4 * 256);
  if (b > (size_t)148 * 8) b = 148 * 8;
  return b < 1 ? 1 : (int)b;
}

// One iteration on the lane-per-row kernels (nb <= 8).
template <int NB>
static int cg_iteration_rows(CgRun& r, cudaStream_t s, const hf_cg_config& cf, bool fp32) {
  const int* act = &r.a.sc->active;
  const int rb = row_blocks(r.a.nk, RowGroup<NB>::KPW);
  const int eb = perk_blocks(r.a.nk);
  k_cgr_density<NB><<<rb, 32 * kRowWarps, 0, s>>>(r.a, 0);
  HF_LAUNCH_CHECK("k_cgr_density");
  int st = cg_project(r, s);
  if (st) return st;
  if ((st = cg_fock(r, s, fp32, act))) return st;
  if ((st = cg_energy(r, s, &r.a.sc->E, act))) return st;
  k_cgr_grad1<NB><<<rb, 32 * kRowWarps, 0, s>>>(r.a);
  HF_LAUNCH_CHECK("k_cgr_grad1");
  const int gb = elem_blocks((size_t)r.a.nk * NB * NB);
  k_cg_grad2_t<NB><<<gb, 256, 0, s>>>(r.a);
  HF_LAUNCH_CHECK("k_cg_grad2");
  k_cg_dir_t<NB><<<gb, 256, 0, s>>>(r.a);
  HF_LAUNCH_CHECK("k_cg_dir");
  const int bt = cf.bt_max;
  if (bt >= 1) {
    k_cgr_trials<NB, 1><<<rb, 32 * kRowWarps, 0, s>>>(r.a, 0, 1, bt == 1);
    HF_LAUNCH_CHECK("k_cgr_trials");
    for (int i0 = 1; i0 < bt; i0 += 8) {
      const int i1 = i0 + 8 < bt ? i0 + 8 : bt;
      k_cgr_trials<NB, 8><<<rb, 32 * kRowWarps, 0, s>>>(r.a, i0, i1, i1 == bt);
      HF_LAUNCH_CHECK("k_cgr_trials");
    }
  }
  k_cgr_update<NB><<<rb, 32 * kRowWarps, 0, s>>>(r.a);
  HF_LAUNCH_CHECK("k_cgr_update");
  if ((st = cg_mu(r, s, cf.mu_maxiter, act))) return st;
  k_cg_step_end<<<1, 1, 0, s>>>(r.a, fp32 ? cf.fp32_switch_rel : 0.0);
  HF_LAUNCH_CHECK("k_cg_step_end");
  return HF_OK;
}

template <int NB>
static int cg_density_rows(CgRun& r, cudaStream_t s, int force) {
  k_cgr_density<NB><<<row_blocks(r.a.nk, RowGroup<NB>::KPW), 32 * kRowWarps, 0, s>>>(r.a, force);
  HF_LAUNCH_CHECK("k_cgr_density");
  return HF_OK;
}

static int cg_density(CgRun& r, cudaStream_t s, int force) {
  switch (r.a.nb) {
#define HF_NB_CASE(N) case N: return cg_density_rows<N>(r, s, force);
    HF_NB_CASE(1) HF_NB_CASE(2) HF_NB_CASE(3) HF_NB_CASE(4) HF_NB_CASE(5) HF_NB_CASE(6) HF_NB_CASE(7) HF_NB_CASE(8)
#undef HF_NB_CASE
    default: break;
  }
  const int nb = r.a.nb, nb2 = nb * nb;
  k_cg_density<<<r.nblk, 32 * kSolverWarps, (2 * (size_t)nb2 + nb) * 16 * kSolverWarps, s>>>(r.a, force);
  HF_LAUNCH_CHECK("k_cg_density");
  return HF_OK;
}

template <int NB>
static int cg_eig_rows(CgRun& r, cudaStream_t s, const double2* A, int rotate) {
  const int per_block = kEigWarps * RowGroup<NB>::KPW;
  int b = (r.a.nk + per_block - 1) / per_block;
  if (b > 148 * 32) b = 148 * 32;
  k_cgr_eig<NB><<<b < 1 ? 1 : b, 32 * kEigWarps, 0, s>>>(r.a, A, rotate, kEigTol);
  HF_LAUNCH_CHECK("k_cgr_eig");
  return HF_OK;
}

// eps, Q <- eigh(A) (init) or eigh(Q^H F Q) with Q <- Q V (finalize)
static int cg_eig(CgRun& r, cudaStream_t s, const double2* A, int rotate) {
  switch (r.a.nb) {
#define HF_NB_CASE(N) case N: return cg_eig_rows<N>(r, s, A, rotate);
    HF_NB_CASE(1) HF_NB_CASE(2) HF_NB_CASE(3) HF_NB_CASE(4) HF_NB_CASE(5) HF_NB_CASE(6) HF_NB_CASE(7) HF_NB_CASE(8)
#undef HF_NB_CASE
    default: break;
  }
  const int nb = r.a.nb;
  k_cg_eig<<<r.nblk, 32 * kSolverWarps, smem_eig(nb), s>>>(r.a, A, rotate);
  HF_LAUNCH_CHECK("k_cg_eig");
  return HF_OK;
}

template <int NB>
static int rows_density_launch(cudaStream_t s, int nk, const double2* Q, const double* p, double2* P) {
  k_rows_density<NB><<<row_blocks(nk, RowGroup<NB>::KPW), 32 * kRowWarps, 0, s>>>(nk, Q, p, P);
  HF_LAUNCH_CHECK("k_rows_density");
  return HF_OK;
}

int rows_density(void* stream, int nk, int nb, const void* Q, const double* p, void* P) {
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  auto q = static_cast<const double2*>(Q);
  auto o = static_cast<double2*>(P);
  switch (nb) {
#define HF_NB_CASE(N) case N: return rows_density_launch<N>(s, nk, q, p, o);
    HF_NB_CASE(1) HF_NB_CASE(2) HF_NB_CASE(3) HF_NB_CASE(4) HF_NB_CASE(5) HF_NB_CASE(6) HF_NB_CASE(7) HF_NB_CASE(8)
#undef HF_NB_CASE
    default: break;
  }
  return fail(HF_ERR_UNSUPPORTED, "rows_density: nb > 8");
}

template <int NB>
static int eig_cols_launch(cudaStream_t s, int nk, const double2* A, const double2* Qin, double2* Qout,
                           double* eps, int mode = 0) {
  const int per_block = kEigWarps * RowGroup<NB>::KPW;
  int b = (nk + per_block - 1) / per_block;
  if (b > 148 * 32) b = 148 * 32;
  k_eig_cols<NB><<<b < 1 ? 1 : b, 32 * kEigWarps, 0, s>>>(nk, A, Qin, Qout, eps, kEigTol, mode);
  HF_LAUNCH_CHECK("k_eig_cols");
  return HF_OK;
}

// hf_eigh / hf_cayley_spectral for complex128 with nb <= 8 (perk.cu): the lane-per-column
// Jacobi from the identity; mode 1 decomposes herm(i A)
int eigh_cols(void* stream, int nk, int nb, const void* A, double* w, void* V, int mode) {
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  auto a = static_cast<const double2*>(A);
  auto v = static_cast<double2*>(V);
  switch (nb) {
#define HF_NB_CASE(N) case N: return eig_cols_launch<N>(s, nk, a, nullptr, v, w, mode);
    HF_NB_CASE(1) HF_NB_CASE(2) HF_NB_CASE(3) HF_NB_CASE(4) HF_NB_CASE(5) HF_NB_CASE(6) HF_NB_CASE(7) HF_NB_CASE(8)
#undef HF_NB_CASE
    default: break;
  }
  return fail(HF_ERR_UNSUPPORTED, "eigh_cols: nb > 8");
}

static int cg_iteration_warp(CgRun& r, cudaStream_t s, const hf_cg_config& cf, bool fp32);

static int cg_iteration(CgRun& r, cudaStream_t s, const hf_cg_config& cf, bool fp32) {
  switch (r.a.nb) {
#define HF_NB_CASE(N) case N: return cg_iteration_rows<N>(r, s, cf, fp32);
    HF_NB_CASE(1) HF_NB_CASE(2) HF_NB_CASE(3) HF_NB_CASE(4) HF_NB_CASE(5) HF_NB_CASE(6) HF_NB_CASE(7) HF_NB_CASE(8)
#undef HF_NB_CASE
    default: return cg_iteration_warp(r, s, cf, fp32);
  }
}

// One iteration on the warp-per-k kernels (9 <= nb <= 16; spectral Cayley).
static int cg_iteration_warp(CgRun& r, cudaStream_t s, const hf_cg_config& cf, bool fp32) {
  const double phase_rel = fp32 ? cf.fp32_switch_rel : 0.0;
  const int nb = r.pb->nb, nb2 = nb * nb;
  const int* act = &r.a.sc->active;
  const dim3 blk(32 * kSolverWarps);
  const size_t sm_den = (2 * (size_t)nb2 + nb) * 16 * kSolverWarps;
  k_cg_density<<<r.nblk, blk, sm_den, s>>>(r.a, 0);
  HF_LAUNCH_CHECK("k_cg_density");
  int st = cg_project(r, s);
  if (st) return st;
  st = cg_fock(r, s, fp32, act);
  if (st) return st;
  st = cg_energy(r, s, &r.a.sc->E, act);
  if (st) return st;
  const size_t sm_g1 = 3 * (size_t)nb2 * 16 * kSolverWarps;
  k_cg_grad1<<<r.nblk, blk, sm_g1, s>>>(r.a);
  HF_LAUNCH_CHECK("k_cg_grad1");
  k_cg_grad2<<<r.nblk, 256, 0, s>>>(r.a);
  HF_LAUNCH_CHECK("k_cg_grad2");
  k_cg_dir<<<r.nblk, blk, smem_eig(nb), s>>>(r.a);
  HF_LAUNCH_CHECK("k_cg_dir");
  const size_t sm_tr = (2 * (size_t)nb2 + nb) * 16 * kSolverWarps;
  const int bt = cf.bt_max;
  if (bt >= 1) {
    k_cg_trials<1><<<r.nblk, blk, sm_tr, s>>>(r.a, 0, 1, bt == 1);
    HF_LAUNCH_CHECK("k_cg_trials");
    for (int i0 = 1; i0 < bt; i0 += 8) {
      const int i1 = i0 + 8 < bt ? i0 + 8 : bt;
      k_cg_trials<8><<<r.nblk, blk, sm_tr, s>>>(r.a, i0, i1, i1 == bt);
      HF_LAUNCH_CHECK("k_cg_trials");
    }
  }
  const size_t sm_up = (4 * (size_t)nb2 + nb) * 16 * kSolverWarps;
  k_cg_update<<<r.nblk, blk, sm_up, s>>>(r.a);
  HF_LAUNCH_CHECK("k_cg_update");
  st = cg_mu(r, s, cf.mu_maxiter, act);
  if (st) return st;
  k_cg_step_end<<<1, 1, 0, s>>>(r.a, phase_rel);
  HF_LAUNCH_CHECK("k_cg_step_end");
  return HF_OK;
}

// ------------------------------------------------------------ one solve ---
// A solve as a host-side state machine over one stream: start() enqueues the
// init and the first chunk of iterations, each chunk ends with an async copy of
// the device scalars to `hs`; once that copy has landed, advance() enqueues the
// next chunk, the FP32 -> FP64 switch, or the finalize (which writes
// scalars_out on the device).  hf_cg_solve drives one of these with blocking
// waits; hf_cg_solve_batch drives many, one per stream, by polling events.
struct CgSolver {
  CgRun r{};
  CgLayout L{};
  const hf_cg_problem* pb = nullptr;
  const hf_cg_config* cf = nullptr;
  cudaStream_t s = nullptr;
  double* scalars_out = nullptr;
  CgScalars* hs = nullptr;
  bool graphs = false, fp32 = false, finalizing = false;
  int switched_at = -1, chunk = 4;
  cudaGraphExec_t exec[2] = {nullptr, nullptr};

  int setup(const hf_cg_problem* pb_, const hf_cg_config* cf_, void* Q, void* p, void* density, void* fock,
            double* hist_E, double* hist_grad, double* scalars_out_, void* workspace, cudaStream_t s_,
            CgScalars* host_slot);
  int init_ops(const void* P0);
  int finalize_ops(bool device_switch);
  int start(const void* P0);
  int launch_chunk();
  int advance(bool* finished);
  int launch_finalize();
  int get_exec(bool f32, cudaGraphExec_t* out);
  void release() {
    for (auto& e : exec)
      if (e) { cudaGraphExecDestroy(e); e = nullptr; }
  }
  ~CgSolver() { release(); }
};

static int cg_check(const hf_cg_problem* pb, const hf_cg_config* cf) {
  if (!pb || !cf) return fail(HF_ERR_INVALID, "NULL problem/config");
  if (pb->nk1 < 1 || pb->nk2 < 1 || pb->nb < 1) return fail(HF_ERR_INVALID, "bad shape");
  if (pb->nb > 16) return fail(HF_ERR_UNSUPPORTED, "the device CG solver supports nb <= 16");
  if (cf->max_iter < 0 || cf->bt_max < 0 || cf->cg_restart < 1)
    return fail(HF_ERR_INVALID, "bad solver configuration");
  return HF_OK;
}

}  // namespace hf

using namespace hf;

extern "C" int hf_cg_workspace_size(const hf_cg_problem* pb, const hf_cg_config* cf, size_t* bytes) {
  int st = cg_check(pb, cf);
  if (st) return st;
  size_t fws = 0, f2 = 0, rws = 0;
  if ((st = fock_ws_size(*pb, fock_flags(*pb, false), &fws))) return st;
  if ((st = fock_ws_size(*pb, fock_flags(*pb, true), &f2))) return st;
  if ((st = hf_reduce_workspace_size(pb->nk1, pb->nk2, pb->nb, &rws))) return st;
  CgLayout L;
  *bytes = cg_layout(*pb, fws > f2 ? fws : f2, rws, L) + (size_t)cf->max_iter * 16 + 256;
  return HF_OK;
}

namespace hf {

int CgSolver::setup(const hf_cg_problem* pb_, const hf_cg_config* cf_, void* Q, void* p, void* density,
                    void* fock, double* hist_E, double* hist_grad, double* scalars_out_, void* workspace,
                    cudaStream_t s_, CgScalars* host_slot) {
  pb = pb_;
  cf = cf_;
  s = s_;
  hs = host_slot;
  scalars_out = scalars_out_;
  size_t fws = 0, f2 = 0, rws = 0;
  int st;
  if ((st = fock_ws_size(*pb, fock_flags(*pb, false), &fws))) return st;
  if ((st = fock_ws_size(*pb, fock_flags(*pb, true), &f2))) return st;
  if ((st = hf_reduce_workspace_size(pb->nk1, pb->nk2, pb->nb, &rws))) return st;
  cg_layout(*pb, fws > f2 ? fws : f2, rws, L);
  char* ws = static_cast<char*>(workspace);
  r.pb = pb;
  r.cf = cf;
  CgArgs& a = r.a;
  a.nk = pb->nk1 * pb->nk2;
  a.nb = pb->nb;
  a.max_iter = cf->max_iter;
  a.cg_restart = cf->cg_restart;
  a.bt_max = cf->bt_max;
  a.plateau_window = cf->plateau_window;
  a.T_r = fmax(pb->T, 1e-12);
  a.tol_E = cf->tol_E;
  a.tol_grad = cf->tol_grad;
  a.denom_scale = cf->denom_scale;
  a.max_step = cf->max_step;
  a.bt_shrink = cf->bt_shrink;
  a.n_target_norm = pb->n_electrons / fmax(pb->weight_sum, 1e-30);
  a.Q = static_cast<double2*>(Q);
  a.P = static_cast<double2*>(density);
  a.F = static_cast<double2*>(fock);
  a.p = static_cast<double*>(p);
  a.Ft = reinterpret_cast<double2*>(ws + L.off[0]);
  a.G0 = reinterpret_cast<double2*>(ws + L.off[1]);
  a.G1 = reinterpret_cast<double2*>(ws + L.off[2]);
  a.dQ = reinterpret_cast<double2*>(ws + L.off[3]);
  a.Vd = reinterpret_cast<double2*>(ws + L.off[4]);
  a.Fe = reinterpret_cast<double2*>(ws + L.off[5]);
  r.Sigma = pb->sigma_buf ? static_cast<double2*>(pb->sigma_buf) : reinterpret_cast<double2*>(ws + L.off[6]);
  a.eps = reinterpret_cast<double*>(ws + L.off[7]);
  a.epsF = reinterpret_cast<double*>(ws + L.off[8]);
  a.gp0 = reinterpret_cast<double*>(ws + L.off[9]);
  a.gp1 = reinterpret_cast<double*>(ws + L.off[10]);
  a.dp = reinterpret_cast<double*>(ws + L.off[11]);
  a.lamd = reinterpret_cast<double*>(ws + L.off[12]);
  a.w_norm = reinterpret_cast<double*>(ws + L.off[13]);
  r.H = pb->h_buf ? static_cast<double2*>(pb->h_buf) : reinterpret_cast<double2*>(ws + L.off[14]);
  a.sc = reinterpret_cast<CgScalars*>(ws + L.off[15]);
  a.counter = reinterpret_cast<unsigned*>(ws + L.off[16]);
  a.part = reinterpret_cast<double*>(ws + L.off[17]);
  r.fock_ws = ws + L.off[18];
  r.fock_ws_bytes = fws > f2 ? fws : f2;
  r.red_ws = ws + L.off[19];
  r.red_ws_bytes = rws;
  a.hist_E = hist_E ? hist_E : reinterpret_cast<double*>(ws + L.total);
  a.hist_G = hist_grad ? hist_grad : reinterpret_cast<double*>(ws + L.total) + cf->max_iter;
  r.nblk = perk_blocks(a.nk);
  fp32 = cf->fp32_exchange != 0;
  chunk = cf->chunk > 0 ? cf->chunk : 4;
  graphs = cf->fock_cb == nullptr && cf->project_cb == nullptr && s != nullptr;
  const int nb = pb->nb, nb2 = nb * nb;
  if ((st = set_smem((const void*)k_cg_eig, smem_eig(nb)))) return st;
  if ((st = set_smem((const void*)k_cg_dir, smem_eig(nb)))) return st;
  if ((st = set_smem((const void*)k_cg_update, (4 * (size_t)nb2 + nb) * 16 * kSolverWarps))) return st;
  if ((st = set_smem((const void*)k_cg_grad1, 3 * (size_t)nb2 * 16 * kSolverWarps))) return st;
  return HF_OK;
}

int CgSolver::start(const void* P0) {
  const int st = init_ops(P0);
  if (st) return st;
  return cf->max_iter > 0 ? launch_chunk() : launch_finalize();
}

int CgSolver::init_ops(const void* P0) {
  CgArgs& a = r.a;
  const int nb = pb->nb, nb2 = nb * nb;
  int st;
  HF_CUDA(cudaMemsetAsync(r.H, 0, sizeof(double2) * nb2, s));  // H stays zero without Hartree
  if (cf->max_iter > 0) HF_CUDA(cudaMemsetAsync(a.hist_E, 0, sizeof(double) * cf->max_iter, s));
  if (cf->max_iter > 0) HF_CUDA(cudaMemsetAsync(a.hist_G, 0, sizeof(double) * cf->max_iter, s));
  // ---- init (solver.py:377-394) ----
  k_cg_init<<<r.nblk, 256, 0, s>>>(a, static_cast<const double2*>(P0), static_cast<const double*>(pb->w2d),
                                   pb->weight_sum);
  HF_LAUNCH_CHECK("k_cg_init");
  if ((st = cg_fock(r, s, false, nullptr))) return st;
  if ((st = cg_eig(r, s, a.F, 0))) return st;
  return cg_mu(r, s, cf->mu_maxiter, nullptr);
}

// One iteration captured into a CUDA graph per precision phase (no host
// callbacks); every kernel of it returns at once once the device stop flag is
// clear, so a chunk may overrun convergence at no cost.
int CgSolver::get_exec(bool f32, cudaGraphExec_t* out) {
  cudaGraphExec_t& e = exec[f32 ? 1 : 0];
  if (!e) {
    cudaGraph_t g = nullptr;
    HF_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    const int st2 = cg_iteration(r, s, *cf, f32);
    const cudaError_t ce = cudaStreamEndCapture(s, &g);
    if (st2 != HF_OK) {
      if (g) cudaGraphDestroy(g);
      return st2;
    }
    if (ce != cudaSuccess) return cuda_check(ce, "cudaStreamEndCapture");
    const cudaError_t ie = cudaGraphInstantiate(&e, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) return cuda_check(ie, "cudaGraphInstantiate");
  }
  *out = e;
  return HF_OK;
}

// ---- loop (solver.py:603-604): `chunk` iterations, then the scalars to the host ----
int CgSolver::launch_chunk() {
  int st;
  if (graphs) {
    cudaGraphExec_t e = nullptr;
    if ((st = get_exec(fp32, &e))) return st;
    for (int c = 0; c < chunk; ++c) HF_CUDA(cudaGraphLaunch(e, s));
  } else {
    for (int c = 0; c < chunk; ++c)
      if ((st = cg_iteration(r, s, *cf, fp32))) return st;
  }
  HF_CUDA(cudaMemcpyAsync(hs, r.a.sc, sizeof(CgScalars), cudaMemcpyDeviceToHost, s));
  return HF_OK;
}

int CgSolver::advance(bool* finished) {
  *finished = false;
  if (finalizing) {
    *finished = true;
    return HF_OK;
  }
  const int host_k = hs->k;
  int host_active = hs->active;
  if (!std::isfinite(hs->E)) {
    host_active = 0;
  } else if (fp32 && host_k < cf->max_iter && (!host_active || host_k >= cf->max_iter / 2)) {
    // mixed precision: FP32 exchange until the windowed energy change reaches the FP32
    // noise floor (or half the iteration budget), then FP64 defect-correction builds
    // continue from the same state to the requested tolerance.
    fp32 = false;
    switched_at = host_k;
    k_cg_rearm<<<1, 1, 0, s>>>(r.a);
    HF_LAUNCH_CHECK("k_cg_rearm");
    host_active = 1;
  }
  return host_active ? launch_chunk() : launch_finalize();
}

// ---- finalize (solver.py:613-648) ----
int CgSolver::launch_finalize() {
  finalizing = true;
  const int st = finalize_ops(false);
  if (st) return st;
  HF_CUDA(cudaMemcpyAsync(hs, r.a.sc, sizeof(CgScalars), cudaMemcpyDeviceToHost, s));
  return HF_OK;
}

int CgSolver::finalize_ops(bool device_switch) {
  CgArgs& a = r.a;
  int st;
  if ((st = cg_density(r, s, 1))) return st;
  if ((st = cg_project(r, s))) return st;
  if ((st = cg_fock(r, s, false, nullptr))) return st;
  if ((st = cg_eig(r, s, a.F, 1))) return st;  // reads the current Q, writes the caller's buffer
  k_cg_qsel_reset<<<1, 1, 0, s>>>(a);
  HF_LAUNCH_CHECK("k_cg_qsel_reset");
  if ((st = cg_mu(r, s, cf->mu_maxiter, nullptr))) return st;
  if ((st = cg_density(r, s, 1))) return st;
  if ((st = cg_project(r, s))) return st;
  if ((st = cg_fock(r, s, false, nullptr))) return st;
  if ((st = cg_energy(r, s, &a.sc->E_fin, nullptr))) return st;
  k_cg_converged<<<1, 1, 0, s>>>(a, device_switch ? -2 : switched_at, scalars_out);
  HF_LAUNCH_CHECK("k_cg_converged");
  return HF_OK;
}

// A non-blocking stream that starts after `user` and that `user` waits for at
// the end (legacy default streams cannot be captured).
struct LaneStream {
  cudaStream_t s = nullptr;
  cudaEvent_t ev = nullptr;
  int open(cudaStream_t user) {
    HF_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    HF_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    HF_CUDA(cudaEventRecord(ev, user));
    HF_CUDA(cudaStreamWaitEvent(s, ev, 0));
    return HF_OK;
  }
  int join(cudaStream_t user) {
    HF_CUDA(cudaEventRecord(ev, s));
    HF_CUDA(cudaStreamWaitEvent(user, ev, 0));
    return HF_OK;
  }
  ~LaneStream() {
    if (s) {
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
    if (ev) cudaEventDestroy(ev);
  }
};

}  // namespace hf

extern "C" int hf_cg_solve(void* stream, const hf_cg_problem* pb, const hf_cg_config* cf, const void* P0,
                           void* Q, void* p, void* density, void* fock, double* hist_E, double* hist_grad,
                           double* scalars_out, void* workspace, size_t workspace_bytes) {
  int st = cg_check(pb, cf);
  if (st) return st;
  if (!P0 || !Q || !p || !density || !fock || !scalars_out || !workspace)
    return fail(HF_ERR_INVALID, "NULL argument");
  size_t need = 0;
  if ((st = hf_cg_workspace_size(pb, cf, &need))) return st;
  if (workspace_bytes < need) return fail(HF_ERR_WORKSPACE, "CG workspace too small: need " + std::to_string(need));
  cudaStream_t user = static_cast<cudaStream_t>(stream);
  // host callbacks enqueue on the caller's stream; otherwise a private stream
  // (capturable) ordered after it
  const bool callbacks = cf->fock_cb != nullptr || cf->project_cb != nullptr;
  LaneStream lane;
  if (!callbacks && (st = lane.open(user))) return st;
  const cudaStream_t s = callbacks ? user : lane.s;
  CgScalars hs{};
  CgSolver sv;
  if ((st = sv.setup(pb, cf, Q, p, density, fock, hist_E, hist_grad, scalars_out, workspace, s, &hs))) return st;
  if ((st = sv.start(P0))) return st;
  bool finished = false;
  while (!finished) {
    HF_CUDA(cudaStreamSynchronize(s));
    if ((st = sv.advance(&finished))) return st;
  }
  return callbacks ? HF_OK : lane.join(user);
}

extern "C" int hf_cg_batch_workspace_size(const hf_cg_batch_item* items, int n_items, const hf_cg_config* cf,
                                          size_t* bytes_per_lane) {
  if (!items || n_items < 1 || !cf || !bytes_per_lane) return fail(HF_ERR_INVALID, "bad batch arguments");
  size_t mx = 0;
  for (int i = 0; i < n_items; ++i) {
    size_t b = 0;
    const int st = hf_cg_workspace_size(&items[i].problem, cf, &b);
    if (st) return st;
    mx = b > mx ? b : mx;
  }
  *bytes_per_lane = align_up(mx, 256);  // every lane's workspace starts 256-byte aligned
  return HF_OK;
}

extern "C" int hf_cg_solve_batch(void* stream, const hf_cg_batch_item* items, int n_items, const hf_cg_config* cf,
                                 int n_lanes, void* workspace, size_t bytes_per_lane, double* solve_ms) {
  if (!items || n_items < 1 || !cf || !workspace || n_lanes < 1) return fail(HF_ERR_INVALID, "bad batch arguments");
  if (cf->fock_cb || cf->project_cb) return fail(HF_ERR_INVALID, "the batched CG driver takes no host callbacks");
  size_t need = 0;
  int st = hf_cg_batch_workspace_size(items, n_items, cf, &need);
  if (st) return st;
  if (bytes_per_lane < need) return fail(HF_ERR_WORKSPACE, "CG batch workspace too small: need " + std::to_string(need) + " per lane");
  for (int i = 0; i < n_items; ++i) {
    const hf_cg_batch_item& it = items[i];
    if (!it.P0 || !it.Q || !it.p || !it.density || !it.fock || !it.scalars_out)
      return fail(HF_ERR_INVALID, "NULL argument in batch item " + std::to_string(i));
  }
  if (n_lanes > n_items) n_lanes = n_items;
  cudaStream_t user = static_cast<cudaStream_t>(stream);

  // longest first (per-k work ~ nk nb^3, FFT ~ nk nb^2 log nk): a greedy list schedule
  std::vector<int> order(n_items);
  for (int i = 0; i < n_items; ++i) order[i] = i;
  auto cost = [&](int i) {
    const hf_cg_problem& q = items[i].problem;
    return (double)q.nk1 * q.nk2 * q.nb * q.nb * (q.nb + 8.0);
  };
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cost(x) > cost(y); });

  CgScalars* hslots = nullptr;
  HF_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&hslots), sizeof(CgScalars) * n_lanes, cudaHostAllocDefault));
  struct Lane {
    LaneStream ls;
    cudaEvent_t ready = nullptr, t0 = nullptr, t1 = nullptr;
    CgSolver* sv = nullptr;
    int item = -1;
  };
  std::vector<Lane> lanes(n_lanes);
  auto cleanup = [&]() {
    for (auto& l : lanes) {
      if (l.ls.s) cudaStreamSynchronize(l.ls.s);
      delete l.sv;
      l.sv = nullptr;
      if (l.ready) cudaEventDestroy(l.ready);
      if (l.t0) cudaEventDestroy(l.t0);
      if (l.t1) cudaEventDestroy(l.t1);
      l.ready = l.t0 = l.t1 = nullptr;
    }
    cudaFreeHost(hslots);
  };
  auto run = [&]() -> int {
    for (auto& l : lanes) {
      int e;
      if ((e = l.ls.open(user))) return e;
      HF_CUDA(cudaEventCreateWithFlags(&l.ready, cudaEventDisableTiming));
      HF_CUDA(cudaEventCreate(&l.t0));
      HF_CUDA(cudaEventCreate(&l.t1));
    }
    int next = 0, busy = 0;
    for (;;) {
      bool progressed = false;
      for (int li = 0; li < n_lanes; ++li) {
        Lane& l = lanes[li];
        char* ws = static_cast<char*>(workspace) + (size_t)li * bytes_per_lane;
        if (!l.sv) {
          if (next >= n_items) continue;
          const int i = order[next++];
          const hf_cg_batch_item& it = items[i];
          l.sv = new CgSolver();
          l.item = i;
          int e;
          if ((e = l.sv->setup(&it.problem, cf, it.Q, it.p, it.density, it.fock, it.hist_E, it.hist_grad,
                               it.scalars_out, ws, l.ls.s, &hslots[li])))
            return e;
          HF_CUDA(cudaEventRecord(l.t0, l.ls.s));
          if ((e = l.sv->start(it.P0))) return e;
          HF_CUDA(cudaEventRecord(l.ready, l.ls.s));
          ++busy;
          progressed = true;
          continue;
        }
        const cudaError_t q = cudaEventQuery(l.ready);
        if (q == cudaErrorNotReady) continue;
        if (q != cudaSuccess) return cuda_check(q, "cudaEventQuery");
        bool finished = false;
        int e;
        if ((e = l.sv->advance(&finished))) return e;
        if (finished) {
          HF_CUDA(cudaEventRecord(l.t1, l.ls.s));
          if (solve_ms) {
            HF_CUDA(cudaEventSynchronize(l.t1));
            float ms = 0.f;
            HF_CUDA(cudaEventElapsedTime(&ms, l.t0, l.t1));
            solve_ms[l.item] = ms;
          }
          delete l.sv;
          l.sv = nullptr;
          l.item = -1;
          --busy;
        } else {
          HF_CUDA(cudaEventRecord(l.ready, l.ls.s));
        }
        progressed = true;
      }
      if (busy == 0 && next >= n_items) break;
      if (!progressed) std::this_thread::yield();
    }
    for (auto& l : lanes) {
      int e;
      if ((e = l.ls.join(user))) return e;
    }
    return HF_OK;
  };
  st = run();
  cleanup();
  return st;
}

// Eigendecomposition of nk Hermitian nb x nb matrices (nb <= 8) by the lane-per-column
// cyclic Jacobi of the CG driver, optionally from a starting basis (see the header).
extern "C" int hf_eigh_warm(void* stream, int nk, int nb, const void* A, const void* Qin, void* Qout, void* eps) {
  if (nk < 1 || nb < 1 || nb > 8) return fail(HF_ERR_UNSUPPORTED, "hf_eigh_warm: needs nk >= 1 and 1 <= nb <= 8");
  if (!A || !Qout || !eps) return fail(HF_ERR_INVALID, "hf_eigh_warm: NULL argument");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const double2* a = static_cast<const double2*>(A);
  const double2* qi = static_cast<const double2*>(Qin);
  double2* qo = static_cast<double2*>(Qout);
  double* e = static_cast<double*>(eps);
  switch (nb) {
#define HF_NB_CASE(N) case N: return eig_cols_launch<N>(s, nk, a, qi, qo, e);
    HF_NB_CASE(1) HF_NB_CASE(2) HF_NB_CASE(3) HF_NB_CASE(4) HF_NB_CASE(5) HF_NB_CASE(6) HF_NB_CASE(7) HF_NB_CASE(8)
#undef HF_NB_CASE
    default: break;
  }
  return fail(HF_ERR_UNSUPPORTED, "hf_eigh_warm: nb > 8");
}

// The whole batch as ONE CUDA graph: every solve is an independent branch
//   init -> [WHILE: FP32 iteration] -> [switch] -> WHILE: FP64 iteration -> finalize
// whose loops are conditional WHILE nodes: the last kernel of an iteration body sets
// the loop's condition on the device (k_cg_graph_cond), so no host round trip happens
// between the launch and the end of the last solve.  Each solve has its own workspace
// (bytes_per_item from hf_cg_batch_workspace_size, n_items of them back to back), so
// all solves may run at once; the GPU interleaves the branches' kernels.  Per-solve
// times come from event nodes at each branch's ends.  Loop tests run after every
// iteration (the stream driver tests every `chunk` iterations), so a solve whose FP32
// phase ends at the half-budget limit may switch a few iterations earlier than there.
// The graph reads P0 and writes the outputs through the items' pointers, so a built
// batch can be launched again after new starting densities are written to the P0s.
struct CgBatchGraph {
  int n = 0;
  cudaGraph_t G = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t run = nullptr;  // the stream the graph runs on, ordered after the caller's
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  std::vector<cudaEvent_t> t0, t1;
  ~CgBatchGraph() {
    if (run) cudaStreamSynchronize(run);  // never free a graph that may still run
    if (exec) cudaGraphExecDestroy(exec);
    if (run) cudaStreamDestroy(run);
    if (ev_in) cudaEventDestroy(ev_in);
    if (ev_out) cudaEventDestroy(ev_out);
    if (G) cudaGraphDestroy(G);
    for (auto e : t0)
      if (e) cudaEventDestroy(e);
    for (auto e : t1)
      if (e) cudaEventDestroy(e);
  }
};

extern "C" int hf_cg_batch_graph_create(const hf_cg_batch_item* items, int n_items, const hf_cg_config* cf,
                                        void* workspace, size_t bytes_per_item, void** handle) {
  if (!items || n_items < 1 || !cf || !workspace || !handle) return fail(HF_ERR_INVALID, "bad batch arguments");
  *handle = nullptr;
  if (cf->fock_cb || cf->project_cb) return fail(HF_ERR_INVALID, "the batched CG driver takes no host callbacks");
  size_t need = 0;
  int st = hf_cg_batch_workspace_size(items, n_items, cf, &need);
  if (st) return st;
  if (bytes_per_item < need)
    return fail(HF_ERR_WORKSPACE, "CG batch workspace too small: need " + std::to_string(need) + " per solve");
  for (int i = 0; i < n_items; ++i) {
    const hf_cg_batch_item& it = items[i];
    if (!it.P0 || !it.Q || !it.p || !it.density || !it.fock || !it.scalars_out)
      return fail(HF_ERR_INVALID, "NULL argument in batch item " + std::to_string(i));
  }
  auto* bg = new CgBatchGraph();
  bg->n = n_items;
  bg->t0.assign(n_items, nullptr);
  bg->t1.assign(n_items, nullptr);
  cudaStream_t cap = nullptr;
  CgScalars unused{};
  auto capture_into = [&](cudaGraph_t g, const std::vector<cudaGraphNode_t>& deps) -> int {
    HF_CUDA(cudaStreamBeginCaptureToGraph(cap, g, deps.empty() ? nullptr : deps.data(), nullptr, deps.size(),
                                          cudaStreamCaptureModeThreadLocal));
    return HF_OK;
  };
  // ends a capture and returns its terminal nodes (the next stage's dependencies)
  auto end_capture = [&](std::vector<cudaGraphNode_t>* tail) -> int {
    if (tail) {
      cudaStreamCaptureStatus cs;
      const cudaGraphNode_t* d = nullptr;
      size_t nd = 0;
      HF_CUDA(cudaStreamGetCaptureInfo(cap, &cs, nullptr, nullptr, &d, &nd));
      tail->assign(d, d + nd);
    }
    cudaGraph_t g = nullptr;
    HF_CUDA(cudaStreamEndCapture(cap, &g));
    return HF_OK;
  };
  auto build = [&]() -> int {
    int e;
    HF_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    HF_CUDA(cudaGraphCreate(&bg->G, 0));
    cudaGraph_t G = bg->G;
    for (int i = 0; i < n_items; ++i) {
      const hf_cg_batch_item& it = items[i];
      CgSolver v;
      char* ws = static_cast<char*>(workspace) + (size_t)i * bytes_per_item;
      if ((e = v.setup(&it.problem, cf, it.Q, it.p, it.density, it.fock, it.hist_E, it.hist_grad, it.scalars_out,
                       ws, cap, &unused)))
        return e;
      HF_CUDA(cudaEventCreate(&bg->t0[i]));
      HF_CUDA(cudaEventCreate(&bg->t1[i]));
      std::vector<cudaGraphNode_t> tail;
      // init
      if ((e = capture_into(G, tail))) return e;
      HF_CUDA(cudaEventRecordWithFlags(bg->t0[i], cap, cudaEventRecordExternal));
      k_cg_graph_begin<<<1, 1, 0, cap>>>(v.r.a);
      HF_LAUNCH_CHECK("k_cg_graph_begin");
      if ((e = v.init_ops(it.P0))) return e;
      if ((e = end_capture(&tail))) return e;
      // iteration loops
      if (cf->max_iter > 0) {
        const bool mixed = cf->fp32_exchange != 0;
        for (int phase = mixed ? 0 : 1; phase < 2; ++phase) {
          const bool f32 = phase == 0;
          if (mixed && !f32) {  // the FP32 -> FP64 switch between the two loops
            if ((e = capture_into(G, tail))) return e;
            k_cg_graph_switch<<<1, 1, 0, cap>>>(v.r.a);
            HF_LAUNCH_CHECK("k_cg_graph_switch");
            if ((e = end_capture(&tail))) return e;
          }
          cudaGraphConditionalHandle h;
          HF_CUDA(cudaGraphConditionalHandleCreate(&h, G, 1u, cudaGraphCondAssignDefault));
          cudaGraphNodeParams np = {};
          np.type = cudaGraphNodeTypeConditional;
          np.conditional.handle = h;
          np.conditional.type = cudaGraphCondTypeWhile;
          np.conditional.size = 1;
          cudaGraphNode_t loop = nullptr;
          HF_CUDA(cudaGraphAddNode(&loop, G, tail.empty() ? nullptr : tail.data(), tail.size(), &np));
          cudaGraph_t body = np.conditional.phGraph_out[0];
          if ((e = capture_into(body, {}))) return e;
          if ((e = cg_iteration(v.r, cap, *cf, f32))) return e;
          k_cg_graph_cond<<<1, 1, 0, cap>>>(h, v.r.a, f32 ? cf->max_iter / 2 : cf->max_iter);
          HF_LAUNCH_CHECK("k_cg_graph_cond");
          if ((e = end_capture(nullptr))) return e;
          tail.assign(1, loop);
        }
      }
      // finalize
      if ((e = capture_into(G, tail))) return e;
      if ((e = v.finalize_ops(true))) return e;
      HF_CUDA(cudaEventRecordWithFlags(bg->t1[i], cap, cudaEventRecordExternal));
      if ((e = end_capture(nullptr))) return e;
    }
    HF_CUDA(cudaGraphInstantiate(&bg->exec, G, 0));
    HF_CUDA(cudaStreamCreateWithFlags(&bg->run, cudaStreamNonBlocking));
    HF_CUDA(cudaEventCreateWithFlags(&bg->ev_in, cudaEventDisableTiming));
    HF_CUDA(cudaEventCreateWithFlags(&bg->ev_out, cudaEventDisableTiming));
    return HF_OK;
  };
  st = build();
  if (cap) {
    if (st != HF_OK) {  // leave no capture open on an error path
      cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
      if (cudaStreamIsCapturing(cap, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(cap, &g);
      }
      cudaGetLastError();
    }
    cudaStreamDestroy(cap);
  }
  if (st != HF_OK) {
    delete bg;
    return st;
  }
  *handle = bg;
  return HF_OK;
}

// Runs a built batch after the work already queued on `stream` and makes `stream` wait
// for it; with solve_ms (n_items entries) it waits for the batch and fills each solve's
// device time from its start to its final scalars.
extern "C" int hf_cg_batch_graph_launch(void* handle, void* stream, double* solve_ms) {
  if (!handle) return fail(HF_ERR_INVALID, "NULL batch graph");
  auto* bg = static_cast<CgBatchGraph*>(handle);
  cudaStream_t user = static_cast<cudaStream_t>(stream);
  HF_CUDA(cudaEventRecord(bg->ev_in, user));
  HF_CUDA(cudaStreamWaitEvent(bg->run, bg->ev_in, 0));
  HF_CUDA(cudaGraphLaunch(bg->exec, bg->run));
  HF_CUDA(cudaEventRecord(bg->ev_out, bg->run));
  HF_CUDA(cudaStreamWaitEvent(user, bg->ev_out, 0));
  if (solve_ms) {
    HF_CUDA(cudaStreamSynchronize(bg->run));
    for (int i = 0; i < bg->n; ++i) {
      float ms = 0.f;
      HF_CUDA(cudaEventElapsedTime(&ms, bg->t0[i], bg->t1[i]));
      solve_ms[i] = ms;
    }
  }
  return HF_OK;
}

extern "C" int hf_cg_batch_graph_destroy(void* handle) {
  delete static_cast<CgBatchGraph*>(handle);
  return HF_OK;
}

extern "C" int hf_cg_solve_batch_graph(void* stream, const hf_cg_batch_item* items, int n_items,
                                       const hf_cg_config* cf, void* workspace, size_t bytes_per_item,
                                       double* solve_ms) {
  void* h = nullptr;
  int st = hf_cg_batch_graph_create(items, n_items, cf, workspace, bytes_per_item, &h);
  if (st) return st;
  st = hf_cg_batch_graph_launch(h, stream, solve_ms);
  if (st == HF_OK && !solve_ms) {
    const cudaError_t e = cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) st = cuda_check(e, "cudaStreamSynchronize");
  }
  hf_cg_batch_graph_destroy(h);
  return st;
}
