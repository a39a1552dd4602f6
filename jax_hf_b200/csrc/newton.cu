// Native trust-region Newton driver (solver.py:686-1078, optimizer="newton"; with
// project_fn=None, block_sizes=None and the built-in Fock build), complex128.
//
// Steihaug truncated CG on the joint (Q, p) Hessian; every Hessian-vector product
// is a Fock build of the linear response (refP = 0) between hf_newton_dP and
// hf_newton_hvp.  All vectors stay on the device.  The host keeps the scalar
// logic of the reference loop body (trust-region ratio, boundary step, CG
// stopping tests) and reads the reductions it needs in batches: each inner CG
// step makes two reads (d.Hd, d.d, v.d, v.v after the product; |v + a d|^2,
// |r - a Hd|^2 and r.z after the update), the outer step one for the
// preconditioner scale, one for the model terms and one (two with deflation) for
// the trial state.  Every reduction is the same device operation that the Python
// loop over the library (newton.py) calls, in the same order, so the two drivers
// take the same steps.
#include <cmath>
#include <cstring>
#include <utility>
#include <vector>

#include "common.cuh"

namespace hf {
namespace {

// complex (nk nb^2), real (nk nb) and other buffers of the workspace
enum {
  cP, cSG, cF, cFR, cDP, cG, cGT, cFT0, cFT1, cQ0, cQ1, cRX0, cRX1, cZX, cVX0, cVX1, cHVX, cDX, cHDX, cVV, cU,
  cFTF, cDIFF, cSPEN, rP0, rP1, rEPS, rEPST, rRP0, rRP1, rZP, rVP0, rVP1, rHVP, rDP, rHDP, rLAM, oH, oWN, oSCAL,
  oFOCKWS, oREDWS, oOPSWS, kNewtonBufs
};
constexpr int kFirstReal = rP0, kFirstOther = oH;

// device scalars: E, |G|^2, mu, trial mu, mu seed, wsum, dots[8], deflation distances[n]
constexpr int sE = 0, sG2 = 1, sMu = 2, sMuT = 3, sMu0 = 4, sWsum = 5, sDot = 6, sD2 = 14;

struct NewtonLayout {
  size_t off[kNewtonBufs];
  size_t total;
};

unsigned response_flags(unsigned f) { return f & ~(unsigned)HF_FOCK_HAS_REFP; }

size_t newton_layout(const hf_cg_problem& pb, const hf_newton_config& cf, size_t fock_ws, size_t red_ws,
                     size_t ops_ws, NewtonLayout& L) {
  const size_t nk = (size_t)pb.nk1 * pb.nk2, nb = pb.nb, nq = nk * nb * nb, nv = nk * nb;
  size_t o = 0;
  for (int i = 0; i < kNewtonBufs; ++i) {
    size_t sz = 256;
    if (i < kFirstReal) sz = nq * 16;
    else if (i < kFirstOther) sz = nv * 8;
    else if (i == oH) sz = nb * nb * 16;
    else if (i == oWN) sz = nk * 8;
    else if (i == oSCAL) sz = (size_t)(sD2 + (cf.n_deflation > 0 ? cf.n_deflation : 0) + 2) * 8;
    else if (i == oFOCKWS) sz = fock_ws;
    else if (i == oREDWS) sz = red_ws;
    else if (i == oOPSWS) sz = ops_ws;
    L.off[i] = o;
    o += align_up(sz > 0 ? sz : 256, 256);
  }
  L.total = o;
  return o;
}

struct Newton {
  cudaStream_t s;
  const hf_cg_problem* pb;
  const hf_newton_config* cf;
  unsigned char* base;
  NewtonLayout L;
  size_t fock_ws, red_ws;
  int nk, nb;
  size_t nq, nv;
  double T_r, tol_g, n_target_norm, occ_den;
  bool defl;
  double inv2L2, dsig;
  int n_builds = 0;

  template <typename T>
  T* at(int i) const { return reinterpret_cast<T*>(base + L.off[i]); }
  double* sc() const { return at<double>(oSCAL); }
  void* ops() const { return at<void>(oOPSWS); }
  const double* w2d() const { return static_cast<const double*>(pb->w2d); }

  int read(double* host, const double* dev, int n) {
    HF_CUDA(cudaMemcpyAsync(host, dev, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    HF_CUDA(cudaStreamSynchronize(s));
    return HF_OK;
  }
  // fock_full: the kernel's own build (refP included); fock_response: refP = 0
  int fock(const void* P, void* F, bool response) {
    ++n_builds;
    const unsigned flags = response ? response_flags(pb->fock_flags) : pb->fock_flags;
    return hf_fock_build(s, HF_C128, flags, pb->nk1, pb->nk2, nb, P, pb->h, pb->VR, response ? nullptr : pb->refP,
                         pb->HH, pb->w2d, pb->n_contact, pb->contact_g, pb->contact_Oi, pb->contact_Oj,
                         at<void>(cSG), at<void>(oH), F, at<void>(oFOCKWS), fock_ws);
  }
  // ip_matrix(aX, bX, ones) + ip_vec(ap, bp, w2d)  (solver.py:783-784)
  int jip(const void* aX, const double* ap, const void* bX, const double* bp, double* out) {
    return hf_jdot(s, (size_t)nk, nb, aX, bX, nullptr, ap, bp, w2d(), out, ops());
  }
  // n of them in one pass, each equal to jip's
  int jip_multi(int n, const void* const* aX, const double* const* ap, const void* const* bX,
                const double* const* bp, double* out) {
    const double* wx[4] = {nullptr, nullptr, nullptr, nullptr};
    const double* wp[4] = {w2d(), w2d(), w2d(), w2d()};
    return jdot_multi(s, (size_t)nk, nb, n, aX, bX, wx, ap, bp, wp, out, ops());
  }
  // solver._solve_mu (solver.py:62-101) from the device seed mu0
  int solve_mu(const double* eps, const double* mu0, double* mu_out) {
    return hf_find_mu(s, HF_C128, 2, nk, 1, nb, eps, at<double>(oWN), n_target_norm, T_r, cf->mu_maxiter, mu0,
                      mu_out);
  }
  int occupations(const double* eps, const double* mu, double* p) {
    return hf_fermi(s, nv, eps, mu, T_r, 1, 0.0, p);
  }
  // z = M^-1 r with the occupation block projected (solver.py:907-913, 224-233)
  int prec(const void* rX, const double* rp, const double* eps, const double* p, double lam, void* zX, double* zp) {
    int st;
    if ((st = hf_newton_prec(s, (size_t)nk, nb, rX, rp, eps, p, lam, T_r, kOccClip, w2d(), zX, zp, sc() + sWsum,
                             ops())))
      return st;
    return hf_sub_scalar(s, nv, zp, sc() + sWsum, 1.0 / occ_den);
  }
  // joint Hessian-vector product (solver.py:916-930)
  int hvp(const void* Q, const void* Ft, const double* p, const void* X, const double* dp, double pen, void* HX,
          double* Hp) {
    int st;
    if ((st = hf_newton_dP(s, nk, nb, Q, X, dp, p, at<void>(cDP)))) return st;
    if ((st = fock(at<void>(cDP), at<void>(cFR), true))) return st;
    if ((st = hf_newton_hvp(s, nk, nb, Q, Ft, X, dp, p, at<void>(cFR), pb->h, T_r, kOccClip, defl ? pen : 0.0,
                            defl ? at<void>(cDP) : nullptr, HX, Hp, w2d(), sc() + sWsum, ops())))
      return st;
    return hf_sub_scalar(s, nv, Hp, sc() + sWsum, 1.0 / occ_den);
  }
  const void* target(int i) const {
    return static_cast<const unsigned char*>(cf->deflation_targets) + (size_t)i * nq * 16;
  }
  // state at (Q, p) (solver.py:814-837): density, Fock build, energy, deflation bias,
  // Ft = Q^H F Q and |G| under the normalised weights
  int eval_state(const void* Q, const double* p, void* Ft, double* E, double* g, double* pen) {
    int st;
    void* P = at<void>(cP);
    void* F = at<void>(cF);
    if ((st = hf_density_from_Qp(s, HF_C128, nk, nb, Q, p, P))) return st;
    if ((st = fock(P, F, false))) return st;
    if ((st = hf_energy(s, HF_C128, pb->nk1, pb->nk2, nb, P, pb->h, at<void>(cSG), at<void>(oH), 1, pb->w2d,
                        sc() + sE, at<void>(oREDWS), red_ws)))
      return st;
    double Phi = 0.0, pn = 0.0;
    if (defl) {  // Gaussian bias of solver.py:804-812, targets in order
      const int n = cf->n_deflation;
      for (int i = 0; i < n; ++i) {
        if ((st = hf_axpby(s, (size_t)nk, nb, 1.0, P, -1.0, target(i), 0, at<void>(cDIFF)))) return st;
        if ((st = hf_jdot(s, (size_t)nk, nb, at<void>(cDIFF), at<void>(cDIFF), w2d(), nullptr, nullptr, nullptr,
                          sc() + sD2 + i, ops())))
          return st;
      }
      std::vector<double> d2(n);
      if ((st = read(d2.data(), sc() + sD2, n))) return st;
      HF_CUDA(cudaMemsetAsync(at<void>(cSPEN), 0, nq * 16, s));
      for (int i = 0; i < n; ++i) {
        const double phi = dsig * std::exp(-d2[i] * inv2L2);
        const double phip = -phi * inv2L2;
        if ((st = hf_axpby(s, (size_t)nk, nb, 1.0, P, -1.0, target(i), 0, at<void>(cDIFF)))) return st;
        if ((st = hf_axpby(s, (size_t)nk, nb, 2.0 * phip, at<void>(cDIFF), 1.0, at<void>(cSPEN), 0,
                           at<void>(cSPEN))))
          return st;
        Phi += phi;
        pn += 2.0 * phip;
      }
      if ((st = hf_axpby(s, (size_t)nk, nb, 1.0, F, 1.0, at<void>(cSPEN), 0, F))) return st;
    }
    if ((st = hf_fock_orbital(s, HF_C128, nk, nb, Q, F, Ft))) return st;
    if ((st = hf_orbital_grad(s, (size_t)nk, nb, Ft, p, at<void>(cGT), nullptr))) return st;
    if ((st = hf_jdot(s, (size_t)nk, nb, at<void>(cGT), at<void>(cGT), at<double>(oWN), nullptr, nullptr, nullptr,
                      sc() + sG2, ops())))
      return st;
    double v[2];
    if ((st = read(v, sc() + sE, 2))) return st;
    *E = v[0] + (defl ? Phi : 0.0);
    *g = std::sqrt(std::fmax(0.0, v[1]));
    *pen = pn;
    return HF_OK;
  }

  static constexpr double kOccClip = 1e-8;
};

}  // namespace
}  // namespace hf

using namespace hf;

static int newton_check(const hf_cg_problem* pb, const hf_newton_config* cf) {
  if (!pb || !cf) return fail(HF_ERR_INVALID, "hf_newton: null problem or config");
  if (pb->nk1 < 1 || pb->nk2 < 1 || pb->nb < 1 || pb->nb > 16)
    return fail(HF_ERR_INVALID, "hf_newton: bad mesh or band count (nb <= 16)");
  if (cf->max_iter < 0) return fail(HF_ERR_INVALID, "max_iter must be non-negative");
  if (cf->tr_cg_max < 0) return fail(HF_ERR_INVALID, "tr_cg_max must be non-negative");
  if (cf->n_deflation < 0 || (cf->n_deflation > 0 && !cf->deflation_targets))
    return fail(HF_ERR_INVALID, "hf_newton: deflation targets missing");
  if (cf->n_deflation > 64) return fail(HF_ERR_UNSUPPORTED, "hf_newton: more than 64 deflation targets");
  return HF_OK;
}

static int newton_sizes(const hf_cg_problem* pb, size_t* fock_ws, size_t* red_ws, size_t* ops_ws) {
  int st;
  size_t a = 0, b = 0;
  if ((st = hf_fock_workspace_size(HF_C128, pb->fock_flags, pb->nk1, pb->nk2, pb->nb, &a))) return st;
  if ((st = hf_fock_workspace_size(HF_C128, response_flags(pb->fock_flags), pb->nk1, pb->nk2, pb->nb, &b)))
    return st;
  *fock_ws = a > b ? a : b;
  if ((st = hf_reduce_workspace_size(pb->nk1, pb->nk2, pb->nb, red_ws))) return st;
  return hf_ops_workspace_size(ops_ws);
}

extern "C" int hf_newton_workspace_size(const hf_cg_problem* pb, const hf_newton_config* cf, size_t* bytes) {
  int st;
  if ((st = newton_check(pb, cf))) return st;
  if (!bytes) return fail(HF_ERR_INVALID, "hf_newton_workspace_size: null output");
  size_t f = 0, r = 0, o = 0;
  if ((st = newton_sizes(pb, &f, &r, &o))) return st;
  NewtonLayout L;
  *bytes = newton_layout(*pb, *cf, f, r, o, L);
  return HF_OK;
}

extern "C" int hf_newton_solve(void* stream, const hf_cg_problem* pb, const hf_newton_config* cf, const void* P0,
                               void* Q_out, void* p_out, void* density, void* fock, double* hist_E, double* hist_G,
                               double* scalars_out, void* workspace, size_t workspace_bytes) {
  int st;
  if ((st = newton_check(pb, cf))) return st;
  if (!P0 || !Q_out || !p_out || !density || !fock || !scalars_out || !workspace)
    return fail(HF_ERR_INVALID, "hf_newton_solve: null buffer");
  Newton N;
  N.s = static_cast<cudaStream_t>(stream);
  N.pb = pb;
  N.cf = cf;
  N.base = static_cast<unsigned char*>(workspace);
  N.nk = pb->nk1 * pb->nk2;
  N.nb = pb->nb;
  N.nq = (size_t)N.nk * N.nb * N.nb;
  N.nv = (size_t)N.nk * N.nb;
  size_t ops_ws = 0;
  if ((st = newton_sizes(pb, &N.fock_ws, &N.red_ws, &ops_ws))) return st;
  if (newton_layout(*pb, *cf, N.fock_ws, N.red_ws, ops_ws, N.L) > workspace_bytes)
    return fail(HF_ERR_WORKSPACE, "hf_newton_solve: workspace too small");
  const cudaStream_t s = N.s;
  const int nk = N.nk, nb = N.nb;
  const size_t nq = N.nq, nv = N.nv;
  constexpr double tiny = 1e-30, delta_min = 1e-10;
  const double ws_sum = pb->weight_sum;
  N.T_r = std::fmax(pb->T, 1e-12);
  N.tol_g = cf->tol_grad > 0.0 ? cf->tol_grad : 1e-6;  // solver.py:1191
  N.n_target_norm = pb->n_electrons / std::fmax(ws_sum, tiny);
  N.occ_den = ws_sum * nb;
  N.defl = cf->n_deflation > 0 && cf->deflation_sigma > 0.0;
  N.inv2L2 = 1.0 / (2.0 * std::pow(std::fmax(cf->deflation_length, 1e-12), 2));
  N.dsig = cf->deflation_sigma;
  const double noise_floor = std::fmax(1e-12, 4500.0 * 2.220446049250313e-16);
  double* sc = N.sc();
  const double* w2d = N.w2d();

  // normalised weights, device scalars
  if ((st = hf_axpby_real(s, (size_t)nk, 1.0 / std::fmax(ws_sum, tiny), w2d, 0.0, nullptr, N.at<double>(oWN))))
    return st;
  HF_CUDA(cudaMemsetAsync(sc, 0, (size_t)sD2 * 8, s));

  // ---- init (solver.py:840-877) ----
  // current state: Q, p, Ft in slot `cur` of each double buffer; trial in 1 - cur
  int cur = 0;
  auto Qb = [&](int i) { return N.at<void>(i ? cQ1 : cQ0); };
  auto pb_ = [&](int i) { return N.at<double>(i ? rP1 : rP0); };
  auto Ftb = [&](int i) { return N.at<void>(i ? cFT1 : cFT0); };
  if ((st = hf_axpby(s, (size_t)nk, nb, 1.0, P0, 0.0, nullptr, 1, N.at<void>(cP)))) return st;
  if ((st = N.fock(N.at<void>(cP), N.at<void>(cF), false))) return st;
  if ((st = hf_eigh(s, HF_C128, nk, nb, N.at<void>(cF), N.at<double>(rEPS), Qb(cur)))) return st;
  if ((st = N.solve_mu(N.at<double>(rEPS), sc + sMu0, sc + sMu))) return st;
  if ((st = N.occupations(N.at<double>(rEPS), sc + sMu, pb_(cur)))) return st;
  double E = 0.0, grad_norm = 0.0, pen = 0.0;
  if ((st = N.eval_state(Qb(cur), pb_(cur), Ftb(cur), &E, &grad_norm, &pen))) return st;
  if (grad_norm <= N.tol_g) {  // occupation refinement at fixed orbitals
    for (int it = 0; it < 30; ++it) {
      if ((st = hf_density_from_Qp(s, HF_C128, nk, nb, Qb(cur), pb_(cur), N.at<void>(cP)))) return st;
      if ((st = N.fock(N.at<void>(cP), N.at<void>(cF), false))) return st;
      if ((st = hf_fock_orbital(s, HF_C128, nk, nb, Qb(cur), N.at<void>(cF), N.at<void>(cFTF)))) return st;
      if ((st = hf_real_diag(s, (size_t)nk, nb, N.at<void>(cFTF), N.at<double>(rEPST)))) return st;
      HF_CUDA(cudaMemcpyAsync(sc + sMu0, sc + sMu, 8, cudaMemcpyDeviceToDevice, s));
      if ((st = N.solve_mu(N.at<double>(rEPST), sc + sMu0, sc + sMu))) return st;
      if ((st = N.occupations(N.at<double>(rEPST), sc + sMu, pb_(cur)))) return st;
    }
    if ((st = N.eval_state(Qb(cur), pb_(cur), Ftb(cur), &E, &grad_norm, &pen))) return st;
  }

  int k = 0;
  double Delta = cf->tr_delta0;
  void* G = N.at<void>(cG);
  double* eps = N.at<double>(rEPS);
  double* dots = sc + sDot;
  while (k < cf->max_iter && grad_norm > N.tol_g && Delta > delta_min) {
    if (hist_E) hist_E[k] = E;
    if (hist_G) hist_G[k] = grad_norm;
    void* Q = Qb(cur);
    double* p = pb_(cur);
    void* Ft = Ftb(cur);
    if ((st = hf_orbital_grad(s, (size_t)nk, nb, Ft, p, G, eps))) return st;
    if ((st = hf_jdot(s, (size_t)nk, nb, nullptr, nullptr, nullptr, eps, eps, nullptr, dots, N.ops()))) return st;
    double es = 0.0;
    if ((st = N.read(&es, dots, 1))) return st;
    const double eps_scale = std::sqrt(es / ((double)nk * nb) + tiny);
    const double lam_pc = std::fmax(N.T_r, cf->denom_scale * eps_scale);

    // ---- Steihaug truncated CG (solver.py:932-992) ----
    // r = -G, rp = 0; d = z = M^-1 r; v = Hv = 0.  Double buffers: r / r + a Hd and v / v + a d.
    int ri = 0, vi = 0;
    auto RX = [&](int i) { return N.at<void>(i ? cRX1 : cRX0); };
    auto RP = [&](int i) { return N.at<double>(i ? rRP1 : rRP0); };
    auto VX = [&](int i) { return N.at<void>(i ? cVX1 : cVX0); };
    auto VP = [&](int i) { return N.at<double>(i ? rVP1 : rVP0); };
    void* dX = N.at<void>(cDX);
    double* dp = N.at<double>(rDP);
    void* HdX = N.at<void>(cHDX);
    double* Hdp = N.at<double>(rHDP);
    void* HvX = N.at<void>(cHVX);
    double* Hvp = N.at<double>(rHVP);
    void* zX = N.at<void>(cZX);
    double* zp = N.at<double>(rZP);
    if ((st = hf_axpby(s, (size_t)nk, nb, -1.0, G, 0.0, nullptr, 0, RX(ri)))) return st;
    HF_CUDA(cudaMemsetAsync(RP(ri), 0, nv * 8, s));
    if ((st = N.prec(RX(ri), RP(ri), eps, p, lam_pc, dX, dp))) return st;
    if ((st = N.jip(RX(ri), RP(ri), dX, dp, dots))) return st;
    double rz = 0.0;
    if ((st = N.read(&rz, dots, 1))) return st;
    HF_CUDA(cudaMemsetAsync(VX(vi), 0, nq * 16, s));
    HF_CUDA(cudaMemsetAsync(VP(vi), 0, nv * 8, s));
    HF_CUDA(cudaMemsetAsync(HvX, 0, nq * 16, s));
    HF_CUDA(cudaMemsetAsync(Hvp, 0, nv * 8, s));
    int cg = 0;
    bool done = false;
    while (cg < cf->tr_cg_max && !done) {
      if ((st = N.hvp(Q, Ft, p, dX, dp, pen, HdX, Hdp))) return st;
      {  // d.Hd, d.d, v.d, v.v in one pass
        const void* ax[4] = {dX, dX, VX(vi), VX(vi)};
        const void* bx[4] = {HdX, dX, dX, VX(vi)};
        const double* apv[4] = {dp, dp, VP(vi), VP(vi)};
        const double* bpv[4] = {Hdp, dp, dp, VP(vi)};
        if ((st = N.jip_multi(4, ax, apv, bx, bpv, dots + 0))) return st;
      }
      double d4[4];
      if ((st = N.read(d4, dots, 4))) return st;
      const double dHd = d4[0], dd = d4[1];
      const bool neg = dHd <= 1e-14 * dd;
      const double b = 2.0 * d4[2];
      const double cc = d4[3] - Delta * Delta;
      const double disc = std::fmax(b * b - 4.0 * dd * cc, 0.0);
      const double t_bd = (-b + std::sqrt(disc)) / (2.0 * dd + 1e-30);
      const double alpha = rz / (neg ? 1.0 : dHd);
      const int va = 1 - vi, ra = 1 - ri;
      if ((st = hf_axpby(s, (size_t)nk, nb, 1.0, VX(vi), alpha, dX, 0, VX(va)))) return st;
      if ((st = hf_axpby_real(s, nv, 1.0, VP(vi), alpha, dp, VP(va)))) return st;
      if ((st = hf_axpby(s, (size_t)nk, nb, 1.0, RX(ri), -alpha, HdX, 0, RX(ra)))) return st;
      if ((st = hf_axpby_real(s, nv, 1.0, RP(ri), -alpha, Hdp, RP(ra)))) return st;
      if ((st = N.prec(RX(ra), RP(ra), eps, p, lam_pc, zX, zp))) return st;
      {  // |v + a d|^2, |r - a Hd|^2, r.z in one pass
        const void* ax[3] = {VX(va), RX(ra), RX(ra)};
        const void* bx[3] = {VX(va), RX(ra), zX};
        const double* apv[3] = {VP(va), RP(ra), RP(ra)};
        const double* bpv[3] = {VP(va), RP(ra), zp};
        if ((st = N.jip_multi(3, ax, apv, bx, bpv, dots + 4))) return st;
      }
      double d3[3];
      if ((st = N.read(d3, dots + 4, 3))) return st;
      const bool cross = std::sqrt(std::fmax(0.0, d3[0])) >= Delta;
      const bool take_bd = neg || cross;
      const double rn = std::sqrt(std::fmax(0.0, d3[1]));
      const bool inner = rn < 0.05 * grad_norm;
      const double rz_new = d3[2];
      const double beta = rz_new / (std::fabs(rz) > tiny ? rz : 1.0);
      const bool stop = take_bd || inner;
      if (take_bd) {
        if ((st = hf_axpby(s, (size_t)nk, nb, 1.0, VX(vi), t_bd, dX, 0, VX(vi)))) return st;
        if ((st = hf_axpby_real(s, nv, 1.0, VP(vi), t_bd, dp, VP(vi)))) return st;
        if ((st = hf_axpby(s, (size_t)nk, nb, 1.0, HvX, t_bd, HdX, 0, HvX))) return st;
        if ((st = hf_axpby_real(s, nv, 1.0, Hvp, t_bd, Hdp, Hvp))) return st;
      } else {
        vi = va;
        if ((st = hf_axpby(s, (size_t)nk, nb, 1.0, HvX, alpha, HdX, 0, HvX))) return st;
        if ((st = hf_axpby_real(s, nv, 1.0, Hvp, alpha, Hdp, Hvp))) return st;
        ri = ra;
      }
      if (!stop) {
        if ((st = hf_axpby(s, (size_t)nk, nb, 1.0, zX, beta, dX, 0, dX))) return st;
        if ((st = hf_axpby_real(s, nv, 1.0, zp, beta, dp, dp))) return st;
        rz = rz_new;
      }
      ++cg;
      done = stop;
    }

    // ---- predicted reduction and trial step (solver.py:998-1046) ----
    void* vX = VX(vi);
    double* vp = VP(vi);
    {  // g.v, v.Hv, v.v in one pass
      const void* ax[3] = {G, vX, vX};
      const void* bx[3] = {vX, HvX, vX};
      const double* wxv[3] = {w2d, w2d, nullptr};
      const double* apv[3] = {nullptr, vp, vp};
      const double* bpv[3] = {nullptr, Hvp, vp};
      const double* wpv[3] = {nullptr, w2d, w2d};
      if ((st = jdot_multi(s, (size_t)nk, nb, 3, ax, bx, wxv, apv, bpv, wpv, dots + 0, N.ops()))) return st;
    }
    double m3[3];
    if ((st = N.read(m3, dots, 3))) return st;
    const double pred = -(m3[0] + 0.5 * m3[1]);
    const int tr = 1 - cur;
    if ((st = hf_cayley_spectral(s, HF_C128, nk, nb, vX, N.at<void>(cVV), N.at<double>(rLAM)))) return st;
    if ((st = hf_cayley_unitary(s, HF_C128, nk, nb, N.at<void>(cVV), N.at<double>(rLAM), -1.0, N.at<void>(cU))))
      return st;
    if ((st = hf_matmul(s, nk, nb, Q, N.at<void>(cU), Qb(tr)))) return st;
    if ((st = hf_fock_orbital(s, HF_C128, nk, nb, N.at<void>(cU), Ft, N.at<void>(cFTF)))) return st;
    if ((st = hf_real_diag(s, (size_t)nk, nb, N.at<void>(cFTF), N.at<double>(rEPST)))) return st;
    if ((st = N.solve_mu(N.at<double>(rEPST), sc + sMu, sc + sMuT))) return st;
    if ((st = N.occupations(N.at<double>(rEPST), sc + sMuT, pb_(tr)))) return st;
    double E_t = 0.0, g_t = 0.0, pen_t = 0.0;
    if ((st = N.eval_state(Qb(tr), pb_(tr), Ftb(tr), &E_t, &g_t, &pen_t))) return st;
    const double noise = noise_floor * std::fmax(std::fabs(E), 1.0);
    const bool use_g = pred <= noise;
    const bool accept_g = g_t <= grad_norm && E_t <= E + noise;
    const double Delta_g = accept_g ? Delta : 0.5 * Delta;
    const double ratio = (E - E_t) / (use_g ? 1.0 : pred);
    const double step_norm = std::sqrt(std::fmax(0.0, m3[2]));
    double Delta_r = Delta;
    if (ratio < 0.25) Delta_r = 0.25 * Delta;
    else if (ratio > 0.75 && step_norm > 0.9 * Delta) Delta_r = std::fmin(2.0 * Delta, 5.0);
    const bool accept = use_g ? accept_g : ratio > 0.1;
    Delta = use_g ? Delta_g : Delta_r;
    if (accept) {
      cur = tr;
      E = E_t;
      grad_norm = g_t;
      pen = pen_t;
      HF_CUDA(cudaMemcpyAsync(sc + sMu, sc + sMuT, 8, cudaMemcpyDeviceToDevice, s));
    }
    ++k;
  }

  // ---- final state (solver.py:1062-1066) ----
  if ((st = hf_density_from_Qp(s, HF_C128, nk, nb, Qb(cur), pb_(cur), density))) return st;
  if ((st = N.fock(density, fock, false))) return st;
  if ((st = hf_energy(s, HF_C128, pb->nk1, pb->nk2, nb, density, pb->h, N.at<void>(cSG), N.at<void>(oH), 1,
                      pb->w2d, sc + sE, N.at<void>(oREDWS), N.red_ws)))
    return st;
  HF_CUDA(cudaMemcpyAsync(Q_out, Qb(cur), nq * 16, cudaMemcpyDeviceToDevice, s));
  HF_CUDA(cudaMemcpyAsync(p_out, pb_(cur), nv * 8, cudaMemcpyDeviceToDevice, s));
  double fin[3];
  if ((st = N.read(fin, sc, 3))) return st;  // E, |G|^2 (unused), mu
  scalars_out[0] = fin[sMu];
  scalars_out[1] = fin[sE];
  scalars_out[2] = (double)k;
  scalars_out[3] = grad_norm <= N.tol_g ? 1.0 : 0.0;
  scalars_out[4] = grad_norm;
  scalars_out[5] = (double)N.n_builds;
  return HF_OK;
}
