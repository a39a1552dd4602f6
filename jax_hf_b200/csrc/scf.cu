// Native SCF driver (reference_scf.py:124-365, solve_scf with project_fn=None
// and the built-in Fock build): Roothaan iteration with linear mixing, Pulay
// C-DIIS or ODA, level shift and trust-radius clip, complex128.
//
// Every array step is one of the library's device operations (Fock build,
// energy, Jacobi eigh, bisection mu, occupations, density, residuals, DIIS
// Gram matrix, extrapolation).  The host keeps the loop's scalar decisions, as
// the reference does in its traced loop, and reads them in one small
// device->host copy per iteration (residual sums, energy, Gram matrix; plus
// the second energy of an ODA step and the step norm of a trust-radius clip).
// The bordered (n+1)^2 DIIS system is solved on the host by LU with partial
// pivoting (the algorithm of LAPACK gesv behind numpy.linalg.solve).
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"

namespace hf {
namespace {

struct ScfLayout {
  size_t off[24];
  size_t total;
};

enum {
  kDH, kSG, kH, kF, kPN, kDELTA, kUPD, kFX, kFD, kFH, kPD, kSTEP, kV, kEV, kSH, kOCC, kRH, kFHIST, kSCAL,
  kFOCKWS, kREDWS, kOPSWS, kDEV, kNBUF
};

// Loop state of the device-resident SCF loop (batch graphs): what the host loop keeps in
// its locals, plus the DIIS Gram matrix B (nh x nh, nh <= 16)
struct ScfDev {
  int k, base, slot, converged, fp32, switch_iter, use_diis, pad;
  double d_prev;
  double B[16 * 16];
};

// device scalar block (float64): mu_raw, mu, E, E_new, sums[3], red[1], gram[21], coeff[n]
constexpr int kSMuRaw = 0, kSMu = 1, kSE = 2, kSEnew = 3, kSSums = 4, kSRed = 7, kSGram = 8, kSCoeff = 29;
static_assert(kSGram + 21 <= kSCoeff, "the Gram slots hold 21 entries (n = 6 upper triangle, or a row of n <= 16)");

size_t scf_layout(const hf_cg_problem& pb, const hf_scf_config& cf, size_t fock_ws, size_t red_ws, size_t ops_ws,
                  ScfLayout& L) {
  const size_t nk = (size_t)pb.nk1 * pb.nk2, nb = pb.nb, nq = nk * nb * nb, nv = nk * nb;
  const size_t nh = cf.acceleration == 1 ? (size_t)cf.diis_size : 1;
  size_t sizes[kNBUF] = {};
  sizes[kDH] = sizes[kSG] = sizes[kF] = sizes[kPN] = sizes[kDELTA] = sizes[kUPD] = nq * 16;
  sizes[kFX] = sizes[kFD] = sizes[kFH] = sizes[kPD] = sizes[kSTEP] = sizes[kV] = nq * 16;
  sizes[kH] = nb * nb * 16;
  sizes[kEV] = sizes[kSH] = sizes[kOCC] = nv * 8;
  sizes[kRH] = nh * nq * 16;
  sizes[kFHIST] = cf.acceleration == 1 ? nh * nq * 16 : 256;
  sizes[kSCAL] = (kSCoeff + nh + 8) * 8;
  sizes[kFOCKWS] = fock_ws;
  sizes[kREDWS] = red_ws;
  sizes[kOPSWS] = ops_ws;
  sizes[kDEV] = sizeof(ScfDev);
  size_t o = 0;
  for (int i = 0; i < kNBUF; ++i) {
    L.off[i] = o;
    o += align_up(sizes[i] > 0 ? sizes[i] : 256, 256);
  }
  L.total = o;
  return o;
}

// Solves A x = b (n <= 16) by LU with partial pivoting (first maximum |a| as the
// pivot row, as idamax); returns false on an exactly singular pivot.
bool lu_solve(std::vector<double> A, std::vector<double> b, int n, std::vector<double>& x) {
  for (int j = 0; j < n; ++j) {
    int p = j;
    double best = std::fabs(A[j * n + j]);
    for (int i = j + 1; i < n; ++i)
      if (std::fabs(A[i * n + j]) > best) { best = std::fabs(A[i * n + j]); p = i; }
    if (A[p * n + j] == 0.0) return false;
    if (p != j) {
      for (int c = 0; c < n; ++c) std::swap(A[j * n + c], A[p * n + c]);
      std::swap(b[j], b[p]);
    }
    const double inv = 1.0 / A[j * n + j];
    for (int i = j + 1; i < n; ++i) {
      const double l = A[i * n + j] * inv;
      A[i * n + j] = l;
      for (int c = j + 1; c < n; ++c) A[i * n + c] -= l * A[j * n + c];
    }
  }
  for (int i = 0; i < n; ++i)  // L y = P b (unit diagonal)
    for (int c = 0; c < i; ++c) b[i] -= A[i * n + c] * b[c];
  x.assign(n, 0.0);
  for (int i = n - 1; i >= 0; --i) {
    double s = b[i];
    for (int c = i + 1; c < n; ++c) s -= A[i * n + c] * x[c];
    x[i] = s / A[i * n + i];
  }
  return true;
}

struct Scf {
  cudaStream_t s;
  const hf_cg_problem* pb;
  const hf_scf_config* cf;
  unsigned char* base;
  ScfLayout L;
  size_t fock_ws, red_ws;
  int nk, nb;
  size_t nq;

  template <typename T>
  T* at(int i) const { return reinterpret_cast<T*>(base + L.off[i]); }
  double* scal() const { return at<double>(kSCAL); }

  int herm_axpby(double a, const void* x, double b, const void* y, void* out) {
    return hf_axpby(s, (size_t)nk, nb, a, x, b, y, 1, out);
  }
  bool fp32 = false;    // this build runs the exchange FFT in FP32
  bool mu_warm = false;  // a previous mu exists: the Newton-bracket start, or the bisection's hint
  bool eig_warm = false; // eigh started from the eigenvectors in kV (the previous decomposition)
  bool eig_cols = false; // eigh by the lane-per-column Jacobi (warm_eigh mode, nb <= 8)
  // herm(project(X)) in place (the caller's projector), or nothing without one
  int project(void* X) {
    if (!cf->project_cb) return HF_OK;
    if (cf->project_cb(cf->cb_user, s, X) != 0) return fail(HF_ERR_ABORTED, "hf_scf_solve: project callback failed");
    return HF_OK;
  }
  // out = herm(project(a x + b y)) (reference_scf.py:275-276 with a projector)
  int herm_proj_axpby(double a, const void* x, double b, const void* y, void* out) {
    if (!cf->project_cb) return herm_axpby(a, x, b, y, out);
    int st;
    if ((st = hf_axpby(s, (size_t)nk, nb, a, x, b, y, 0, out))) return st;
    return project(out);
  }
  int fock(const void* P, void* Sg, void* H, void* F) {
    int st;
    if (cf->fock_cb) {
      if (cf->fock_cb(cf->cb_user, s, P, Sg, H, F) != 0)
        return fail(HF_ERR_ABORTED, "hf_scf_solve: Fock callback failed");
    } else {
      const unsigned flags = pb->fock_flags | (fp32 ? HF_FOCK_FFT_FP32 : 0u);
      if ((st = hf_fock_build(s, HF_C128, flags, pb->nk1, pb->nk2, nb, P, pb->h, pb->VR, pb->refP, pb->HH,
                              pb->w2d, pb->n_contact, pb->contact_g, pb->contact_Oi, pb->contact_Oj, Sg, H, F,
                              at<void>(kFOCKWS), fock_ws)))
        return st;
    }
    return project(F);  // build_fock(project_fn=...) returns herm(project(F))
  }
  int energy(const void* P, const void* Sg, const void* H, double* E) {
    // H from hf_fock_build is one nb x nb matrix for all k (H_mode 1); zero without Hartree
    return hf_energy(s, HF_C128, pb->nk1, pb->nk2, nb, P, pb->h, Sg, H, 1, pb->w2d, E, at<void>(kREDWS), red_ws);
  }
  // reference_scf.py:87-96: eigh, bisection mu, level shift, occupations, density
  int density_from_fock(const void* F, void* P_out) {
    int st;
    double* sc = scal();
    if (eig_cols) {  // lane-per-column Jacobi, from the previous eigenvectors when there are any
      if ((st = hf_eigh_warm(s, nk, nb, F, eig_warm ? at<void>(kV) : nullptr, at<void>(kV), at<double>(kEV))))
        return st;
    } else if ((st = hf_eigh(s, HF_C128, nk, nb, F, at<double>(kEV), at<void>(kV)))) {
      return st;
    }
    // mu_method 2: Newton-bracket solver, from mu = 0 in the first call and from the previous
    // mu afterwards; mu_method 0: the bisection, given the previous mu as a hint that decides
    // most levels without evaluations (same result).  The kernel reads that word before it
    // overwrites it.
    if ((st = hf_find_mu(s, HF_C128, cf->mu_method == 2 ? 2 : 0, nk, 1, nb, at<double>(kEV), pb->w2d,
                         pb->n_electrons, pb->T, 0, mu_warm ? sc + kSMuRaw : nullptr, sc + kSMuRaw)))
      return st;
    const double* shifted = at<double>(kEV);
    const double* mu = sc + kSMuRaw;
    if (cf->level_shift != 0.0) {
      if ((st = hf_fermi(s, (size_t)nk * nb, at<double>(kEV), sc + kSMuRaw, pb->T, 2, cf->level_shift,
                         at<double>(kSH))))
        return st;
      if ((st = hf_find_mu(s, HF_C128, 0, nk, 1, nb, at<double>(kSH), pb->w2d, pb->n_electrons, pb->T, 0,
                           mu_warm ? sc + kSMu : nullptr, sc + kSMu)))
        return st;
      shifted = at<double>(kSH);
      mu = sc + kSMu;
    } else {
      HF_CUDA(cudaMemcpyAsync(sc + kSMu, sc + kSMuRaw, sizeof(double), cudaMemcpyDeviceToDevice, s));
    }
    if ((st = hf_fermi(s, (size_t)nk * nb, shifted, mu, pb->T, 0, 0.0, at<double>(kOCC)))) return st;
    return hf_density_from_Qp(s, HF_C128, nk, nb, at<void>(kV), at<double>(kOCC), P_out);
  }
  // reference_scf.py:78-84: herm(density) -> build -> energy -> next density
  int build_and_occupy(const void* dens, void* F, void* Pn) {
    int st;
    if ((st = herm_proj_axpby(1.0, dens, 0.0, nullptr, at<void>(kDH)))) return st;
    if ((st = fock(at<void>(kDH), at<void>(kSG), at<void>(kH), F))) return st;
    if ((st = energy(at<void>(kDH), at<void>(kSG), at<void>(kH), scal() + kSE))) return st;
    if ((st = density_from_fock(F, Pn))) return st;
    return project(Pn);
  }
  int read(double* host, const double* dev, int n) {
    HF_CUDA(cudaMemcpyAsync(host, dev, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    HF_CUDA(cudaStreamSynchronize(s));
    return HF_OK;
  }
};

}  // namespace
}  // namespace hf

using namespace hf;

static int scf_check(const hf_cg_problem* pb, const hf_scf_config* cf) {
  if (!pb || !cf) return fail(HF_ERR_INVALID, "hf_scf: null problem or config");
  if (pb->nk1 < 1 || pb->nk2 < 1 || pb->nb < 1 || pb->nb > 32)
    return fail(HF_ERR_INVALID, "hf_scf: bad mesh or band count");
  if (cf->max_iter <= 0) return fail(HF_ERR_INVALID, "max_iter must be positive");
  if (cf->acceleration < 0 || cf->acceleration > 2)
    return fail(HF_ERR_INVALID, "SCFConfig.acceleration must be 'linear', 'diis', or 'oda'");
  if (cf->diis_size <= 0) return fail(HF_ERR_INVALID, "diis_size must be positive");
  if (cf->acceleration == 1 && cf->diis_size > 16) return fail(HF_ERR_UNSUPPORTED, "hf_scf: diis_size > 16");
  if (cf->mu_method != 0 && cf->mu_method != 2) return fail(HF_ERR_INVALID, "hf_scf: mu_method must be 0 or 2");
  if (cf->mu_method == 2 && cf->level_shift != 0.0)
    return fail(HF_ERR_INVALID, "hf_scf: mu_method 2 needs level_shift = 0");
  if (cf->fp32_exchange && !(pb->fock_flags & HF_FOCK_EXCHANGE))
    return fail(HF_ERR_INVALID, "hf_scf: fp32_exchange needs the exchange term");
  if (cf->fp32_exchange && cf->fock_cb)
    return fail(HF_ERR_INVALID, "hf_scf: fp32_exchange applies to the built-in Fock build only");
  return HF_OK;
}

static int scf_sizes(const hf_cg_problem* pb, const hf_scf_config* cf, size_t* fock_ws, size_t* red_ws,
                     size_t* ops_ws) {
  int st;
  if ((st = hf_fock_workspace_size(HF_C128, pb->fock_flags, pb->nk1, pb->nk2, pb->nb, fock_ws))) return st;
  if ((st = hf_reduce_workspace_size(pb->nk1, pb->nk2, pb->nb, red_ws))) return st;
  return hf_ops_workspace_size(ops_ws);
}

extern "C" int hf_scf_workspace_size(const hf_cg_problem* pb, const hf_scf_config* cf, size_t* bytes) {
  int st;
  if ((st = scf_check(pb, cf))) return st;
  if (!bytes) return fail(HF_ERR_INVALID, "hf_scf_workspace_size: null output");
  size_t f = 0, r = 0, o = 0;
  if ((st = scf_sizes(pb, cf, &f, &r, &o))) return st;
  ScfLayout L;
  *bytes = scf_layout(*pb, *cf, f, r, o, L);
  return HF_OK;
}

extern "C" int hf_scf_solve(void* stream, const hf_cg_problem* pb, const hf_scf_config* cf, const void* P0,
                            void* density, void* fock, double* hist_E, double* hist_D, double* hist_C,
                            double* scalars_out, void* workspace, size_t workspace_bytes) {
  int st;
  if ((st = scf_check(pb, cf))) return st;
  if (!P0 || !density || !fock || !scalars_out || !workspace)
    return fail(HF_ERR_INVALID, "hf_scf_solve: null buffer");
  Scf S;
  S.s = static_cast<cudaStream_t>(stream);
  S.pb = pb;
  S.cf = cf;
  S.base = static_cast<unsigned char*>(workspace);
  S.nk = pb->nk1 * pb->nk2;
  S.nb = pb->nb;
  S.nq = (size_t)S.nk * pb->nb * pb->nb;
  size_t ops_ws = 0;
  if ((st = scf_sizes(pb, cf, &S.fock_ws, &S.red_ws, &ops_ws))) return st;
  if (scf_layout(*pb, *cf, S.fock_ws, S.red_ws, ops_ws, S.L) > workspace_bytes)
    return fail(HF_ERR_INVALID, "hf_scf_solve: workspace too small");
  const cudaStream_t s = S.s;
  const int nk = S.nk, nb = S.nb;
  const size_t nq = S.nq, qbytes = nq * 16;
  const bool diis = cf->acceleration == 1, oda = cf->acceleration == 2;
  const int nh = diis ? cf->diis_size : 1;
  const double wsum = std::fmax(pb->weight_sum, 1e-30);
  double* sc = S.scal();
  void* ops = S.at<void>(kOPSWS);
  const double* w2d = static_cast<const double*>(pb->w2d);

  HF_CUDA(cudaMemcpyAsync(density, P0, qbytes, cudaMemcpyDeviceToDevice, s));
  if (diis) {
    HF_CUDA(cudaMemsetAsync(S.at<void>(kRH), 0, (size_t)nh * qbytes, s));
    HF_CUDA(cudaMemsetAsync(S.at<void>(kFHIST), 0, (size_t)nh * qbytes, s));
  }
  std::vector<double> hv(kSCoeff + 8, 0.0);
  // B is kept here between iterations and only the replaced slot's row is refreshed per step
  // (hf_gram_row; each entry bit-identical to the full hf_gram's)
  std::vector<double> Bkeep(diis ? (size_t)nh * nh : 0, 0.0);
  int k = 0, base = 0, switch_iter = -1;  // base: first iteration of the current DIIS history
  bool converged = false;
  double d_prev = INFINITY;
  S.fp32 = cf->fp32_exchange != 0;
  while (k < cf->max_iter && !converged) {
    void* F = S.at<void>(kF);
    void* Pn = S.at<void>(kPN);
    if (S.fp32 && d_prev <= cf->fp32_switch_density) {  // FP64 from here on, with a fresh DIIS history
      S.fp32 = false;
      switch_iter = k;
      base = k;
      if (diis) {
        HF_CUDA(cudaMemsetAsync(S.at<void>(kRH), 0, (size_t)nh * qbytes, s));
        HF_CUDA(cudaMemsetAsync(S.at<void>(kFHIST), 0, (size_t)nh * qbytes, s));
        std::fill(Bkeep.begin(), Bkeep.end(), 0.0);
      }
    }
    S.mu_warm = k > 0;
    S.eig_cols = cf->warm_eigh != 0 && nb <= 8;
    S.eig_warm = S.eig_cols && k > 0;
    if ((st = S.build_and_occupy(density, F, Pn))) return st;
    const int kd = k - base;  // index in the current DIIS history
    void* R_out = diis ? (void*)(S.at<unsigned char>(kRH) + (size_t)(kd % nh) * qbytes) : (void*)S.at<void>(kRH);
    if ((st = hf_scf_residuals(s, nk, nb, F, density, Pn, w2d, R_out, S.at<void>(kDELTA), sc + kSSums, ops)))
      return st;
    if (diis) {
      HF_CUDA(cudaMemcpyAsync(S.at<unsigned char>(kFHIST) + (size_t)(kd % nh) * qbytes, F, qbytes,
                              cudaMemcpyDeviceToDevice, s));
      if ((st = hf_gram_row(s, nh, kd % nh, nq, nk, nb, S.at<void>(kRH), w2d, sc + kSGram, ops))) return st;
    }
    if ((st = S.read(hv.data(), sc, kSCoeff))) return st;
    const double E_host = hv[kSE];
    const double d_res = std::sqrt(hv[kSSums] / wsum), c_res = std::sqrt(hv[kSSums + 1] / wsum);
    converged = !S.fp32 && d_res <= cf->density_tol && c_res <= cf->comm_tol;
    d_prev = d_res;
    void* updated = S.at<void>(kUPD);
    if (diis) {
      // B_ij = sum_k w Re tr(R_i^H R_j) over every history slot (zeros where unused)
      const int slot = kd % nh;
      for (int j = 0; j < nh; ++j) Bkeep[(size_t)slot * nh + j] = Bkeep[(size_t)j * nh + slot] = hv[kSGram + j];
      const std::vector<double>& B = Bkeep;
      double bmax = 0.0;
      for (double v : B) bmax = std::fmax(bmax, std::fabs(v));
      bmax = std::fmax(bmax, 1e-30);
      const int count = kd + 1 < nh ? kd + 1 : nh;
      const int m = nh + 1;
      std::vector<double> A((size_t)m * m, 0.0), rhs(m, 0.0), sol;
      for (int i = 0; i < nh; ++i) {
        const double act = i < count ? 1.0 : 0.0;
        for (int j = 0; j < nh; ++j) A[i * m + j] = B[i * nh + j] / bmax;
        A[i * m + i] += 1.0 - act;
        A[i * m + nh] = -act;
        A[nh * m + i] = -act;
      }
      rhs[nh] = -1.0;
      bool ok = lu_solve(A, rhs, m, sol);
      if (ok)
        for (double v : sol) ok = ok && std::isfinite(v);
      const int start = cf->diis_start > 2 ? cf->diis_start : 2;
      if (count >= start && ok) {
        // from pageable memory: the values are staged before the call returns
        HF_CUDA(cudaMemcpyAsync(sc + kSCoeff, sol.data(), nh * sizeof(double), cudaMemcpyHostToDevice, s));
        if ((st = hf_lincomb(s, nh, nq, nq, S.at<void>(kFHIST), sc + kSCoeff, S.at<void>(kFX)))) return st;
        const void* Fx = S.at<void>(kFX);
        const double damp = std::fmin(std::fmax(cf->diis_damping, 0.0), 1.0);
        if (damp != 1.0) {
          if ((st = hf_axpby(s, (size_t)nk, nb, damp, Fx, 1.0 - damp, F, 0, S.at<void>(kFD)))) return st;
          Fx = S.at<void>(kFD);
        }
        if ((st = S.herm_axpby(1.0, Fx, 0.0, nullptr, S.at<void>(kFH)))) return st;
        if ((st = S.density_from_fock(S.at<void>(kFH), updated))) return st;
        if ((st = S.project(updated))) return st;
      } else {
        if ((st = S.herm_proj_axpby(1.0, density, cf->mixing, S.at<void>(kDELTA), updated))) return st;
      }
    } else if (oda) {
      if ((st = S.fock(Pn, S.at<void>(kSG), S.at<void>(kH), S.at<void>(kFX)))) return st;
      if ((st = S.energy(Pn, S.at<void>(kSG), S.at<void>(kH), sc + kSEnew))) return st;
      double E_new = 0.0;
      if ((st = S.read(&E_new, sc + kSEnew, 1))) return st;
      const double c1 = hv[kSSums + 2];
      const double c2 = (E_new - E_host) - c1;
      double lam;
      if (c2 > 1e-12) lam = std::fmin(std::fmax(-c1 / (2.0 * c2), 0.0), 1.0);
      else lam = c1 < 0.0 ? 1.0 : 0.0;
      if ((st = S.herm_proj_axpby(1.0, density, lam, S.at<void>(kDELTA), updated))) return st;
    } else {
      if ((st = S.herm_proj_axpby(1.0, density, cf->mixing, S.at<void>(kDELTA), updated))) return st;
    }
    if (cf->trust_radius > 0.0) {  // reference_scf.py:333-339
      if ((st = hf_axpby(s, (size_t)nk, nb, 1.0, updated, -1.0, density, 0, S.at<void>(kSTEP)))) return st;
      if ((st = hf_jdot(s, (size_t)nk, nb, S.at<void>(kSTEP), S.at<void>(kSTEP), w2d, nullptr, nullptr,
                        nullptr, sc + kSRed, ops)))
        return st;
      double red = 0.0;
      if ((st = S.read(&red, sc + kSRed, 1))) return st;
      const double sn = std::sqrt(red / wsum);
      if (sn > cf->trust_radius) {
        const double scale = cf->trust_radius / std::fmax(sn, 1e-30);
        if ((st = S.herm_proj_axpby(1.0, density, scale, S.at<void>(kSTEP), updated))) return st;
      }
    }
    HF_CUDA(cudaMemcpyAsync(density, converged ? Pn : updated, qbytes, cudaMemcpyDeviceToDevice, s));
    if (hist_E) hist_E[k] = E_host;
    if (hist_D) hist_D[k] = d_res;
    if (hist_C) hist_C[k] = c_res;
    ++k;
  }
  // final build at the returned density (reference_scf.py:345-347), FP64 in every mode
  S.fp32 = false;
  S.mu_warm = k > 0;
  S.eig_cols = cf->warm_eigh != 0 && nb <= 8;
  S.eig_warm = S.eig_cols && k > 0;
  if ((st = S.build_and_occupy(density, fock, S.at<void>(kPN)))) return st;
  double fin[3] = {0.0, 0.0, 0.0};
  if ((st = S.read(fin, sc, 3))) return st;
  scalars_out[0] = fin[kSE];
  scalars_out[1] = fin[kSMu];
  scalars_out[2] = (double)k;
  scalars_out[3] = converged ? 1.0 : 0.0;
  if (cf->fp32_exchange) scalars_out[4] = (double)switch_iter;
  return HF_OK;
}

// ====================================================== device-resident SCF loop ====
// The SCF loop of hf_scf_solve with its host decisions moved onto the device, so that a
// batch of solves runs as one CUDA graph (hf_scf_batch_graph_*): the loop state lives in
// an ScfDev in the workspace, the DIIS bordered system is solved by a one-thread kernel
// with the host's LU (every multiply and subtract rounded separately, as on the host,
// where nothing is contracted into an FMA), the DIIS-or-mixing choice is a conditional IF
// node and the iteration loops are conditional WHILE nodes.  DIIS and linear mixing
// (with damping, level shift, Newton-bracket mu, warm eigh and the FP32-exchange phase);
// ODA and the trust-radius clip read extra values per iteration and stay with the host
// driver.
namespace hf {
namespace {

struct ScfStepArgs {
  double wsum, density_tol, comm_tol, switch_density;
  int nh, diis, diis_start, max_iter;
  double *hist_E, *hist_D, *hist_C;
};

__global__ void k_scf_dev_begin(ScfDev* d, int fp32) {
  d->k = 0;
  d->base = 0;
  d->slot = 0;
  d->converged = 0;
  d->fp32 = fp32;
  d->switch_iter = -1;
  d->use_diis = 0;
  d->d_prev = INFINITY;
  for (int i = 0; i < 16 * 16; ++i) d->B[i] = 0.0;
}

__global__ void k_scf_dev_iter_begin(ScfDev* d, int nh) { d->slot = (d->k - d->base) % nh; }

// reference_scf.py:291-329 after the residuals: convergence test, history, DIIS solve
__global__ void k_scf_dev_step(ScfDev* d, double* sc, ScfStepArgs a, cudaGraphConditionalHandle hif) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double E = sc[kSE];
  const double d_res = sqrt(sc[kSSums] / a.wsum), c_res = sqrt(sc[kSSums + 1] / a.wsum);
  d->converged = (!d->fp32 && d_res <= a.density_tol && c_res <= a.comm_tol) ? 1 : 0;
  d->d_prev = d_res;
  if (a.hist_E) a.hist_E[d->k] = E;
  if (a.hist_D) a.hist_D[d->k] = d_res;
  if (a.hist_C) a.hist_C[d->k] = c_res;
  if (!a.diis) return;
  const int nh = a.nh, slot = d->slot, kd = d->k - d->base, m = nh + 1;
  for (int j = 0; j < nh; ++j) d->B[slot * nh + j] = d->B[j * nh + slot] = sc[kSGram + j];
  double bmax = 0.0;
  for (int i = 0; i < nh * nh; ++i) bmax = fmax(bmax, fabs(d->B[i]));
  bmax = fmax(bmax, 1e-30);
  const int count = kd + 1 < nh ? kd + 1 : nh;
  double A[17 * 17], b[17], x[17];
  for (int i = 0; i < m * m; ++i) A[i] = 0.0;
  for (int i = 0; i < m; ++i) b[i] = 0.0;
  for (int i = 0; i < nh; ++i) {
    const double act = i < count ? 1.0 : 0.0;
    for (int j = 0; j < nh; ++j) A[i * m + j] = __ddiv_rn(d->B[i * nh + j], bmax);
    A[i * m + i] = __dadd_rn(A[i * m + i], __dsub_rn(1.0, act));
    A[i * m + nh] = -act;
    A[nh * m + i] = -act;
  }
  b[nh] = -1.0;
  bool ok = true;
  for (int j = 0; j < m && ok; ++j) {  // LU with partial pivoting, the host's lu_solve
    int p = j;
    double best = fabs(A[j * m + j]);
    for (int i = j + 1; i < m; ++i)
      if (fabs(A[i * m + j]) > best) {
        best = fabs(A[i * m + j]);
        p = i;
      }
    if (A[p * m + j] == 0.0) {
      ok = false;
      break;
    }
    if (p != j) {
      for (int c = 0; c < m; ++c) {
        const double t = A[j * m + c];
        A[j * m + c] = A[p * m + c];
        A[p * m + c] = t;
      }
      const double t = b[j];
      b[j] = b[p];
      b[p] = t;
    }
    const double inv = __ddiv_rn(1.0, A[j * m + j]);
    for (int i = j + 1; i < m; ++i) {
      const double l = __dmul_rn(A[i * m + j], inv);
      A[i * m + j] = l;
      for (int c = j + 1; c < m; ++c) A[i * m + c] = __dsub_rn(A[i * m + c], __dmul_rn(l, A[j * m + c]));
    }
  }
  if (ok) {
    for (int i = 0; i < m; ++i)
      for (int c = 0; c < i; ++c) b[i] = __dsub_rn(b[i], __dmul_rn(A[i * m + c], b[c]));
    for (int i = m - 1; i >= 0; --i) {
      double t = b[i];
      for (int c = i + 1; c < m; ++c) t = __dsub_rn(t, __dmul_rn(A[i * m + c], x[c]));
      x[i] = __ddiv_rn(t, A[i * m + i]);
    }
    for (int i = 0; i < m; ++i) ok = ok && isfinite(x[i]);
  }
  const int start = a.diis_start > 2 ? a.diis_start : 2;
  const bool use = count >= start && ok;
  if (use)
    for (int i = 0; i < nh; ++i) sc[kSCoeff + i] = x[i];
  d->use_diis = use ? 1 : 0;
  cudaGraphSetConditional(hif, use ? 1u : 0u);
}

// density <- (converged ? Pn : updated)   (reference_scf.py:341)
__global__ void k_scf_dev_select(size_t n, const ScfDev* d, const double2* __restrict__ Pn,
                                 const double2* __restrict__ upd, double2* __restrict__ density) {
  const double2* src = d->converged ? Pn : upd;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
    density[e] = src[e];
}

// end of an iteration: k += 1 and the condition of the loop that runs next
__global__ void k_scf_dev_next(ScfDev* d, cudaGraphConditionalHandle h, int max_iter, int fp32_phase,
                               double switch_density) {
  d->k += 1;
  bool go;
  if (fp32_phase) go = d->k < max_iter && !(d->d_prev <= switch_density);
  else go = !d->converged && d->k < max_iter;
  cudaGraphSetConditional(h, go ? 1u : 0u);
}

// between the FP32 and the FP64 loops: FP64 from here on with a fresh DIIS history
// (reference loop: the top of the iteration after the residual fell below the switch)
__global__ void k_scf_dev_switch(ScfDev* d, cudaGraphConditionalHandle h, int max_iter, double switch_density) {
  if (d->fp32 && d->k < max_iter && d->d_prev <= switch_density) {
    d->fp32 = 0;
    d->switch_iter = d->k;
    d->base = d->k;
    for (int i = 0; i < 16 * 16; ++i) d->B[i] = 0.0;
  }
  cudaGraphSetConditional(h, (!d->fp32 && !d->converged && d->k < max_iter) ? 1u : 0u);
}

__global__ void k_scf_dev_out(const ScfDev* d, const double* sc, double* out) {
  out[0] = sc[kSE];
  out[1] = sc[kSMu];
  out[2] = (double)d->k;
  out[3] = d->converged ? 1.0 : 0.0;
  out[4] = (double)d->switch_iter;
}

struct Capture {
  cudaStream_t s = nullptr;
  int into(cudaGraph_t g, const std::vector<cudaGraphNode_t>& deps) {
    HF_CUDA(cudaStreamBeginCaptureToGraph(s, g, deps.empty() ? nullptr : deps.data(), nullptr, deps.size(),
                                          cudaStreamCaptureModeThreadLocal));
    return HF_OK;
  }
  int end(std::vector<cudaGraphNode_t>* tail) {
    if (tail) {
      cudaStreamCaptureStatus cs;
      const cudaGraphNode_t* dn = nullptr;
      size_t nd = 0;
      HF_CUDA(cudaStreamGetCaptureInfo(s, &cs, nullptr, nullptr, &dn, &nd));
      tail->assign(dn, dn + nd);
    }
    cudaGraph_t g = nullptr;
    HF_CUDA(cudaStreamEndCapture(s, &g));
    return HF_OK;
  }
};

int add_conditional(cudaGraph_t g, const std::vector<cudaGraphNode_t>& deps, cudaGraphConditionalHandle h,
                    cudaGraphConditionalNodeType type, unsigned size, cudaGraphNode_t* node, cudaGraph_t* bodies) {
  cudaGraphNodeParams np = {};
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = h;
  np.conditional.type = type;
  np.conditional.size = size;
  HF_CUDA(cudaGraphAddNode(node, g, deps.empty() ? nullptr : deps.data(), deps.size(), &np));
  for (unsigned i = 0; i < size; ++i) bodies[i] = np.conditional.phGraph_out[i];
  return HF_OK;
}

// One SCF iteration captured into graph g after `deps` (its terminal nodes returned in
// `deps`): build, residuals, history slot, DIIS step, then an IF node between the DIIS
// extrapolation and linear mixing, then the density update and the next loop condition.
int scf_iteration_dev(Scf& S, Capture& cap, cudaGraph_t g, std::vector<cudaGraphNode_t>& deps, bool fp32_phase,
                      bool warm, cudaGraphConditionalHandle h_next, int next_fp32_phase,
                      const ScfStepArgs& args) {
  const hf_scf_config* cf = S.cf;
  const hf_cg_problem* pb = S.pb;
  const int nk = S.nk, nb = S.nb, nh = args.nh;
  const size_t nq = S.nq;
  const bool diis = args.diis != 0;
  ScfDev* d = S.at<ScfDev>(kDEV);
  double* sc = S.scal();
  void* ops = S.at<void>(kOPSWS);
  const double* w2d = static_cast<const double*>(pb->w2d);
  void* density = S.at<void>(kPD);
  void* F = S.at<void>(kF);
  void* Pn = S.at<void>(kPN);
  void* updated = S.at<void>(kUPD);
  int st;
  if ((st = cap.into(g, deps))) return st;
  k_scf_dev_iter_begin<<<1, 1, 0, cap.s>>>(d, nh);
  HF_LAUNCH_CHECK("k_scf_dev_iter_begin");
  S.fp32 = fp32_phase;
  S.mu_warm = warm;
  S.eig_cols = cf->warm_eigh != 0 && nb <= 8;
  S.eig_warm = S.eig_cols && warm;
  if ((st = S.build_and_occupy(density, F, Pn))) return st;
  if ((st = scf_residuals_slot(cap.s, nk, nb, F, density, Pn, w2d, S.at<void>(kRH), nq, &d->slot,
                               S.at<void>(kDELTA), sc + kSSums, ops)))
    return st;
  if (diis) {
    if ((st = copy_to_slot(cap.s, nq, F, S.at<void>(kFHIST), &d->slot))) return st;
    if ((st = gram_row_slot(cap.s, nh, &d->slot, nq, nk, nb, S.at<void>(kRH), w2d, sc + kSGram, ops))) return st;
  }
  cudaGraphConditionalHandle hif = 0;
  if (diis) HF_CUDA(cudaGraphConditionalHandleCreate(&hif, g, 0u, cudaGraphCondAssignDefault));
  k_scf_dev_step<<<1, 1, 0, cap.s>>>(d, sc, args, hif);
  HF_LAUNCH_CHECK("k_scf_dev_step");
  if (diis) {
    std::vector<cudaGraphNode_t> tail;
    if ((st = cap.end(&tail))) return st;
    cudaGraphNode_t ifn = nullptr;
    cudaGraph_t br[2] = {nullptr, nullptr};
    if ((st = add_conditional(g, tail, hif, cudaGraphCondTypeIf, 2, &ifn, br))) return st;
    // then: F_x = sum c_i F_i, damping, herm, next density from F_x (reference_scf.py:305-314)
    if ((st = cap.into(br[0], {}))) return st;
    if ((st = hf_lincomb(cap.s, nh, nq, nq, S.at<void>(kFHIST), sc + kSCoeff, S.at<void>(kFX)))) return st;
    const void* Fx = S.at<void>(kFX);
    const double damp = std::fmin(std::fmax(cf->diis_damping, 0.0), 1.0);
    if (damp != 1.0) {
      if ((st = hf_axpby(cap.s, (size_t)nk, nb, damp, Fx, 1.0 - damp, F, 0, S.at<void>(kFD)))) return st;
      Fx = S.at<void>(kFD);
    }
    if ((st = hf_axpby(cap.s, (size_t)nk, nb, 1.0, Fx, 0.0, nullptr, 1, S.at<void>(kFH)))) return st;
    if ((st = S.density_from_fock(S.at<void>(kFH), updated))) return st;
    if ((st = cap.end(nullptr))) return st;
    // else: linear mixing
    if ((st = cap.into(br[1], {}))) return st;
    if ((st = hf_axpby(cap.s, (size_t)nk, nb, 1.0, density, cf->mixing, S.at<void>(kDELTA), 1, updated))) return st;
    if ((st = cap.end(nullptr))) return st;
    if ((st = cap.into(g, {ifn}))) return st;
  } else {
    if ((st = hf_axpby(cap.s, (size_t)nk, nb, 1.0, density, cf->mixing, S.at<void>(kDELTA), 1, updated))) return st;
  }
  k_scf_dev_select<<<148 * 4, 256, 0, cap.s>>>(nq, d, static_cast<const double2*>(Pn),
                                              static_cast<const double2*>(updated), static_cast<double2*>(density));
  HF_LAUNCH_CHECK("k_scf_dev_select");
  k_scf_dev_next<<<1, 1, 0, cap.s>>>(d, h_next, cf->max_iter, next_fp32_phase, cf->fp32_switch_density);
  HF_LAUNCH_CHECK("k_scf_dev_next");
  return cap.end(&deps);
}

struct ScfBatchGraph {
  int n = 0;
  cudaGraph_t G = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t run = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  std::vector<cudaEvent_t> t0, t1;
  ~ScfBatchGraph() {
    if (run) cudaStreamSynchronize(run);
    if (exec) cudaGraphExecDestroy(exec);
    if (G) cudaGraphDestroy(G);
    if (run) cudaStreamDestroy(run);
    if (ev_in) cudaEventDestroy(ev_in);
    if (ev_out) cudaEventDestroy(ev_out);
    for (auto e : t0)
      if (e) cudaEventDestroy(e);
    for (auto e : t1)
      if (e) cudaEventDestroy(e);
  }
};

}  // namespace
}  // namespace hf

static int scf_graph_check(const hf_scf_config* cf) {
  if (cf->fock_cb || cf->project_cb) return fail(HF_ERR_INVALID, "hf_scf_batch_graph: no host callbacks");
  if (cf->acceleration == 2) return fail(HF_ERR_UNSUPPORTED, "hf_scf_batch_graph: ODA reads values per iteration");
  if (cf->trust_radius > 0.0)
    return fail(HF_ERR_UNSUPPORTED, "hf_scf_batch_graph: the trust-radius clip reads values per iteration");
  return HF_OK;
}

extern "C" int hf_scf_batch_workspace_size(const hf_scf_batch_item* items, int n_items, const hf_scf_config* cf,
                                           size_t* bytes_per_item) {
  if (!items || n_items < 1 || !cf || !bytes_per_item) return fail(HF_ERR_INVALID, "bad batch arguments");
  size_t mx = 0;
  for (int i = 0; i < n_items; ++i) {
    size_t b = 0;
    const int st = hf_scf_workspace_size(&items[i].problem, cf, &b);
    if (st) return st;
    mx = b > mx ? b : mx;
  }
  *bytes_per_item = align_up(mx, 256);
  return HF_OK;
}

extern "C" int hf_scf_batch_graph_create(const hf_scf_batch_item* items, int n_items, const hf_scf_config* cf,
                                         void* workspace, size_t bytes_per_item, void** handle) {
  if (!items || n_items < 1 || !cf || !workspace || !handle) return fail(HF_ERR_INVALID, "bad batch arguments");
  *handle = nullptr;
  int st;
  if ((st = scf_graph_check(cf))) return st;
  size_t need = 0;
  if ((st = hf_scf_batch_workspace_size(items, n_items, cf, &need))) return st;
  if (bytes_per_item < need)
    return fail(HF_ERR_WORKSPACE, "SCF batch workspace too small: need " + std::to_string(need) + " per solve");
  for (int i = 0; i < n_items; ++i) {
    const hf_scf_batch_item& it = items[i];
    if ((st = scf_check(&it.problem, cf))) return st;
    if (!it.P0 || !it.density || !it.fock || !it.scalars_out)
      return fail(HF_ERR_INVALID, "NULL argument in batch item " + std::to_string(i));
  }
  auto* bg = new ScfBatchGraph();
  bg->n = n_items;
  bg->t0.assign(n_items, nullptr);
  bg->t1.assign(n_items, nullptr);
  Capture cap;
  auto build = [&]() -> int {
    int e;
    HF_CUDA(cudaStreamCreateWithFlags(&cap.s, cudaStreamNonBlocking));
    HF_CUDA(cudaGraphCreate(&bg->G, 0));
    cudaGraph_t G = bg->G;
    for (int i = 0; i < n_items; ++i) {
      const hf_scf_batch_item& it = items[i];
      const hf_cg_problem* pb = &it.problem;
      Scf S;
      S.s = cap.s;
      S.pb = pb;
      S.cf = cf;
      S.base = static_cast<unsigned char*>(workspace) + (size_t)i * bytes_per_item;
      S.nk = pb->nk1 * pb->nk2;
      S.nb = pb->nb;
      S.nq = (size_t)S.nk * pb->nb * pb->nb;
      size_t ops_ws = 0;
      if ((e = scf_sizes(pb, cf, &S.fock_ws, &S.red_ws, &ops_ws))) return e;
      scf_layout(*pb, *cf, S.fock_ws, S.red_ws, ops_ws, S.L);
      const bool diis = cf->acceleration == 1;
      const int nh = diis ? cf->diis_size : 1;
      const size_t qbytes = S.nq * 16;
      ScfDev* d = S.at<ScfDev>(kDEV);
      ScfStepArgs args;
      args.wsum = std::fmax(pb->weight_sum, 1e-30);
      args.density_tol = cf->density_tol;
      args.comm_tol = cf->comm_tol;
      args.switch_density = cf->fp32_switch_density;
      args.nh = nh;
      args.diis = diis ? 1 : 0;
      args.diis_start = cf->diis_start;
      args.max_iter = cf->max_iter;
      args.hist_E = it.hist_E;
      args.hist_D = it.hist_D;
      args.hist_C = it.hist_C;
      const bool mixed = cf->fp32_exchange != 0;
      HF_CUDA(cudaEventCreate(&bg->t0[i]));
      HF_CUDA(cudaEventCreate(&bg->t1[i]));
      cudaGraphConditionalHandle hA = 0, hB = 0;
      if (mixed) HF_CUDA(cudaGraphConditionalHandleCreate(&hA, G, 0u, cudaGraphCondAssignDefault));
      HF_CUDA(cudaGraphConditionalHandleCreate(&hB, G, 0u, cudaGraphCondAssignDefault));
      std::vector<cudaGraphNode_t> tail;
      // init (reference_scf.py:222-240)
      if ((e = cap.into(G, tail))) return e;
      HF_CUDA(cudaEventRecordWithFlags(bg->t0[i], cap.s, cudaEventRecordExternal));
      HF_CUDA(cudaMemcpyAsync(S.at<void>(kPD), it.P0, qbytes, cudaMemcpyDeviceToDevice, cap.s));
      if (diis) {
        HF_CUDA(cudaMemsetAsync(S.at<void>(kRH), 0, (size_t)nh * qbytes, cap.s));
        HF_CUDA(cudaMemsetAsync(S.at<void>(kFHIST), 0, (size_t)nh * qbytes, cap.s));
      }
      k_scf_dev_begin<<<1, 1, 0, cap.s>>>(d, mixed ? 1 : 0);
      HF_LAUNCH_CHECK("k_scf_dev_begin");
      if ((e = cap.end(&tail))) return e;
      if (cf->max_iter > 0) {
        // iteration 0 (cold eigensolve and mu), then the loops
        if ((e = scf_iteration_dev(S, cap, G, tail, mixed, false, mixed ? hA : hB, mixed ? 1 : 0, args))) return e;
        if (mixed) {
          cudaGraphNode_t loop = nullptr;
          cudaGraph_t body = nullptr;
          if ((e = add_conditional(G, tail, hA, cudaGraphCondTypeWhile, 1, &loop, &body))) return e;
          std::vector<cudaGraphNode_t> bt;
          if ((e = scf_iteration_dev(S, cap, body, bt, true, true, hA, 1, args))) return e;
          tail.assign(1, loop);
          if ((e = cap.into(G, tail))) return e;
          if (diis) {
            HF_CUDA(cudaMemsetAsync(S.at<void>(kRH), 0, (size_t)nh * qbytes, cap.s));
            HF_CUDA(cudaMemsetAsync(S.at<void>(kFHIST), 0, (size_t)nh * qbytes, cap.s));
          }
          k_scf_dev_switch<<<1, 1, 0, cap.s>>>(d, hB, cf->max_iter, cf->fp32_switch_density);
          HF_LAUNCH_CHECK("k_scf_dev_switch");
          if ((e = cap.end(&tail))) return e;
        }
        cudaGraphNode_t loop = nullptr;
        cudaGraph_t body = nullptr;
        if ((e = add_conditional(G, tail, hB, cudaGraphCondTypeWhile, 1, &loop, &body))) return e;
        std::vector<cudaGraphNode_t> bt;
        if ((e = scf_iteration_dev(S, cap, body, bt, false, true, hB, 0, args))) return e;
        tail.assign(1, loop);
      }
      // final build at the returned density, FP64 (reference_scf.py:345-347)
      if ((e = cap.into(G, tail))) return e;
      S.fp32 = false;
      S.mu_warm = cf->max_iter > 0;
      S.eig_cols = cf->warm_eigh != 0 && S.nb <= 8;
      S.eig_warm = S.eig_cols && cf->max_iter > 0;
      HF_CUDA(cudaMemcpyAsync(it.density, S.at<void>(kPD), qbytes, cudaMemcpyDeviceToDevice, cap.s));
      if ((e = S.build_and_occupy(it.density, it.fock, S.at<void>(kPN)))) return e;
      k_scf_dev_out<<<1, 1, 0, cap.s>>>(d, S.scal(), it.scalars_out);
      HF_LAUNCH_CHECK("k_scf_dev_out");
      HF_CUDA(cudaEventRecordWithFlags(bg->t1[i], cap.s, cudaEventRecordExternal));
      if ((e = cap.end(nullptr))) return e;
    }
    HF_CUDA(cudaGraphInstantiate(&bg->exec, G, 0));
    HF_CUDA(cudaStreamCreateWithFlags(&bg->run, cudaStreamNonBlocking));
    HF_CUDA(cudaEventCreateWithFlags(&bg->ev_in, cudaEventDisableTiming));
    HF_CUDA(cudaEventCreateWithFlags(&bg->ev_out, cudaEventDisableTiming));
    return HF_OK;
  };
  st = build();
  if (cap.s) {
    if (st != HF_OK) {  // leave no capture open on an error path
      cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
      if (cudaStreamIsCapturing(cap.s, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(cap.s, &g);
      }
      cudaGetLastError();
    }
    cudaStreamDestroy(cap.s);
  }
  if (st != HF_OK) {
    delete bg;
    return st;
  }
  *handle = bg;
  return HF_OK;
}

extern "C" int hf_scf_batch_graph_launch(void* handle, void* stream, double* solve_ms) {
  if (!handle) return fail(HF_ERR_INVALID, "NULL batch graph");
  auto* bg = static_cast<ScfBatchGraph*>(handle);
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

extern "C" int hf_scf_batch_graph_destroy(void* handle) {
  delete static_cast<ScfBatchGraph*>(handle);
  return HF_OK;
}
