// Reverse-mode pieces of the Fock build and the HF objective (complex128).
//
// The exchange self-energy is a C-linear map of dP = P - refP,
//   Sigma = A(dP) = -IFFT2(VR . FFT2(dP))          (utils.py:164-173),
// so its vector-Jacobian product is the Hermitian adjoint
//   A^H(X) = -IFFT2(conj(VR) . FFT2(X)),
// i.e. the same Fock-build kernels run on the cotangent with conj(VR)
// (VR itself when it is real).  F = herm(h + Sigma + H) (fock.py:94) is
// self-adjoint in the real inner product Re tr(X^H Y), so the cotangent that
// reaches Sigma is Sigma_bar + herm(F_bar) and h_bar = herm(F_bar).
// Gradients follow torch's convention for complex leaves (d/dRe + i d/dIm).
//
// hf_energy_vjp / hf_free_energy_vjp differentiate fock.py:100-129;
// hf_fourier_coeffs gives the h_R gradients of an energy whose h(k) is the
// Fourier series sum_R h_R e^{i k.R} (the synthetic Hamiltonians of the
// benchmarks, with k on the centred grid 2 pi (m - n/2) / n).
#include <cmath>

#include "common.cuh"

namespace hf {

int fock_build_internal(void* stream, int dtype, unsigned flags, int nk1, int nk2, int nb, const void* P,
                        const void* h, const void* VR, const void* refP, const void* HH, const void* w2d,
                        int n_contact, const void* contact_g, const void* contact_Oi, const void* contact_Oj,
                        void* Sigma, void* H, void* F, void* workspace, size_t workspace_bytes,
                        const int* active);

constexpr int kAdjThreads = 256;

static int adj_blocks(size_t n) {
  size_t b = (n + kAdjThreads - 1) / kAdjThreads;
  if (b > (size_t)148 * 16) b = 148 * 16;
  return b < 1 ? 1 : (int)b;
}

static unsigned vjp_flags(unsigned flags) {
  // exchange of an arbitrary (non-Hermitian) cotangent: every channel, no refP, no Hartree
  return (flags & (HF_FOCK_EXCHANGE | HF_FOCK_VR_SCALAR | HF_FOCK_VR_REAL | HF_FOCK_GENERIC_FFT));
}

// X = Sigma_bar + herm(F_bar); h_bar = herm(F_bar)
__global__ void k_vjp_xbar(size_t nk, int nb, const double2* __restrict__ Sb, const double2* __restrict__ Fb,
                           double2* __restrict__ X, double2* __restrict__ hb) {
  const size_t nb2 = (size_t)nb * nb, n = nk * nb2;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const size_t k = e / nb2;
    const int r = (int)(e - k * nb2), i = r / nb, j = r - i * nb;
    double2 hf = make_double2(0.0, 0.0);
    if (Fb) {
      const double2 a = Fb[e], b = Fb[k * nb2 + (size_t)j * nb + i];
      hf = make_double2(0.5 * (a.x + b.x), 0.5 * (a.y - b.y));
    }
    const double2 s = Sb ? Sb[e] : make_double2(0.0, 0.0);
    X[e] = make_double2(s.x + hf.x, s.y + hf.y);
    if (hb) hb[e] = hf;
  }
}

// E = Re sum_k w_k sum_ij (h + (Sigma + H)/2)_ij P_ji  ->  P_bar = Eb w A^H, h_bar = Eb w P^H,
// Sigma_bar = Eb w P^H / 2 (the shared H's cotangent is a k-sum formed by the caller).
__global__ void k_energy_vjp(size_t nk, int nb, const double2* __restrict__ P, const double2* __restrict__ h,
                             const double2* __restrict__ S, const double2* __restrict__ H, int H_mode,
                             const double* __restrict__ w, double Eb, double2* __restrict__ Pb,
                             double2* __restrict__ hb, double2* __restrict__ Sb) {
  const size_t nb2 = (size_t)nb * nb, n = nk * nb2;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const size_t k = e / nb2;
    const int r = (int)(e - k * nb2), i = r / nb, j = r - i * nb;
    const size_t t = k * nb2 + (size_t)j * nb + i;  // transposed element
    const double s = Eb * w[k];
    if (Pb) {  // Pb_ij = s conj(A_ji)
      double ax = S[t].x, ay = S[t].y;
      if (H_mode == 1) {
        ax += H[(size_t)j * nb + i].x;
        ay += H[(size_t)j * nb + i].y;
      } else if (H_mode == 2) {
        ax += H[t].x;
        ay += H[t].y;
      }
      ax = h[t].x + 0.5 * ax;
      ay = h[t].y + 0.5 * ay;
      Pb[e] = make_double2(s * ax, -s * ay);
    }
    const double2 pt = P[t];  // (P^H)_ij = conj(P_ji)
    if (hb) hb[e] = make_double2(s * pt.x, -s * pt.y);
    if (Sb) Sb[e] = make_double2(0.5 * s * pt.x, -0.5 * s * pt.y);
  }
}

// Omega = E - max(T, 1e-14) S(p), S = -sum_k wn_k sum_i s(clip(p)), s(p) = p log p + (1-p) log1p(-p):
// p_bar = Ob T wn (log p - log1p(-p)) inside the clip range, 0 outside (fock.py:114-129).
__global__ void k_free_energy_vjp(size_t n, int nb, const double* __restrict__ p, const double* __restrict__ wn,
                                  double T, double Ob, double* __restrict__ pb) {
  const double Tm = fmax(T, 1e-14);
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const double pv = p[e];
    double g = 0.0;
    if (pv > 1e-14 && pv < 1.0 - 1e-14) g = Ob * Tm * wn[e / nb] * (log(pv) - log1p(-pv));
    pb[e] = g;
  }
}

// out[R][i][j] = sum_k w_k e^{-i k.R} P_k[i][j]; one CTA per (R, i, j), compensated sums.
__global__ void __launch_bounds__(kAdjThreads)
k_fourier_coeffs(int nk1, int nk2, int nb, const double2* __restrict__ P, const double* __restrict__ w,
                 const int* __restrict__ R, double2* __restrict__ out) {
  __shared__ double sm[64];
  const int ij = blockIdx.x, rid = blockIdx.y;
  const int Rx = R[2 * rid], Ry = R[2 * rid + 1];
  const int nb2 = nb * nb, nk = nk1 * nk2;
  const int c1 = nk1 / 2, c2 = nk2 / 2;
  KSum re, im;
  for (int k = threadIdx.x; k < nk; k += blockDim.x) {
    const int m1 = k / nk2, m2 = k - m1 * nk2;
    // phase / pi = -2 ((m1 - c1) Rx / nk1 + (m2 - c2) Ry / nk2), reduced exactly in integers first
    const long long a1 = (long long)(m1 - c1) * Rx, a2 = (long long)(m2 - c2) * Ry;
    const double t = -2.0 * ((double)(((a1 % nk1) + nk1) % nk1) / nk1 + (double)(((a2 % nk2) + nk2) % nk2) / nk2);
    double sn, cs;
    sincospi(t, &sn, &cs);
    const double2 pv = P[(size_t)k * nb2 + ij];
    const double wk = w[k];
    re.add(wk * (cs * pv.x - sn * pv.y));
    im.add(wk * (cs * pv.y + sn * pv.x));
  }
  const KSum rr = block_reduce(re, sm);
  __syncthreads();
  const KSum ri = block_reduce(im, sm);
  if (threadIdx.x == 0) out[(size_t)rid * nb2 + ij] = make_double2(rr.value(), ri.value());
}

}  // namespace hf

using namespace hf;

extern "C" int hf_fock_vjp_workspace_size(int dtype, unsigned flags, int nk1, int nk2, int nb, size_t* bytes) {
  if (!bytes) return fail(HF_ERR_INVALID, "bytes is NULL");
  if (dtype != HF_C128) return fail(HF_ERR_UNSUPPORTED, "the Fock-build VJP is complex128 only");
  if (nk1 < 1 || nk2 < 1 || nb < 1) return fail(HF_ERR_INVALID, "bad shape");
  size_t fws = 0;
  if (flags & HF_FOCK_EXCHANGE) {
    const int st = hf_fock_workspace_size(dtype, vjp_flags(flags), nk1, nk2, nb, &fws);
    if (st) return st;
  }
  const size_t nq = (size_t)nk1 * nk2 * nb * nb * sizeof(double2);
  *bytes = align_up(fws, 256) + 2 * align_up(nq, 256);
  return HF_OK;
}

extern "C" int hf_fock_build_vjp(void* stream, int dtype, unsigned flags, int nk1, int nk2, int nb,
                                 const void* Sigma_bar, const void* F_bar, const void* VR_adj, void* P_bar,
                                 void* h_bar, void* workspace, size_t workspace_bytes) {
  size_t need = 0;
  int st = hf_fock_vjp_workspace_size(dtype, flags, nk1, nk2, nb, &need);
  if (st) return st;
  if (!P_bar || (!Sigma_bar && !F_bar)) return fail(HF_ERR_INVALID, "P_bar and a cotangent must be non-NULL");
  if ((flags & HF_FOCK_EXCHANGE) && !VR_adj) return fail(HF_ERR_INVALID, "VR_adj must be non-NULL");
  if (!workspace || workspace_bytes < need)
    return fail(HF_ERR_WORKSPACE, "workspace too small: need " + std::to_string(need) + " bytes");
  if (reinterpret_cast<uintptr_t>(workspace) % 256 != 0)
    return fail(HF_ERR_WORKSPACE, "workspace must be 256-byte aligned");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t nk = (size_t)nk1 * nk2, nq = nk * nb * nb;
  size_t fws = 0;
  if (flags & HF_FOCK_EXCHANGE) hf_fock_workspace_size(dtype, vjp_flags(flags), nk1, nk2, nb, &fws);
  char* ws = static_cast<char*>(workspace);
  double2* X = reinterpret_cast<double2*>(ws + align_up(fws, 256));
  double2* Fs = X + align_up(nq * sizeof(double2), 256) / sizeof(double2);
  k_vjp_xbar<<<adj_blocks(nq), kAdjThreads, 0, s>>>(nk, nb, static_cast<const double2*>(Sigma_bar),
                                                   static_cast<const double2*>(F_bar), X,
                                                   static_cast<double2*>(h_bar));
  HF_LAUNCH_CHECK("k_vjp_xbar");
  if (!(flags & HF_FOCK_EXCHANGE)) {
    HF_CUDA(cudaMemsetAsync(P_bar, 0, nq * sizeof(double2), s));
    return HF_OK;
  }
  // P_bar = A^H(X): the Sigma output of a build of X with conj(VR); its F output (scratch) is discarded
  return fock_build_internal(stream, HF_C128, vjp_flags(flags), nk1, nk2, nb, X, X, VR_adj, nullptr, nullptr,
                             nullptr, 0, nullptr, nullptr, nullptr, P_bar, nullptr, Fs, ws, fws, nullptr);
}

extern "C" int hf_energy_vjp(void* stream, int nk1, int nk2, int nb, const void* P, const void* h,
                             const void* Sigma, const void* H, int H_mode, const double* w2d, double E_bar,
                             void* P_bar, void* h_bar, void* Sigma_bar) {
  if (nk1 < 1 || nk2 < 1 || nb < 1) return fail(HF_ERR_INVALID, "bad shape");
  if (!P || !w2d) return fail(HF_ERR_INVALID, "P and w2d must be non-NULL");
  if (H_mode < 0 || H_mode > 2) return fail(HF_ERR_INVALID, "H_mode must be 0, 1 or 2");
  if (P_bar && (!h || !Sigma || (H_mode != 0 && !H))) return fail(HF_ERR_INVALID, "P_bar needs h, Sigma and H");
  const size_t nq = (size_t)nk1 * nk2 * nb * nb;
  k_energy_vjp<<<adj_blocks(nq), kAdjThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      (size_t)nk1 * nk2, nb, static_cast<const double2*>(P), static_cast<const double2*>(h),
      static_cast<const double2*>(Sigma), static_cast<const double2*>(H), H_mode, w2d, E_bar,
      static_cast<double2*>(P_bar), static_cast<double2*>(h_bar), static_cast<double2*>(Sigma_bar));
  HF_LAUNCH_CHECK("k_energy_vjp");
  return HF_OK;
}

extern "C" int hf_free_energy_vjp(void* stream, int nk1, int nk2, int nb, const double* p, const double* w_norm,
                                  double T, double Omega_bar, double* p_bar) {
  if (nk1 < 1 || nk2 < 1 || nb < 1) return fail(HF_ERR_INVALID, "bad shape");
  if (!p || !w_norm || !p_bar) return fail(HF_ERR_INVALID, "NULL argument");
  const size_t n = (size_t)nk1 * nk2 * nb;
  k_free_energy_vjp<<<adj_blocks(n), kAdjThreads, 0, static_cast<cudaStream_t>(stream)>>>(n, nb, p, w_norm, T,
                                                                                          Omega_bar, p_bar);
  HF_LAUNCH_CHECK("k_free_energy_vjp");
  return HF_OK;
}

extern "C" int hf_fourier_coeffs(void* stream, int nk1, int nk2, int nb, const void* P, const double* w2d,
                                 int nR, const int* R, void* out) {
  if (nk1 < 1 || nk2 < 1 || nb < 1 || nR < 1) return fail(HF_ERR_INVALID, "bad shape");
  if (!P || !w2d || !R || !out) return fail(HF_ERR_INVALID, "NULL argument");
  if (nb * nb > 65535 || nR > 65535) return fail(HF_ERR_UNSUPPORTED, "too many channels or lattice vectors");
  const dim3 grid(nb * nb, nR);
  k_fourier_coeffs<<<grid, kAdjThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      nk1, nk2, nb, static_cast<const double2*>(P), w2d, R, static_cast<double2*>(out));
  HF_LAUNCH_CHECK("k_fourier_coeffs");
  return HF_OK;
}
