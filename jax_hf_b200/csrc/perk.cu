// Per-k small nb x nb kernels: one warp per matrix, matrices staged in shared
// memory (double precision internally, storage precision at the boundary).
//
// Eigendecomposition: cyclic Jacobi with complex Hermitian rotations in the
// round-robin parallel ordering (Jacobi 1846; Golub & Van Loan, Matrix
// Computations, sec. 8.5): each round applies nb/2 disjoint rotations at once
// (lanes over rows/columns), sweeps repeat until no off-diagonal entry exceeds
// 1e-17 ||A||_F (1e-8 in single precision) or 60 sweeps.  Eigenvalues are
// returned ascending, eigenvectors as columns (A = V diag(w) V^H), like LAPACK
// heevd; the input is hermitised first, as jnp.linalg.eigh does.
#include "common.cuh"
#include "perk.cuh"

namespace hf {

// ---------------------------------------------------------------- loads ----
template <typename RT>
__device__ __forceinline__ void load_mat(double2* dst, const cpx_t<RT>* src, int nb2, int lane) {
  for (int e = lane; e < nb2; e += 32) dst[e] = cvt<double2>(src[e]);
}
template <typename RT>
__device__ __forceinline__ void store_mat(cpx_t<RT>* dst, const double2* src, int nb2, int lane) {
  for (int e = lane; e < nb2; e += 32) dst[e] = cvt<cpx_t<RT>>(src[e]);
}

// ------------------------------------------------------------- density -----
template <typename RT>
__global__ void k_density(int batch, int nb, const cpx_t<RT>* __restrict__ Q, const RT* __restrict__ p,
                          cpx_t<RT>* __restrict__ P) {
  extern __shared__ double2 sm[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const int nb2 = nb * nb;
  double2* q = sm + (size_t)w * (2 * nb2 + nb);
  double2* t = q + nb2;
  double* pp = reinterpret_cast<double*>(t + nb2);
  for (int m = blockIdx.x * wpb + w; m < batch; m += gridDim.x * wpb) {
    load_mat<RT>(q, Q + (size_t)m * nb2, nb2, lane);
    for (int e = lane; e < nb; e += 32) pp[e] = (double)p[(size_t)m * nb + e];
    __syncwarp();
    warp_density(q, pp, t, nb, lane);
    __syncwarp();
    for (int e = lane; e < nb2; e += 32) {
      const int i = e / nb, j = e - i * nb;
      const double2 a = t[e], b = t[j * nb + i];
      P[(size_t)m * nb2 + e] = mk<cpx_t<RT>>(0.5 * (a.x + b.x), 0.5 * (a.y - b.y));
    }
    __syncwarp();
  }
}

// ----------------------------------------------------- Ft = Q^H F Q --------
template <typename RT>
__global__ void k_fock_orbital(int batch, int nb, const cpx_t<RT>* __restrict__ Q,
                               const cpx_t<RT>* __restrict__ F, cpx_t<RT>* __restrict__ Ft) {
  extern __shared__ double2 sm[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const int nb2 = nb * nb;
  double2* q = sm + (size_t)w * 3 * nb2;
  double2* f = q + nb2;
  double2* t = f + nb2;
  for (int m = blockIdx.x * wpb + w; m < batch; m += gridDim.x * wpb) {
    load_mat<RT>(q, Q + (size_t)m * nb2, nb2, lane);
    load_mat<RT>(f, F + (size_t)m * nb2, nb2, lane);
    __syncwarp();
    warp_qhaq(q, f, t, nb, lane);  // f <- Q^H F Q (t scratch)
    __syncwarp();
    store_mat<RT>(Ft + (size_t)m * nb2, f, nb2, lane);
    __syncwarp();
  }
}

// ---------------------------------------------------------------- eigh -----
template <typename RT>
__global__ void k_eigh(int batch, int nb, int mode, const cpx_t<RT>* __restrict__ A, RT* __restrict__ wout,
                       cpx_t<RT>* __restrict__ Vout) {
  extern __shared__ double2 sm[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const int nb2 = nb * nb;
  double2* a = sm + (size_t)w * jacobi_smem_elems(nb);
  double2* v = a + nb2;
  double2* scr = v + nb2;
  const double tol = sizeof(RT) == 8 ? 1e-17 : 1e-8;
  for (int m = blockIdx.x * wpb + w; m < batch; m += gridDim.x * wpb) {
    const cpx_t<RT>* src = A + (size_t)m * nb2;
    // hermitise (mode 0) or form herm(i d) (mode 1, Cayley spectral setup)
    for (int e = lane; e < nb2; e += 32) {
      const int i = e / nb, j = e - i * nb;
      double2 x = cvt<double2>(src[e]), y = cvt<double2>(src[j * nb + i]);
      if (mode == 1) { x = mul_pi(x); y = mul_pi(y); }
      a[e] = make_double2(0.5 * (x.x + y.x), 0.5 * (x.y - y.y));
    }
    __syncwarp();
    double* wv = reinterpret_cast<double*>(scr);
    warp_jacobi_eigh(a, v, scr + nb, nb, lane, tol);
    for (int e = lane; e < nb; e += 32) wv[e] = a[e * nb + e].x;
    __syncwarp();
    // ascending order (stable), eigenvectors as columns
    for (int i = lane; i < nb; i += 32) {
      const double wi = wv[i];
      int r = 0;
      for (int j = 0; j < nb; ++j) r += (wv[j] < wi) || (wv[j] == wi && j < i);
      wout[(size_t)m * nb + r] = (RT)wi;
      for (int row = 0; row < nb; ++row)
        Vout[(size_t)m * nb2 + row * nb + r] = cvt<cpx_t<RT>>(v[row * nb + i]);
    }
    __syncwarp();
  }
}

// ------------------------------------------------------- Cayley (LU) -------
template <typename RT>
__global__ void k_cayley_lu(int batch, int nb, const cpx_t<RT>* __restrict__ d, double tau,
                            const double* __restrict__ tau_dev, cpx_t<RT>* __restrict__ U) {
  extern __shared__ double2 sm[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const int nb2 = nb * nb;
  double2* M = sm + (size_t)w * 2 * nb2;
  double2* B = M + nb2;
  const double t = tau_dev ? tau_dev[0] : tau;
  for (int m = blockIdx.x * wpb + w; m < batch; m += gridDim.x * wpb) {
    for (int e = lane; e < nb2; e += 32) {
      const int i = e / nb, j = e - i * nb;
      double2 x = cvt<double2>(d[(size_t)m * nb2 + e]);
      x = make_double2(0.5 * t * x.x, 0.5 * t * x.y);
      const double id = (i == j) ? 1.0 : 0.0;
      M[e] = make_double2(id + x.x, x.y);
      B[e] = make_double2(id - x.x, -x.y);
    }
    __syncwarp();
    warp_lu_solve(M, B, nb, lane);
    store_mat<RT>(U + (size_t)m * nb2, B, nb2, lane);
    __syncwarp();
  }
}

// ------------------------------------------- Cayley from the spectrum ------
template <typename RT>
__global__ void k_cayley_unitary(int batch, int nb, const cpx_t<RT>* __restrict__ V, const RT* __restrict__ lam,
                                 double tau, const double* __restrict__ tau_dev, cpx_t<RT>* __restrict__ U) {
  extern __shared__ double2 sm[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const int nb2 = nb * nb;
  double2* v = sm + (size_t)w * (nb2 + nb);
  double2* c = v + nb2;
  const double t = tau_dev ? tau_dev[0] : tau;
  for (int m = blockIdx.x * wpb + w; m < batch; m += gridDim.x * wpb) {
    load_mat<RT>(v, V + (size_t)m * nb2, nb2, lane);
    for (int e = lane; e < nb; e += 32) c[e] = cayley_factor(t, (double)lam[(size_t)m * nb + e]);
    __syncwarp();
    for (int e = lane; e < nb2; e += 32) {
      const int i = e / nb, j = e - i * nb;
      double2 acc = make_double2(0.0, 0.0);
      for (int n = 0; n < nb; ++n) acc = cadd(acc, cmulc(cmul(v[i * nb + n], c[n]), v[j * nb + n]));
      U[(size_t)m * nb2 + e] = cvt<cpx_t<RT>>(acc);
    }
    __syncwarp();
  }
}

template <typename RT>
__global__ void k_diag_ufu(int batch, int nb, const cpx_t<RT>* __restrict__ V, const cpx_t<RT>* __restrict__ Fe,
                           const RT* __restrict__ lam, double tau, const double* __restrict__ tau_dev,
                           RT* __restrict__ out) {
  extern __shared__ double2 sm[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const int nb2 = nb * nb;
  double2* v = sm + (size_t)w * (2 * nb2 + nb);
  double2* f = v + nb2;
  double2* c = f + nb2;
  const double t = tau_dev ? tau_dev[0] : tau;
  for (int m = blockIdx.x * wpb + w; m < batch; m += gridDim.x * wpb) {
    load_mat<RT>(v, V + (size_t)m * nb2, nb2, lane);
    load_mat<RT>(f, Fe + (size_t)m * nb2, nb2, lane);
    for (int e = lane; e < nb; e += 32) c[e] = cayley_factor(t, (double)lam[(size_t)m * nb + e]);
    __syncwarp();
    for (int i = lane; i < nb; i += 32) out[(size_t)m * nb + i] = (RT)diag_ufu_row(v, f, c, nb, i);
    __syncwarp();
  }
}

// ---------------------------------------------------------- QR retract -----
template <typename RT>
__global__ void k_qr_retract(int batch, int nb, const cpx_t<RT>* __restrict__ G, double tau,
                             cpx_t<RT>* __restrict__ U) {
  extern __shared__ double2 sm[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  const int nb2 = nb * nb;
  double2* x = sm + (size_t)w * 2 * nb2;
  double2* q = x + nb2;
  for (int m = blockIdx.x * wpb + w; m < batch; m += gridDim.x * wpb) {
    for (int e = lane; e < nb2; e += 32) {
      const int i = e / nb, j = e - i * nb;
      double2 g = cvt<double2>(G[(size_t)m * nb2 + e]);
      x[e] = make_double2((i == j ? 1.0 : 0.0) - tau * g.x, -tau * g.y);
    }
    __syncwarp();
    warp_qr_cgs2(x, q, nb, lane);
    store_mat<RT>(U + (size_t)m * nb2, q, nb2, lane);
    __syncwarp();
  }
}

// ------------------------------------------------------------ launching ----
static int warps_per_block(size_t per_warp_bytes) {
  int wpb = 8;
  while (wpb > 1 && per_warp_bytes * wpb > 96 * 1024) wpb >>= 1;
  return wpb;
}

static int check_perk(int dtype, int batch, int nb) {
  if (dtype != HF_C128 && dtype != HF_C64) return fail(HF_ERR_INVALID, "bad dtype");
  if (batch < 0 || nb < 1) return fail(HF_ERR_INVALID, "bad shape");
  if (nb > 32) return fail(HF_ERR_UNSUPPORTED, "nb > 32 is not supported by this build");
  return HF_OK;
}

struct Launch {
  dim3 grid, block;
  size_t smem;
};

static Launch warp_launch(int batch, size_t per_warp_elems) {
  Launch L;
  const size_t bytes = per_warp_elems * sizeof(double2);
  const int wpb = warps_per_block(bytes);
  int blocks = (batch + wpb - 1) / wpb;
  if (blocks < 1) blocks = 1;
  if (blocks > 148 * 32) blocks = 148 * 32;
  L.grid = dim3(blocks);
  L.block = dim3(32 * wpb);
  L.smem = bytes * wpb;
  return L;
}

#define HF_SET_SMEM(kern, L) HF_SMEM_CAP(kern)

}  // namespace hf

using namespace hf;

extern "C" int hf_density_from_Qp(void* stream, int dtype, int batch, int nb, const void* Q, const void* p,
                                  void* P) {
  int st = check_perk(dtype, batch, nb);
  if (st) return st;
  if (batch == 0) return HF_OK;
  if (!Q || !p || !P) return fail(HF_ERR_INVALID, "NULL argument");
  // complex128 with nb <= 8: a group of lanes per k-point, one matrix column per lane
  if (dtype == HF_C128 && nb <= 8) return hf::rows_density(stream, batch, nb, Q, static_cast<const double*>(p), P);
  Launch L = warp_launch(batch, 2 * nb * nb + nb);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (dtype == HF_C128) {
    HF_SET_SMEM(k_density<double>, L);
    k_density<double><<<L.grid, L.block, L.smem, s>>>(batch, nb, (const double2*)Q, (const double*)p, (double2*)P);
  } else {
    HF_SET_SMEM(k_density<float>, L);
    k_density<float><<<L.grid, L.block, L.smem, s>>>(batch, nb, (const float2*)Q, (const float*)p, (float2*)P);
  }
  HF_LAUNCH_CHECK("k_density");
  return HF_OK;
}

extern "C" int hf_fock_orbital(void* stream, int dtype, int batch, int nb, const void* Q, const void* F,
                               void* Ft) {
  int st = check_perk(dtype, batch, nb);
  if (st) return st;
  if (batch == 0) return HF_OK;
  if (!Q || !F || !Ft) return fail(HF_ERR_INVALID, "NULL argument");
  Launch L = warp_launch(batch, 3 * nb * nb);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (dtype == HF_C128) {
    HF_SET_SMEM(k_fock_orbital<double>, L);
    k_fock_orbital<double><<<L.grid, L.block, L.smem, s>>>(batch, nb, (const double2*)Q, (const double2*)F, (double2*)Ft);
  } else {
    HF_SET_SMEM(k_fock_orbital<float>, L);
    k_fock_orbital<float><<<L.grid, L.block, L.smem, s>>>(batch, nb, (const float2*)Q, (const float2*)F, (float2*)Ft);
  }
  HF_LAUNCH_CHECK("k_fock_orbital");
  return HF_OK;
}

static int eigh_common(void* stream, int dtype, int batch, int nb, int mode, const void* A, void* w, void* V) {
  int st = check_perk(dtype, batch, nb);
  if (st) return st;
  if (batch == 0) return HF_OK;
  if (!A || !w || !V) return fail(HF_ERR_INVALID, "NULL argument");
  // complex128 with nb <= 8: a group of lanes per matrix, one column per lane
  if (dtype == HF_C128 && nb <= 8) return hf::eigh_cols(stream, batch, nb, A, static_cast<double*>(w), V, mode);
  Launch L = warp_launch(batch, jacobi_smem_elems(nb));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (dtype == HF_C128) {
    HF_SET_SMEM(k_eigh<double>, L);
    k_eigh<double><<<L.grid, L.block, L.smem, s>>>(batch, nb, mode, (const double2*)A, (double*)w, (double2*)V);
  } else {
    HF_SET_SMEM(k_eigh<float>, L);
    k_eigh<float><<<L.grid, L.block, L.smem, s>>>(batch, nb, mode, (const float2*)A, (float*)w, (float2*)V);
  }
  HF_LAUNCH_CHECK("k_eigh");
  return HF_OK;
}

extern "C" int hf_eigh(void* stream, int dtype, int batch, int nb, const void* A, void* w, void* V) {
  return eigh_common(stream, dtype, batch, nb, 0, A, w, V);
}

extern "C" int hf_cayley_spectral(void* stream, int dtype, int batch, int nb, const void* d, void* V,
                                  void* lam) {
  return eigh_common(stream, dtype, batch, nb, 1, d, lam, V);
}

extern "C" int hf_cayley_retract(void* stream, int dtype, int batch, int nb, const void* d, double tau,
                                 void* U) {
  int st = check_perk(dtype, batch, nb);
  if (st) return st;
  if (batch == 0) return HF_OK;
  if (!d || !U) return fail(HF_ERR_INVALID, "NULL argument");
  Launch L = warp_launch(batch, 2 * nb * nb);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (dtype == HF_C128) {
    HF_SET_SMEM(k_cayley_lu<double>, L);
    k_cayley_lu<double><<<L.grid, L.block, L.smem, s>>>(batch, nb, (const double2*)d, tau, nullptr, (double2*)U);
  } else {
    HF_SET_SMEM(k_cayley_lu<float>, L);
    k_cayley_lu<float><<<L.grid, L.block, L.smem, s>>>(batch, nb, (const float2*)d, tau, nullptr, (float2*)U);
  }
  HF_LAUNCH_CHECK("k_cayley_lu");
  return HF_OK;
}

extern "C" int hf_cayley_unitary(void* stream, int dtype, int batch, int nb, const void* V, const void* lam,
                                 double tau, void* U) {
  int st = check_perk(dtype, batch, nb);
  if (st) return st;
  if (batch == 0) return HF_OK;
  if (!V || !lam || !U) return fail(HF_ERR_INVALID, "NULL argument");
  Launch L = warp_launch(batch, nb * nb + nb);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (dtype == HF_C128) {
    HF_SET_SMEM(k_cayley_unitary<double>, L);
    k_cayley_unitary<double><<<L.grid, L.block, L.smem, s>>>(batch, nb, (const double2*)V, (const double*)lam, tau,
                                                             nullptr, (double2*)U);
  } else {
    HF_SET_SMEM(k_cayley_unitary<float>, L);
    k_cayley_unitary<float><<<L.grid, L.block, L.smem, s>>>(batch, nb, (const float2*)V, (const float*)lam, tau,
                                                            nullptr, (float2*)U);
  }
  HF_LAUNCH_CHECK("k_cayley_unitary");
  return HF_OK;
}

extern "C" int hf_diag_UFU(void* stream, int dtype, int batch, int nb, const void* V, const void* Ft_eig,
                           const void* lam, double tau, void* diag) {
  int st = check_perk(dtype, batch, nb);
  if (st) return st;
  if (batch == 0) return HF_OK;
  if (!V || !Ft_eig || !lam || !diag) return fail(HF_ERR_INVALID, "NULL argument");
  Launch L = warp_launch(batch, 2 * nb * nb + nb);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (dtype == HF_C128) {
    HF_SET_SMEM(k_diag_ufu<double>, L);
    k_diag_ufu<double><<<L.grid, L.block, L.smem, s>>>(batch, nb, (const double2*)V, (const double2*)Ft_eig,
                                                       (const double*)lam, tau, nullptr, (double*)diag);
  } else {
    HF_SET_SMEM(k_diag_ufu<float>, L);
    k_diag_ufu<float><<<L.grid, L.block, L.smem, s>>>(batch, nb, (const float2*)V, (const float2*)Ft_eig,
                                                      (const float*)lam, tau, nullptr, (float*)diag);
  }
  HF_LAUNCH_CHECK("k_diag_ufu");
  return HF_OK;
}

extern "C" int hf_qr_retract(void* stream, int dtype, int batch, int nb, const void* G, double tau, void* U) {
  int st = check_perk(dtype, batch, nb);
  if (st) return st;
  if (batch == 0) return HF_OK;
  if (!G || !U) return fail(HF_ERR_INVALID, "NULL argument");
  Launch L = warp_launch(batch, 2 * nb * nb);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (dtype == HF_C128) {
    HF_SET_SMEM(k_qr_retract<double>, L);
    k_qr_retract<double><<<L.grid, L.block, L.smem, s>>>(batch, nb, (const double2*)G, tau, (double2*)U);
  } else {
    HF_SET_SMEM(k_qr_retract<float>, L);
    k_qr_retract<float><<<L.grid, L.block, L.smem, s>>>(batch, nb, (const float2*)G, tau, (float2*)U);
  }
  HF_LAUNCH_CHECK("k_qr_retract");
  return HF_OK;
}
