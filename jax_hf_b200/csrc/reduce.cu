// Compensated objective reductions: hf_energy, occupation entropy, free energy.
//
// fock.py:100-129.  Two launches per reduction: a grid of CTAs forms Neumaier
// partial sums over a grid-stride range, a single CTA then combines the
// partials in a fixed order, so the result is deterministic for a given shape.
#include "common.cuh"

namespace hf {

constexpr int kRedThreads = 256;
constexpr int kRedMaxBlocks = 148 * 8;

static int red_blocks(size_t n) {
  size_t b = (n + kRedThreads * 4 - 1) / (kRedThreads * 4);
  if (b < 1) b = 1;
  if (b > (size_t)kRedMaxBlocks) b = kRedMaxBlocks;
  return (int)b;
}

__global__ void k_red_final(const double* __restrict__ part, int nparts, int mode, double T,
                            const double* __restrict__ E, double* __restrict__ out, const int* active) {
  if (active && !*active) return;
  __shared__ double sm[64];
  KSum acc;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) {
    acc.add(part[2 * i]);
    acc.add(part[2 * i + 1]);
  }
  KSum r = block_reduce(acc, sm);
  if (threadIdx.x == 0) {
    double v = r.value();
    if (mode == 1) v = -v;                                  // entropy S
    if (mode == 2) v = E[0] - fmax(T, 1e-14) * (-v);        // free energy
    out[0] = v;
  }
}

template <typename RT>
__global__ void __launch_bounds__(kRedThreads)
k_energy_part(int nk, int nb, const cpx_t<RT>* __restrict__ P, const cpx_t<RT>* __restrict__ h,
              const cpx_t<RT>* __restrict__ S, const cpx_t<RT>* __restrict__ H, int H_mode,
              const RT* __restrict__ w, double* __restrict__ part, const int* active) {
  if (active && !*active) return;
  __shared__ double sm[64];
  const int nb2 = nb * nb;
  const size_t n = (size_t)nk * nb2;
  KSum acc;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const size_t k = e / nb2;
    const int rem = (int)(e - k * nb2);
    const int i = rem / nb, j = rem - (rem / nb) * nb;
    const cpx_t<RT> hv = h[e], sv = S[e];
    double xr = (double)sv.x, xi = (double)sv.y;
    if (H_mode == 1) { xr += (double)H[rem].x; xi += (double)H[rem].y; }
    else if (H_mode == 2) { xr += (double)H[e].x; xi += (double)H[e].y; }
    xr = (double)hv.x + 0.5 * xr;
    xi = (double)hv.y + 0.5 * xi;
    const cpx_t<RT> pv = P[k * nb2 + (size_t)j * nb + i];
    const double wk = (double)w[k];
    acc.add(wk * (xr * (double)pv.x - xi * (double)pv.y));
  }
  KSum r = block_reduce(acc, sm);
  if (threadIdx.x == 0) { part[2 * blockIdx.x] = r.s; part[2 * blockIdx.x + 1] = r.c; }
}

// sum_k w_k sum_i [p log p + (1-p) log1p(-p)], p clipped to [1e-14, 1-1e-14]
template <typename RT>
__global__ void __launch_bounds__(kRedThreads)
k_entropy_part(int nk, int nb, const RT* __restrict__ p, const RT* __restrict__ w,
               double* __restrict__ part) {
  __shared__ double sm[64];
  const size_t n = (size_t)nk * nb;
  KSum acc;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    double ps = fmin(fmax((double)p[e], 1e-14), 1.0 - 1e-14);
    double s = ps * log(ps) + (1.0 - ps) * log1p(-ps);
    acc.add((double)w[e / nb] * s);
  }
  KSum r = block_reduce(acc, sm);
  if (threadIdx.x == 0) { part[2 * blockIdx.x] = r.s; part[2 * blockIdx.x + 1] = r.c; }
}

static int check_ws(void* ws, size_t bytes, int nblocks) {
  if (!ws || bytes < (size_t)nblocks * 2 * sizeof(double))
    return fail(HF_ERR_WORKSPACE, "reduction workspace too small");
  return HF_OK;
}

}  // namespace hf

using namespace hf;

extern "C" int hf_reduce_workspace_size(int nk1, int nk2, int nb, size_t* bytes) {
  if (!bytes) return fail(HF_ERR_INVALID, "bytes is NULL");
  (void)nk1; (void)nk2; (void)nb;
  *bytes = (size_t)kRedMaxBlocks * 2 * sizeof(double);
  return HF_OK;
}

namespace hf {
int energy_internal(void* stream, int dtype, int nk1, int nk2, int nb, const void* P, const void* h,
                    const void* Sigma, const void* H, int H_mode, const void* w2d, double* E_out,
                    void* workspace, size_t workspace_bytes, const int* active);
}

extern "C" int hf_energy(void* stream, int dtype, int nk1, int nk2, int nb, const void* P,
                         const void* h, const void* Sigma, const void* H, int H_mode,
                         const void* w2d, double* E_out, void* workspace, size_t workspace_bytes) {
  return hf::energy_internal(stream, dtype, nk1, nk2, nb, P, h, Sigma, H, H_mode, w2d, E_out, workspace,
                             workspace_bytes, nullptr);
}

int hf::energy_internal(void* stream, int dtype, int nk1, int nk2, int nb, const void* P, const void* h,
                        const void* Sigma, const void* H, int H_mode, const void* w2d, double* E_out,
                        void* workspace, size_t workspace_bytes, const int* active) {
  if (dtype != HF_C128 && dtype != HF_C64) return fail(HF_ERR_INVALID, "bad dtype");
  if (nk1 < 1 || nk2 < 1 || nb < 1) return fail(HF_ERR_INVALID, "bad shape");
  if (!P || !h || !Sigma || !w2d || !E_out) return fail(HF_ERR_INVALID, "NULL argument");
  if (H_mode < 0 || H_mode > 2 || (H_mode > 0 && !H)) return fail(HF_ERR_INVALID, "bad H_mode");
  const int nk = nk1 * nk2;
  const int nbk = red_blocks((size_t)nk * nb * nb);
  int st = check_ws(workspace, workspace_bytes, nbk);
  if (st) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double* part = static_cast<double*>(workspace);
  if (dtype == HF_C128)
    k_energy_part<double><<<nbk, kRedThreads, 0, s>>>(nk, nb, (const double2*)P, (const double2*)h,
                                                      (const double2*)Sigma, (const double2*)H, H_mode,
                                                      (const double*)w2d, part, active);
  else
    k_energy_part<float><<<nbk, kRedThreads, 0, s>>>(nk, nb, (const float2*)P, (const float2*)h,
                                                     (const float2*)Sigma, (const float2*)H, H_mode,
                                                     (const float*)w2d, part, active);
  HF_LAUNCH_CHECK("k_energy_part");
  k_red_final<<<1, 256, 0, s>>>(part, nbk, 0, 0.0, nullptr, E_out, active);
  HF_LAUNCH_CHECK("k_red_final");
  return HF_OK;
}

static int entropy_common(void* stream, int dtype, int nk1, int nk2, int nb, const void* p,
                          const void* w_norm, int mode, double T, const double* E, double* out,
                          void* workspace, size_t workspace_bytes) {
  if (dtype != HF_C128 && dtype != HF_C64) return fail(HF_ERR_INVALID, "bad dtype");
  if (nk1 < 1 || nk2 < 1 || nb < 1) return fail(HF_ERR_INVALID, "bad shape");
  if (!p || !w_norm || !out) return fail(HF_ERR_INVALID, "NULL argument");
  const int nk = nk1 * nk2;
  const int nbk = red_blocks((size_t)nk * nb);
  int st = check_ws(workspace, workspace_bytes, nbk);
  if (st) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double* part = static_cast<double*>(workspace);
  if (dtype == HF_C128)
    k_entropy_part<double><<<nbk, kRedThreads, 0, s>>>(nk, nb, (const double*)p, (const double*)w_norm, part);
  else
    k_entropy_part<float><<<nbk, kRedThreads, 0, s>>>(nk, nb, (const float*)p, (const float*)w_norm, part);
  HF_LAUNCH_CHECK("k_entropy_part");
  k_red_final<<<1, 256, 0, s>>>(part, nbk, mode, T, E, out, nullptr);
  HF_LAUNCH_CHECK("k_red_final");
  return HF_OK;
}

extern "C" int hf_occupation_entropy(void* stream, int dtype, int nk1, int nk2, int nb, const void* p,
                                     const void* w_norm, double* S_out, void* workspace,
                                     size_t workspace_bytes) {
  return entropy_common(stream, dtype, nk1, nk2, nb, p, w_norm, 1, 0.0, nullptr, S_out, workspace,
                        workspace_bytes);
}

extern "C" int hf_free_energy(void* stream, int dtype, int nk1, int nk2, int nb, const double* E,
                              const void* p, const void* w_norm, double T, double* Omega_out,
                              void* workspace, size_t workspace_bytes) {
  if (!E) return fail(HF_ERR_INVALID, "E is NULL");
  return entropy_common(stream, dtype, nk1, nk2, nb, p, w_norm, 2, T, E, Omega_out, workspace,
                        workspace_bytes);
}
