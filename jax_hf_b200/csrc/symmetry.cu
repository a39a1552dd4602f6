// Symmetry averaging of (nk1, nk2, nb, nb) k-grid matrices (symmetry.py:22-150):
// group averages out(k) = (1/N) sum_g U_g A(k_g) U_g^H over elements applied at
// the same k and elements applied at a mapped k (axis flip, periodic negation
// or a per-element index map), and the time-reversal average
// out(k) = (A(k) + U conj(A(-k)) U^H) / 2.  A mask leaves A(k) unchanged where
// it is zero (finite patches whose orbit leaves the sampled region).
//
// A CTA of 256 threads takes KPB = 256 / nb^2 k-points (at least one); each
// thread owns up to four matrix elements of one k-point.  For every group
// element the CTA stages U_g and the gathered A(k_g) in shared memory, forms
// T = U_g A(k_g), then accumulates (T U_g^H)_ab in registers: 2 nb complex
// multiply-adds per element and group element, reads of A are whole matrices.
#include "common.cuh"

namespace hf {

constexpr int kSymThreads = 256;
constexpr int kSymMaxNb = 32;

struct SymArgs {
  int nk1, nk2, nb, kpb;
  int n_same, n_mapped;
  const void* G_same;    // (n_same, nb, nb)
  const void* G_mapped;  // (n_mapped, nb, nb)
  int k_mode, flip_axes;
  const int* idx_i;      // (n_mapped, nk1, nk2) or (nk1, nk2) for time reversal
  const int* idx_j;
  const unsigned char* mask;
  int time_reversal;
};

__device__ __forceinline__ int map_axis(int i, int n, int mode, bool on) {
  if (!on) return i;
  return mode == HF_K_FLIP ? n - 1 - i : (n - i) % n;
}

template <typename R>
__global__ void __launch_bounds__(kSymThreads) k_sym_average(const __grid_constant__ SymArgs s, const cpx_t<R>* __restrict__ A,
                                                             cpx_t<R>* __restrict__ out) {
  using C = cpx_t<R>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int nb = s.nb, nb2 = nb * nb, kpb = s.kpb;
  C* U = reinterpret_cast<C*>(smem_raw);  // nb2
  C* As = U + nb2;                        // kpb * nb2
  C* Ts = As + kpb * nb2;                 // kpb * nb2
  const int nk = s.nk1 * s.nk2;
  const int per = kpb * nb2;
  const int N = s.n_same + s.n_mapped;
  const C* Gs = static_cast<const C*>(s.G_same);
  const C* Gm = static_cast<const C*>(s.G_mapped);
  for (int k0 = blockIdx.x * kpb; k0 < nk; k0 += gridDim.x * kpb) {
    C acc[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) acc[r] = mk<C>(0.0, 0.0);
    for (int g = 0; g < N; ++g) {
      const bool same = g < s.n_same;
      const int gm = g - s.n_same;
      const C* Ug = same ? Gs + (size_t)g * nb2 : Gm + (size_t)gm * nb2;
      __syncthreads();  // the previous element's U, A, T are no longer read
      for (int e = threadIdx.x; e < nb2; e += kSymThreads) U[e] = Ug[e];
      for (int e = threadIdx.x; e < per; e += kSymThreads) {
        const int kl = e / nb2, c = e - kl * nb2, k = k0 + kl;
        C v = mk<C>(0.0, 0.0);
        if (k < nk) {
          const int i = k / s.nk2, j = k - i * s.nk2;
          int ii = i, jj = j;
          if (!same) {
            if (s.k_mode == HF_K_INDEX_MAP) {
              const size_t off = (s.time_reversal ? 0 : (size_t)gm * nk) + k;
              ii = s.idx_i[off];
              jj = s.idx_j[off];
              if (ii < 0 || ii >= s.nk1 || jj < 0 || jj >= s.nk2) {  // out-of-range entry: identity map
                ii = i;
                jj = j;
              }
            } else {
              ii = map_axis(i, s.nk1, s.k_mode, (s.flip_axes & 1) != 0);
              jj = map_axis(j, s.nk2, s.k_mode, (s.flip_axes & 2) != 0);
            }
          }
          v = A[((size_t)ii * s.nk2 + jj) * nb2 + c];
          if (s.time_reversal) v.y = -v.y;
        }
        As[e] = v;
      }
      __syncthreads();
      for (int e = threadIdx.x; e < per; e += kSymThreads) {  // T = U A
        const int kl = e / nb2, c = e - kl * nb2, a = c / nb, b = c - a * nb;
        const C* Ak = As + kl * nb2;
        C t = mk<C>(0.0, 0.0);
        for (int q = 0; q < nb; ++q) t = cadd(t, cmul(U[a * nb + q], Ak[q * nb + b]));
        Ts[e] = t;
      }
      __syncthreads();
      int r = 0;
      for (int e = threadIdx.x; e < per; e += kSymThreads, ++r) {  // acc += T U^H
        const int kl = e / nb2, c = e - kl * nb2, a = c / nb, b = c - a * nb;
        const C* Tk = Ts + kl * nb2;
        C t = mk<C>(0.0, 0.0);
        for (int q = 0; q < nb; ++q) t = cadd(t, cmulc(Tk[a * nb + q], U[b * nb + q]));
        acc[r] = cadd(acc[r], t);
      }
    }
    int r = 0;
    for (int e = threadIdx.x; e < per; e += kSymThreads, ++r) {
      const int kl = e / nb2, c = e - kl * nb2, k = k0 + kl;
      if (k >= nk) continue;
      const size_t o = (size_t)k * nb2 + c;
      const C a0 = A[o];
      C v;
      if (s.mask && !s.mask[k]) {
        v = a0;
      } else if (s.time_reversal) {
        v = mk<C>(R(0.5) * (a0.x + acc[r].x), R(0.5) * (a0.y + acc[r].y));
      } else {
        v = mk<C>(acc[r].x / (R)N, acc[r].y / (R)N);
      }
      out[o] = v;
    }
  }
}

template <typename R>
static int launch_sym(const SymArgs& s, const void* A, void* out, cudaStream_t stream) {
  const size_t sm = (size_t)(s.nb * s.nb + 2 * s.kpb * s.nb * s.nb) * sizeof(cpx_t<R>);
  const int nk = s.nk1 * s.nk2;
  int grid = (nk + s.kpb - 1) / s.kpb;
  if (grid > 148 * 8) grid = 148 * 8;
  k_sym_average<R><<<grid, kSymThreads, sm, stream>>>(s, static_cast<const cpx_t<R>*>(A), static_cast<cpx_t<R>*>(out));
  HF_LAUNCH_CHECK("k_sym_average");
  return HF_OK;
}

static int sym_common(int dtype, int nk1, int nk2, int nb, const void* A, const void* out, int k_mode) {
  if (dtype != HF_C128 && dtype != HF_C64) return fail(HF_ERR_INVALID, "dtype must be HF_C128 or HF_C64");
  if (nk1 <= 0 || nk2 <= 0 || nb <= 0) return fail(HF_ERR_INVALID, "nk1, nk2 and nb must be positive");
  if (nb > kSymMaxNb) return fail(HF_ERR_UNSUPPORTED, "symmetry averaging supports nb <= 32");
  if (!A || !out) return fail(HF_ERR_INVALID, "A and out must be non-NULL");
  if (A == out) return fail(HF_ERR_INVALID, "A and out must not alias (A is read at other k-points)");
  if (k_mode != HF_K_FLIP && k_mode != HF_K_MOD && k_mode != HF_K_INDEX_MAP)
    return fail(HF_ERR_INVALID, "k_convention must be 'mod' or 'flip'");
  return HF_OK;
}

static int kpb_for(int nb) {
  const int k = kSymThreads / (nb * nb);
  return k < 1 ? 1 : k;
}

}  // namespace hf

using namespace hf;

extern "C" int hf_sym_group_average(void* stream, int dtype, int nk1, int nk2, int nb, const void* A, void* out,
                                    int n_same, const void* G_same, int n_mapped, const void* G_mapped, int k_mode,
                                    int flip_axes, const int* idx_i, const int* idx_j, const unsigned char* mask) {
  int st = sym_common(dtype, nk1, nk2, nb, A, out, k_mode);
  if (st) return st;
  if (n_same < 0 || n_mapped < 0 || n_same + n_mapped < 1) return fail(HF_ERR_INVALID, "the group has no elements");
  if ((n_same > 0 && !G_same) || (n_mapped > 0 && !G_mapped)) return fail(HF_ERR_INVALID, "group matrices are NULL");
  if (n_mapped > 0 && k_mode == HF_K_INDEX_MAP && (!idx_i || !idx_j))
    return fail(HF_ERR_INVALID, "index-map mode needs idx_i and idx_j");
  SymArgs s{nk1, nk2, nb, kpb_for(nb), n_same, n_mapped, G_same, G_mapped, k_mode, flip_axes, idx_i, idx_j, mask, 0};
  cudaStream_t cs = static_cast<cudaStream_t>(stream);
  return dtype == HF_C128 ? launch_sym<double>(s, A, out, cs) : launch_sym<float>(s, A, out, cs);
}

extern "C" int hf_sym_time_reversal(void* stream, int dtype, int nk1, int nk2, int nb, const void* A, void* out,
                                    const void* U, int k_mode, int flip_axes, const int* idx_i, const int* idx_j,
                                    const unsigned char* valid) {
  int st = sym_common(dtype, nk1, nk2, nb, A, out, k_mode);
  if (st) return st;
  if (!U) return fail(HF_ERR_INVALID, "time-reversal U is NULL");
  if (k_mode == HF_K_INDEX_MAP && (!idx_i || !idx_j || !valid))
    return fail(HF_ERR_INVALID, "index-map mode needs idx_i, idx_j and valid");
  SymArgs s{nk1, nk2, nb, kpb_for(nb), 0, 1, nullptr, U, k_mode, flip_axes, idx_i, idx_j, valid, 1};
  cudaStream_t cs = static_cast<cudaStream_t>(stream);
  return dtype == HF_C128 ? launch_sym<double>(s, A, out, cs) : launch_sym<float>(s, A, out, cs);
}
