// Off-block check of block-diagonal exchange specs (utils.py:252-309): for every
// spec, max over k and off-block channels of |P - refP|, and the overall maximum,
// in one pass over the density; the caller reads all of them with one copy and
// picks the first spec whose off-block maximum is within atol + rtol * max.
//
// Maxima of non-negative doubles are order-independent, so they are combined with
// 64-bit integer atomicMax on the bit patterns (monotone for non-negative IEEE
// values).  A NaN anywhere is kept as the canonical quiet NaN, the largest pattern,
// so the maximum is NaN and the caller's comparison fails, as jnp.max propagates it.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "common.cuh"

namespace hf {
namespace {

constexpr int kMaxSpecs = 8;
constexpr int kMaxNbBlocks = 32;  // nb limit of the Fock build
constexpr int kMaskWords = kMaxNbBlocks * kMaxNbBlocks / 64;

struct SpecMasks {
  unsigned long long off[kMaxSpecs][kMaskWords];  // bit c set: channel c is off-block in spec i
};

__device__ __forceinline__ unsigned long long max_bits(double v) {
  if (v != v) return 0x7FF8000000000000ull;
  return (unsigned long long)__double_as_longlong(v);
}

// n < 2^31 elements (checked by the host); each thread takes four elements per step
// and issues their loads before any of the arithmetic.
template <typename SC>
__global__ void k_block_offmax(unsigned n, int nb2, int n_specs, const __grid_constant__ SpecMasks m,
                               const SC* __restrict__ P, const SC* __restrict__ refP,
                               unsigned long long* __restrict__ out) {
  constexpr int U = 4;
  unsigned long long best[kMaxSpecs + 1];
#pragma unroll
  for (int i = 0; i <= kMaxSpecs; ++i) best[i] = 0ull;
  const unsigned stride = gridDim.x * blockDim.x;
  for (unsigned e0 = blockIdx.x * blockDim.x + threadIdx.x; e0 < n; e0 += U * stride) {
    SC x[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const unsigned e = e0 + u * stride;
      x[u] = e < n ? P[e] : SC{0, 0};
      if (refP && e < n) {
        const SC r = refP[e];
        x[u].x -= r.x;
        x[u].y -= r.y;
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const unsigned e = e0 + u * stride;
      if (e >= n) break;
      const unsigned long long v = max_bits(hypot((double)x[u].x, (double)x[u].y));
      best[0] = v > best[0] ? v : best[0];
      const unsigned c = e % (unsigned)nb2;
#pragma unroll
      for (int i = 0; i < kMaxSpecs; ++i)
        if (i < n_specs && ((m.off[i][c >> 6] >> (c & 63)) & 1ull)) best[i + 1] = v > best[i + 1] ? v : best[i + 1];
    }
  }
#pragma unroll
  for (int i = 0; i <= kMaxSpecs; ++i) {
    if (i > n_specs) break;
    unsigned long long v = best[i];
    for (int o = 16; o > 0; o >>= 1) {
      const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
      v = w > v ? w : v;
    }
    if ((threadIdx.x & 31) == 0 && v) atomicMax(out + i, v);
  }
}

}  // namespace
}  // namespace hf

using namespace hf;

extern "C" int hf_block_offdiag_max(void* stream, int dtype, size_t nk, int nb, const void* P, const void* refP,
                                    int n_specs, const unsigned char* inblock, double* out) {
  if (!P || !out || (n_specs > 0 && !inblock)) return fail(HF_ERR_INVALID, "hf_block_offdiag_max: bad argument");
  if (dtype != HF_C128 && dtype != HF_C64) return fail(HF_ERR_INVALID, "dtype must be HF_C128 or HF_C64");
  if (nb < 1 || nb > kMaxNbBlocks) return fail(HF_ERR_UNSUPPORTED, "hf_block_offdiag_max: nb > 32");
  if (n_specs < 0 || n_specs > kMaxSpecs) return fail(HF_ERR_UNSUPPORTED, "hf_block_offdiag_max: at most 8 specs");
  SpecMasks m;
  memset(&m, 0, sizeof(m));
  const int nb2 = nb * nb;
  for (int i = 0; i < n_specs; ++i)
    for (int c = 0; c < nb2; ++c)
      if (!inblock[(size_t)i * nb2 + c]) m.off[i][c >> 6] |= 1ull << (c & 63);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  HF_CUDA(cudaMemsetAsync(out, 0, (size_t)(n_specs + 1) * sizeof(double), s));
  const size_t n = nk * (size_t)nb2;
  if (n == 0) return HF_OK;
  if (n >= (1ull << 31)) return fail(HF_ERR_UNSUPPORTED, "hf_block_offdiag_max: more than 2^31 elements");
  const int blocks = (int)std::min<size_t>((n + 1023) / 1024, (size_t)148 * 8);
  auto* o = reinterpret_cast<unsigned long long*>(out);
  if (dtype == HF_C128)
    k_block_offmax<double2><<<blocks, 256, 0, s>>>((unsigned)n, nb2, n_specs, m, static_cast<const double2*>(P),
                                                   static_cast<const double2*>(refP), o);
  else
    k_block_offmax<float2><<<blocks, 256, 0, s>>>((unsigned)n, nb2, n_specs, m, static_cast<const float2*>(P),
                                                  static_cast<const float2*>(refP), o);
  HF_LAUNCH_CHECK("k_block_offmax");
  return HF_OK;
}
