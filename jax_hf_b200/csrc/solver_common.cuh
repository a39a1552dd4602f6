// Shared device-side machinery of the solvers: block partial sums finalised by
// the last CTA to finish (atomic ticket, no spin-wait), and per-k launch shapes.
#pragma once

#include "common.cuh"

namespace hf {

constexpr int kSolverWarps = 4;  // warps (k-points in flight) per CTA for per-k kernels
constexpr int kMaxSums = 20;     // partial sums per reduction

// Per-block compensated partials of NS quantities: part[blk][NS][2].
// Returns true in every thread of the CTA that finished last; that CTA then
// reads all partials (fixed order -> deterministic) through L2.
template <int NS>
__device__ __forceinline__ bool publish_partials(KSum (&acc)[NS], double* __restrict__ part,
                                                 unsigned* __restrict__ counter, double* sm) {
  for (int q = 0; q < NS; ++q) {
    KSum r = block_reduce(acc[q], sm);
    if (threadIdx.x == 0) {
      part[((size_t)blockIdx.x * NS + q) * 2] = r.s;
      part[((size_t)blockIdx.x * NS + q) * 2 + 1] = r.c;
    }
  }
  __shared__ bool s_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned t = atomicAdd(counter, 1u);
    s_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  return s_last;
}

// In the last CTA: totals[q] = sum over blocks.  Every thread sums a fixed
// strided subset of the block partials, then one compensated block reduction per
// quantity (fixed assignment and tree -> deterministic for a launch shape).
template <int NS>
__device__ __forceinline__ void gather_partials(const double* __restrict__ part, unsigned* __restrict__ counter,
                                                double* totals, double* sm) {
  KSum t[NS];
  for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
#pragma unroll
    for (int q = 0; q < NS; ++q) {
      t[q].add(__ldcg(part + ((size_t)b * NS + q) * 2));
      t[q].add(__ldcg(part + ((size_t)b * NS + q) * 2 + 1));
    }
  }
#pragma unroll
  for (int q = 0; q < NS; ++q) {
    const KSum r = block_reduce(t[q], sm);
    if (threadIdx.x == 0) totals[q] = r.value();
  }
  __syncthreads();
  if (threadIdx.x == 0) *counter = 0u;
}

__device__ __forceinline__ double sigmoid(double x) { return 1.0 / (1.0 + exp(-x)); }

// p log p + (1-p) log1p(-p) with the 1e-14 clip of occupation_entropy (fock.py:114-118)
__device__ __forceinline__ double ent_term(double p) {
  const double ps = fmin(fmax(p, 1e-14), 1.0 - 1e-14);
  return ps * log(ps) + (1.0 - ps) * log1p(-ps);
}

__device__ __forceinline__ double clip(double x, double lo, double hi) { return fmin(fmax(x, lo), hi); }

inline int perk_blocks(int nk) {
  int b = (nk + kSolverWarps - 1) / kSolverWarps;
  if (b > 148 * 16) b = 148 * 16;
  if (b < 1) b = 1;
  return b;
}

}  // namespace hf
