// Fast Fock-build passes for compile-time mesh lengths (see fft_reg.cuh).
//
// Thread layout of every pass: 16 slot lanes x TPL line parts; lane s of a
// half-warp owns band-pair slot s of the group, part t = threadIdx.x / 16.
// Global loads/stores go straight between HBM/L2 and registers: for a fixed
// element index the 16 lanes touch 16 consecutive slots (scratch) or one
// k-point's channel tiles (P, h, Sigma, F), so every access is a few whole
// 32-byte sectors.  Streamed operands use cache-streaming hints (__ldcs /
// __stcs) so that the spectrum scratch, which is re-read by the next pass,
// keeps its place in L2.
//   row_fwd : P - refP (pattern A along k2) -> FFT -> scratch (pattern B)
//   col     : scratch column (pattern A along k1) -> FFT -> x(-VR/N) -> IFFT -> scratch
//   row_inv : scratch (pattern B) -> IFFT -> epilogue (contact, Hartree, herm via a
//             lane shuffle with the transposed channel, + h) -> Sigma, F
// With the rows plan (nb <= 8, no packing) a slot group holds whole matrix rows,
// so the P, h, Sigma and F accesses of a k-point are contiguous, and the inverse
// row pass runs as clusters of ngroups CTAs that exchange the herm partners
// through distributed shared memory (k_fast_row_inv_rows).
#pragma once

#include <cooperative_groups.h>

#include <type_traits>

#include "fft_reg.cuh"
#include "fock_params.cuh"

namespace hf {

template <typename C>
__device__ __forceinline__ C ld_stream(const C* p) { return __ldcs(p); }
template <typename C>
__device__ __forceinline__ void st_stream(C* p, C v) { __stcs(p, v); }

// cp.async helpers: 16/8-byte global->shared copies that bypass registers.
// src_bytes = 0 zero-fills the destination (padding slots).
__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void cp_async16(void* dst, const void* src, bool valid) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(dst)), "l"(src),
               "r"(valid ? 16 : 0));
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src, bool valid) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(smem_u32(dst)), "l"(src),
               "r"(valid ? 8 : 0));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Programmatic dependent launch: the column and inverse row passes are launched
// with programmatic stream serialization, so their CTAs may start (twiddle
// tables, index setup) while the previous pass finishes; pdl_wait()
// (griddepcontrol.wait: the previous grid has completed and its writes are
// visible) comes before the first read of anything an earlier kernel wrote.
// Without the launch attribute griddepcontrol.wait returns at once.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }

// Launches kernel<<<grid, block, smem, stream>>>(p) with programmatic stream
// serialization (and a cluster shape when csize > 0).
template <typename K>
inline cudaError_t launch_pass(K kernel, int grid, int block, size_t smem, cudaStream_t stream, const FockParams& p,
                               int csize = 0) {
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[2];
  int na = 0;
  attr[na].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[na].val.programmaticStreamSerializationAllowed = 1;
  ++na;
  if (csize > 0) {
    attr[na].id = cudaLaunchAttributeClusterDimension;
    attr[na].val.clusterDim.x = (unsigned)csize;
    attr[na].val.clusterDim.y = 1;
    attr[na].val.clusterDim.z = 1;
    ++na;
  }
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cfg.attrs = attr;
  cfg.numAttrs = na;
  return cudaLaunchKernelEx(&cfg, kernel, p);
}

// Each fast pass is a persistent kernel: CTA b handles items b, b + grid, ...
// (item = slot group g + ngroups * line), and while it transforms one item the
// copies of the next one are already in flight into `stage`.  Every thread
// copies exactly the elements it later reads, so completion needs no barrier.

// Stages the pattern-A elements of row k1 (P - refP along k2) for one thread.
template <typename ST, typename FT, class S>
__device__ __forceinline__ void stage_row_fwd(const FockParams& p, cpx_t<FT>* stage, int k1, int c, int t, int s) {
  using SC = cpx_t<ST>;
  const SC* P = static_cast<const SC*>(p.P) + (size_t)k1 * S::N * p.nb2 + (c < 0 ? 0 : c);
  if constexpr (sizeof(SC) == sizeof(cpx_t<FT>)) {
#pragma unroll
    for (int i = 0; i < S::E1; ++i)
#pragma unroll
      for (int n1 = 0; n1 < S::N1; ++n1) {
        const int n = S::idxA(t, i, n1);
        if constexpr (sizeof(SC) == 16) cp_async16(stage + n * 16 + s, P + (size_t)n * p.nb2, c >= 0);
        else cp_async8(stage + n * 16 + s, P + (size_t)n * p.nb2, c >= 0);
      }
  }
  cp_async_commit();
}

template <typename ST, typename FT, class S>
__global__ void __launch_bounds__(16 * S::TPL) k_fast_row_fwd(const __grid_constant__ FockParams p) {
  if (p.active && !*p.active) return;
  pdl_launch_dependents();
  using SC = cpx_t<ST>;
  using FC = cpx_t<FT>;
  constexpr bool kStage = sizeof(SC) == sizeof(FC);  // mixed precision converts in registers
  extern __shared__ __align__(16) unsigned char smem_raw[];
  FC* twf = reinterpret_cast<FC*>(smem_raw);
  FC* twi = twf + S::TPL * S::TS;
  FC* buf = twi + S::TPL * S::TS;
  FC* stage = buf + 16 * S::N;
  const int t = threadIdx.x >> 4, s = threadIdx.x & 15, LS = p.LS;
  const int nitems = p.ngroups * p.nk1;
  build_line_twiddles<S, FT>(twf, twi);
  const bool has_ref = (p.flags & HF_FOCK_HAS_REFP) != 0;
  int item = blockIdx.x;
  if (kStage && item < nitems) {
    const int g = item % p.ngroups;
    stage_row_fwd<ST, FT, S>(p, stage, item / p.ngroups, s < LS ? p.chan[g * LS + s] : -1, t, s);
  }
  __syncthreads();
  for (; item < nitems; item += gridDim.x) {
    const int g = item % p.ngroups, k1 = item / p.ngroups;
    const int c = s < LS ? p.chan[g * LS + s] : -1;
    FC x[S::E];
    if constexpr (kStage) {
      cp_async_wait_all();
#pragma unroll
      for (int i = 0; i < S::E1; ++i)
#pragma unroll
        for (int n1 = 0; n1 < S::N1; ++n1) x[i * S::N1 + n1] = stage[S::idxA(t, i, n1) * 16 + s];
      const int nx = item + gridDim.x;
      if (nx < nitems) {
        const int g2 = nx % p.ngroups;
        stage_row_fwd<ST, FT, S>(p, stage, nx / p.ngroups, s < LS ? p.chan[g2 * LS + s] : -1, t, s);
      }
    } else {
      const SC* P = static_cast<const SC*>(p.P) + (size_t)k1 * S::N * p.nb2 + (c < 0 ? 0 : c);
#pragma unroll
      for (int i = 0; i < S::E1; ++i)
#pragma unroll
        for (int n1 = 0; n1 < S::N1; ++n1)
          x[i * S::N1 + n1] = c >= 0 ? cvt<FC>(ld_stream(P + (size_t)S::idxA(t, i, n1) * p.nb2)) : mk<FC>(0.0, 0.0);
    }
    if (has_ref && c >= 0) {
      const SC* R = static_cast<const SC*>(p.refP) + (size_t)k1 * S::N * p.nb2 + c;
#pragma unroll
      for (int i = 0; i < S::E1; ++i)
#pragma unroll
        for (int n1 = 0; n1 < S::N1; ++n1)
          x[i * S::N1 + n1] = csub(x[i * S::N1 + n1], cvt<FC>(ld_stream(R + (size_t)S::idxA(t, i, n1) * p.nb2)));
    }
    fwd_AB<S>(x, buf, twf + t * S::TS, t, s);
    if (s < LS) {
      FC* out = static_cast<FC*>(p.scratch) + ((size_t)g * p.nk1 + k1) * S::N * LS + s;
#pragma unroll
      for (int j = 0; j < S::E2; ++j)
#pragma unroll
        for (int k2 = 0; k2 < S::N2; ++k2) __stcg(out + S::idxB(t, j, k2) * LS, x[j * S::N2 + k2]);
    }
    __syncthreads();  // buf is rewritten by the next item
  }
}

template <typename FT, class S>
__device__ __forceinline__ void stage_col(const FockParams& p, cpx_t<FT>* stage, int g, int k2c, int t, int s) {
  using FC = cpx_t<FT>;
  const int LS = p.LS;
  const FC* col = static_cast<const FC*>(p.scratch) + ((size_t)g * p.nk1 * p.nk2 + k2c) * LS + (s < LS ? s : 0);
  const size_t rs = (size_t)p.nk2 * LS;
#pragma unroll
  for (int i = 0; i < S::E1; ++i)
#pragma unroll
    for (int n1 = 0; n1 < S::N1; ++n1) {
      const int n = S::idxA(t, i, n1);
      if constexpr (sizeof(FC) == 16) cp_async16(stage + n * 16 + s, col + n * rs, s < LS);
      else cp_async8(stage + n * 16 + s, col + n * rs, s < LS);
    }
  cp_async_commit();
}

// VREAL: the shifted V-hat is real (HF_FOCK_VR_REAL), one ST per entry.  With an FP32
// transform the shared memory of a CTA is half as large, so three CTAs share an SM.
template <typename ST, typename FT, class S, bool VREAL>
__global__ void __launch_bounds__(16 * S::TPL, sizeof(FT) == 4 ? 3 : 2) k_fast_col(const __grid_constant__ FockParams p) {
  pdl_launch_dependents();
  using SC = cpx_t<ST>;
  using FC = cpx_t<FT>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  FC* twf = reinterpret_cast<FC*>(smem_raw);
  FC* twi = twf + S::TPL * S::TS;
  FC* buf = twi + S::TPL * S::TS;
  FC* stage = buf + 16 * S::N;
  const int t = threadIdx.x >> 4, s = threadIdx.x & 15, LS = p.LS;
  const int nitems = p.ngroups * p.nk2;
  build_line_twiddles<S, FT>(twf, twi);
  const bool vr_scalar = (p.flags & HF_FOCK_VR_SCALAR) != 0;
  const size_t vstride = vr_scalar ? 1 : (size_t)p.nb2;
  const size_t rs = (size_t)p.nk2 * LS;
  int item = blockIdx.x;
  pdl_wait();  // the row pass has finished writing the scratch
  if (p.active && !*p.active) return;
  if (item < nitems) stage_col<FT, S>(p, stage, item % p.ngroups, item / p.ngroups, t, s);
  __syncthreads();
  for (; item < nitems; item += gridDim.x) {
    const int g = item % p.ngroups, k2c = item / p.ngroups;
    const int c = s < LS ? p.chan[g * LS + s] : -1;
    const int vc = vr_scalar ? 0 : (c < 0 ? 0 : c);
    // V-hat for the pattern-B frequencies of this thread, issued before the FFT and
    // scaled only where it is used, so that the loads stay in flight across the transform
    using VT = std::conditional_t<VREAL, ST, SC>;
    VT vq[S::E];
#pragma unroll
    for (int j = 0; j < S::E2; ++j)
#pragma unroll
      for (int k2 = 0; k2 < S::N2; ++k2) {
        const size_t q = (size_t)S::idxB(t, j, k2) * p.nk2 + k2c;
        vq[j * S::N2 + k2] = ld_stream(static_cast<const VT*>(p.VR) + q * vstride + vc);
      }
    cp_async_wait_all();
    FC x[S::E];
#pragma unroll
    for (int i = 0; i < S::E1; ++i)
#pragma unroll
      for (int n1 = 0; n1 < S::N1; ++n1) x[i * S::N1 + n1] = stage[S::idxA(t, i, n1) * 16 + s];
    const int nx = item + gridDim.x;
    if (nx < nitems) stage_col<FT, S>(p, stage, nx % p.ngroups, nx / p.ngroups, t, s);
    fwd_AB<S>(x, buf, twf + t * S::TS, t, s);
#pragma unroll
    for (int e = 0; e < S::E; ++e) {
      const FC v = x[e];
      if constexpr (VREAL) {
        const FT w = (FT)((double)vq[e] * p.scale);
        x[e] = c < 0 ? mk<FC>(0.0, 0.0) : mk<FC>(v.x * w, v.y * w);
      } else {
        const FT wr = (FT)((double)vq[e].x * p.scale), wi = (FT)((double)vq[e].y * p.scale);
        x[e] = c < 0 ? mk<FC>(0.0, 0.0) : mk<FC>(v.x * wr - v.y * wi, v.x * wi + v.y * wr);
      }
    }
    __syncthreads();  // buf is reused by the inverse transform
    inv_BA<S>(x, buf, twi + t * S::TS, t, s);
    if (s < LS) {
      FC* col = static_cast<FC*>(p.scratch) + ((size_t)g * p.nk1 * p.nk2 + k2c) * LS + s;
#pragma unroll
      for (int i = 0; i < S::E1; ++i)
#pragma unroll
        for (int n1 = 0; n1 < S::N1; ++n1) __stcg(col + S::idxA(t, i, n1) * rs, x[i * S::N1 + n1]);
    }
    __syncthreads();
  }
}

template <typename FT, class S>
__device__ __forceinline__ void stage_row_inv(const FockParams& p, cpx_t<FT>* stage, int g, int k1, int t, int s) {
  using FC = cpx_t<FT>;
  const int LS = p.LS;
  const FC* row = static_cast<const FC*>(p.scratch) + ((size_t)g * p.nk1 + k1) * S::N * LS + (s < LS ? s : 0);
#pragma unroll
  for (int j = 0; j < S::E2; ++j)
#pragma unroll
    for (int k2 = 0; k2 < S::N2; ++k2) {
      const int n = S::idxB(t, j, k2);
      if constexpr (sizeof(FC) == 16) cp_async16(stage + n * 16 + s, row + n * LS, s < LS);
      else cp_async8(stage + n * 16 + s, row + n * LS, s < LS);
    }
  cp_async_commit();
}

template <typename ST, typename FT, class S>
__global__ void __launch_bounds__(16 * S::TPL, 2) k_fast_row_inv(const __grid_constant__ FockParams p) {
  using SC = cpx_t<ST>;
  using FC = cpx_t<FT>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  FC* twf = reinterpret_cast<FC*>(smem_raw);
  FC* twi = twf + S::TPL * S::TS;
  FC* buf = twi + S::TPL * S::TS;
  FC* stage = buf + 16 * S::N;
  const int t = threadIdx.x >> 4, s = threadIdx.x & 15;
  const int lane = threadIdx.x & 31;
  const int LS = p.LS, nb = p.nb;
  const int nitems = p.ngroups * p.nk1;
  const bool exch = (p.flags & HF_FOCK_EXCHANGE) != 0;
  const bool packing = (p.flags & HF_FOCK_PACKING) != 0;
  const bool consts = p.sigc != nullptr;
  const SC* h = static_cast<const SC*>(p.h);
  SC* Sg = static_cast<SC*>(p.Sigma);
  SC* F = static_cast<SC*>(p.F);
  build_line_twiddles<S, FT>(twf, twi);
  int item = blockIdx.x;
  pdl_wait();  // the column pass has finished writing the scratch
  if (p.active && !*p.active) return;
  if (exch && item < nitems) stage_row_inv<FT, S>(p, stage, item % p.ngroups, item / p.ngroups, t, s);
  __syncthreads();
  for (; item < nitems; item += gridDim.x) {
    const int g = item % p.ngroups, k1 = item / p.ngroups;
    const int c = s < LS ? p.chan[g * LS + s] : -1;
    const int plane = (lane & 16) | (s < LS ? p.partner[g * LS + s] : s);
    const int a = c >= 0 ? c / nb : 0, b = c >= 0 ? c - (c / nb) * nb : 0;
    const size_t row0 = (size_t)k1 * S::N * p.nb2;
    // h for this thread's k-points, issued before the transform
    SC hv[S::E];
#pragma unroll
    for (int i = 0; i < S::E1; ++i)
#pragma unroll
      for (int m1 = 0; m1 < S::N1; ++m1)
        hv[i * S::N1 + m1] = c >= 0 ? ld_stream(h + row0 + (size_t)S::idxA(t, i, m1) * p.nb2 + a * nb + b)
                                    : mk<SC>(0.0, 0.0);
    FC x[S::E];
    if (exch) {
      cp_async_wait_all();
#pragma unroll
      for (int j = 0; j < S::E2; ++j)
#pragma unroll
        for (int k2 = 0; k2 < S::N2; ++k2) x[j * S::N2 + k2] = stage[S::idxB(t, j, k2) * 16 + s];
      const int nx = item + gridDim.x;
      if (nx < nitems) stage_row_inv<FT, S>(p, stage, nx % p.ngroups, nx / p.ngroups, t, s);
      inv_BA<S>(x, buf, twi + t * S::TS, t, s);
    } else {
#pragma unroll
      for (int e = 0; e < S::E; ++e) x[e] = mk<FC>(0.0, 0.0);
    }
    SC cab = mk<SC>(0.0, 0.0), cba = mk<SC>(0.0, 0.0);
    double hd = 0.0;
    if (consts && c >= 0) {
      cab = cvt<SC>(p.sigc[a * nb + b]);
      cba = cvt<SC>(p.sigc[b * nb + a]);
      if (a == b) hd = p.hdiag[a];
    }
#pragma unroll
    for (int i = 0; i < S::E1; ++i)
#pragma unroll
      for (int m1 = 0; m1 < S::N1; ++m1) {
        const FC mine = x[i * S::N1 + m1];
        const SC hab = hv[i * S::N1 + m1];
        // every lane takes part in both shuffles (padding lanes included)
        FC other;
        other.x = __shfl_sync(0xffffffffu, mine.x, plane);
        other.y = __shfl_sync(0xffffffffu, mine.y, plane);
        SC hsh;
        hsh.x = __shfl_sync(0xffffffffu, hab.x, plane);
        hsh.y = __shfl_sync(0xffffffffu, hab.y, plane);
        if (c < 0) continue;
        const size_t base = row0 + (size_t)S::idxA(t, i, m1) * p.nb2;
        SC sab = cvt<SC>(mine);
        SC sba = packing ? (a == b ? sab : conj(sab)) : cvt<SC>(other);
        sab = cadd(sab, cab);
        sba = cadd(sba, cba);
        const SC hba = packing ? ld_stream(h + base + b * nb + a) : hsh;
        SC f = mk<SC>(0.5 * ((double)hab.x + (double)hba.x) + 0.5 * ((double)sab.x + (double)sba.x),
                      0.5 * ((double)hab.y - (double)hba.y) + 0.5 * ((double)sab.y - (double)sba.y));
        f.x += (ST)hd;
        st_stream(Sg + base + a * nb + b, sab);
        st_stream(F + base + a * nb + b, f);
        if (packing && a != b) {
          st_stream(Sg + base + b * nb + a, sba);
          st_stream(F + base + b * nb + a, conj(f));
        }
      }
    __syncthreads();
  }
}

// Cluster barrier halves (all threads of every CTA of the cluster take part).
__device__ __forceinline__ void cluster_arrive() { asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory"); }
__device__ __forceinline__ void cluster_wait() { asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory"); }
// Arrival without release semantics, for a barrier that only says "my reads of
// the other CTAs' shared memory are done" (their values have been consumed, so
// no later write can change them); it does not wait for this thread's global
// stores to complete, as a release would.
__device__ __forceinline__ void cluster_arrive_relaxed() {
  asm volatile("barrier.cluster.arrive.relaxed.aligned;\n" ::: "memory");
}

// Inverse row pass of the rows plan (see the file comment).  Cluster q of the
// grid takes rows k1 = q, q + nclusters, ...; CTA rank g of the cluster is slot
// group g.  Per row: inverse FFT of the group's spectrum row (direct L2 loads,
// no stage; 2 CTAs per SM without register spills), Sigma = result + contact, M = h + Sigma into shared
// memory, cluster barrier A, F = (M + M_partner^H) / 2 + Hartree with M_partner
// read from the partner group's CTA (partner = (group << 8) | slot), arrival at
// cluster barrier B.  The wait on B (the partners have read the buffer) comes
// in the next row after its loads and first FFT step, just before the buffer
// is overwritten, and once more before the CTA exits.
template <typename ST, typename FT, class S>
__global__ void __launch_bounds__(16 * S::TPL, 2) k_fast_row_inv_rows(const __grid_constant__ FockParams p) {
  namespace cg = cooperative_groups;
  using SC = cpx_t<ST>;
  using FC = cpx_t<FT>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  FC* twf = reinterpret_cast<FC*>(smem_raw);
  FC* twi = twf + S::TPL * S::TS;
  FC* buf = twi + S::TPL * S::TS;  // FFT exchange, then M
  SC* mbuf = reinterpret_cast<SC*>(buf);
  FC* stage = reinterpret_cast<FC*>(mbuf + 16 * S::N);  // cp.async stage of the next spectrum row
  cg::cluster_group cluster = cg::this_cluster();
  const int g = (int)cluster.block_rank();
  const int ncl = gridDim.x / p.ngroups, cl = blockIdx.x / p.ngroups;
  const int t = threadIdx.x >> 4, s = threadIdx.x & 15;
  const int LS = p.LS, nb = p.nb;
  const bool exch = (p.flags & HF_FOCK_EXCHANGE) != 0;
  const SC* h = static_cast<const SC*>(p.h);
  SC* Sg = static_cast<SC*>(p.Sigma);
  SC* F = static_cast<SC*>(p.F);
  build_line_twiddles<S, FT>(twf, twi);
  const int c = s < LS ? p.chan[g * LS + s] : -1;
  const int pe = c >= 0 ? p.partner[g * LS + s] : ((g << 8) | s);
  const SC* pbuf = cluster.map_shared_rank(mbuf, pe >> 8) + (pe & 255);
  pdl_wait();  // scratch, contact sigma and Hartree diagonal come from earlier kernels
  if (p.active && !*p.active) return;  // the flag is uniform over the grid
  const int cc = c >= 0 ? c : 0;
  SC cab = mk<SC>(0.0, 0.0);
  double hd = 0.0;
  if (p.sigc != nullptr && c >= 0) {
    cab = cvt<SC>(p.sigc[c]);
    if (cc / nb == cc % nb) hd = p.hdiag[cc / nb];
  }
  if (exch && cl < p.nk1) stage_row_inv<FT, S>(p, stage, g, cl, t, s);
  __syncthreads();
  bool pending = false;  // arrived at barrier B, not yet waited
  for (int k1 = cl; k1 < p.nk1; k1 += ncl) {
    const size_t base = ((size_t)k1 * S::N + t) * p.nb2 + cc;
    // h for this thread's k-points, issued before the transform
    SC m[S::E];
#pragma unroll
    for (int i = 0; i < S::E1; ++i)
#pragma unroll
      for (int m1 = 0; m1 < S::N1; ++m1)
        m[i * S::N1 + m1] = c >= 0 ? ld_stream(h + base + (size_t)(S::TPL * i + S::N2 * m1) * p.nb2) : mk<SC>(0.0, 0.0);
    FC x[S::E];
    if (exch) {
      cp_async_wait_all();  // this thread's copies of the row (no barrier: it reads only what it copied)
#pragma unroll
      for (int j = 0; j < S::E2; ++j)
#pragma unroll
        for (int k2 = 0; k2 < S::N2; ++k2) x[j * S::N2 + k2] = stage[S::idxB(t, j, k2) * 16 + s];
      if (k1 + ncl < p.nk1) stage_row_inv<FT, S>(p, stage, g, k1 + ncl, t, s);
      inv_BA<S>(x, buf, twi + t * S::TS, t, s, [&] {
        if (pending) cluster_wait();
        pending = false;
      });
    } else {
#pragma unroll
      for (int e = 0; e < S::E; ++e) x[e] = mk<FC>(0.0, 0.0);
      if (pending) cluster_wait();
      pending = false;
    }
    __syncthreads();  // the exchange reads of buf are done: it now takes M
#pragma unroll
    for (int i = 0; i < S::E1; ++i)
#pragma unroll
      for (int m1 = 0; m1 < S::N1; ++m1) {
        const int e = i * S::N1 + m1;
        const SC sab = cadd(cvt<SC>(x[e]), cab);
        m[e] = cadd(m[e], sab);
        mbuf[S::idxA(t, i, m1) * 16 + s] = m[e];
      }
    cluster_arrive();  // barrier A: M of every group is in shared memory
#pragma unroll
    for (int i = 0; i < S::E1; ++i)
#pragma unroll
      for (int m1 = 0; m1 < S::N1; ++m1)
        if (c >= 0) st_stream(Sg + base + (size_t)(S::TPL * i + S::N2 * m1) * p.nb2, cadd(cvt<SC>(x[i * S::N1 + m1]), cab));
    cluster_wait();
#pragma unroll
    for (int i = 0; i < S::E1; ++i) {
      // every partner load of the batch is issued before its F stores: a global store
      // may alias the generic pbuf address, so interleaving them would serialise the
      // distributed-shared-memory round trips
      SC mo[S::N1];
#pragma unroll
      for (int m1 = 0; m1 < S::N1; ++m1) mo[m1] = pbuf[S::idxA(t, i, m1) * 16];
#pragma unroll
      for (int m1 = 0; m1 < S::N1; ++m1) {
        const int e = i * S::N1 + m1;
        if (c >= 0)
          st_stream(F + base + (size_t)(S::TPL * i + S::N2 * m1) * p.nb2,
                    mk<SC>(0.5 * ((double)m[e].x + (double)mo[m1].x) + hd, 0.5 * ((double)m[e].y - (double)mo[m1].y)));
      }
    }
    cluster_arrive_relaxed();  // barrier B: this CTA's reads of the partners' buffers are done
    pending = true;
  }
  if (pending) cluster_wait();  // no CTA exits while a partner may read its buffer
}

template <class S, typename FT>
constexpr size_t fast_smem() {
  return (size_t)(2 * S::TPL * S::TS + 32 * S::N) * sizeof(cpx_t<FT>);  // twiddle rows, exchange buffer, stage
}
// k_fast_row_inv_rows: twiddle rows, one buffer of 16 N entries (FFT exchange, then M), the stage
template <class S, typename ST, typename FT>
constexpr size_t fast_smem_rows() {
  constexpr size_t e = sizeof(cpx_t<ST>) > sizeof(cpx_t<FT>) ? sizeof(cpx_t<ST>) : sizeof(cpx_t<FT>);
  return (size_t)(2 * S::TPL * S::TS) * sizeof(cpx_t<FT>) + 16 * (size_t)S::N * e + 16 * (size_t)S::N * sizeof(cpx_t<FT>);
}

// Persistent grid: CTAs resident on the device (2 per SM for the large shapes).
template <typename K>
inline int persistent_grid(K kernel, int threads, size_t smem, int items) {
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  const int g = sms * per_sm;
  return items < g ? items : g;
}

// Launches the three passes when both mesh lengths have a fast shape; returns
// HF_OK and sets *handled, or leaves *handled false for the generic engine.
template <typename ST, typename FT>
int fast_fock(FockParams& p, cudaStream_t stream, bool* handled) {
  *handled = false;
  if (p.LS > 16 || !fast_length(p.nk1) || !fast_length(p.nk2)) return HF_OK;
  const bool exch = (p.flags & HF_FOCK_EXCHANGE) != 0;
  int st = HF_OK;
  auto row = [&](auto shape) {
    using S = decltype(shape);
    constexpr size_t sm = fast_smem<S, FT>();
    if (exch) {
      cudaFuncSetAttribute(k_fast_row_fwd<ST, FT, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
      const int grid = persistent_grid(k_fast_row_fwd<ST, FT, S>, 16 * S::TPL, sm, p.ngroups * p.nk1);
      k_fast_row_fwd<ST, FT, S><<<grid, 16 * S::TPL, sm, stream>>>(p);
    }
  };
  auto col = [&](auto shape) {
    using S = decltype(shape);
    constexpr size_t sm = fast_smem<S, FT>();
    auto kern = (p.flags & HF_FOCK_VR_REAL) ? k_fast_col<ST, FT, S, true> : k_fast_col<ST, FT, S, false>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    const int grid = persistent_grid(kern, 16 * S::TPL, sm, p.ngroups * p.nk2);
    const cudaError_t e = launch_pass(kern, grid, 16 * S::TPL, sm, stream, p);
    if (e != cudaSuccess) st = cuda_check(e, "k_fast_col");
  };
  auto inv = [&](auto shape) {
    using S = decltype(shape);
    if (p.rows_plan) {
      constexpr size_t sm = fast_smem_rows<S, ST, FT>();
      auto kern = k_fast_row_inv_rows<ST, FT, S>;
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
      cudaLaunchConfig_t cfg = {};
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = (unsigned)p.ngroups;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.gridDim = dim3((unsigned)p.ngroups);
      cfg.blockDim = dim3(16 * S::TPL);
      cfg.dynamicSmemBytes = sm;
      cfg.stream = stream;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      int ncl = 0;
      if (cudaOccupancyMaxActiveClusters(&ncl, kern, &cfg) != cudaSuccess || ncl < 1) ncl = 1;
      if (ncl > p.nk1) ncl = p.nk1;
      const cudaError_t e = launch_pass(kern, ncl * p.ngroups, 16 * S::TPL, sm, stream, p, p.ngroups);
      if (e != cudaSuccess) st = cuda_check(e, "k_fast_row_inv_rows");
      return;
    }
    constexpr size_t sm = fast_smem<S, FT>();
    cudaFuncSetAttribute(k_fast_row_inv<ST, FT, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    const int grid = persistent_grid(k_fast_row_inv<ST, FT, S>, 16 * S::TPL, sm, p.ngroups * p.nk1);
    const cudaError_t e = launch_pass(k_fast_row_inv<ST, FT, S>, grid, 16 * S::TPL, sm, stream, p);
    if (e != cudaSuccess) st = cuda_check(e, "k_fast_row_inv");
  };
  switch (p.nk2) {
#define HF_CASE(N, A, B, T) case N: row(LineShape<N, A, B, T>{}); break;
    HF_FAST_SHAPES(HF_CASE)
#undef HF_CASE
  }
  HF_LAUNCH_CHECK("k_fast_row_fwd");
  if (exch) {
    switch (p.nk1) {
#define HF_CASE(N, A, B, T) case N: col(LineShape<N, A, B, T>{}); break;
      HF_FAST_SHAPES(HF_CASE)
#undef HF_CASE
    }
    HF_LAUNCH_CHECK("k_fast_col");
  }
  switch (p.nk2) {
#define HF_CASE(N, A, B, T) case N: inv(LineShape<N, A, B, T>{}); break;
    HF_FAST_SHAPES(HF_CASE)
#undef HF_CASE
  }
  HF_LAUNCH_CHECK("k_fast_row_inv");
  *handled = true;
  return st;
}

}  // namespace hf
