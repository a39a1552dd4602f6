// Bulk-copy pipelined Fock passes (sm_100a) for the rows plan with nb in {4, 8}.
//
// Same arithmetic as the register passes of fock_fast.cuh (two-level line FFT of
// fft_reg.cuh, compile-time twiddles), organised around Blackwell's
// asynchronous copy engine instead of per-thread cp.async:
//
//   * one persistent CTA per SM with a ring of NS shared-memory stages; every
//     item's input arrives with ONE asynchronous copy: a tensor copy (TMA) of a
//     2D / 3D box for the strided row and column reads, a contiguous bulk copy
//     for the inverse row pass, completion counted in bytes on the stage's
//     mbarrier (128-byte bulk copies per k-point, one per chunk, ran at ~2% of
//     HBM bandwidth);
//   * NG consumer groups of GT = SL * TPL threads (SL slot lanes x TPL line
//     parts), about twelve warps per SM, take the CTA's items round robin; a
//     group transforms its item in registers, using its own stage as the FFT
//     exchange buffer (group-local named barriers); after its last read of the
//     stage the group's leader issues the copy of the item NS places ahead into
//     it, and the group stores its result straight from registers;
//   * so the copies of NS - NG items stay in flight while the groups compute.
//     There is no producer warp: with one, three warps of some SM
//     sub-partitions would cap the consumers' registers at the same 168 with
//     a third fewer consumer warps.
//
// An item is SL consecutive channels (whole matrix rows) of one line: 128-byte
// runs at every k-point of P, Sigma and F.  Passes:
//   k_pipe_row_fwd : (P - refP) row k1 -> FFT along k2 -> scratch [g][k1][k2][SL]
//   k_pipe_col     : scratch column -> FFT along k1, x (-VR / (nk1 nk2)), IFFT -> scratch
//   k_pipe_row_inv : scratch row -> IFFT along k2 (+ contact sigma) -> Sigma
//   k_pipe_herm    : F = herm(h + Sigma) + Hartree diagonal, k-point tiles in shared memory
// The herm partner of a channel lives in another item, so F is formed by the
// fourth, streaming pass (Sigma is re-read from L2, where the third pass left it).
//
// Every mbarrier wait is bounded (kPipeWaitNs of %globaltimer); a wait that
// runs out records a code in *p.fault, and every group of the CTA leaves its
// loop (a group decides together through a barrier reduction, so no thread is
// left in a named barrier).  Thread 0 then waits, again bounded, for the copies
// still in flight before the CTA exits.
#pragma once

#include <cudaTypedefs.h>

#include "fft_reg.cuh"
#include "fock_params.cuh"

namespace hf {

constexpr int kPipeMaxStages = 16;
constexpr unsigned long long kPipeWaitNs = 2000000000ull;  // 2 s

// ------------------------------------------------------------- PTX wrappers --
__device__ __forceinline__ unsigned pipe_saddr(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(pipe_saddr(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(pipe_saddr(b)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint64_t* b, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(pipe_saddr(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t* b, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(pipe_saddr(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ unsigned long long pipe_now_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
  return t;
}
// Waits until the phase of the given parity of *b has completed.  Gives up
// after kPipeWaitNs, or at once when another warp has recorded a fault, and
// returns false; a timeout records `code` in *fault.
// Waits until *slot == want (a shared-memory word written by another thread of
// the CTA); bounded like mbar_wait.
static __device__ __noinline__ bool smem_wait_eq(const int* slot, int want, int* fault, int code) {
  const volatile int* v = slot;
  if (*v == want) return true;
  const unsigned long long t0 = pipe_now_ns();
  for (;;) {
#pragma unroll 1
    for (int i = 0; i < 64; ++i)
      if (*v == want) return true;
    if (fault && *reinterpret_cast<volatile int*>(fault) != 0) return false;
    if (pipe_now_ns() - t0 > kPipeWaitNs) {
      if (fault) atomicCAS(fault, 0, code);
      return false;
    }
    __nanosleep(64);
  }
}
static __device__ __noinline__ bool mbar_wait(uint64_t* b, unsigned parity, int* fault, int code) {
  if (mbar_test(b, parity)) return true;
  const unsigned long long t0 = pipe_now_ns();
  for (;;) {
#pragma unroll 1
    for (int i = 0; i < 32; ++i)
      if (mbar_test(b, parity)) return true;
    if (fault && *reinterpret_cast<volatile int*>(fault) != 0) return false;
    if (pipe_now_ns() - t0 > kPipeWaitNs) {
      if (fault) atomicCAS(fault, 0, code);
      return false;
    }
  }
}
__device__ __forceinline__ uint64_t pipe_policy_evict_first() {
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;\n" : "=l"(pol));
  return pol;
}
// Bulk global -> shared copy of `bytes` (multiple of 16, both addresses 16-byte
// aligned), completion counted on *bar, with an L2 eviction policy.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, uint64_t* bar, uint64_t pol) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;\n" ::"r"(
          pipe_saddr(dst)),
      "l"(src), "r"(bytes), "r"(pipe_saddr(bar)), "l"(pol)
      : "memory");
}
// Tensor copies (TMA) of a box of the tensor map (a __grid_constant__ kernel
// parameter) into shared memory, completion counted on *bar.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar,
                                            uint64_t pol) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
      " [%0], [%1, {%2, %3}], [%4], %5;\n" ::"r"(pipe_saddr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(pipe_saddr(bar)), "l"(pol)
      : "memory");
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(pipe_saddr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(pipe_saddr(bar))
      : "memory");
}
__device__ __forceinline__ void named_bar(int id, int n) { asm volatile("bar.sync %0, %1;\n" ::"r"(id), "r"(n) : "memory"); }
// Barrier over the n threads of named barrier `id` that also returns whether
// `ok` holds on every one of them.
__device__ __forceinline__ bool named_bar_all(int id, int n, bool ok) {
  unsigned r;
  asm volatile(
      "{\n .reg .pred p, q;\n setp.ne.u32 p, %1, 0;\n bar.red.and.pred q, %2, %3, p;\n selp.u32 %0, 1, 0, q;\n}\n"
      : "=r"(r)
      : "r"((unsigned)ok), "r"(id), "r"(n)
      : "memory");
  return r != 0;
}
// Orders this thread's generic-proxy shared-memory accesses before later
// asynchronous-proxy writes (the next bulk copy into the stage).
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// ----------------------------------------------------------- group shapes --
// SL slot lanes (channels per item: 128 bytes of storage), TPL line parts.
template <typename SC, class S_, int NG_>
struct PipeShape {
  using S = S_;
  static constexpr int SL = 128 / (int)sizeof(SC);
  static constexpr int GT = SL * S::TPL;  // threads per consumer group
  static constexpr int GW = GT / 32;      // warps per consumer group
  static constexpr int NG = NG_;
  static constexpr int kThreads = NG * GW * 32;
};
// consumer groups per CTA: about twelve warps (three per SM sub-partition, 168 registers each)
template <typename SC, class S>
constexpr int pipe_groups() {
  constexpr int gw = (128 / (int)sizeof(SC)) * S::TPL / 32;
  return gw < 1 ? 12 : (12 / gw < 1 ? 1 : 12 / gw);
}
template <typename SC, class S>
constexpr bool pipe_shape_ok() {
  return ((128 / (int)sizeof(SC)) * S::TPL) % 32 == 0;
}
// shared memory in front of the stages: twiddle rows, the barriers and the armed-item
// table, 128-byte aligned
template <class S, typename FT>
__host__ __device__ constexpr size_t pipe_head_bytes() {
  return ((size_t)2 * S::TPL * S::TS * sizeof(cpx_t<FT>) + kPipeMaxStages * (sizeof(uint64_t) + sizeof(int)) + 127) /
         128 * 128;
}

// ----------------------------------------------- line FFT through a stage --
// As fwd_AB / inv_BA of fft_reg.cuh, with the exchange in the group's stage
// (index stride SL) and group barriers.  `rel` runs after the last read of buf.
template <class S, int SL, typename C, typename Bar, typename Rel>
__device__ __forceinline__ void pipe_fwd_AB(C* x, C* __restrict__ buf, const C* __restrict__ tw, int t, int s, Bar bar,
                                            Rel rel) {
#pragma unroll
  for (int i = 0; i < S::E1; ++i) {
    rdft<S::N1, S::N, false>(x + i * S::N1, tw);
#pragma unroll
    for (int k1 = 1; k1 < S::N1; ++k1) x[i * S::N1 + k1] = cmul(x[i * S::N1 + k1], tw[i * S::N1 + k1]);
  }
  bar();  // every thread of the group has read its inputs from buf
#pragma unroll
  for (int i = 0; i < S::E1; ++i) {
    const int n2 = t + S::TPL * i;
#pragma unroll
    for (int k1 = 0; k1 < S::N1; ++k1) buf[(k1 * S::N2 + n2) * SL + s] = x[i * S::N1 + k1];
  }
  bar();
#pragma unroll
  for (int j = 0; j < S::E2; ++j) {
    const int k1 = t + S::TPL * j;
#pragma unroll
    for (int n2 = 0; n2 < S::N2; ++n2) x[j * S::N2 + n2] = buf[(k1 * S::N2 + n2) * SL + s];
  }
  rel();
#pragma unroll
  for (int j = 0; j < S::E2; ++j) rdft<S::N2, S::N, false>(x + j * S::N2, tw);
}

template <class S, int SL, typename C, typename Bar, typename Rel>
__device__ __forceinline__ void pipe_inv_BA(C* x, C* __restrict__ buf, const C* __restrict__ tw, int t, int s, Bar bar,
                                            Rel rel) {
#pragma unroll
  for (int j = 0; j < S::E2; ++j) {
    rdft<S::N2, S::N, true>(x + j * S::N2, tw);
#pragma unroll
    for (int m2 = 1; m2 < S::N2; ++m2) x[j * S::N2 + m2] = cmulc(x[j * S::N2 + m2], tw[j * S::N2 + m2]);
  }
  bar();  // buf is free
#pragma unroll
  for (int j = 0; j < S::E2; ++j) {
    const int k1 = t + S::TPL * j;
#pragma unroll
    for (int m2 = 0; m2 < S::N2; ++m2) buf[(k1 * S::N2 + m2) * SL + s] = x[j * S::N2 + m2];
  }
  bar();
#pragma unroll
  for (int i = 0; i < S::E1; ++i) {
    const int m2 = t + S::TPL * i;
#pragma unroll
    for (int k1 = 0; k1 < S::N1; ++k1) x[i * S::N1 + k1] = buf[(k1 * S::N2 + m2) * SL + s];
  }
  rel();
#pragma unroll
  for (int i = 0; i < S::E1; ++i) rdft<S::N1, S::N, true>(x + i * S::N1, tw);
}

// Common prologue: twiddle rows, one "full" barrier per stage.  Returns the stage base.
template <class S, typename FT>
__device__ __forceinline__ unsigned char* pipe_prologue(unsigned char* smem, int ns, uint64_t*& full, int*& armed) {
  using FC = cpx_t<FT>;
  FC* twf = reinterpret_cast<FC*>(smem);
  FC* twi = twf + S::TPL * S::TS;
  full = reinterpret_cast<uint64_t*>(twi + S::TPL * S::TS);
  armed = reinterpret_cast<int*>(full + kPipeMaxStages);
  build_line_twiddles<S, FT>(twf, twi);
  if (threadIdx.x == 0) {
    for (int i = 0; i < ns; ++i) {
      mbar_init(full + i, 1);
      armed[i] = -1;
    }
    mbar_fence_init();
  }
  __syncthreads();
  return smem + pipe_head_bytes<S, FT>();
}

// The ring of one CTA.  Its items are blockIdx.x + li * gridDim.x (li = 0, 1, ...);
// item li lives in stage li % ns, and its copy completes phase li / ns of that
// stage's barrier.  Thread 0 fills the ring; consumer group g takes li = g,
// g + NG, ...; after the last read of its stage the group fences its shared
// memory writes (the FFT exchange) against the asynchronous proxy, meets at its
// named barrier, and its leader arms and issues the copy of item li + ns into
// the same stage.  Consecutive uses of a stage may belong to different groups,
// so a group first waits until the stage's armed-item entry names its own item:
// a parity wait alone cannot tell phase li / ns from phase li / ns - 2 when the
// copy in between has not been armed yet.  issue(item, stage, bar) issues the
// copies of one item.
// body(li, item, stage, rel) transforms one item and calls rel() right after its
// last read of the stage.  On a fault every group leaves its loop; then thread 0
// waits (bounded) until the last copy armed on every stage has landed, so no
// copy is still writing the CTA's shared memory when it exits.
template <int NG, int GT, typename Issue, typename Body>
__device__ __forceinline__ void pipe_run(int nitems, int ns, unsigned char* stages, unsigned sb, uint64_t* full,
                                         int* armed, int* fault, Issue issue, Body body) {
  const int nloc = (int)blockIdx.x < nitems ? (nitems - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
  auto arm = [&](int li) {
    const int st = li % ns;
    *reinterpret_cast<volatile int*>(armed + st) = li;
    mbar_arrive_tx(full + st, sb);
    issue((int)blockIdx.x + li * (int)gridDim.x, stages + (size_t)st * sb, full + st);
  };
  if (threadIdx.x == 0)
    for (int li = 0; li < ns && li < nloc; ++li) arm(li);
  const int grp = threadIdx.x / GT, r = threadIdx.x - grp * GT, bid = 1 + grp;
  for (int li = grp; li < nloc; li += NG) {
    const int st = li % ns;
    const bool ok = smem_wait_eq(armed + st, li, fault, 3) && mbar_wait(full + st, (unsigned)(li / ns) & 1u, fault, 2);
    if (!named_bar_all(bid, GT, ok)) break;
    body(li, (int)blockIdx.x + li * (int)gridDim.x, stages + (size_t)st * sb, [&] {
      fence_proxy_async_smem();
      named_bar(bid, GT);
      if (r == 0 && li + ns < nloc) arm(li + ns);
    });
  }
  __syncthreads();
  if (threadIdx.x == 0 && *reinterpret_cast<volatile int*>(fault) != 0)
    for (int st = 0; st < ns && st < nloc; ++st) mbar_wait(full + st, (unsigned)(armed[st] / ns) & 1u, nullptr, 0);
}

// ------------------------------------------------------------------ passes --
template <typename ST, typename FT, class S, int NG>
__global__ void __launch_bounds__(PipeShape<cpx_t<ST>, S, NG>::kThreads, 1)
    k_pipe_row_fwd(const __grid_constant__ FockParams p) {
  using SC = cpx_t<ST>;
  using FC = cpx_t<FT>;
  using PS = PipeShape<SC, S, NG>;
  constexpr int SL = PS::SL;
  constexpr unsigned SB = (unsigned)(S::N * SL * sizeof(SC));
  if (p.active && !*p.active) return;
  pdl_launch_dependents();
  extern __shared__ __align__(128) unsigned char smem_pipe[];
  uint64_t* full;
  int* armed;
  const int ns = p.pipe_ns;
  unsigned char* stages = pipe_prologue<S, FT>(smem_pipe, ns, full, armed);
  const FC* twf = reinterpret_cast<const FC*>(smem_pipe);
  const int ng = p.nb2 / SL, nitems = ng * p.nk1;
  const int grp = threadIdx.x / PS::GT, r = threadIdx.x - grp * PS::GT;
  const int s = r % SL, t = r / SL, bid = 1 + grp;
  const bool has_ref = (p.flags & HF_FOCK_HAS_REFP) != 0;
  const uint64_t pol = pipe_policy_evict_first();
  auto bar = [&] { named_bar(bid, PS::GT); };
  pipe_run<NG, PS::GT>(
      nitems, ns, stages, SB, full, armed, p.fault,
      [&](int item, unsigned char* dst, uint64_t* b) {
        tma_load_2d(dst, &p.tmap_row, (item % ng) * SL * (int)sizeof(SC) / 4, (item / ng) * S::N, b, pol);
      },
      [&](int, int item, unsigned char* stage, auto rel) {
        const int g = item % ng, k1 = item / ng;
        const SC* stg = reinterpret_cast<const SC*>(stage);
        FC* xb = reinterpret_cast<FC*>(stage);
        FC x[S::E];
#pragma unroll
        for (int i = 0; i < S::E1; ++i)
#pragma unroll
          for (int n1 = 0; n1 < S::N1; ++n1) x[i * S::N1 + n1] = cvt<FC>(stg[S::idxA(t, i, n1) * SL + s]);
        if (has_ref) {
          const SC* R = static_cast<const SC*>(p.refP) + (size_t)k1 * S::N * p.nb2 + g * SL + s;
#pragma unroll
          for (int i = 0; i < S::E1; ++i)
#pragma unroll
            for (int n1 = 0; n1 < S::N1; ++n1)
              x[i * S::N1 + n1] = csub(x[i * S::N1 + n1], cvt<FC>(ld_stream(R + (size_t)S::idxA(t, i, n1) * p.nb2)));
        }
        pipe_fwd_AB<S, SL>(x, xb, twf + t * S::TS, t, s, bar, rel);
        FC* out = static_cast<FC*>(p.scratch) + ((size_t)g * p.nk1 + k1) * S::N * SL + s;
#pragma unroll
        for (int j = 0; j < S::E2; ++j)
#pragma unroll
          for (int k2 = 0; k2 < S::N2; ++k2) __stcg(out + S::idxB(t, j, k2) * SL, x[j * S::N2 + k2]);
      });
}

template <typename ST, typename FT, class S, int NG, bool VREAL>
__global__ void __launch_bounds__(PipeShape<cpx_t<ST>, S, NG>::kThreads, 1)
    k_pipe_col(const __grid_constant__ FockParams p) {
  using SC = cpx_t<ST>;
  using FC = cpx_t<FT>;
  using PS = PipeShape<SC, S, NG>;
  constexpr int SL = PS::SL;
  constexpr unsigned SB = (unsigned)(S::N * SL * sizeof(FC));
  pdl_launch_dependents();
  extern __shared__ __align__(128) unsigned char smem_pipe[];
  uint64_t* full;
  int* armed;
  const int ns = p.pipe_ns;
  unsigned char* stages = pipe_prologue<S, FT>(smem_pipe, ns, full, armed);
  const FC* twf = reinterpret_cast<const FC*>(smem_pipe);
  const FC* twi = twf + S::TPL * S::TS;
  const int ng = p.nb2 / SL, nitems = ng * p.nk2;
  const int grp = threadIdx.x / PS::GT, r = threadIdx.x - grp * PS::GT;
  const int s = r % SL, t = r / SL, bid = 1 + grp;
  const bool vr_scalar = (p.flags & HF_FOCK_VR_SCALAR) != 0;
  const size_t vstride = vr_scalar ? 1 : (size_t)p.nb2;
  const size_t rs = (size_t)p.nk2 * SL;
  auto bar = [&] { named_bar(bid, PS::GT); };
  pdl_wait();  // the row pass has finished writing the scratch
  if (p.active && !*p.active) return;
  pipe_run<NG, PS::GT>(
      nitems, ns, stages, SB, full, armed, p.fault,
      [&](int item, unsigned char* dst, uint64_t* b) {
        tma_load_3d(dst, &p.tmap_col, 0, item / ng, (item % ng) * p.nk1, b);
      },
      [&](int, int item, unsigned char* stage, auto rel) {
        const int g = item % ng, k2c = item / ng;
        const int vc = vr_scalar ? 0 : g * SL + s;
        // V-hat at this thread's pattern-B frequencies, in flight across the forward FFT
        using VT = std::conditional_t<VREAL, ST, SC>;
        VT vq[S::E];
#pragma unroll
        for (int j = 0; j < S::E2; ++j)
#pragma unroll
          for (int k2 = 0; k2 < S::N2; ++k2) {
            const size_t q = (size_t)S::idxB(t, j, k2) * p.nk2 + k2c;
            vq[j * S::N2 + k2] = ld_stream(static_cast<const VT*>(p.VR) + q * vstride + vc);
          }
        FC* xb = reinterpret_cast<FC*>(stage);
        FC x[S::E];
#pragma unroll
        for (int i = 0; i < S::E1; ++i)
#pragma unroll
          for (int n1 = 0; n1 < S::N1; ++n1) x[i * S::N1 + n1] = xb[S::idxA(t, i, n1) * SL + s];
        pipe_fwd_AB<S, SL>(x, xb, twf + t * S::TS, t, s, bar, [] {});
#pragma unroll
        for (int e = 0; e < S::E; ++e) {
          const FC v = x[e];
          if constexpr (VREAL) {
            const FT w = (FT)((double)vq[e] * p.scale);
            x[e] = mk<FC>(v.x * w, v.y * w);
          } else {
            const FT wr = (FT)((double)vq[e].x * p.scale), wi = (FT)((double)vq[e].y * p.scale);
            x[e] = mk<FC>(v.x * wr - v.y * wi, v.x * wi + v.y * wr);
          }
        }
        pipe_inv_BA<S, SL>(x, xb, twi + t * S::TS, t, s, bar, rel);
        FC* col = static_cast<FC*>(p.scratch) + ((size_t)g * p.nk1 * p.nk2 + k2c) * SL + s;
#pragma unroll
        for (int i = 0; i < S::E1; ++i)
#pragma unroll
          for (int n1 = 0; n1 < S::N1; ++n1) __stcg(col + S::idxA(t, i, n1) * rs, x[i * S::N1 + n1]);
      });
}

template <typename ST, typename FT, class S, int NG>
__global__ void __launch_bounds__(PipeShape<cpx_t<ST>, S, NG>::kThreads, 1)
    k_pipe_row_inv(const __grid_constant__ FockParams p) {
  using SC = cpx_t<ST>;
  using FC = cpx_t<FT>;
  using PS = PipeShape<SC, S, NG>;
  constexpr int SL = PS::SL;
  constexpr unsigned SB = (unsigned)(S::N * SL * sizeof(FC));
  pdl_launch_dependents();
  extern __shared__ __align__(128) unsigned char smem_pipe[];
  uint64_t* full;
  int* armed;
  const int ns = p.pipe_ns;
  unsigned char* stages = pipe_prologue<S, FT>(smem_pipe, ns, full, armed);
  const FC* twi = reinterpret_cast<const FC*>(smem_pipe) + S::TPL * S::TS;
  const int ng = p.nb2 / SL, nitems = ng * p.nk1;
  const int grp = threadIdx.x / PS::GT, r = threadIdx.x - grp * PS::GT;
  const int s = r % SL, t = r / SL, bid = 1 + grp;
  const uint64_t pol = pipe_policy_evict_first();
  auto bar = [&] { named_bar(bid, PS::GT); };
  SC* Sg = static_cast<SC*>(p.Sigma);
  const FC* scr = static_cast<const FC*>(p.scratch);
  pdl_wait();  // the column pass has finished writing the scratch
  if (p.active && !*p.active) return;
  pipe_run<NG, PS::GT>(
      nitems, ns, stages, SB, full, armed, p.fault,
      [&](int item, unsigned char* dst, uint64_t* b) {
        bulk_load(dst, scr + ((size_t)(item % ng) * p.nk1 + item / ng) * S::N * SL, SB, b, pol);
      },
      [&](int, int item, unsigned char* stage, auto rel) {
        const int g = item % ng, k1 = item / ng;
        const int c = g * SL + s;
        const SC cab = p.sigc != nullptr ? cvt<SC>(p.sigc[c]) : mk<SC>(0.0, 0.0);
        FC* xb = reinterpret_cast<FC*>(stage);
        FC x[S::E];
#pragma unroll
        for (int j = 0; j < S::E2; ++j)
#pragma unroll
          for (int k2 = 0; k2 < S::N2; ++k2) x[j * S::N2 + k2] = xb[S::idxB(t, j, k2) * SL + s];
        pipe_inv_BA<S, SL>(x, xb, twi + t * S::TS, t, s, bar, rel);
        // Sigma keeps the default L2 policy: the herm pass reads it back
        SC* out = Sg + (size_t)k1 * S::N * p.nb2 + c;
#pragma unroll
        for (int i = 0; i < S::E1; ++i)
#pragma unroll
          for (int m1 = 0; m1 < S::N1; ++m1)
            out[(size_t)S::idxA(t, i, m1) * p.nb2] = cadd(cvt<SC>(x[i * S::N1 + m1]), cab);
      });
}

// F = herm(h + Sigma) + diag(Hartree): tiles of kHermTile consecutive elements
// (whole k-point blocks, nb^2 | kHermTile), M = h + Sigma in shared memory, the
// transposed element read back from the tile.
constexpr int kHermThreads = 256, kHermPer = 4, kHermTile = kHermThreads * kHermPer;

template <typename ST>
__global__ void __launch_bounds__(kHermThreads) k_pipe_herm(const __grid_constant__ FockParams p) {
  using SC = cpx_t<ST>;
  __shared__ SC m[kHermTile];
  pdl_launch_dependents();
  pdl_wait();  // Sigma comes from the previous pass
  if (p.active && !*p.active) return;
  const int nb = p.nb, nb2 = p.nb2;
  const size_t total = (size_t)p.nk1 * p.nk2 * nb2;
  const SC* h = static_cast<const SC*>(p.h);
  const SC* Sg = static_cast<const SC*>(p.Sigma);
  SC* F = static_cast<SC*>(p.F);
  const double* hd = p.hdiag;
  for (size_t base = (size_t)blockIdx.x * kHermTile; base < total; base += (size_t)gridDim.x * kHermTile) {
    SC hv[kHermPer], sv[kHermPer];
#pragma unroll
    for (int u = 0; u < kHermPer; ++u) {
      const size_t e = base + u * kHermThreads + threadIdx.x;
      if (e < total) {
        hv[u] = ld_stream(h + e);
        sv[u] = __ldcs(Sg + e);
      }
    }
#pragma unroll
    for (int u = 0; u < kHermPer; ++u) {
      const size_t e = base + u * kHermThreads + threadIdx.x;
      if (e < total) m[u * kHermThreads + threadIdx.x] = cadd(hv[u], sv[u]);
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < kHermPer; ++u) {
      const int l = u * kHermThreads + threadIdx.x;
      const size_t e = base + l;
      if (e < total) {
        const int c = (int)(e % (size_t)nb2), a = c / nb, b = c - a * nb;
        const SC mab = m[l], mba = m[l - c + b * nb + a];
        SC f = mk<SC>(0.5 * ((double)mab.x + (double)mba.x), 0.5 * ((double)mab.y - (double)mba.y));
        if (hd != nullptr && a == b) f.x += (ST)hd[a];
        st_stream(F + e, f);
      }
    }
    __syncthreads();
  }
}

// Launches the four pipelined passes when they are asked for (HF_FOCK_PIPE) and apply (rows plan, exchange on,
// nb^2 a multiple of the slot lanes with whole rows per item, both mesh lengths
// with a pipelined shape, 16-byte aligned operands); otherwise leaves *handled
// false for the register passes.
template <typename ST, typename FT>
int pipe_fock(FockParams& p, cudaStream_t stream, bool* handled) {
  using SC = cpx_t<ST>;
  using FC = cpx_t<FT>;
  constexpr int SL = 128 / (int)sizeof(SC);
  *handled = false;
  if (!p.rows_plan || !(p.flags & HF_FOCK_EXCHANGE) || !(p.flags & HF_FOCK_PIPE)) return HF_OK;
  if (p.nb2 % SL != 0 || SL % p.nb != 0 || !p.fault) return HF_OK;
  const void* ptrs[] = {p.P, p.h, p.Sigma, p.F, p.scratch, p.VR};
  for (const void* q : ptrs)
    if (reinterpret_cast<uintptr_t>(q) % 16 != 0) return HF_OK;
  int dev = 0, sms = 148, optin = 0;
  HF_CUDA(cudaGetDevice(&dev));
  HF_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  HF_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  // stages per pass: as many as fit, at most kPipeMaxStages, at least groups + 1
  auto stages_for = [&](size_t head, size_t sb, int ng) {
    long long n = ((long long)optin - (long long)head) / (long long)sb;
    if (n > kPipeMaxStages) n = kPipeMaxStages;
    return n >= ng + 1 ? (int)n : 0;
  };
  int ns_row = 0, ns_inv = 0, ns_col = 0;
  bool row_ok = false, col_ok = false;
  auto probe_row = [&](auto shape) {
    using S = decltype(shape);
    if constexpr (pipe_shape_ok<SC, S>()) {
      constexpr int NG = pipe_groups<SC, S>();
      ns_row = stages_for(pipe_head_bytes<S, FT>(), (size_t)S::N * SL * sizeof(SC), NG);
      ns_inv = stages_for(pipe_head_bytes<S, FT>(), (size_t)S::N * SL * sizeof(FC), NG);
      row_ok = ns_row > 0 && ns_inv > 0;
    }
  };
  auto probe_col = [&](auto shape) {
    using S = decltype(shape);
    if constexpr (pipe_shape_ok<SC, S>()) {
      constexpr int NG = pipe_groups<SC, S>();
      ns_col = stages_for(pipe_head_bytes<S, FT>(), (size_t)S::N * SL * sizeof(FC), NG);
      col_ok = ns_col > 0;
    }
  };
  switch (p.nk2) {
#define HF_CASE(N, A, B, T) case N: probe_row(LineShape<N, A, B, T>{}); break;
    HF_FAST_SHAPES(HF_CASE)
#undef HF_CASE
  }
  switch (p.nk1) {
#define HF_CASE(N, A, B, T) case N: probe_col(LineShape<N, A, B, T>{}); break;
    HF_FAST_SHAPES(HF_CASE)
#undef HF_CASE
  }
  if (!row_ok || !col_ok) return HF_OK;
  // tensor maps of the row pass (P) and the column pass (scratch), in 4-byte words
  static PFN_cuTensorMapEncodeTiled_v12000 encode = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  }();
  if (!encode) return HF_OK;
  {
    const cuuint64_t esz = sizeof(SC), fsz = sizeof(FC), ng = (cuuint64_t)(p.nb2 / SL);
    const cuuint64_t gd_r[2] = {(cuuint64_t)p.nb2 * esz / 4, (cuuint64_t)p.nk1 * p.nk2};
    const cuuint64_t gs_r[1] = {(cuuint64_t)p.nb2 * esz};
    const cuuint32_t bx_r[2] = {(cuuint32_t)(SL * esz / 4), (cuuint32_t)p.nk2};
    const cuuint64_t gd_c[3] = {SL * fsz / 4, (cuuint64_t)p.nk2, ng * p.nk1};
    const cuuint64_t gs_c[2] = {SL * fsz, (cuuint64_t)p.nk2 * SL * fsz};
    const cuuint32_t bx_c[3] = {(cuuint32_t)(SL * fsz / 4), 1u, (cuuint32_t)p.nk1};
    const cuuint32_t es[3] = {1u, 1u, 1u};
    if (encode(&p.tmap_row, CU_TENSOR_MAP_DATA_TYPE_UINT32, 2, const_cast<void*>(p.P), gd_r, gs_r, bx_r, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS ||
        encode(&p.tmap_col, CU_TENSOR_MAP_DATA_TYPE_UINT32, 3, p.scratch, gd_c, gs_c, bx_c, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return HF_OK;  // not encodable here: the register passes take the build
  }
  int st = HF_OK;
  auto launch = [&](auto kern, int threads, int ns, size_t sb, size_t head, int nitems, bool pdl, const char* what) {
    if (st != HF_OK) return;
    const size_t smem = head + (size_t)ns * sb;
    st = allow_max_dynamic_smem((const void*)kern);
    if (st != HF_OK) return;
    p.pipe_ns = ns;
    const int grid = nitems < sms ? nitems : sms;
    cudaError_t e;
    if (pdl) e = launch_pass(kern, grid, threads, smem, stream, p);
    else {
      kern<<<grid, threads, smem, stream>>>(p);
      e = cudaGetLastError();
    }
    if (e != cudaSuccess) st = cuda_check(e, what);
  };
  auto row = [&](auto shape) {
    using S = decltype(shape);
    if constexpr (pipe_shape_ok<SC, S>()) {
      constexpr int NG = pipe_groups<SC, S>();
      using PS = PipeShape<SC, S, NG>;
      launch(k_pipe_row_fwd<ST, FT, S, NG>, PS::kThreads, ns_row, (size_t)S::N * SL * sizeof(SC),
             pipe_head_bytes<S, FT>(), p.nb2 / SL * p.nk1, false, "k_pipe_row_fwd");
    }
  };
  auto col = [&](auto shape) {
    using S = decltype(shape);
    if constexpr (pipe_shape_ok<SC, S>()) {
      constexpr int NG = pipe_groups<SC, S>();
      using PS = PipeShape<SC, S, NG>;
      auto kern = (p.flags & HF_FOCK_VR_REAL) ? k_pipe_col<ST, FT, S, NG, true> : k_pipe_col<ST, FT, S, NG, false>;
      launch(kern, PS::kThreads, ns_col, (size_t)S::N * SL * sizeof(FC), pipe_head_bytes<S, FT>(),
             p.nb2 / SL * p.nk2, true, "k_pipe_col");
    }
  };
  auto inv = [&](auto shape) {
    using S = decltype(shape);
    if constexpr (pipe_shape_ok<SC, S>()) {
      constexpr int NG = pipe_groups<SC, S>();
      using PS = PipeShape<SC, S, NG>;
      launch(k_pipe_row_inv<ST, FT, S, NG>, PS::kThreads, ns_inv, (size_t)S::N * SL * sizeof(FC),
             pipe_head_bytes<S, FT>(), p.nb2 / SL * p.nk1, true, "k_pipe_row_inv");
    }
  };
  switch (p.nk2) {
#define HF_CASE(N, A, B, T) case N: row(LineShape<N, A, B, T>{}); break;
    HF_FAST_SHAPES(HF_CASE)
#undef HF_CASE
  }
  switch (p.nk1) {
#define HF_CASE(N, A, B, T) case N: col(LineShape<N, A, B, T>{}); break;
    HF_FAST_SHAPES(HF_CASE)
#undef HF_CASE
  }
  switch (p.nk2) {
#define HF_CASE(N, A, B, T) case N: inv(LineShape<N, A, B, T>{}); break;
    HF_FAST_SHAPES(HF_CASE)
#undef HF_CASE
  }
  if (st != HF_OK) return st;
  {
    const size_t tiles = ((size_t)p.nk1 * p.nk2 * p.nb2 + kHermTile - 1) / kHermTile;
    int per_sm = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pipe_herm<ST>, kHermThreads, 0) != cudaSuccess ||
        per_sm < 1)
      per_sm = 1;
    const size_t cap = (size_t)sms * per_sm;
    const int grid = (int)(tiles < cap ? tiles : cap);
    const cudaError_t e = launch_pass(k_pipe_herm<ST>, grid, kHermThreads, 0, stream, p);
    if (e != cudaSuccess) return cuda_check(e, "k_pipe_herm");
  }
  *handled = true;
  return HF_OK;
}

}  // namespace hf
