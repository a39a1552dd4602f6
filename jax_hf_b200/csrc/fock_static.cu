// Fock build whose scratch is a library-owned static device array.
//
// Who needs it: callers that must not allocate device memory during a call.
// Examples are a framework custom-call handler whose framework owns every
// device buffer (it hands kernels only the operands and results), and code
// inside CUDA stream capture, where a cudaMalloc either is rejected or
// silently synchronises the device.  Such callers cannot provide the
// workspace that hf_fock_build requires, so this entry point brings its own.
//
// The scratch is one file-scope array of HF_FOCK_STATIC_SCRATCH_BYTES (40 MiB).
// The driver allocates it when it loads this library module on a device (with
// lazy module loading: on the first call of this entry point on that device)
// and it stays allocated until the context is destroyed.  Host code cannot use
// the array's name as a device address, so the first call in each CUDA context
// looks the address up with cudaGetSymbolAddress and caches it under the
// context's unique id; make that first call before any stream capture.  After a
// cudaDeviceReset the runtime creates a new context with a new id, and the
// next call looks the address up again.
//
// Every call on a device uses the same array.  Calls that overlap on the GPU
// (different streams, or host threads with no ordering) race on it and must be
// serialised by the caller.  Nothing in the array has to start at zero: the
// row pass writes every spectrum entry, and the density partial sums and the
// constant terms are fully rewritten before they are read.
#include "common.cuh"

namespace hf {
int fock_build_internal(void* stream, int dtype, unsigned flags, int nk1, int nk2, int nb, const void* P,
                        const void* h, const void* VR, const void* refP, const void* HH, const void* w2d,
                        int n_contact, const void* contact_g, const void* contact_Oi, const void* contact_Oj,
                        void* Sigma, void* H, void* F, void* workspace, size_t workspace_bytes,
                        const int* active);
}

static __device__ __align__(256) unsigned char g_fock_static_scratch[HF_FOCK_STATIC_SCRATCH_BYTES];


extern "C" int hf_fock_build_static_scratch(void* stream, int dtype, unsigned flags, int nk1, int nk2, int nb,
                                            const void* P, const void* h, const void* VR, const void* refP,
                                            const void* HH, const void* w2d, int n_contact,
                                            const void* contact_g, const void* contact_Oi,
                                            const void* contact_Oj, void* Sigma, void* H, void* F) {
  size_t need = 0;
  int st = hf_fock_workspace_size(dtype, flags, nk1, nk2, nb, &need);
  if (st != HF_OK) return st;
  if (need > (size_t)HF_FOCK_STATIC_SCRATCH_BYTES)
    return hf::fail(HF_ERR_WORKSPACE,
                    "hf_fock_build_static_scratch: this mesh needs " + std::to_string(need) +
                        " bytes of scratch, more than the fixed " +
                        std::to_string((size_t)HF_FOCK_STATIC_SCRATCH_BYTES) +
                        " bytes of the static array; use hf_fock_build with a workspace");
  void* scratch = nullptr;
  st = hf::symbol_address(reinterpret_cast<const void*>(g_fock_static_scratch), &scratch);
  if (st != HF_OK) return st;
  return hf::fock_build_internal(stream, dtype, flags, nk1, nk2, nb, P, h, VR, refP, HH, w2d, n_contact,
                                 contact_g, contact_Oi, contact_Oj, Sigma, H, F, scratch,
                                 (size_t)HF_FOCK_STATIC_SCRATCH_BYTES, nullptr);
}
