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
// and it stays allocated until the process exits.  Host code cannot use the
// array's name as a device address, so the first call on each device looks
// the address up with cudaGetSymbolAddress while that device is current and
// caches it; make that first call before any stream capture.
//
// Every call on a device uses the same array.  Calls that overlap on the GPU
// (different streams, or host threads with no ordering) race on it and must be
// serialised by the caller.  Nothing in the array has to start at zero: the
// row pass writes every spectrum entry, and the density partial sums and the
// constant terms are fully rewritten before they are read.
#include <mutex>

#include "common.cuh"

namespace hf {
int fock_build_internal(void* stream, int dtype, unsigned flags, int nk1, int nk2, int nb, const void* P,
                        const void* h, const void* VR, const void* refP, const void* HH, const void* w2d,
                        int n_contact, const void* contact_g, const void* contact_Oi, const void* contact_Oj,
                        void* Sigma, void* H, void* F, void* workspace, size_t workspace_bytes,
                        const int* active);
}

static __device__ __align__(256) unsigned char g_fock_static_scratch[HF_FOCK_STATIC_SCRATCH_BYTES];

namespace {
constexpr int kMaxDevices = 128;
std::mutex g_scratch_mutex;
void* g_scratch_ptr[kMaxDevices] = {};
}  // namespace

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
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return hf::cuda_check(e, "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) return hf::fail(HF_ERR_UNSUPPORTED, "device ordinal out of range");
  void* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_ptr[dev]) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_fock_static_scratch);
      if (e != cudaSuccess) return hf::cuda_check(e, "cudaGetSymbolAddress(g_fock_static_scratch)");
      g_scratch_ptr[dev] = p;
    }
    scratch = g_scratch_ptr[dev];
  }
  return hf::fock_build_internal(stream, dtype, flags, nk1, nk2, nb, P, h, VR, refP, HH, w2d, n_contact,
                                 contact_g, contact_Oi, contact_Oj, Sigma, H, F, scratch,
                                 (size_t)HF_FOCK_STATIC_SCRATCH_BYTES, nullptr);
}
