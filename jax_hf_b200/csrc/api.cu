// Error reporting and version of the hf_b200 C ABI.
#include <cuda.h>

#include <map>
#include <mutex>
#include <set>
#include <string>

#include "common.cuh"

namespace hf {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

int fail(int status, const std::string& msg) {
  g_last_error = msg;
  return status;
}

int cuda_check(cudaError_t e, const char* what) {
  g_last_error = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
  return HF_ERR_CUDA;
}

// The unique id (cuCtxGetId) of the CUDA context current on this thread.  Per-device
// state the library caches (symbol addresses, kernel attributes) is keyed on it: a
// context that cudaDeviceReset tears down and the runtime creates again has a new id,
// so nothing cached for the old one (a device address, a raised smem cap) is reused.
// The driver functions come through cudaGetDriverEntryPoint (no libcuda link).  When
// no context is current yet, the device's primary context is made current first.
int context_id(unsigned long long* id) {
  using GetCurrent = CUresult (*)(CUcontext*);
  using GetId = CUresult (*)(CUcontext, unsigned long long*);
  static const std::pair<GetCurrent, GetId> fns = [] {
    void* a = nullptr;
    void* b = nullptr;
    cudaDriverEntryPointQueryResult qa, qb;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa) != cudaSuccess ||
        qa != cudaDriverEntryPointSuccess)
      a = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb) != cudaSuccess ||
        qb != cudaDriverEntryPointSuccess)
      b = nullptr;
    return std::make_pair(reinterpret_cast<GetCurrent>(a), reinterpret_cast<GetId>(b));
  }();
  if (!fns.first || !fns.second) return fail(HF_ERR_CUDA, "cuCtxGetCurrent / cuCtxGetId not available");
  CUcontext c = nullptr;
  if (fns.first(&c) != CUDA_SUCCESS) return fail(HF_ERR_CUDA, "cuCtxGetCurrent failed");
  if (!c) {
    int dev = 0;
    HF_CUDA(cudaGetDevice(&dev));
    HF_CUDA(cudaSetDevice(dev));  // initialises and binds the primary context
    if (fns.first(&c) != CUDA_SUCCESS || !c) return fail(HF_ERR_CUDA, "no CUDA context current");
  }
  if (fns.second(c, id) != CUDA_SUCCESS) return fail(HF_ERR_CUDA, "cuCtxGetId failed");
  return HF_OK;
}

// Lifts a kernel's dynamic shared-memory cap to the device's opt-in maximum, once
// per (kernel, context).  The cap only bounds launches (occupancy follows each
// launch's own size); a per-call cap could drop below the size of a launch that
// another stream (a batch lane, a captured graph) still has to make.
int allow_max_dynamic_smem(const void* fn) {
  static std::mutex mu;
  static std::set<std::pair<const void*, unsigned long long>> done;
  unsigned long long ctx = 0;
  int st = context_id(&ctx);
  if (st) return st;
  std::lock_guard<std::mutex> lock(mu);
  if (done.count({fn, ctx})) return HF_OK;
  int dev = 0, optin = 0;
  HF_CUDA(cudaGetDevice(&dev));
  HF_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  cudaFuncAttributes fa;
  HF_CUDA(cudaFuncGetAttributes(&fa, fn));
  HF_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes));
  done.insert({fn, ctx});
  return HF_OK;
}

// Device address of a __device__ variable in the current context, looked up once per
// (variable, context) with cudaGetSymbolAddress.  The first lookup of a variable may
// load the library's module on the device, so it belongs outside stream capture.
int symbol_address(const void* symbol, void** out) {
  static std::mutex mu;
  static std::map<std::pair<const void*, unsigned long long>, void*> cache;
  unsigned long long ctx = 0;
  int st = context_id(&ctx);
  if (st) return st;
  std::lock_guard<std::mutex> lock(mu);
  auto it = cache.find({symbol, ctx});
  if (it == cache.end()) {
    void* p = nullptr;
    HF_CUDA(cudaGetSymbolAddress(&p, symbol));
    it = cache.emplace(std::make_pair(symbol, ctx), p).first;
  }
  *out = it->second;
  return HF_OK;
}

}  // namespace hf

extern "C" const char* hf_last_error(void) { return hf::g_last_error.c_str(); }

extern "C" const char* hf_status_string(int status) {
  switch (status) {
    case HF_OK: return "ok";
    case HF_ERR_INVALID: return "invalid argument";
    case HF_ERR_UNSUPPORTED: return "unsupported size";
    case HF_ERR_CUDA: return "CUDA error";
    case HF_ERR_WORKSPACE: return "workspace too small";
    case HF_ERR_NONFINITE: return "non-finite value";
    case HF_ERR_MAXITER: return "iteration cap reached";
    case HF_ERR_ABORTED: return "aborted";
    default: return "unknown status";
  }
}

extern "C" int hf_version(void) { return 1; }
