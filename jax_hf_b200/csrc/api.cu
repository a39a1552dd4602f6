// Error reporting and version of the hf_b200 C ABI.
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

// Lifts a kernel's dynamic shared-memory cap to the device's opt-in maximum, once
// per (kernel, device).  The cap only bounds launches (occupancy follows each
// launch's own size); a per-call cap could drop below the size of a launch that
// another stream (a batch lane, a captured graph) still has to make.
int allow_max_dynamic_smem(const void* fn) {
  static std::mutex mu;
  static std::set<std::pair<const void*, int>> done;
  int dev = 0;
  HF_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  if (done.count({fn, dev})) return HF_OK;
  int optin = 0;
  HF_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  cudaFuncAttributes fa;
  HF_CUDA(cudaFuncGetAttributes(&fa, fn));
  HF_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes));
  done.insert({fn, dev});
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
