// Error reporting and version of the hf_b200 C ABI.
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
