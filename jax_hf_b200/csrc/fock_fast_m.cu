// Fast Fock passes, storage double / FFT float (instantiation unit).
#include "fock_fast.cuh"

namespace hf {
template int fast_fock<double, float>(FockParams&, cudaStream_t, bool*);
}  // namespace hf
