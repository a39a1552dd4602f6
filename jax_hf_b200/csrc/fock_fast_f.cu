// Fast Fock passes, storage float / FFT float (instantiation unit).
#include "fock_fast.cuh"

namespace hf {
template int fast_fock<float, float>(FockParams&, cudaStream_t, bool*);
}  // namespace hf
