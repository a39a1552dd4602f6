// Fast Fock passes, storage double / FFT double (instantiation unit).
#include "fock_fast.cuh"

namespace hf {
template int fast_fock<double, double>(FockParams&, cudaStream_t, bool*);
}  // namespace hf
