// Pipelined Fock passes, storage float / FFT float (instantiation unit).
#include "fock_fast.cuh"
#include "fock_pipe.cuh"

namespace hf {
template int pipe_fock<float, float>(FockParams&, cudaStream_t, bool*);
}  // namespace hf
