// Pipelined Fock passes, storage double / FFT double (instantiation unit).
#include "fock_fast.cuh"
#include "fock_pipe.cuh"

namespace hf {
template int pipe_fock<double, double>(FockParams&, cudaStream_t, bool*);
}  // namespace hf
