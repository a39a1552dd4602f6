// Parameters of the Fock-build kernels (shared by the generic and fast paths).
#pragma once

#include <cuda.h>

#include "fft_engine.cuh"

namespace hf {

constexpr int kMaxNb = 32;
constexpr int kMaxSlotTable = 1280;
constexpr int kThreads = 256;

struct FockParams {
  int nk1, nk2, nb, nb2, LS, ngroups;
  unsigned flags;
  int n_contact;
  double scale;  // -1 / (nk1 nk2)
  FftPlan1D row, col;
  const void* P;
  const void* h;
  const void* VR;
  const void* refP;
  const void* w2d;
  const void* HH;
  const void* cg;
  const void* cOi;
  const void* cOj;
  void* Sigma;
  void* F;
  void* Hout;
  void* scratch;
  double2* rho_part;  // [nk1][ngroups*LS]
  double2* sigc;      // [nb*nb] contact sigma
  double* hdiag;      // [nb] Hartree diagonal
  const int* active;  // optional device flag: kernels return at once when *active == 0
  int rows_plan;      // slot groups are whole matrix rows; partner = (group << 8) | slot
  int pipe_ns;        // stages of the pipelined passes (set per launch)
  int* fault;         // device word: a bounded wait of a pipelined pass that ran out records a code here
  CUtensorMap tmap_row;  // pipelined row pass: P as [nk1 nk2][nb^2] 4-byte words, box = SL channels x nk2 k-points
  CUtensorMap tmap_col;  // pipelined column pass: scratch as [group nk1][nk2][SL], box = one column
  int16_t chan[kMaxSlotTable];
  int16_t partner[kMaxSlotTable];
};

// Mesh lengths with a specialised register-FFT pass: N = N1 * N2 split over TPL
// threads per line (see fft_reg.cuh).
#define HF_FAST_SHAPES(X) \
  X(12, 4, 3, 1)          \
  X(16, 4, 4, 4)          \
  X(24, 4, 6, 2)          \
  X(32, 4, 8, 4)          \
  X(36, 6, 6, 6)          \
  X(48, 4, 12, 4)         \
  X(64, 8, 8, 8)          \
  X(72, 6, 12, 6)         \
  X(96, 8, 12, 4)         \
  X(128, 8, 16, 8)        \
  X(144, 12, 12, 12)      \
  X(192, 8, 24, 8)

inline bool fast_length(int n) {
  switch (n) {
#define HF_CASE(N, A, B, T) case N:
    HF_FAST_SHAPES(HF_CASE)
#undef HF_CASE
    return true;
    default: return false;
  }
}

// Launches the fast passes when both mesh lengths have a fast shape.
template <typename ST, typename FT>
int fast_fock(FockParams& p, cudaStream_t stream, bool* handled);
// Launches the bulk-copy pipelined passes (fock_pipe.cuh) where they apply.
template <typename ST, typename FT>
int pipe_fock(FockParams& p, cudaStream_t stream, bool* handled);

}  // namespace hf
