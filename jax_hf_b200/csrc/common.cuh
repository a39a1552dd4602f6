// Shared device/host helpers for the hf_b200 CUDA library (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>
#include <string>

#include "../../include/hf_b200.h"

namespace hf {

// ---------------------------------------------------------------- errors ----
void set_error(const std::string& msg);
int fail(int status, const std::string& msg);
int cuda_check(cudaError_t e, const char* what);
int allow_max_dynamic_smem(const void* fn);
int context_id(unsigned long long* id);
// Slot-indexed DIIS steps for the device-resident SCF loop (ops.cu): the history slot is
// a device int, so one captured iteration serves every slot
int scf_residuals_slot(void* stream, int nk, int nb, const void* F, const void* P, const void* Pn, const double* w,
                       void* R, size_t stride, const int* slot, void* delta, double* sums3, void* ws);
int copy_to_slot(void* stream, size_t n, const void* x, void* hist, const int* slot);
// n <= 4 inner products of hf_jdot's form in one pass, each equal to hf_jdot's (ops.cu)
int jdot_multi(void* stream, size_t nk, int nb, int n, const void* const* aX, const void* const* bX,
               const double* const* wX, const double* const* ap, const double* const* bp, const double* const* wp,
               double* out, void* ws);
int gram_row_slot(void* stream, int n, const int* slot, size_t stride, int nk, int nb, const void* R,
                  const double* w, double* b_out, void* ws);
// eigh of herm(A) (mode 0) or herm(i A) (mode 1), complex128, nb <= 8, ascending, the
// lane-per-column Jacobi (solver_cg.cu)
int eigh_cols(void* stream, int nk, int nb, const void* A, double* w, void* V, int mode);
// P = herm(Q diag(p) Q^H), complex128, nb <= 8, lane-per-column kernel (solver_cg.cu)
int rows_density(void* stream, int nk, int nb, const void* Q, const double* p, void* P);
int symbol_address(const void* symbol, void** out);

#define HF_SMEM_CAP(...)                                              \
  do {                                                                \
    const int _st = ::hf::allow_max_dynamic_smem((const void*)(__VA_ARGS__));  \
    if (_st) return _st;                                              \
  } while (0)

#define HF_CUDA(call)                                            \
  do {                                                           \
    cudaError_t _e = (call);                                     \
    if (_e != cudaSuccess) return ::hf::cuda_check(_e, #call);   \
  } while (0)

#define HF_LAUNCH_CHECK(what)                                    \
  do {                                                           \
    cudaError_t _e = cudaGetLastError();                         \
    if (_e != cudaSuccess) return ::hf::cuda_check(_e, what);    \
  } while (0)

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// --------------------------------------------------------------- complex ----
template <typename T> struct Cpx;
template <> struct Cpx<double> { using type = double2; };
template <> struct Cpx<float> { using type = float2; };
template <typename T> using cpx_t = typename Cpx<T>::type;

template <typename C> __host__ __device__ __forceinline__ C mk(double x, double y) {
  C r; r.x = x; r.y = y; return r;
}
template <typename C, typename T> __host__ __device__ __forceinline__ C make_c(T x, T y) {
  C r; r.x = x; r.y = y; return r;
}
__host__ __device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
__host__ __device__ __forceinline__ double2 cmulc(double2 a, double2 b) {
  return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__host__ __device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
  return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__host__ __device__ __forceinline__ double2 conj(double2 a) { return make_double2(a.x, -a.y); }
__host__ __device__ __forceinline__ float2 conj(float2 a) { return make_float2(a.x, -a.y); }
__host__ __device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
// multiply by -i (forward) / +i
__host__ __device__ __forceinline__ double2 mul_mi(double2 a) { return make_double2(a.y, -a.x); }
__host__ __device__ __forceinline__ float2 mul_mi(float2 a) { return make_float2(a.y, -a.x); }
__host__ __device__ __forceinline__ double2 mul_pi(double2 a) { return make_double2(-a.y, a.x); }
__host__ __device__ __forceinline__ float2 mul_pi(float2 a) { return make_float2(-a.y, a.x); }

template <typename To, typename From> __device__ __forceinline__ To cvt(From a) {
  To r; r.x = a.x; r.y = a.y; return r;
}

// ------------------------------------------------- compensated summation ----
// Neumaier (1974) running sum: s + c carries the exact sum of the added terms
// to within O(eps^2) relative error, independent of the number of terms.
struct KSum {
  double s, c;
  __device__ __forceinline__ KSum() : s(0.0), c(0.0) {}
  __device__ __forceinline__ void add(double x) {
    double t = s + x;
    if (fabs(s) >= fabs(x)) c += (s - t) + x; else c += (x - t) + s;
    s = t;
  }
  __device__ __forceinline__ void merge(const KSum& o) { add(o.s); add(o.c); }
  __device__ __forceinline__ double value() const { return s + c; }
};

__device__ __forceinline__ KSum warp_reduce(KSum v) {
  for (int off = 16; off > 0; off >>= 1) {
    KSum o;
    o.s = __shfl_xor_sync(0xffffffffu, v.s, off);
    o.c = __shfl_xor_sync(0xffffffffu, v.c, off);
    v.merge(o);
  }
  return v;
}

__device__ __forceinline__ double warp_sum(double v) {
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

// Block-wide compensated reduction; result valid in thread 0.  `sm` needs
// 2*32 doubles.  Deterministic for a fixed launch shape.
__device__ __forceinline__ KSum block_reduce(KSum v, double* sm) {
  v = warp_reduce(v);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
  __syncthreads();
  if (lane == 0) { sm[2 * wid] = v.s; sm[2 * wid + 1] = v.c; }
  __syncthreads();
  KSum r;
  if (wid == 0) {
    if (lane < nw) { r.s = sm[2 * lane]; r.c = sm[2 * lane + 1]; }
    r = warp_reduce(r);
  }
  return r;
}

}  // namespace hf
