// Coarse -> fine k-grid resampling for multigrid continuation
// (utils.py:477-535 resample_kgrid, continuation.py:47-50 _resample_density).
//
// The two leading axes are a periodic k-grid stored centered (k = 0 at index
// n // 2).  Output index j of an axis maps to the input position
// u = (j - m/2) (n/m) + n/2 (integer halves), taken in the array's real
// precision with every operation rounded separately (as the reference
// evaluates it), and the value is (1 - f) x[floor(u) mod n] + f x[floor(u)+1
// mod n], f = u - floor(u); the first axis is interpolated first, then the
// second.  An axis whose length does not change is copied.  One thread per
// output component, grid-stride; the reads of a k-point are contiguous.
#include "common.cuh"

namespace hf {

template <typename R>
struct AxisMap {
  int i0, i1;
  R f;
  bool copy;
};

template <typename R>
__device__ __forceinline__ AxisMap<R> axis_map(int j, int n, int m) {
  AxisMap<R> a;
  if (n == m) {
    a.i0 = a.i1 = j;
    a.f = R(0);
    a.copy = true;
    return a;
  }
  R u;
  if constexpr (sizeof(R) == 8) {
    u = __dadd_rn(__dmul_rn(__dsub_rn((double)j, (double)(m / 2)), __ddiv_rn((double)n, (double)m)), (double)(n / 2));
  } else {
    u = __fadd_rn(__fmul_rn(__fsub_rn((float)j, (float)(m / 2)), __fdiv_rn((float)n, (float)m)), (float)(n / 2));
  }
  const R fl = floor(u);
  int i0 = (int)fl % n;
  if (i0 < 0) i0 += n;
  a.i0 = i0;
  a.i1 = (i0 + 1) % n;
  a.f = u - fl;
  a.copy = false;
  return a;
}

template <typename R>
__device__ __forceinline__ R lerp_ref(R a, R b, R f) {  // (1 - f) a + f b, separately rounded
  if constexpr (sizeof(R) == 8) return __dadd_rn(__dmul_rn(__dsub_rn(1.0, f), a), __dmul_rn(f, b));
  else return __fadd_rn(__fmul_rn(__fsub_rn(1.0f, f), a), __fmul_rn(f, b));
}

// value of component e at output k-point (j1, j2)
template <typename R>
__device__ __forceinline__ R resample_at(const R* __restrict__ x, int n1, int n2, long long nc, const AxisMap<R>& A,
                                         const AxisMap<R>& B, long long e) {
  auto at = [&](int a, int b) { return x[((long long)a * n2 + b) * nc + e]; };
  const R t0 = A.copy ? at(A.i0, B.i0) : lerp_ref(at(A.i0, B.i0), at(A.i1, B.i0), A.f);
  if (B.copy) return t0;
  const R t1 = A.copy ? at(A.i0, B.i1) : lerp_ref(at(A.i0, B.i1), at(A.i1, B.i1), A.f);
  return lerp_ref(t0, t1, B.f);
}

template <typename R>
__global__ void k_resample(int n1, int n2, int m1, int m2, long long nc, const R* __restrict__ x, R* __restrict__ y) {
  const long long total = (long long)m1 * m2 * nc;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total; q += (long long)gridDim.x * blockDim.x) {
    const long long e = q % nc, kp = q / nc;
    const int j2 = (int)(kp % m2), j1 = (int)(kp / m2);
    y[q] = resample_at(x, n1, n2, nc, axis_map<R>(j1, n1, m1), axis_map<R>(j2, n2, m2), e);
  }
}

// hermitised density: out_ab = (Q_ab + conj(Q_ba)) / 2, Q = resampled P (complex, nb x nb per k-point)
template <typename R>
__global__ void k_resample_density(int n1, int n2, int m1, int m2, int nb, const R* __restrict__ x, R* __restrict__ y) {
  const long long nc = 2LL * nb * nb;
  const long long total = (long long)m1 * m2 * nb * nb;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total; q += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(q % (nb * nb));
    const long long kp = q / (nb * nb);
    const int j2 = (int)(kp % m2), j1 = (int)(kp / m2);
    const int a = c / nb, b = c - a * nb, ct = b * nb + a;
    const AxisMap<R> A = axis_map<R>(j1, n1, m1), B = axis_map<R>(j2, n2, m2);
    const R re = resample_at(x, n1, n2, nc, A, B, 2LL * c), im = resample_at(x, n1, n2, nc, A, B, 2LL * c + 1);
    const R ret = resample_at(x, n1, n2, nc, A, B, 2LL * ct), imt = resample_at(x, n1, n2, nc, A, B, 2LL * ct + 1);
    y[2 * q] = R(0.5) * (re + ret);
    y[2 * q + 1] = R(0.5) * (im - imt);
  }
}

static int resample_check(int dtype, int n1, int n2, int m1, int m2, long long nc, const void* x, const void* y) {
  if (dtype != HF_C128 && dtype != HF_C64) return fail(HF_ERR_INVALID, "dtype must be HF_C128 or HF_C64");
  if (n1 <= 0 || n2 <= 0) return fail(HF_ERR_INVALID, "input k-grid dimensions must be positive");
  if (m1 <= 0 || m2 <= 0) return fail(HF_ERR_INVALID, "n_new must be a positive integer.");
  if (nc <= 0) return fail(HF_ERR_INVALID, "components per k-point must be positive");
  if (!x || !y) return fail(HF_ERR_INVALID, "x and y must be non-NULL");
  if (x == y) return fail(HF_ERR_INVALID, "x and y must not alias");
  return HF_OK;
}

static int grid_for(long long total) {
  long long g = (total + 255) / 256;
  return (int)(g < 148 * 16 ? (g < 1 ? 1 : g) : 148 * 16);
}

}  // namespace hf

using namespace hf;

extern "C" int hf_resample_kgrid(void* stream, int dtype, int n1, int n2, int m1, int m2, long long ncomp,
                                 const void* x, void* y) {
  int st = resample_check(dtype, n1, n2, m1, m2, ncomp, x, y);
  if (st) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int g = grid_for((long long)m1 * m2 * ncomp);
  if (dtype == HF_C128)
    k_resample<double><<<g, 256, 0, s>>>(n1, n2, m1, m2, ncomp, static_cast<const double*>(x), static_cast<double*>(y));
  else
    k_resample<float><<<g, 256, 0, s>>>(n1, n2, m1, m2, ncomp, static_cast<const float*>(x), static_cast<float*>(y));
  HF_LAUNCH_CHECK("k_resample");
  return HF_OK;
}

extern "C" int hf_resample_density(void* stream, int dtype, int n1, int n2, int m1, int m2, int nb, const void* P,
                                   void* out) {
  if (nb <= 0) return fail(HF_ERR_INVALID, "nb must be positive");
  int st = resample_check(dtype, n1, n2, m1, m2, 2LL * nb * nb, P, out);
  if (st) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int g = grid_for((long long)m1 * m2 * nb * nb);
  if (dtype == HF_C128)
    k_resample_density<double><<<g, 256, 0, s>>>(n1, n2, m1, m2, nb, static_cast<const double*>(P), static_cast<double*>(out));
  else
    k_resample_density<float><<<g, 256, 0, s>>>(n1, n2, m1, m2, nb, static_cast<const float*>(P), static_cast<float*>(out));
  HF_LAUNCH_CHECK("k_resample_density");
  return HF_OK;
}
