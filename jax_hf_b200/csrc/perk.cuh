// Warp-level nb x nb complex routines (matrices in shared memory, double).
// A warp owns one matrix; lanes stride over elements / rows / rotation pairs.
#pragma once

#include "common.cuh"

namespace hf {

__host__ __device__ inline size_t jacobi_smem_elems(int nb) { return (size_t)2 * nb * nb + nb + 40; }

__device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
  // Smith's algorithm
  if (fabs(b.x) >= fabs(b.y)) {
    const double r = b.y / b.x, den = b.x + b.y * r;
    return make_double2((a.x + a.y * r) / den, (a.y - a.x * r) / den);
  }
  const double r = b.x / b.y, den = b.x * r + b.y;
  return make_double2((a.x * r + a.y) / den, (a.y * r - a.x) / den);
}

// c(tau, lam) = (1 + i x)/(1 - i x), x = tau lam / 2   (solver.py:169-175)
__device__ __forceinline__ double2 cayley_factor(double tau, double lam) {
  const double x = tau * lam * 0.5;
  const double d = 1.0 + x * x;
  return make_double2((1.0 - x * x) / d, 2.0 * x / d);
}

// t[i,j] = sum_n q[i,n] p[n] conj(q[j,n])
__device__ __forceinline__ void warp_density(const double2* q, const double* p, double2* t, int nb, int lane) {
  const int nb2 = nb * nb;
  for (int e = lane; e < nb2; e += 32) {
    const int i = e / nb, j = e - i * nb;
    double2 acc = make_double2(0.0, 0.0);
    for (int n = 0; n < nb; ++n) acc = cadd(acc, cscale(cmulc(q[i * nb + n], q[j * nb + n]), p[n]));
    t[e] = acc;
  }
}

// f <- Q^H F Q   (t: nb*nb scratch)
__device__ __forceinline__ void warp_qhaq(const double2* q, double2* f, double2* t, int nb, int lane) {
  const int nb2 = nb * nb;
  for (int e = lane; e < nb2; e += 32) {
    const int i = e / nb, m = e - i * nb;
    double2 acc = make_double2(0.0, 0.0);
    for (int j = 0; j < nb; ++j) acc = cadd(acc, cmul(f[i * nb + j], q[j * nb + m]));
    t[e] = acc;
  }
  __syncwarp();
  for (int e = lane; e < nb2; e += 32) {
    const int n = e / nb, m = e - n * nb;
    double2 acc = make_double2(0.0, 0.0);
    for (int i = 0; i < nb; ++i) acc = cadd(acc, cmulc(t[i * nb + m], q[i * nb + n]));
    f[e] = acc;
  }
}

// Cyclic Jacobi on Hermitian a (overwritten by its diagonalised form), v <- eigenvectors
// (columns, unsorted).  rot: scratch of >= 2*(nb/2+1) double2.
__device__ inline void warp_jacobi_eigh(double2* a, double2* v, double2* rot, int nb, int lane, double tol) {
  const int nb2 = nb * nb;
  double fro = 0.0;
  for (int e = lane; e < nb2; e += 32) {
    const int i = e / nb, j = e - i * nb;
    v[e] = make_double2(i == j ? 1.0 : 0.0, 0.0);
    fro += a[e].x * a[e].x + a[e].y * a[e].y;
  }
  fro = sqrt(warp_sum(fro));
  const double thr = fmax(tol * fro, 1e-300);
  const int m = nb + (nb & 1);
  const int npairs = m / 2;
  __syncwarp();
  if (nb == 1) return;
  for (int sweep = 0; sweep < 60; ++sweep) {
    bool any_sweep = false;
    for (int r = 0; r < m - 1; ++r) {
      bool act = false;
      if (lane < npairs) {
        const int pa = lane == 0 ? 0 : 1 + ((lane - 1 + r) % (m - 1));
        const int pbpos = m - 1 - lane;
        const int pb = 1 + ((pbpos - 1 + r) % (m - 1));
        const int p = min(pa, pb), q = max(pa, pb);
        double c = 1.0;
        double2 sp = make_double2(0.0, 0.0);
        if (q < nb) {
          const double2 apq = a[p * nb + q];
          const double mag = hypot(apq.x, apq.y);
          if (mag > thr) {
            const double app = a[p * nb + p].x, aqq = a[q * nb + q].x;
            const double tau = (aqq - app) / (2.0 * mag);
            const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
            c = 1.0 / sqrt(1.0 + t * t);
            const double s = t * c;
            sp = make_double2(s * apq.x / mag, s * apq.y / mag);
            act = true;
          }
        }
        rot[2 * lane] = make_double2(c, __longlong_as_double((long long)(p | (q << 8) | ((act ? 1 : 0) << 16))));
        rot[2 * lane + 1] = sp;
      }
      const bool any = __any_sync(0xffffffffu, act);
      __syncwarp();
      if (!any) continue;
      any_sweep = true;
      // A <- A G and V <- V G   (columns p, q of every row)
      for (int it = lane; it < nb * npairs; it += 32) {
        const int k = it % npairs, i = it / npairs;
        const long long code = __double_as_longlong(rot[2 * k].y);
        if (!((code >> 16) & 1)) continue;
        const int p = (int)(code & 255), q = (int)((code >> 8) & 255);
        const double c = rot[2 * k].x;
        const double2 sp = rot[2 * k + 1];
        double2 x = a[i * nb + p], y = a[i * nb + q];
        a[i * nb + p] = csub(cscale(x, c), cmulc(y, sp));
        a[i * nb + q] = cadd(cmul(sp, x), cscale(y, c));
        x = v[i * nb + p];
        y = v[i * nb + q];
        v[i * nb + p] = csub(cscale(x, c), cmulc(y, sp));
        v[i * nb + q] = cadd(cmul(sp, x), cscale(y, c));
      }
      __syncwarp();
      // A <- G^H A   (rows p, q of every column)
      for (int it = lane; it < nb * npairs; it += 32) {
        const int k = it % npairs, j = it / npairs;
        const long long code = __double_as_longlong(rot[2 * k].y);
        if (!((code >> 16) & 1)) continue;
        const int p = (int)(code & 255), q = (int)((code >> 8) & 255);
        const double c = rot[2 * k].x;
        const double2 sp = rot[2 * k + 1];
        const double2 x = a[p * nb + j], y = a[q * nb + j];
        a[p * nb + j] = csub(cscale(x, c), cmul(sp, y));
        a[q * nb + j] = cadd(cmulc(x, sp), cscale(y, c));
      }
      __syncwarp();
      if (lane < npairs) {
        const long long code = __double_as_longlong(rot[2 * lane].y);
        if ((code >> 16) & 1) {
          const int p = (int)(code & 255), q = (int)((code >> 8) & 255);
          a[p * nb + q] = make_double2(0.0, 0.0);
          a[q * nb + p] = make_double2(0.0, 0.0);
          a[p * nb + p].y = 0.0;
          a[q * nb + q].y = 0.0;
        }
      }
      __syncwarp();
    }
    if (!any_sweep) break;
  }
}

// Solves M X = B in place (B <- X) by LU with partial pivoting (|re|+|im| pivots, as LAPACK).
__device__ inline void warp_lu_solve(double2* M, double2* B, int nb, int lane) {
  for (int j = 0; j < nb; ++j) {
    double best = -1.0;
    int bi = j;
    for (int i = j + lane; i < nb; i += 32) {
      const double val = fabs(M[i * nb + j].x) + fabs(M[i * nb + j].y);
      if (val > best) { best = val; bi = i; }
    }
    for (int off = 16; off > 0; off >>= 1) {
      const double ob = __shfl_xor_sync(0xffffffffu, best, off);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
      if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
    }
    if (bi != j) {
      for (int k = lane; k < nb; k += 32) {
        double2 t = M[j * nb + k]; M[j * nb + k] = M[bi * nb + k]; M[bi * nb + k] = t;
        t = B[j * nb + k]; B[j * nb + k] = B[bi * nb + k]; B[bi * nb + k] = t;
      }
    }
    __syncwarp();
    const double2 piv = M[j * nb + j];
    for (int i = j + 1 + lane; i < nb; i += 32) M[i * nb + j] = cdiv(M[i * nb + j], piv);
    __syncwarp();
    const int rows = nb - j - 1;
    for (int it = lane; it < rows * nb; it += 32) {
      const int i = j + 1 + it / nb, k = it % nb;
      const double2 l = M[i * nb + j];
      if (k > j) M[i * nb + k] = csub(M[i * nb + k], cmul(l, M[j * nb + k]));
      B[i * nb + k] = csub(B[i * nb + k], cmul(l, B[j * nb + k]));
    }
    __syncwarp();
  }
  for (int j = nb - 1; j >= 0; --j) {
    for (int k = lane; k < nb; k += 32) {
      double2 s = B[j * nb + k];
      for (int c = j + 1; c < nb; ++c) s = csub(s, cmul(M[j * nb + c], B[c * nb + k]));
      B[j * nb + k] = cdiv(s, M[j * nb + j]);
    }
    __syncwarp();
  }
}

// Re sum_j (V M)_ij conj(V_ij),  M_ab = conj(c_a) F_ab c_b   (solver.py:185-197)
__device__ __forceinline__ double diag_ufu_row(const double2* v, const double2* f, const double2* c, int nb, int i) {
  double acc = 0.0;
  for (int j = 0; j < nb; ++j) {
    double2 aij = make_double2(0.0, 0.0);
    for (int a = 0; a < nb; ++a) aij = cadd(aij, cmul(v[i * nb + a], cmulc(f[a * nb + j], c[a])));
    aij = cmul(aij, c[j]);
    const double2 z = cmulc(aij, v[i * nb + j]);
    acc += z.x;
  }
  return acc;
}

// q <- orthonormal factor of x with a positive real diagonal of R (classical
// Gram-Schmidt, applied twice), i.e. LAPACK's QR with the diag(R) phase fixed.
__device__ inline void warp_qr_cgs2(const double2* x, double2* q, int nb, int lane) {
  for (int j = 0; j < nb; ++j) {
    double2 vi = lane < nb ? x[lane * nb + j] : make_double2(0.0, 0.0);
    for (int pass = 0; pass < 2; ++pass) {
      for (int c = 0; c < j; ++c) {
        double2 z = lane < nb ? cmulc(vi, q[lane * nb + c]) : make_double2(0.0, 0.0);  // conj(q) v
        z.x = warp_sum(z.x);
        z.y = warp_sum(z.y);
        if (lane < nb) vi = csub(vi, cmul(q[lane * nb + c], z));
      }
    }
    double nn = lane < nb ? vi.x * vi.x + vi.y * vi.y : 0.0;
    nn = sqrt(warp_sum(nn));
    if (lane < nb) q[lane * nb + j] = nn > 0.0 ? cscale(vi, 1.0 / nn) : vi;
    __syncwarp();
  }
}

}  // namespace hf
