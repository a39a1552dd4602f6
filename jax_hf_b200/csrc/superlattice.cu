// Streaming superlattice Fock exchange on the extended momentum grid
// (superlattice.py:167-229): for every difference DG = G_a - G_b the density
// blocks rho[(a, alpha), (b, beta)](k) of the pairs with that DG are placed as
// tiles of an (N_ext_x, N_ext_y) grid at the offsets of G_a, convolved with
// the lag Coulomb kernel (Sigma = -IFFT2(FFT2(tile grid) * V_lag_hat)) and the
// same tiles are read back into sigma.  Here the DG channels go through the
// library's exchange build in chunks: a scatter kernel lays up to 32^2 channels
// (n DG values x dim_orb^2 orbital channels, zero padded) out as one
// (N_ext_x, N_ext_y, nbp, nbp) array, one hf_fock_build with a scalar VR
// transforms all of them, and a gather kernel writes the tiles back.
#include "common.cuh"

namespace hf {
int fock_build_internal(void* stream, int dtype, unsigned flags, int nk1, int nk2, int nb, const void* P,
                        const void* h, const void* VR, const void* refP, const void* HH, const void* w2d,
                        int n_contact, const void* contact_g, const void* contact_Oi, const void* contact_Oj,
                        void* Sigma, void* H, void* F, void* workspace, size_t workspace_bytes, const int* active);

struct SlDims {
  int nkx, nky, nG, dorb, Nx, Ny, TX, TY, n_delta;
};

// big[x][y][c], c = (d - d0) dorb^2 + alpha dorb + beta for d < d0 + nd, else 0
__global__ void k_sl_scatter(SlDims s, int d0, int nd, int nbp, const int* __restrict__ tile_owner,
                             const double2* __restrict__ rho, double2* __restrict__ big) {
  const int nc = nbp * nbp, do2 = s.dorb * s.dorb, D = s.nG * s.dorb;
  const long long total = (long long)s.Nx * s.Ny * nc;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total; q += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(q % nc);
    const long long xy = q / nc;
    const int y = (int)(xy % s.Ny), x = (int)(xy / s.Ny);
    double2 v = make_double2(0.0, 0.0);
    const int dl = c / do2;
    if (dl < nd) {
      const int d = d0 + dl, ab = c - dl * do2, al = ab / s.dorb, be = ab - al * s.dorb;
      const int owner = tile_owner[((size_t)d * s.TX + x / s.nkx) * s.TY + y / s.nky];
      if (owner >= 0) {
        const int i = owner / s.nG, j = owner - i * s.nG;
        const int kx = x % s.nkx, ky = y % s.nky;
        v = rho[(((size_t)kx * s.nky + ky) * D + (i * s.dorb + al)) * D + j * s.dorb + be];
      }
    }
    big[q] = v;
  }
}

// sigma[k][(i, alpha)][(j, beta)] = sig_big[G_a offset of i + k][channel of (pair_to_delta(i, j), alpha, beta)]
__global__ void k_sl_gather(SlDims s, int d0, int nd, int nbp, const int* __restrict__ g_off,
                            const int* __restrict__ pair_to_delta, const double2* __restrict__ sig_big,
                            double2* __restrict__ sigma) {
  const int D = s.nG * s.dorb, do2 = s.dorb * s.dorb, nc = nbp * nbp;
  const long long total = (long long)s.nkx * s.nky * D * D;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total; q += (long long)gridDim.x * blockDim.x) {
    const int J = (int)(q % D);
    const long long r = q / D;
    const int I = (int)(r % D);
    const long long kk = r / D;
    const int ky = (int)(kk % s.nky), kx = (int)(kk / s.nky);
    const int i = I / s.dorb, al = I - i * s.dorb, j = J / s.dorb, be = J - j * s.dorb;
    const int d = pair_to_delta[i * s.nG + j];
    if (d < d0 || d >= d0 + nd) continue;
    const int x = s.nkx * g_off[2 * i] + kx, y = s.nky * g_off[2 * i + 1] + ky;
    sigma[q] = sig_big[((size_t)x * s.Ny + y) * nc + (d - d0) * do2 + al * s.dorb + be];
  }
}

static int sl_nbp(int n_delta, int dorb) {
  int nbp = 1;
  while (nbp < 32 && nbp * nbp < n_delta * dorb * dorb) ++nbp;
  return nbp;
}

struct SlLayout {
  size_t big, fws, hb, total;
};

static int sl_layout(const SlDims& s, int nbp, SlLayout& L) {
  size_t fws = 0;
  const int st = hf_fock_workspace_size(HF_C128, HF_FOCK_EXCHANGE | HF_FOCK_VR_SCALAR, s.Nx, s.Ny, nbp, &fws);
  if (st) return st;
  L.big = align_up((size_t)s.Nx * s.Ny * nbp * nbp * sizeof(double2), 256);
  L.fws = align_up(fws, 256);
  L.hb = align_up((size_t)nbp * nbp * sizeof(double2), 256);
  L.total = 3 * L.big + L.fws + L.hb;  // tile grid, Sigma, F, Fock workspace, H
  return HF_OK;
}

static int sl_check(int nkx, int nky, int nG, int dorb, int Nx, int Ny, int n_delta) {
  if (nkx <= 0 || nky <= 0 || nG <= 0 || dorb <= 0 || n_delta <= 0)
    return fail(HF_ERR_INVALID, "superlattice dimensions must be positive");
  if (Nx % nkx || Ny % nky) return fail(HF_ERR_INVALID, "extended grid must be a whole number of k tiles");
  if (Nx > 768 || Ny > 768) return fail(HF_ERR_UNSUPPORTED, "extended grid above 768 points per axis");
  if (dorb * dorb > 1024) return fail(HF_ERR_UNSUPPORTED, "dim_orb above 32");
  return HF_OK;
}

}  // namespace hf

using namespace hf;

extern "C" int hf_sl_fock_workspace_size(int nkx, int nky, int n_G, int dim_orb, int N_ext_x, int N_ext_y,
                                         int n_delta, size_t* bytes) {
  if (!bytes) return fail(HF_ERR_INVALID, "bytes is NULL");
  int st = sl_check(nkx, nky, n_G, dim_orb, N_ext_x, N_ext_y, n_delta);
  if (st) return st;
  SlDims s{nkx, nky, n_G, dim_orb, N_ext_x, N_ext_y, N_ext_x / nkx, N_ext_y / nky, n_delta};
  SlLayout L;
  if ((st = sl_layout(s, sl_nbp(n_delta, dim_orb), L))) return st;
  *bytes = L.total;
  return HF_OK;
}

extern "C" int hf_sl_fock(void* stream, int nkx, int nky, int n_G, int dim_orb, int N_ext_x, int N_ext_y,
                          int n_delta, const int* tile_owner, const int* g_a_off, const int* pair_to_delta,
                          const void* V_lag_fft, const void* rho, void* sigma, void* workspace,
                          size_t workspace_bytes) {
  int st = sl_check(nkx, nky, n_G, dim_orb, N_ext_x, N_ext_y, n_delta);
  if (st) return st;
  if (!tile_owner || !g_a_off || !pair_to_delta || !V_lag_fft || !rho || !sigma)
    return fail(HF_ERR_INVALID, "superlattice arrays must be non-NULL");
  SlDims s{nkx, nky, n_G, dim_orb, N_ext_x, N_ext_y, N_ext_x / nkx, N_ext_y / nky, n_delta};
  const int nbp = sl_nbp(n_delta, dim_orb);
  SlLayout L;
  if ((st = sl_layout(s, nbp, L))) return st;
  if (!workspace || workspace_bytes < L.total)
    return fail(HF_ERR_WORKSPACE, "workspace too small: need " + std::to_string(L.total) + " bytes");
  if (reinterpret_cast<uintptr_t>(workspace) % 256 != 0) return fail(HF_ERR_WORKSPACE, "workspace must be 256-byte aligned");
  char* ws = static_cast<char*>(workspace);
  double2* big = reinterpret_cast<double2*>(ws);
  double2* sbig = reinterpret_cast<double2*>(ws + L.big);
  double2* fbig = reinterpret_cast<double2*>(ws + 2 * L.big);
  void* fws = ws + 3 * L.big;
  void* Hb = ws + 3 * L.big + L.fws;
  cudaStream_t cs = static_cast<cudaStream_t>(stream);
  const int per_chunk = (nbp * nbp) / (dim_orb * dim_orb);
  const long long nbig = (long long)N_ext_x * N_ext_y * nbp * nbp;
  const long long nsig = (long long)nkx * nky * (n_G * dim_orb) * (long long)(n_G * dim_orb);
  auto grid = [](long long n) { long long g = (n + 255) / 256; return (int)(g > 148 * 16 ? 148 * 16 : (g < 1 ? 1 : g)); };
  for (int d0 = 0; d0 < n_delta; d0 += per_chunk) {
    const int nd = (n_delta - d0) < per_chunk ? (n_delta - d0) : per_chunk;
    k_sl_scatter<<<grid(nbig), 256, 0, cs>>>(s, d0, nd, nbp, tile_owner, static_cast<const double2*>(rho), big);
    HF_LAUNCH_CHECK("k_sl_scatter");
    // h = the tile grid itself: F = herm(h + Sigma) is written to fbig and not used
    st = fock_build_internal(stream, HF_C128, HF_FOCK_EXCHANGE | HF_FOCK_VR_SCALAR, N_ext_x, N_ext_y, nbp, big, big,
                             V_lag_fft, nullptr, nullptr, nullptr, 0, nullptr, nullptr, nullptr, sbig, Hb, fbig, fws,
                             L.fws, nullptr);
    if (st) return st;
    k_sl_gather<<<grid(nsig), 256, 0, cs>>>(s, d0, nd, nbp, g_a_off, pair_to_delta, sbig, static_cast<double2*>(sigma));
    HF_LAUNCH_CHECK("k_sl_gather");
  }
  return HF_OK;
}
