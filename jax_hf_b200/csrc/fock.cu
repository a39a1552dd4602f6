// Fock build on B200: exchange convolution by batched 2D FFT + fused epilogue.
//
// Replaces jax_hf.fock.build_fock (fock.py:18-97) with
// utils.selfenergy_fft (utils.py:66-173) inside it:
//   Sigma_ab(k) = -IFFT2( FFT2(P - refP)_ab * VR_ab )(k)   (channels independent)
//   F = herm(h + Sigma + H)
//
// Three passes over a slot-grouped spectrum in the caller's workspace
// (layout [group][k1][k2][slot], complex at the FFT precision):
//   K1 row pass     : load (P - refP) row k1 for one slot group, FFT along k2.
//   K2 column pass  : FFT along k1, multiply by -VR/(nk1 nk2), IFFT along k1.
//   K3 row pass     : IFFT along k2, then the epilogue (contact sigma, Hartree
//                     diagonal, herm with the transposed channel, h-add) writes
//                     Sigma and F once.
// A slot group is a set of band-pair channels closed under transposition
// (2x2 channel tiles paired with their transposes), so the hermitisation of
// F needs no extra pass, and each 2x2 tile keeps 32-byte sectors whole.
#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "common.cuh"
#include "fft_engine.cuh"
#include "fock_params.cuh"

namespace hf {

// ------------------------------------------------------------ planning -----
struct SlotPlan {
  int LS = 0, ngroups = 0;
  bool rows = false;  // rows plan of the fast passes (plan_rows)
  std::vector<int16_t> chan, partner;
};

static FftPlan1D make_fft_plan(int n) {
  FftPlan1D p{};
  p.n = n;
  int m = n, k = 0;
  auto push = [&](int r) { p.radix[k++] = r; m /= r; };
  while (m % 8 == 0 && k < kMaxStages) push(8);
  while (m % 4 == 0 && k < kMaxStages) push(4);
  while (m % 2 == 0 && k < kMaxStages) push(2);
  while (m % 5 == 0 && k < kMaxStages) push(5);
  while (m % 3 == 0 && k < kMaxStages) push(3);
  for (int f = 7; m > 1 && k < kMaxStages; f += 2)
    while (m % f == 0 && k < kMaxStages) push(f);
  p.nstages = k;
  return p;
}

// Units are transpose-closed channel sets built from 2x2 tiles; full mode pairs
// tile (I,J) with (J,I); packing mode keeps the upper triangle only.  With an
// in-block mask (nb x nb, symmetric, 1 = in-block) only in-block channels enter a
// unit, so the exchange passes never transform an off-block channel.
static std::vector<std::vector<int>> make_units(int nb, bool packing, const unsigned char* inb = nullptr);

// A block-diagonal mask (every band's in-block row is its own block: the relation is an
// equivalence, as for block_sizes and disjoint block_indices) gets one unit per block,
// C x C channels (upper triangle with packing), so each k-point's channels of a block
// are read and written as whole rows of the block; blocks of more than 16 channels are
// split into 2x2 tile pairs of their own bands.  Returns false for other masks.
static bool block_units(int nb, bool packing, const unsigned char* inb, std::vector<std::vector<int>>& units) {
  std::vector<unsigned> row(nb, 0u);
  for (int a = 0; a < nb; ++a)
    for (int b = 0; b < nb; ++b)
      if (inb[a * nb + b]) row[a] |= 1u << b;
  for (int a = 0; a < nb; ++a) {
    if (!row[a]) continue;
    if (!((row[a] >> a) & 1u)) return false;
    for (int b = 0; b < nb; ++b)
      if (((row[a] >> b) & 1u) && row[b] != row[a]) return false;
  }
  units.clear();
  unsigned seen = 0u;
  for (int a = 0; a < nb; ++a) {
    if (!row[a] || (seen & row[a])) continue;
    seen |= row[a];
    std::vector<int> cls;
    for (int b = 0; b < nb; ++b)
      if ((row[a] >> b) & 1u) cls.push_back(b);
    const int m = (int)cls.size();
    if (m * m <= 16) {
      std::vector<int> u;
      for (int i = 0; i < m; ++i)
        for (int j = packing ? i : 0; j < m; ++j) u.push_back(cls[i] * nb + cls[j]);
      units.push_back(u);
      continue;
    }
    // the tile units of an m-band problem, mapped onto the block's bands
    for (const auto& t : make_units(m, packing)) {
      std::vector<int> u;
      for (int c : t) u.push_back(cls[c / m] * nb + cls[c % m]);
      units.push_back(u);
    }
  }
  return true;
}

static std::vector<std::vector<int>> make_units(int nb, bool packing, const unsigned char* inb) {
  std::vector<std::vector<int>> units;
  if (inb && block_units(nb, packing, inb, units)) return units;
  const int T = (nb + 1) / 2;
  auto tile = [&](int I, int J, bool upper_only) {
    std::vector<int> v;
    for (int a = 2 * I; a < std::min(2 * I + 2, nb); ++a)
      for (int b = 2 * J; b < std::min(2 * J + 2, nb); ++b)
        if ((!upper_only || a <= b) && (!inb || inb[a * nb + b])) v.push_back(a * nb + b);
    return v;
  };
  for (int I = 0; I < T; ++I)
    for (int J = I; J < T; ++J) {
      std::vector<int> u = tile(I, J, packing);
      if (!packing && J > I) {
        std::vector<int> t = tile(J, I, false);
        u.insert(u.end(), t.begin(), t.end());
      }
      if (!u.empty()) units.push_back(u);
    }
  return units;
}

static bool pack_units(const std::vector<std::vector<int>>& units, int LS,
                       std::vector<std::vector<int>>& groups) {
  groups.clear();
  std::vector<int> order(units.size());
  for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
  std::stable_sort(order.begin(), order.end(),
                   [&](int x, int y) { return units[x].size() > units[y].size(); });
  for (int ui : order) {
    const auto& u = units[ui];
    if ((int)u.size() > LS) return false;
    bool placed = false;
    for (auto& g : groups)
      if ((int)(g.size() + u.size()) <= LS) {
        g.insert(g.end(), u.begin(), u.end());
        placed = true;
        break;
      }
    if (!placed) groups.push_back(u);
  }
  return true;
}

template <typename FT>
static size_t fock_smem_bytes(int n, int LS) {
  return (size_t)(2 * n * LS + n) * sizeof(cpx_t<FT>);
}

static int plan_slots(int nb, bool packing, int nmax, size_t celem, int max_ls, SlotPlan& out,
                      const unsigned char* inb = nullptr) {
  auto units = make_units(nb, packing, inb);
  if (units.empty()) {  // no channel to transform (an in-block mask without in-block channels)
    out.LS = 16;
    out.ngroups = 0;
    out.chan.clear();
    out.partner.clear();
    return HF_OK;
  }
  int maxu = 0, total = 0;
  for (auto& u : units) { maxu = std::max<int>(maxu, (int)u.size()); total += (int)u.size(); }
  const size_t kTwoPerSm = 113 * 1024, kOnePerSm = 227 * 1024;
  int best = -1, best_pad = 1 << 30, best_fit2 = 0;
  std::vector<std::vector<int>> groups, best_groups;
  for (int LS = maxu; LS <= max_ls; ++LS) {
    if (!pack_units(units, LS, groups)) continue;
    size_t smem = (size_t)(2 * nmax * LS + nmax) * celem;
    if (smem > kOnePerSm) continue;
    int pad = (int)groups.size() * LS - total;
    int fit2 = smem <= kTwoPerSm ? 1 : 0;
    bool better = false;
    if (best < 0) better = true;
    else if (fit2 != best_fit2) better = fit2 > best_fit2;
    else if (pad != best_pad) better = pad < best_pad;
    else better = std::abs(LS - 16) < std::abs(best - 16);
    if (better) { best = LS; best_pad = pad; best_fit2 = fit2; best_groups = groups; }
  }
  if (best < 0) return HF_ERR_UNSUPPORTED;
  out.LS = best;
  out.ngroups = (int)best_groups.size();
  out.chan.assign(out.LS * out.ngroups, -1);
  out.partner.assign(out.LS * out.ngroups, -1);
  if (inb)  // ascending channels: each k-point's in-block runs are read and written in order
    for (auto& grp : best_groups) std::sort(grp.begin(), grp.end());
  for (int g = 0; g < out.ngroups; ++g) {
    const auto& grp = best_groups[g];
    for (size_t s = 0; s < grp.size(); ++s) out.chan[g * out.LS + s] = (int16_t)grp[s];
    for (size_t s = 0; s < grp.size(); ++s) {
      int a = grp[s] / nb, b = grp[s] % nb;
      int want = b * nb + a;
      int16_t pidx = (int16_t)s;
      if (!packing)
        for (size_t t = 0; t < grp.size(); ++t)
          if (grp[t] == want) pidx = (int16_t)t;
      out.partner[g * out.LS + s] = pidx;
    }
  }
  if ((int)out.chan.size() > kMaxSlotTable) return HF_ERR_UNSUPPORTED;
  return HF_OK;
}

// ------------------------------------------------------------- kernels -----
template <typename ST, typename FT>
__global__ void __launch_bounds__(kThreads) k_fock_row_fwd(const __grid_constant__ FockParams p) {
  if (p.active && !*p.active) return;
  using SC = cpx_t<ST>;
  using FC = cpx_t<FT>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int N = p.nk2, LS = p.LS;
  FC* tw = reinterpret_cast<FC*>(smem_raw);
  FC* b0 = tw + N;
  FC* b1 = b0 + N * LS;
  const int k1 = blockIdx.x, g = blockIdx.y;
  build_twiddles<FT>(tw, N);
  const SC* P = static_cast<const SC*>(p.P);
  const SC* refP = static_cast<const SC*>(p.refP);
  const bool has_ref = (p.flags & HF_FOCK_HAS_REFP) != 0;
  const size_t row0 = (size_t)k1 * N;
  for (int it = threadIdx.x; it < N * LS; it += blockDim.x) {
    const int i = it / LS, s = it - i * LS;
    const int c = p.chan[g * LS + s];
    FC v = mk<FC>(0.0, 0.0);
    if (c >= 0) {
      const size_t idx = (row0 + i) * p.nb2 + c;
      SC x = P[idx];
      if (has_ref) x = csub(x, refP[idx]);
      v = cvt<FC>(x);
    }
    b0[it] = v;
  }
  __syncthreads();
  FC* res = fft_lines<false>(p.row, b0, b1, tw, LS);
  FC* out = static_cast<FC*>(p.scratch) + (((size_t)g * p.nk1 + k1) * N) * LS;
  for (int it = threadIdx.x; it < N * LS; it += blockDim.x) out[it] = res[it];
}

// Weighted density partial sums for Hartree / contact terms: rho_part[k1][slot]
// = sum_{k2} w(k1,k2) (P - refP)(k1,k2)[chan(slot)], accumulated in float64.
template <typename ST>
__global__ void __launch_bounds__(kThreads) k_fock_rho_part(const __grid_constant__ FockParams p) {
  if (p.active && !*p.active) return;
  using SC = cpx_t<ST>;
  __shared__ double2 red[kThreads];
  const int N = p.nk2, LS = p.LS;
  const int k1 = blockIdx.x, g = blockIdx.y;
  const int parts = kThreads / LS;
  const int s = threadIdx.x % LS, part = threadIdx.x / LS;
  const SC* P = static_cast<const SC*>(p.P);
  const SC* refP = static_cast<const SC*>(p.refP);
  const ST* w = static_cast<const ST*>(p.w2d);
  const bool has_ref = (p.flags & HF_FOCK_HAS_REFP) != 0;
  double2 acc = make_double2(0.0, 0.0);
  const int c = p.chan[g * LS + s];
  if (part < parts && c >= 0) {
    for (int i = part; i < N; i += parts) {
      const size_t kk = (size_t)k1 * N + i;
      SC x = P[kk * p.nb2 + c];
      if (has_ref) x = csub(x, refP[kk * p.nb2 + c]);
      const double wk = (double)w[kk];
      acc.x += wk * (double)x.x;
      acc.y += wk * (double)x.y;
    }
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  if (threadIdx.x < LS) {
    double2 t = make_double2(0.0, 0.0);
    for (int q = 0; q < parts; ++q) t = cadd(t, red[q * LS + threadIdx.x]);
    p.rho_part[(size_t)k1 * (p.ngroups * LS) + g * LS + threadIdx.x] = t;
  }
}

template <typename ST, typename FT>
__global__ void __launch_bounds__(kThreads) k_fock_col(const __grid_constant__ FockParams p) {
  if (p.active && !*p.active) return;
  using SC = cpx_t<ST>;
  using FC = cpx_t<FT>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int N = p.nk1, LS = p.LS;
  FC* tw = reinterpret_cast<FC*>(smem_raw);
  FC* b0 = tw + N;
  FC* b1 = b0 + N * LS;
  const int k2 = blockIdx.x, g = blockIdx.y;
  build_twiddles<FT>(tw, N);
  FC* sc = static_cast<FC*>(p.scratch) + ((size_t)g * p.nk1 * p.nk2 + k2) * LS;
  const size_t rstride = (size_t)p.nk2 * LS;
  for (int it = threadIdx.x; it < N * LS; it += blockDim.x) {
    const int i = it / LS, s = it - i * LS;
    b0[it] = sc[i * rstride + s];
  }
  __syncthreads();
  FC* x = fft_lines<false>(p.col, b0, b1, tw, LS);
  const bool vr_scalar = (p.flags & HF_FOCK_VR_SCALAR) != 0;
  const bool vr_real = (p.flags & HF_FOCK_VR_REAL) != 0;
  for (int it = threadIdx.x; it < N * LS; it += blockDim.x) {
    const int q1 = it / LS, s = it - q1 * LS;
    const int c = p.chan[g * LS + s];
    if (c < 0) { x[it] = mk<FC>(0.0, 0.0); continue; }
    const size_t q = (size_t)q1 * p.nk2 + k2;
    const size_t vi = vr_scalar ? q : q * p.nb2 + c;
    FC v = x[it];
    if (vr_real) {
      const FT r = (FT)((double)static_cast<const ST*>(p.VR)[vi] * p.scale);
      v = cscale(v, r);
    } else {
      SC z = static_cast<const SC*>(p.VR)[vi];
      FC zz = mk<FC>((double)z.x * p.scale, (double)z.y * p.scale);
      v = cmul(v, zz);
    }
    x[it] = v;
  }
  __syncthreads();
  FC* other = (x == b0) ? b1 : b0;
  FC* y = fft_lines<true>(p.col, x, other, tw, LS);
  for (int it = threadIdx.x; it < N * LS; it += blockDim.x) {
    const int i = it / LS, s = it - i * LS;
    sc[i * rstride + s] = y[it];
  }
}

// Reduces rho partials and forms the k-independent terms (fock.py:66-92).
template <typename ST>
__global__ void k_fock_consts(const __grid_constant__ FockParams p) {
  if (p.active && !*p.active) return;
  using SC = cpx_t<ST>;
  __shared__ double2 rho[kMaxNb * kMaxNb];
  const int nb = p.nb, nb2 = p.nb2, LS = p.LS, ns = p.ngroups * LS;
  const bool packing = (p.flags & HF_FOCK_PACKING) != 0;
  for (int c = threadIdx.x; c < nb2; c += blockDim.x) rho[c] = make_double2(0.0, 0.0);
  __syncthreads();
  for (int s = threadIdx.x; s < ns; s += blockDim.x) {
    const int c = p.chan[s];
    if (c < 0) continue;
    double2 t = make_double2(0.0, 0.0);
    for (int k1 = 0; k1 < p.nk1; ++k1) t = cadd(t, p.rho_part[(size_t)k1 * ns + s]);
    rho[c] = t;
    const int a = c / nb, b = c % nb;
    if (packing && a != b) rho[b * nb + a] = conj(t);
  }
  __syncthreads();
  // Hartree diagonal: HH @ n, n_a = Re rho_aa (fock.py:66-74)
  if (p.flags & HF_FOCK_HARTREE) {
    const ST* HH = static_cast<const ST*>(p.HH);
    for (int a = threadIdx.x; a < nb; a += blockDim.x) {
      double acc = 0.0;
      for (int b = 0; b < nb; ++b) acc += (double)HH[a * nb + b] * rho[b * nb + b].x;
      p.hdiag[a] = (double)(ST)acc;
    }
  } else {
    for (int a = threadIdx.x; a < nb; a += blockDim.x) p.hdiag[a] = 0.0;
  }
  // contact: sum_t g_t [Oi_t tr(Oj_t rho) - Oi_t rho Oj_t] (fock.py:77-92)
  const SC* Oi = static_cast<const SC*>(p.cOi);
  const SC* Oj = static_cast<const SC*>(p.cOj);
  const ST* gg = static_cast<const ST*>(p.cg);
  for (int c = threadIdx.x; c < nb2; c += blockDim.x) {
    const int i = c / nb, l = c % nb;
    double2 acc = make_double2(0.0, 0.0);
    for (int t = 0; t < p.n_contact; ++t) {
      const SC* oi = Oi + (size_t)t * nb2;
      const SC* oj = Oj + (size_t)t * nb2;
      double2 tr = make_double2(0.0, 0.0);
      for (int a = 0; a < nb; ++a)
        for (int b = 0; b < nb; ++b) tr = cadd(tr, cmul(cvt<double2>(oj[a * nb + b]), rho[b * nb + a]));
      const double gt = (double)gg[t];
      double2 hterm = cscale(cmul(cvt<double2>(oi[i * nb + l]), tr), gt);
      double2 fterm = make_double2(0.0, 0.0);
      for (int j = 0; j < nb; ++j) {
        double2 oir = make_double2(0.0, 0.0);
        for (int k = 0; k < nb; ++k) oir = cadd(oir, cmul(cvt<double2>(oi[i * nb + k]), rho[k * nb + j]));
        fterm = cadd(fterm, cmul(oir, cvt<double2>(oj[j * nb + l])));
      }
      acc = cadd(acc, csub(hterm, cscale(fterm, gt)));
    }
    p.sigc[c] = acc;
  }
  __syncthreads();
  if (p.Hout) {
    SC* Ho = static_cast<SC*>(p.Hout);
    for (int c = threadIdx.x; c < nb2; c += blockDim.x) {
      const int a = c / nb, b = c % nb;
      Ho[c] = mk<SC>(a == b ? p.hdiag[a] : 0.0, 0.0);
    }
  }
}

template <typename ST, typename FT>
__global__ void __launch_bounds__(kThreads) k_fock_row_inv(const __grid_constant__ FockParams p) {
  if (p.active && !*p.active) return;
  using SC = cpx_t<ST>;
  using FC = cpx_t<FT>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int N = p.nk2, LS = p.LS, nb = p.nb;
  FC* tw = reinterpret_cast<FC*>(smem_raw);
  FC* b0 = tw + N;
  FC* b1 = b0 + N * LS;
  const int k1 = blockIdx.x, g = blockIdx.y;
  const bool exch = (p.flags & HF_FOCK_EXCHANGE) != 0;
  const bool packing = (p.flags & HF_FOCK_PACKING) != 0;
  FC* res = b0;
  if (exch) {
    build_twiddles<FT>(tw, N);
    const FC* sc = static_cast<const FC*>(p.scratch) + (((size_t)g * p.nk1 + k1) * N) * LS;
    for (int it = threadIdx.x; it < N * LS; it += blockDim.x) b0[it] = sc[it];
    __syncthreads();
    res = fft_lines<true>(p.row, b0, b1, tw, LS);
  } else {
    for (int it = threadIdx.x; it < N * LS; it += blockDim.x) b0[it] = mk<FC>(0.0, 0.0);
    __syncthreads();
  }
  const SC* h = static_cast<const SC*>(p.h);
  SC* Sg = static_cast<SC*>(p.Sigma);
  SC* F = static_cast<SC*>(p.F);
  const bool consts = p.sigc != nullptr;
  for (int it = threadIdx.x; it < N * LS; it += blockDim.x) {
    const int i = it / LS, s = it - i * LS;
    const int c = p.chan[g * LS + s];
    if (c < 0) continue;
    const int a = c / nb, b = c - (c / nb) * nb;
    const size_t base = ((size_t)k1 * N + i) * p.nb2;
    SC sab = cvt<SC>(res[it]);
    SC sba;
    if (packing) sba = (a == b) ? sab : conj(sab);
    else sba = cvt<SC>(res[i * LS + p.partner[g * LS + s]]);
    if (consts) {
      sab = cadd(sab, cvt<SC>(p.sigc[a * nb + b]));
      sba = cadd(sba, cvt<SC>(p.sigc[b * nb + a]));
    }
    const SC hab = h[base + a * nb + b];
    const SC hba = h[base + b * nb + a];
    SC f = mk<SC>(0.5 * ((double)hab.x + (double)hba.x) + 0.5 * ((double)sab.x + (double)sba.x),
                  0.5 * ((double)hab.y - (double)hba.y) + 0.5 * ((double)sab.y - (double)sba.y));
    if (consts && a == b) f.x += (ST)p.hdiag[a];
    Sg[base + a * nb + b] = sab;
    F[base + a * nb + b] = f;
    if (packing && a != b) {
      Sg[base + b * nb + a] = sba;
      F[base + b * nb + a] = conj(f);
    }
  }
}

// ---------------------------------------------------------- host driver ----
struct WsLayout {
  size_t scratch = 0, rho = 0, sigc = 0, hdiag = 0, total = 0;
};

// rho_slots: slots of the plan that forms the constant terms (-1: the exchange plan's)
static WsLayout ws_layout(const SlotPlan& sp, int nk1, int nk2, int nb, size_t felem, bool exch,
                          int rho_slots = -1) {
  WsLayout w;
  size_t off = 0;
  w.scratch = off;
  if (exch) off += align_up((size_t)sp.ngroups * sp.LS * nk1 * nk2 * felem, 256);
  w.rho = off;
  off += align_up((size_t)nk1 * (rho_slots >= 0 ? rho_slots : sp.ngroups * sp.LS) * sizeof(double2), 256);
  w.sigc = off;
  off += align_up((size_t)nb * nb * sizeof(double2), 256);
  w.hdiag = off;
  off += align_up((size_t)nb * sizeof(double), 256);
  w.total = off;
  return w;
}

static int validate(int dtype, unsigned flags, int nk1, int nk2, int nb) {
  if (dtype != HF_C128 && dtype != HF_C64) return fail(HF_ERR_INVALID, "dtype must be HF_C128 or HF_C64");
  if (nk1 < 1 || nk2 < 1 || nb < 1) return fail(HF_ERR_INVALID, "nk1, nk2, nb must be positive");
  if (nb > kMaxNb) return fail(HF_ERR_UNSUPPORTED, "nb > 32 is not supported by this build");
  if (!(flags & (HF_FOCK_EXCHANGE | HF_FOCK_HARTREE)))
    return fail(HF_ERR_INVALID, "HartreeFockKernel must include at least one of Hartree or exchange.");
  if ((flags & HF_FOCK_PACKING) && !(flags & (HF_FOCK_VR_SCALAR | HF_FOCK_SYM_V)))
    return fail(HF_ERR_INVALID,
                "hermitian_channel_packing requires a scalar interaction kernel with shape (..., 1, 1).");
  if ((flags & HF_FOCK_FFT_FP32) && dtype != HF_C128)
    return fail(HF_ERR_INVALID, "HF_FOCK_FFT_FP32 applies to complex128 storage only");
  return HF_OK;
}

static size_t fft_elem(int dtype, unsigned flags) {
  return (dtype == HF_C64 || (flags & HF_FOCK_FFT_FP32)) ? sizeof(float2) : sizeof(double2);
}

// Rows plan for the fast passes (nb <= 8, no packing): group g holds the whole
// matrix rows [g R, g R + R), R = min(nb, 16 / nb), LS = R nb slots, so every
// k-point's channels of a group are contiguous in memory; the herm partner
// (b, a) of slot (a, b) is in group b / R: partner = (group << 8) | slot.
static void plan_rows(int nb, SlotPlan& out) {
  const int R = std::min(nb, 16 / nb);
  out.rows = true;
  out.LS = R * nb;
  out.ngroups = (nb + R - 1) / R;
  out.chan.assign(out.LS * out.ngroups, -1);
  out.partner.assign(out.LS * out.ngroups, -1);
  for (int c = 0; c < nb * nb; ++c) {
    const int a = c / nb, b = c % nb, cp = b * nb + a, gp = b / R;
    out.chan[c] = (int16_t)c;
    out.partner[c] = (int16_t)((gp << 8) | (cp - gp * out.LS));
  }
}

static int get_plan(int dtype, unsigned flags, int nk1, int nk2, int nb, SlotPlan& sp,
                    const unsigned char* inb = nullptr) {
  const bool packing = (flags & HF_FOCK_PACKING) != 0;
  if (!inb && !packing && nb <= 8 && !(flags & (HF_FOCK_GENERIC_FFT | HF_FOCK_TILE_PLAN)) && fast_length(nk1) &&
      fast_length(nk2)) {
    plan_rows(nb, sp);
    return HF_OK;
  }
  const int max_ls = (fast_length(nk1) && fast_length(nk2)) ? 16 : 32;
  int st = plan_slots(nb, packing, std::max(nk1, nk2), fft_elem(dtype, flags), max_ls, sp, inb);
  if (st != HF_OK) return fail(st, "mesh too large for the shared-memory FFT (nk1, nk2 <= 768 in complex128)");
  return HF_OK;
}

// Sigma and F on the off-block channels of an in-block mask (listed in `off`): no
// exchange there, so Sigma = the contact constant and F = herm(h + Sigma) + the
// Hartree diagonal, the epilogue's formula with a zero exchange term.  One thread per
// (k, off-block channel), channels ascending within a k-point.
struct OffBlockList {
  int16_t ch[kMaxNb * kMaxNb];
  int n;
};

template <typename ST>
__global__ void k_fock_offblock(unsigned nk, int nb, const __grid_constant__ OffBlockList m, const void* hv,
                                const double2* __restrict__ sigc, const double* __restrict__ hdiag, void* Sgv,
                                void* Fv, const int* active) {
  if (active && !*active) return;
  using SC = cpx_t<ST>;
  const SC* h = static_cast<const SC*>(hv);
  SC* Sg = static_cast<SC*>(Sgv);
  SC* F = static_cast<SC*>(Fv);
  constexpr int U = 4;  // elements per thread and step, loads issued first
  const unsigned nb2 = (unsigned)(nb * nb), n = nk * (unsigned)m.n, stride = gridDim.x * blockDim.x;
  for (unsigned j0 = blockIdx.x * blockDim.x + threadIdx.x; j0 < n; j0 += U * stride) {
    SC hab[U], hba[U];
    size_t at[U];
    int cs[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const unsigned j = j0 + u * stride;
      const unsigned k = j < n ? j / (unsigned)m.n : 0u;
      const int c = j < n ? m.ch[j - k * (unsigned)m.n] : 0;
      const int a = c / nb, b = c - a * nb;
      cs[u] = c;
      at[u] = (size_t)k * nb2;
      hab[u] = j < n ? h[at[u] + c] : mk<SC>(0.0, 0.0);
      hba[u] = j < n ? h[at[u] + b * nb + a] : mk<SC>(0.0, 0.0);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (j0 + u * stride >= n) break;
      const int c = cs[u], a = c / nb, b = c - a * nb;
      SC sab = mk<SC>(0.0, 0.0), sba = mk<SC>(0.0, 0.0);
      if (sigc) {
        sab = cvt<SC>(sigc[c]);
        sba = cvt<SC>(sigc[b * nb + a]);
      }
      SC f = mk<SC>(0.5 * ((double)hab[u].x + (double)hba[u].x) + 0.5 * ((double)sab.x + (double)sba.x),
                    0.5 * ((double)hab[u].y - (double)hba[u].y) + 0.5 * ((double)sab.y - (double)sba.y));
      if (hdiag && a == b) f.x += (ST)hdiag[a];
      Sg[at[u] + c] = sab;
      F[at[u] + c] = f;
    }
  }
}

template <typename ST>
static int launch_consts(const FockParams& q, cudaStream_t stream) {
  k_fock_rho_part<ST><<<dim3(q.nk1, q.ngroups), kThreads, 0, stream>>>(q);
  HF_LAUNCH_CHECK("k_fock_rho_part");
  k_fock_consts<ST><<<1, 256, 0, stream>>>(q);
  HF_LAUNCH_CHECK("k_fock_consts");
  return HF_OK;
}

// A side stream and two events per host thread and CUDA context, for forking work off the
// caller's stream and joining it back (also inside stream capture, where the fork and
// join become graph edges).  Per thread, so concurrent callers never share an event.
struct ForkJoin {
  unsigned long long ctx = 0;
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
};

static int fork_join(ForkJoin** out) {
  thread_local ForkJoin fj;
  unsigned long long ctx = 0;
  int st = context_id(&ctx);
  if (st) return st;
  if (!fj.side || fj.ctx != ctx) {  // first use in this context (a reset context's handles are gone)
    HF_CUDA(cudaStreamCreateWithFlags(&fj.side, cudaStreamNonBlocking));
    HF_CUDA(cudaEventCreateWithFlags(&fj.fork, cudaEventDisableTiming));
    HF_CUDA(cudaEventCreateWithFlags(&fj.join, cudaEventDisableTiming));
    fj.ctx = ctx;
  }
  *out = &fj;
  return HF_OK;
}

// pc: the plan for the constant terms when it differs from the exchange plan (an
// in-block mask: the Hartree and contact terms read every channel of the density).
template <typename ST, typename FT>
static int launch_fock(FockParams& p, cudaStream_t stream, bool need_consts, const FockParams* pc = nullptr) {
  const bool exch = (p.flags & HF_FOCK_EXCHANGE) != 0;
  const size_t sm_row = fock_smem_bytes<FT>(p.nk2, p.LS);
  const size_t sm_col = fock_smem_bytes<FT>(p.nk1, p.LS);
  HF_SMEM_CAP(k_fock_row_fwd<ST, FT>);
  HF_SMEM_CAP(k_fock_col<ST, FT>);
  HF_SMEM_CAP(k_fock_row_inv<ST, FT>);
  dim3 grow(p.nk1, p.ngroups), gcol(p.nk2, p.ngroups);
  if (need_consts) {
    const FockParams& q = pc ? *pc : p;
    k_fock_rho_part<ST><<<dim3(q.nk1, q.ngroups), kThreads, 0, stream>>>(q);
    HF_LAUNCH_CHECK("k_fock_rho_part");
    k_fock_consts<ST><<<1, 256, 0, stream>>>(q);
    HF_LAUNCH_CHECK("k_fock_consts");
  }
  if (p.ngroups == 0) return HF_OK;  // an in-block mask without in-block channels
  if (!(p.flags & HF_FOCK_GENERIC_FFT)) {
    bool handled = false;
    int st = pipe_fock<ST, FT>(p, stream, &handled);
    if (st != HF_OK || handled) return st;
    st = fast_fock<ST, FT>(p, stream, &handled);
    if (st != HF_OK || handled) return st;
  }
  if (exch) {
    k_fock_row_fwd<ST, FT><<<grow, kThreads, sm_row, stream>>>(p);
    HF_LAUNCH_CHECK("k_fock_row_fwd");
    k_fock_col<ST, FT><<<gcol, kThreads, sm_col, stream>>>(p);
    HF_LAUNCH_CHECK("k_fock_col");
  }
  k_fock_row_inv<ST, FT><<<grow, kThreads, sm_row, stream>>>(p);
  HF_LAUNCH_CHECK("k_fock_row_inv");
  return HF_OK;
}

// ------------------------------------------------------------ fault word -----
// Written by the bounded waits of the pipelined passes (fock_pipe.cuh).  Its address
// is cached per context (hf::symbol_address), so a device reset gets a fresh lookup.
__device__ int g_fock_fault;

static int fault_word(int** out) {
  void* p = nullptr;
  int st = hf::symbol_address(reinterpret_cast<const void*>(&g_fock_fault), &p);
  *out = static_cast<int*>(p);
  return st;
}

// ------------------------------------------------------------ autotuner -----
// Engine flags chosen by hf_fock_autotune per (device, dtype, flags, nk1, nk2, nb).
constexpr unsigned kEngineFlags = HF_FOCK_TILE_PLAN | HF_FOCK_GENERIC_FFT | HF_FOCK_PIPE;
constexpr int kTuneCands = 4;
// default schedule, 2x2-tile slot plan, generic engine, bulk-copy pipeline
constexpr unsigned kTuneCand[kTuneCands] = {0u, HF_FOCK_TILE_PLAN, HF_FOCK_GENERIC_FFT, HF_FOCK_PIPE};
using TuneKey = std::tuple<int, int, unsigned, int, int, int>;
static std::mutex g_tune_mu;
static std::map<TuneKey, unsigned> g_tune;

static TuneKey tune_key(int dtype, unsigned flags, int nk1, int nk2, int nb) {
  int dev = 0;
  cudaGetDevice(&dev);
  return TuneKey(dev, dtype, flags & ~kEngineFlags, nk1, nk2, nb);
}

// flags with the stored engine choice applied (unless the caller set an engine flag)
static unsigned tuned_flags(int dtype, unsigned flags, int nk1, int nk2, int nb) {
  if (flags & kEngineFlags) return flags;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  if (g_tune.empty()) return flags;
  auto it = g_tune.find(tune_key(dtype, flags, nk1, nk2, nb));
  return it == g_tune.end() ? flags : (flags | it->second);
}

}  // namespace hf

using namespace hf;

extern "C" int hf_fock_workspace_size(int dtype, unsigned flags, int nk1, int nk2, int nb, size_t* bytes) {
  if (!bytes) return fail(HF_ERR_INVALID, "bytes is NULL");
  int st = validate(dtype, flags, nk1, nk2, nb);
  if (st) return st;
  // every schedule the autotuner may pick (they differ only in the slot plan)
  size_t most = 0;
  for (unsigned e : kTuneCand) {
    if ((flags & kEngineFlags) && e != 0) continue;
    SlotPlan sp;
    if ((st = get_plan(dtype, flags | e, nk1, nk2, nb, sp))) return st;
    most = std::max(most, ws_layout(sp, nk1, nk2, nb, fft_elem(dtype, flags), (flags & HF_FOCK_EXCHANGE) != 0).total);
  }
  *bytes = most;
  return HF_OK;
}

namespace hf {
int fock_build_internal(void* stream, int dtype, unsigned flags, int nk1, int nk2, int nb, const void* P,
                        const void* h, const void* VR, const void* refP, const void* HH, const void* w2d,
                        int n_contact, const void* contact_g, const void* contact_Oi, const void* contact_Oj,
                        void* Sigma, void* H, void* F, void* workspace, size_t workspace_bytes,
                        const int* active);
}

extern "C" int hf_fock_build(void* stream, int dtype, unsigned flags, int nk1, int nk2, int nb,
                             const void* P, const void* h, const void* VR, const void* refP,
                             const void* HH, const void* w2d, int n_contact, const void* contact_g,
                             const void* contact_Oi, const void* contact_Oj, void* Sigma, void* H,
                             void* F, void* workspace, size_t workspace_bytes) {
  return hf::fock_build_internal(stream, dtype, flags, nk1, nk2, nb, P, h, VR, refP, HH, w2d, n_contact,
                                 contact_g, contact_Oi, contact_Oj, Sigma, H, F, workspace, workspace_bytes,
                                 nullptr);
}

// Workspace of a build whose exchange covers only the in-block channels of `inb`.
static int masked_ws(int dtype, unsigned flags, int nk1, int nk2, int nb, const unsigned char* inb, SlotPlan& sp,
                     SlotPlan& spc, WsLayout& wl) {
  int st;
  if ((st = get_plan(dtype, flags, nk1, nk2, nb, sp, inb))) return st;
  if ((st = get_plan(dtype, flags & ~kEngineFlags, nk1, nk2, nb, spc))) return st;
  wl = ws_layout(sp, nk1, nk2, nb, fft_elem(dtype, flags), true, spc.ngroups * spc.LS);
  return HF_OK;
}

// The build with exactly these flags (no stored autotuner choice applied).  inb: an
// in-block channel mask (nb x nb, symmetric; NULL = every channel) for the exchange.
static int fock_build_exact(void* stream, int dtype, unsigned flags, int nk1, int nk2, int nb, const void* P,
                            const void* h, const void* VR, const void* refP, const void* HH, const void* w2d,
                            int n_contact, const void* contact_g, const void* contact_Oi,
                            const void* contact_Oj, void* Sigma, void* H, void* F, void* workspace,
                            size_t workspace_bytes, const int* active, const unsigned char* inb = nullptr) {
  int st = validate(dtype, flags, nk1, nk2, nb);
  if (st) return st;
  const bool exch = (flags & HF_FOCK_EXCHANGE) != 0;
  if (!P || !h || !Sigma || !F) return fail(HF_ERR_INVALID, "P, h, Sigma and F must be non-NULL");
  if (exch && !VR) return fail(HF_ERR_INVALID, "VR must be non-NULL when exchange is included");
  if ((flags & HF_FOCK_HAS_REFP) && !refP) return fail(HF_ERR_INVALID, "refP flagged but NULL");
  if ((flags & HF_FOCK_HARTREE) && (!HH || !w2d)) return fail(HF_ERR_INVALID, "Hartree needs HH and w2d");
  if (n_contact < 0) return fail(HF_ERR_INVALID, "n_contact must be >= 0");
  if (n_contact > 0 && (!contact_g || !contact_Oi || !contact_Oj || !w2d))
    return fail(HF_ERR_INVALID, "contact terms need g, O_i, O_j and w2d");
  SlotPlan sp, spc;
  WsLayout wl;
  if (inb) {
    if ((st = masked_ws(dtype, flags, nk1, nk2, nb, inb, sp, spc, wl))) return st;
  } else {
    if ((st = get_plan(dtype, flags, nk1, nk2, nb, sp))) return st;
    wl = ws_layout(sp, nk1, nk2, nb, fft_elem(dtype, flags), exch);
  }
  if (!workspace || workspace_bytes < wl.total)
    return fail(HF_ERR_WORKSPACE, "workspace too small: need " + std::to_string(wl.total) + " bytes");
  if (reinterpret_cast<uintptr_t>(workspace) % 256 != 0)
    return fail(HF_ERR_WORKSPACE, "workspace must be 256-byte aligned");

  FockParams p;
  memset(&p, 0, sizeof(p));
  p.nk1 = nk1; p.nk2 = nk2; p.nb = nb; p.nb2 = nb * nb;
  p.LS = sp.LS; p.ngroups = sp.ngroups; p.rows_plan = sp.rows ? 1 : 0;
  p.flags = flags; p.n_contact = n_contact;
  p.scale = -1.0 / ((double)nk1 * (double)nk2);
  p.row = make_fft_plan(nk2);
  p.col = make_fft_plan(nk1);
  p.P = P; p.h = h; p.VR = VR; p.refP = refP; p.w2d = w2d; p.HH = HH;
  p.cg = contact_g; p.cOi = contact_Oi; p.cOj = contact_Oj;
  p.Sigma = Sigma; p.F = F; p.Hout = H;
  p.active = active;
  if ((st = fault_word(&p.fault))) return st;
  char* ws = static_cast<char*>(workspace);
  p.scratch = ws + wl.scratch;
  const bool need_consts = (flags & HF_FOCK_HARTREE) || n_contact > 0;
  if (need_consts) {
    p.rho_part = reinterpret_cast<double2*>(ws + wl.rho);
    p.sigc = reinterpret_cast<double2*>(ws + wl.sigc);
    p.hdiag = reinterpret_cast<double*>(ws + wl.hdiag);
  }
  std::copy(sp.chan.begin(), sp.chan.end(), p.chan);
  std::copy(sp.partner.begin(), sp.partner.end(), p.partner);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (H && !need_consts && !active) {
    const size_t hb = (size_t)nb * nb * (dtype == HF_C128 ? sizeof(double2) : sizeof(float2));
    HF_CUDA(cudaMemsetAsync(H, 0, hb, s));
  }
  if (!inb) {
    if (dtype == HF_C64) return launch_fock<float, float>(p, s, need_consts);
    if (flags & HF_FOCK_FFT_FP32) return launch_fock<double, float>(p, s, need_consts);
    return launch_fock<double, double>(p, s, need_consts);
  }
  // masked exchange: constant terms from the full plan, then the exchange passes over the
  // in-block plan and, on a forked stream, the off-block channels (independent of the
  // passes: both read only P's constants and h), so the off-block pass fills the SMs the
  // passes leave idle in their last rounds
  FockParams pc = p;
  pc.LS = spc.LS;
  pc.ngroups = spc.ngroups;
  pc.rows_plan = spc.rows ? 1 : 0;
  std::fill(pc.chan, pc.chan + kMaxSlotTable, (int16_t)-1);
  std::copy(spc.chan.begin(), spc.chan.end(), pc.chan);
  std::copy(spc.partner.begin(), spc.partner.end(), pc.partner);
  if (need_consts) {
    if (dtype == HF_C64) st = launch_consts<float>(pc, s);
    else st = launch_consts<double>(pc, s);
    if (st) return st;
  }
  ForkJoin* fj = nullptr;
  if ((st = fork_join(&fj))) return st;
  HF_CUDA(cudaEventRecord(fj->fork, s));
  if (dtype == HF_C64) st = launch_fock<float, float>(p, s, false);
  else if (flags & HF_FOCK_FFT_FP32) st = launch_fock<double, float>(p, s, false);
  else st = launch_fock<double, double>(p, s, false);
  if (st) return st;
  OffBlockList m;
  memset(&m, 0, sizeof(m));
  for (int c = 0; c < nb * nb; ++c)
    if (!inb[c]) m.ch[m.n++] = (int16_t)c;
  if (m.n == 0) return HF_OK;
  const unsigned nk = (unsigned)nk1 * (unsigned)nk2;
  const size_t n = (size_t)nk * m.n;
  if (n >= (1ull << 31)) return fail(HF_ERR_UNSUPPORTED, "mesh too large for the off-block pass");
  const int blocks = (int)std::min<size_t>((n + 1023) / 1024, (size_t)148 * 8);
  const double2* sigc = need_consts ? p.sigc : nullptr;
  const double* hdiag = need_consts ? p.hdiag : nullptr;
  HF_CUDA(cudaStreamWaitEvent(fj->side, fj->fork, 0));
  if (dtype == HF_C64)
    k_fock_offblock<float><<<blocks, 256, 0, fj->side>>>(nk, nb, m, h, sigc, hdiag, Sigma, F, active);
  else
    k_fock_offblock<double><<<blocks, 256, 0, fj->side>>>(nk, nb, m, h, sigc, hdiag, Sigma, F, active);
  HF_LAUNCH_CHECK("k_fock_offblock");
  HF_CUDA(cudaEventRecord(fj->join, fj->side));
  HF_CUDA(cudaStreamWaitEvent(s, fj->join, 0));
  return HF_OK;
}

int hf::fock_build_internal(void* stream, int dtype, unsigned flags, int nk1, int nk2, int nb, const void* P,
                            const void* h, const void* VR, const void* refP, const void* HH, const void* w2d,
                            int n_contact, const void* contact_g, const void* contact_Oi,
                            const void* contact_Oj, void* Sigma, void* H, void* F, void* workspace,
                            size_t workspace_bytes, const int* active) {
  const int st = validate(dtype, flags, nk1, nk2, nb);
  if (st) return st;
  return fock_build_exact(stream, dtype, tuned_flags(dtype, flags, nk1, nk2, nb), nk1, nk2, nb, P, h, VR, refP, HH,
                          w2d, n_contact, contact_g, contact_Oi, contact_Oj, Sigma, H, F, workspace, workspace_bytes,
                          active);
}

static int check_inblock(int nb, const unsigned char* inb) {
  if (!inb) return fail(HF_ERR_INVALID, "inblock mask is NULL");
  for (int a = 0; a < nb; ++a)
    for (int b = 0; b < nb; ++b)
      if ((inb[a * nb + b] != 0) != (inb[b * nb + a] != 0))
        return fail(HF_ERR_INVALID, "inblock mask must be symmetric (blocks are sets of bands)");
  return HF_OK;
}

extern "C" int hf_fock_blocks_workspace_size(int dtype, unsigned flags, int nk1, int nk2, int nb,
                                             const unsigned char* inblock, size_t* bytes) {
  if (!bytes) return fail(HF_ERR_INVALID, "bytes is NULL");
  int st = validate(dtype, flags, nk1, nk2, nb);
  if (st || (st = check_inblock(nb, inblock))) return st;
  if (!(flags & HF_FOCK_EXCHANGE)) return hf_fock_workspace_size(dtype, flags, nk1, nk2, nb, bytes);
  SlotPlan sp, spc;
  WsLayout wl;
  if ((st = masked_ws(dtype, flags & ~(unsigned)HF_FOCK_PIPE, nk1, nk2, nb, inblock, sp, spc, wl))) return st;
  *bytes = wl.total;
  return HF_OK;
}

extern "C" int hf_fock_build_blocks(void* stream, int dtype, unsigned flags, int nk1, int nk2, int nb,
                                    const unsigned char* inblock, const void* P, const void* h, const void* VR,
                                    const void* refP, const void* HH, const void* w2d, int n_contact,
                                    const void* contact_g, const void* contact_Oi, const void* contact_Oj,
                                    void* Sigma, void* H, void* F, void* workspace, size_t workspace_bytes) {
  int st = validate(dtype, flags, nk1, nk2, nb);
  if (st || (st = check_inblock(nb, inblock))) return st;
  const bool all_in = std::all_of(inblock, inblock + nb * nb, [](unsigned char v) { return v != 0; });
  if (!(flags & HF_FOCK_EXCHANGE) || all_in)  // nothing to leave out: the plain build
    return hf::fock_build_internal(stream, dtype, flags, nk1, nk2, nb, P, h, VR, refP, HH, w2d, n_contact,
                                   contact_g, contact_Oi, contact_Oj, Sigma, H, F, workspace, workspace_bytes,
                                   nullptr);
  return fock_build_exact(stream, dtype, flags & ~(unsigned)HF_FOCK_PIPE, nk1, nk2, nb, P, h, VR, refP, HH, w2d,
                          n_contact, contact_g, contact_Oi, contact_Oj, Sigma, H, F, workspace, workspace_bytes,
                          nullptr, inblock);
}

// ------------------------------------------------ block specs on the device -----
// The first spec whose off-block maximum is within atol + rtol * max runs; flag[i] = 1
// for it (flag[n_specs] for the full build when none is compatible, or a NaN maximum).
__global__ void k_block_choose(int n_specs, double atol, double rtol, const double* __restrict__ maxima,
                               int* __restrict__ flag, int* __restrict__ chosen) {
  if (threadIdx.x != 0) return;
  const double tol = atol + rtol * maxima[0];
  int pick = n_specs;
  for (int i = 0; i < n_specs; ++i)
    if (maxima[i + 1] <= tol) {
      pick = i;
      break;
    }
  for (int i = 0; i <= n_specs; ++i) flag[i] = i == pick ? 1 : 0;
  if (chosen) *chosen = pick < n_specs ? pick : -1;
}

constexpr size_t kSpecHead = 256;  // maxima (n_specs + 1 doubles) and flags (n_specs + 1 ints)

static int block_specs_ws(int dtype, unsigned flags, int nk1, int nk2, int nb, int n_specs,
                          const unsigned char* inblock, size_t* bytes) {
  int st;
  size_t most = 0;
  if ((st = hf_fock_workspace_size(dtype, flags, nk1, nk2, nb, &most))) return st;
  for (int i = 0; i < n_specs; ++i) {
    size_t b = 0;
    if ((st = hf_fock_blocks_workspace_size(dtype, flags, nk1, nk2, nb, inblock + (size_t)i * nb * nb, &b)))
      return st;
    most = std::max(most, b);
  }
  *bytes = kSpecHead + most;
  return HF_OK;
}

extern "C" int hf_fock_block_specs_workspace_size(int dtype, unsigned flags, int nk1, int nk2, int nb, int n_specs,
                                                  const unsigned char* inblock, size_t* bytes) {
  if (!bytes) return fail(HF_ERR_INVALID, "bytes is NULL");
  if (n_specs < 1 || n_specs > 8) return fail(HF_ERR_INVALID, "n_specs must be 1..8");
  return block_specs_ws(dtype, flags & ~(unsigned)HF_FOCK_PIPE, nk1, nk2, nb, n_specs, inblock, bytes);
}

extern "C" int hf_fock_build_block_specs(void* stream, int dtype, unsigned flags, int nk1, int nk2, int nb,
                                         int n_specs, const unsigned char* inblock, double atol, double rtol,
                                         const void* P, const void* h, const void* VR, const void* refP,
                                         const void* HH, const void* w2d, int n_contact, const void* contact_g,
                                         const void* contact_Oi, const void* contact_Oj, void* Sigma, void* H,
                                         void* F, void* workspace, size_t workspace_bytes, int* chosen) {
  int st = validate(dtype, flags, nk1, nk2, nb);
  if (st) return st;
  if (n_specs < 1 || n_specs > 8) return fail(HF_ERR_INVALID, "n_specs must be 1..8");
  if (!(flags & HF_FOCK_EXCHANGE)) return fail(HF_ERR_INVALID, "block specs need the exchange term");
  flags &= ~(unsigned)HF_FOCK_PIPE;
  for (int i = 0; i < n_specs; ++i)
    if ((st = check_inblock(nb, inblock + (size_t)i * nb * nb))) return st;
  size_t need = 0;
  if ((st = block_specs_ws(dtype, flags, nk1, nk2, nb, n_specs, inblock, &need))) return st;
  if (!workspace || workspace_bytes < need)
    return fail(HF_ERR_WORKSPACE, "workspace too small: need " + std::to_string(need) + " bytes");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  unsigned char* ws = static_cast<unsigned char*>(workspace);
  double* maxima = reinterpret_cast<double*>(ws);
  int* flag = reinterpret_cast<int*>(ws + 128);
  void* cand_ws = ws + kSpecHead;
  const size_t cand_bytes = workspace_bytes - kSpecHead;
  const bool has_ref = (flags & HF_FOCK_HAS_REFP) != 0;
  if ((st = hf_block_offdiag_max(stream, dtype, (size_t)nk1 * nk2, nb, P, has_ref ? refP : nullptr, n_specs,
                                 inblock, maxima)))
    return st;
  k_block_choose<<<1, 32, 0, s>>>(n_specs, atol, rtol, maxima, flag, chosen);
  HF_LAUNCH_CHECK("k_block_choose");
  if (H) {  // a candidate without constant terms leaves H to this
    const size_t hb = (size_t)nb * nb * (dtype == HF_C128 ? sizeof(double2) : sizeof(float2));
    HF_CUDA(cudaMemsetAsync(H, 0, hb, s));
  }
  // every candidate is queued; its kernels return at once unless its flag is set
  for (int i = 0; i < n_specs; ++i) {
    const unsigned char* m = inblock + (size_t)i * nb * nb;
    const bool all_in = std::all_of(m, m + nb * nb, [](unsigned char v) { return v != 0; });
    st = fock_build_exact(stream, dtype, all_in ? tuned_flags(dtype, flags, nk1, nk2, nb) : flags, nk1, nk2, nb,
                          P, h, VR, refP, HH, w2d, n_contact, contact_g, contact_Oi, contact_Oj, Sigma, H, F,
                          cand_ws, cand_bytes, flag + i, all_in ? nullptr : m);
    if (st) return st;
  }
  return hf::fock_build_internal(stream, dtype, flags, nk1, nk2, nb, P, h, VR, refP, HH, w2d, n_contact, contact_g,
                                 contact_Oi, contact_Oj, Sigma, H, F, cand_ws, cand_bytes, flag + n_specs);
}

extern "C" int hf_fock_autotune(void* stream, int dtype, unsigned flags, int nk1, int nk2, int nb, const void* P,
                                const void* h, const void* VR, const void* refP, const void* HH, const void* w2d,
                                int n_contact, const void* contact_g, const void* contact_Oi,
                                const void* contact_Oj, void* Sigma, void* H, void* F, void* workspace,
                                size_t workspace_bytes, int reps, unsigned* chosen, float* us) {
  using namespace hf;
  int st = validate(dtype, flags, nk1, nk2, nb);
  if (st) return st;
  if (reps < 1) return fail(HF_ERR_INVALID, "reps must be >= 1");
  if (flags & kEngineFlags) return fail(HF_ERR_INVALID, "hf_fock_autotune chooses the engine flags itself");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const unsigned* cands = kTuneCand;
  // the tile and pipeline candidates only differ from the default where the rows plan applies
  SlotPlan sp0;
  if ((st = get_plan(dtype, flags, nk1, nk2, nb, sp0))) return st;
  float times[kTuneCands] = {-1.f, -1.f, -1.f, -1.f};
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  HF_CUDA(cudaEventCreate(&e0));
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return fail(HF_ERR_CUDA, "cudaEventCreate failed");
  }
  int best = -1;
  for (int c = 0; c < kTuneCands && st == HF_OK; ++c) {
    if ((c == 1 || c == 3) && !sp0.rows) continue;
    const unsigned f = flags | cands[c];
    auto run = [&] {
      return fock_build_exact(stream, dtype, f, nk1, nk2, nb, P, h, VR, refP, HH, w2d, n_contact, contact_g,
                              contact_Oi, contact_Oj, Sigma, H, F, workspace, workspace_bytes, nullptr);
    };
    if ((st = run()) != HF_OK) break;
    if (cudaEventRecord(e0, s) != cudaSuccess) { st = fail(HF_ERR_CUDA, "cudaEventRecord failed"); break; }
    for (int r = 0; r < reps && st == HF_OK; ++r) st = run();
    if (st != HF_OK) break;
    if (cudaEventRecord(e1, s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess) {
      st = fail(HF_ERR_CUDA, "timing the autotuner candidates failed");
      break;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    times[c] = 1000.f * ms / (float)reps;
    if (best < 0 || times[c] < times[best]) best = c;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st != HF_OK) return st;
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[tune_key(dtype, flags, nk1, nk2, nb)] = cands[best];
  }
  // the outputs hold the winner's result
  st = fock_build_exact(stream, dtype, flags | cands[best], nk1, nk2, nb, P, h, VR, refP, HH, w2d, n_contact,
                        contact_g, contact_Oi, contact_Oj, Sigma, H, F, workspace, workspace_bytes, nullptr);
  if (st != HF_OK) return st;
  if (chosen) *chosen = cands[best];
  if (us)
    for (int c = 0; c < kTuneCands; ++c) us[c] = times[c];
  return HF_OK;
}

extern "C" int hf_fock_fault_status(int* code, int clear) {
  if (!code) return hf::fail(HF_ERR_INVALID, "code is NULL");
  int* w = nullptr;
  int st = hf::fault_word(&w);
  if (st) return st;
  HF_CUDA(cudaDeviceSynchronize());
  HF_CUDA(cudaMemcpy(code, w, sizeof(int), cudaMemcpyDeviceToHost));
  if (clear) HF_CUDA(cudaMemset(w, 0, sizeof(int)));
  return HF_OK;
}

extern "C" int hf_fock_autotune_reset(void) {
  std::lock_guard<std::mutex> lk(hf::g_tune_mu);
  hf::g_tune.clear();
  return HF_OK;
}
