"""CPU oracle for the Fock-build / HF-objective path (float64 NumPy restatement).

TEST INFRASTRUCTURE ONLY.  Nothing in the shipped package imports this module;
only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` use it, and only as the checker or as
the timed CPU baseline.  The CUDA path never falls back to it.

The reference (jax_hf v2.2.1) is pure Python on JAX; its arithmetic runs in
XLA (``jnp.fft.fftn/ifftn``) and LAPACK (``jnp.linalg.eigh/solve``).  JAX is not
installed here, so this module restates the reference algorithm in NumPy
(pocketfft + LAPACK through numpy/scipy) in float64, following the cited lines
of the reference one step at a time: same clip constants, iteration counts,
bracket formulas and branch order.  Citations are ``file:line`` inside the
reference project (``src/jax_hf/...``).

Parity pin: ``tests/test_oracle.py`` checks ``build_fock`` +
``hf_energy`` against ``tests/data/meshgrid_regression_case_v1.npz`` of the
reference (F_expected / E_expected, 12x12x4, complex64), and the reference's own
unit-test identities (single-k exchange identity, packed == full, mu hits the
target count, Cayley spectral == LU, HVP == finite differences, the bistable
analytic energies).
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Any, Callable

import numpy as np
import scipy.fft as _sfft
from scipy.special import expit

# FFT worker threads for the exchange (scipy's pocketfft; 1 = numpy-equivalent).
FFT_WORKERS = 1


def _fftn(x):
    return _sfft.fftn(x, axes=(0, 1), workers=FFT_WORKERS)


def _ifftn(x):
    return _sfft.ifftn(x, axes=(0, 1), workers=FFT_WORKERS)

# --------------------------------------------------------------------------
# Small helpers  (solver.py:34-49, fock.py:13-15, utils.py:46-63)
# --------------------------------------------------------------------------


def herm(X):
    """0.5 (X + X^H) on the last two axes (fock.py:13-15, solver.py:34-35)."""
    return 0.5 * (X + np.conj(np.swapaxes(X, -1, -2)))


def skew_hermitian(A):
    """0.5 (A - A^H) (solver.py:38-39)."""
    return 0.5 * (A - np.conj(np.swapaxes(A, -1, -2)))


def density_from_Qp(Q, p):
    """P = Q diag(p) Q^H (solver.py:42-44)."""
    return np.einsum("...in,...n,...jn->...ij", Q, p, np.conj(Q))


def fock_in_orbital_basis(Q, F):
    """Ft = Q^H F Q (solver.py:47-49)."""
    return np.einsum("...in,...ij,...jm->...nm", np.conj(Q), F, Q)


def logit(p):
    """log(p) - log1p(-p) with a 1e-6 clip (solver.py:52-55)."""
    ps = np.clip(p, 1e-6, 1.0 - 1e-6)
    return np.log(ps) - np.log1p(-ps)


def fermidirac(x, T):
    """expit(-x / (T + 1e-12)) (utils.py:51-53)."""
    return expit(-np.asarray(x) / (T + 1e-12))


def sigmoid(x):
    return expit(x)


# --------------------------------------------------------------------------
# Electron-count validation (utils.py:21-43)
# --------------------------------------------------------------------------


def validate_electron_count(weights, nbands, n_electrons, *, context="n_electrons"):
    total_weight = float(np.real(np.asarray(weights)).sum())
    target = float(np.asarray(n_electrons))
    max_electrons = total_weight * int(nbands)
    tol = max(1e-8, 1e-6 * max(1.0, abs(max_electrons)))
    if not np.isfinite(target):
        raise ValueError(f"{context} must be finite, got {target!r}.")
    if target < -tol or target > max_electrons + tol:
        raise ValueError(
            f"{context}={target} is outside the physically reachable range "
            f"[0, {max_electrons}] for {int(nbands)} bands and weights.sum()={total_weight}."
        )


# --------------------------------------------------------------------------
# Kernel precompute (problem.py:22-217)
# --------------------------------------------------------------------------


def shift_phase(n0, n1):
    """e^{2 pi i (m0 s0/n0 + m1 s1/n1)} with s = n//2 (problem.py:90-97)."""
    s0, s1 = n0 // 2, n1 // 2
    ph0 = np.exp(2j * np.pi * np.arange(n0) * s0 / n0)
    ph1 = np.exp(2j * np.pi * np.arange(n1) * s1 / n1)
    return (ph0[:, None] * ph1[None, :])[..., None, None]


class Kernel:
    """Restatement of ``HartreeFockKernel.__init__`` (problem.py:22-199)."""

    def __init__(self, weights, hamiltonian, coulomb_q, T, include_hartree=False,
                 include_exchange=True, reference_density=None, hartree_matrix=None,
                 contact_terms=None, embed_reference_potential=False,
                 center_embedded_hartree=True, dtype=np.complex128):
        h = np.asarray(hamiltonian).astype(dtype)
        rdt = np.zeros((), dtype).real.dtype
        self.h = h
        w2d = np.asarray(weights).astype(rdt)
        self.weights_b = w2d[..., None, None]
        self.weight_sum = np.sum(w2d)
        self.w2d = w2d
        Vq = np.asarray(coulomb_q)
        if np.iscomplexobj(Vq):                                   # problem.py:79-84
            if float(np.max(np.abs(np.imag(Vq)))) <= 1e-8:
                Vq = np.real(Vq)
        else:
            Vq = Vq.astype(rdt)
        self.exchange_hermitian_channel_packing = bool(           # problem.py:85-87
            Vq.shape[-2:] == (1, 1) and not np.iscomplexobj(Vq))
        self.VR = np.fft.fftn(self.weights_b * np.asarray(Vq).astype(dtype), axes=(0, 1))
        n0, n1 = h.shape[0], h.shape[1]
        self._VR_shifted = (self.VR * shift_phase(n0, n1)).astype(dtype)   # problem.py:88-98
        self.T = float(T)
        self.include_hartree = bool(include_hartree)
        self.include_exchange = bool(include_exchange)
        if not self.include_hartree and not self.include_exchange:
            raise ValueError("HartreeFockKernel must include at least one of Hartree or exchange.")
        if reference_density is not None:
            ref = np.asarray(reference_density).astype(dtype)
            if ref.shape != h.shape:
                raise ValueError(f"reference_density must have shape {h.shape}, got {ref.shape}")
            self.refP = ref
        else:
            self.refP = np.zeros_like(h)
        if self.include_hartree:
            if hartree_matrix is None:
                raise ValueError("include_hartree=True requires hartree_matrix to be provided")
            if reference_density is None:
                raise ValueError("include_hartree=True requires reference_density to be provided")
            HH = np.asarray(hartree_matrix).astype(rdt)
            if HH.shape != h.shape[-2:]:
                raise ValueError(f"hartree_matrix must have shape {h.shape[-2:]}, got {HH.shape}")
            self.HH = HH
        else:
            self.HH = np.zeros(h.shape[-2:], dtype=rdt)
        n_orb = h.shape[-1]
        if not contact_terms:                                     # problem.py:129-132
            self.contact_g = np.zeros((1,), rdt)
            self.contact_Oi = np.zeros((1, n_orb, n_orb), dtype)
            self.contact_Oj = np.zeros((1, n_orb, n_orb), dtype)
        else:
            gs, Ois, Ojs = [], [], []
            for k, term in enumerate(contact_terms):
                if len(term) != 3:
                    raise ValueError(f"contact_terms[{k}] must be (g, O_i, O_j); got len={len(term)}")
                g_t, Oi_t, Oj_t = term
                Oi_arr = np.asarray(Oi_t).astype(dtype)
                Oj_arr = np.asarray(Oj_t).astype(dtype)
                if Oi_arr.shape != (n_orb, n_orb) or Oj_arr.shape != (n_orb, n_orb):
                    raise ValueError("contact operator shape mismatch")
                gs.append(rdt.type(g_t))
                Ois.append(Oi_arr)
                Ojs.append(Oj_arr)
            self.contact_g = np.stack(gs)
            self.contact_Oi = np.stack(Ois)
            self.contact_Oj = np.stack(Ojs)
        self.embed_reference_potential = bool(embed_reference_potential)
        self.center_embedded_hartree = bool(center_embedded_hartree)
        self.embedded_energy_offset = 0.0
        if self.embed_reference_potential:                        # problem.py:164-199
            if reference_density is None:
                raise ValueError("embed_reference_potential=True requires reference_density.")
            ref = self.refP
            const_J = 0.0
            J_ref_diag = np.zeros(n_orb, rdt)
            if self.include_hartree:
                diag_R = np.einsum("ij,ijaa->a", w2d, ref).real
                J_ref_diag = self.HH @ diag_R
                if self.center_embedded_hartree:
                    J_ref_diag = J_ref_diag - np.mean(J_ref_diag)
                const_J = float(np.sum(J_ref_diag * diag_R))
            const_S = 0.0
            Sigma_ref = None
            if self.include_exchange:
                Sigma_ref = selfenergy_fft(self._VR_shifted, ref, apply_ifftshift=False,
                                           hermitian_channel_packing=self.exchange_hermitian_channel_packing)
                const_S = float(np.einsum("ij,ijab,ijba->", w2d, Sigma_ref, ref).real)
            h_eff = self.h
            if Sigma_ref is not None:
                h_eff = h_eff + Sigma_ref
            h_eff = h_eff + np.diag(J_ref_diag.astype(dtype))[None, None]
            self.h = h_eff
            self.embedded_energy_offset = 0.5 * (const_J + const_S)

    def as_args(self):
        """problem.py:201-217."""
        return dict(h=self.h, weights_b=self.weights_b, weight_sum=self.weight_sum,
                    VR=self._VR_shifted, T=self.T, refP=self.refP, HH=self.HH,
                    include_hartree=self.include_hartree, include_exchange=self.include_exchange,
                    exchange_hermitian_channel_packing=self.exchange_hermitian_channel_packing,
                    contact_g=self.contact_g, contact_Oi=self.contact_Oi, contact_Oj=self.contact_Oj)


# --------------------------------------------------------------------------
# Exchange self-energy (utils.py:66-311)
# --------------------------------------------------------------------------


def _normalize_block_specs(block_specs):
    """Canonical ('sizes', ...) / ('indices', ...) tuples (linalg.py:19-91)."""
    if block_specs is None:
        return None
    items = (block_specs,) if isinstance(block_specs, dict) else block_specs
    out = []
    for spec in items:
        if isinstance(spec, tuple) and len(spec) == 2 and isinstance(spec[0], str):
            kind = spec[0].strip().lower()
            if kind == "sizes":
                out.append(("sizes", tuple(int(x) for x in spec[1])))
            else:
                out.append(("indices", tuple(tuple(int(i) for i in b) for b in spec[1])))
        elif isinstance(spec, dict):
            if "block_sizes" in spec:
                out.append(("sizes", tuple(int(x) for x in spec["block_sizes"])))
            elif "block_indices" in spec:
                out.append(("indices", tuple(tuple(int(i) for i in b) for b in spec["block_indices"])))
            else:
                raise TypeError("Spec dict must contain 'block_sizes' or 'block_indices'.")
        else:
            seq = list(spec)
            if all(isinstance(x, (int, np.integer)) for x in seq):
                out.append(("sizes", tuple(int(x) for x in seq)))
            else:
                out.append(("indices", tuple(tuple(int(i) for i in b) for b in seq)))
    return tuple(out)


def _block_mask(kind, data, n):
    """Off-block mask (utils.py:176-191)."""
    mask = np.ones((n, n), bool)
    if kind == "sizes":
        start = 0
        for s in data:
            mask[start:start + s, start:start + s] = False
            start += s
    else:
        for idx in data:
            idx = np.asarray(idx, int)
            mask[np.ix_(idx, idx)] = False
    return mask


def _selfenergy_fft_full(VR, P, hermitian_channel_packing=False):
    """utils.py:164-173 (and the packed branch 140-161)."""
    if hermitian_channel_packing:
        n = P.shape[-1]
        ti, tj = np.triu_indices(n)
        off = ti != tj
        flat = ti * n + tj
        Pf = P.reshape(P.shape[:-2] + (n * n,))
        packed = Pf[..., flat]
        sig = -_ifftn(_fftn(packed) * VR[..., 0, 0][..., None])
        out = np.zeros_like(Pf)
        out[..., flat] = sig
        out[..., tj[off] * n + ti[off]] = np.conj(sig[..., off])
        return out.reshape(P.shape)
    return -_ifftn(_fftn(P) * VR)


def _slice_vr(VR, idx):
    if VR.shape[-2] == 1 and VR.shape[-1] == 1:
        return VR
    return VR[..., idx, :][..., :, idx]


def selfenergy_fft(VR, P, *, block_specs=None, check_offdiag=None, offdiag_atol=1e-12,
                   offdiag_rtol=0.0, apply_ifftshift=True, hermitian_channel_packing=False):
    """Sigma = -IFFT2(FFT2(P) * VR) with packing / block options (utils.py:66-137, 206-311)."""
    VR = np.asarray(VR)
    P = np.asarray(P)
    if hermitian_channel_packing and VR.shape[-2:] != (1, 1):
        raise ValueError("hermitian_channel_packing requires a scalar interaction kernel "
                         "with shape (..., 1, 1).")
    specs = _normalize_block_specs(block_specs)
    if not specs:
        result = _selfenergy_fft_full(VR, P, hermitian_channel_packing)
    else:
        check = bool(check_offdiag) if check_offdiag is not None else True
        n = P.shape[-1]
        absP = np.abs(P)
        tol = offdiag_atol + offdiag_rtol * absP.max()
        result = None
        for kind, data in specs:                       # first compatible spec wins
            mask = _block_mask(kind, data, n)
            ok = (absP * mask).max() <= tol if check else True
            if ok:
                out = np.zeros_like(P)
                if kind == "sizes":
                    if sum(data) != n:
                        raise ValueError(f"block_sizes must sum to {n}.")
                    blocks = []
                    start = 0
                    for s in data:
                        blocks.append(np.arange(start, start + s))
                        start += s
                else:
                    blocks = [np.asarray(b, int) for b in data]
                for idx in blocks:
                    sub = P[..., idx, :][..., :, idx]
                    sb = _selfenergy_fft_full(_slice_vr(VR, idx), sub, hermitian_channel_packing)
                    out[..., idx[:, None], idx[None, :]] = sb
                result = out
                break
        if result is None:
            result = _selfenergy_fft_full(VR, P, hermitian_channel_packing)
    if apply_ifftshift:
        return np.fft.ifftshift(result, axes=(0, 1))
    return result


# --------------------------------------------------------------------------
# Fock build + objective (fock.py:18-129)
# --------------------------------------------------------------------------


def build_fock(P, *, h, VR, refP, HH, w2d, include_exchange, include_hartree,
               exchange_hermitian_channel_packing, contact_g=None, contact_Oi=None,
               contact_Oj=None, exchange_block_specs=None, exchange_check_offdiag=None,
               exchange_offdiag_atol=1e-12, exchange_offdiag_rtol=0.0, project_fn=None):
    """Returns (Sigma, H, F) with F = herm(h + Sigma + H) (fock.py:18-97)."""
    dP = P - refP
    if include_exchange:
        Sigma = selfenergy_fft(VR, dP, block_specs=exchange_block_specs,
                               check_offdiag=exchange_check_offdiag,
                               offdiag_atol=exchange_offdiag_atol,
                               offdiag_rtol=exchange_offdiag_rtol, apply_ifftshift=False,
                               hermitian_channel_packing=exchange_hermitian_channel_packing)
    else:
        Sigma = np.zeros_like(h)
    if include_hartree:                                             # fock.py:66-74
        diag_real = np.real(np.diagonal(dP, axis1=-2, axis2=-1))
        n_vec = np.sum(w2d[..., None] * diag_real, axis=(0, 1))
        H = np.diag((HH @ n_vec).astype(h.real.dtype))[None, None].astype(h.dtype)
    else:
        H = np.zeros_like(h)
    if contact_g is not None and contact_Oi is not None and contact_Oj is not None:
        rho_bar = np.einsum("ij,ijab->ab", w2d, dP)                 # fock.py:79-92
        tr_Oj_rho = np.einsum("tij,ji->t", contact_Oj, rho_bar)
        s_h = np.einsum("t,tij->ij", contact_g * tr_Oj_rho, contact_Oi)
        oi_rho = np.einsum("tij,jk->tik", contact_Oi, rho_bar)
        oi_rho_oj = np.einsum("tik,tkl->til", oi_rho, contact_Oj)
        s_f = np.einsum("t,tij->ij", -contact_g, oi_rho_oj)
        Sigma = Sigma + (s_h + s_f).astype(h.dtype)[None, None]
    F = herm(h + Sigma + H)
    if project_fn is not None:
        F = herm(np.asarray(project_fn(F), dtype=F.dtype))
    return Sigma, H, F


def hf_energy(P, *, h, Sigma, H, weights_b):
    """E = sum_k w_k Re Tr[(h + (Sigma+H)/2) P] (fock.py:100-111)."""
    return float(np.sum(np.real(np.einsum("...ij,...ji->...", weights_b * (h + 0.5 * (Sigma + H)), P))))


def occupation_entropy(p, w_norm):
    """S = -sum w [p log p + (1-p) log1p(-p)], clip 1e-14 (fock.py:114-118)."""
    ps = np.clip(p, 1e-14, 1.0 - 1e-14)
    s = ps * np.log(ps) + (1.0 - ps) * np.log1p(-ps)
    return float(-np.sum(w_norm[..., None] * s))


def free_energy(E, p, w_norm, T):
    """Omega = E - max(T, 1e-14) S (fock.py:121-129)."""
    return float(E - max(float(T), 1e-14) * occupation_entropy(p, w_norm))


# --------------------------------------------------------------------------
# Chemical potential (utils.py:314-442, solver.py:62-101)
# --------------------------------------------------------------------------


def find_mu_bisection(bands, weights, n_electrons, T, maxiter=None, single=False):
    """Pure bracket bisection (utils.py:353-382)."""
    if maxiter is None:
        maxiter = 30 if single else 54
    bmin, bmax = float(np.min(bands)), float(np.max(bands))
    span = bmax - bmin + 10.0 * max(T, 1e-6)
    lo, hi = bmin - span, bmax + span
    w = np.asarray(weights)[..., None]
    for _ in range(int(maxiter)):
        mid = 0.5 * (lo + hi)
        count = np.sum(w * fermidirac(bands - mid, T))
        if count > n_electrons:
            hi = mid
        else:
            lo = mid
    return 0.5 * (lo + hi)


def find_mu_newton(bands, weights, n_electrons, T, maxiter=None, single=False):
    """Newton with bracket safeguards (utils.py:385-442)."""
    if maxiter is None:
        maxiter = 15 if single else 25
    Tj = max(T, 1e-12)
    bmin, bmax = float(np.min(bands)), float(np.max(bands))
    span = bmax - bmin + 10.0 * max(Tj, 1e-6)
    lo, hi = bmin - span, bmax + span
    mu = 0.5 * (lo + hi)
    w = np.asarray(weights)[..., None]

    def count_and_slope(m):
        p = sigmoid((m - bands) / Tj)
        return np.sum(w * p), np.sum(w * (p * (1.0 - p)) / Tj)

    for _ in range(int(maxiter)):
        N, Z = count_and_slope(mu)
        g = N - n_electrons
        if g < 0:
            lo = mu
        if g > 0:
            hi = mu
        mu_new = mu - g / max(Z, 1e-18)
        mu_bis = 0.5 * (lo + hi)
        if mu_new <= lo or mu_new >= hi:
            mu_new = mu_bis
        mu_new = min(max(mu_new, lo), hi)
        if not np.isfinite(mu_new):
            mu_new = mu_bis
        mu = mu_new
    N, _ = count_and_slope(mu)
    return 0.5 * (lo + hi) if abs(N - n_electrons) > 1e-12 else mu


def find_chemical_potential(bands, weights, n_electrons, T, *, maxiter=None, method="bisection",
                            single=False):
    """utils.py:314-350."""
    validate_electron_count(weights, np.shape(bands)[-1], n_electrons)
    method = str(method).lower()
    if method == "bisection":
        return find_mu_bisection(bands, weights, n_electrons, T, maxiter, single)
    if method == "newton":
        return find_mu_newton(bands, weights, n_electrons, T, maxiter, single)
    raise ValueError(f"method must be 'bisection' or 'newton', got {method!r}")


def solve_mu(eps, w_norm, n_target_norm, mu0, T, maxiter=25):
    """Newton-bracket mu solve of the direct-minimisation solver (solver.py:62-101)."""
    Tj = max(float(T), 1e-12)
    lo = float(np.min(eps)) - 50.0 * Tj
    hi = float(np.max(eps)) + 50.0 * Tj
    mu = min(max(float(mu0), lo), hi)
    w = w_norm[..., None]
    for _ in range(int(maxiter)):
        p = sigmoid((mu - eps) / Tj)
        N = np.sum(w * p)
        Z = np.sum(w * p * (1.0 - p) / Tj)
        g = N - n_target_norm
        if g < 0:
            lo = mu
        if g > 0:
            hi = mu
        mu_new = mu - g / max(Z, 1e-18)
        mu_bis = 0.5 * (lo + hi)
        if mu_new <= lo or mu_new >= hi:
            mu_new = mu_bis
        mu_new = min(max(mu_new, lo), hi)
        if not np.isfinite(mu_new):
            mu_new = mu_bis
        mu = mu_new
    return mu


# --------------------------------------------------------------------------
# Retractions (solver.py:108-197)
# --------------------------------------------------------------------------


def qr_retract(G, tau):
    """U = QR(I - tau G) with diag(R) phase normalisation (solver.py:108-119)."""
    n = G.shape[-1]
    U0 = np.eye(n, dtype=G.dtype) - np.asarray(tau)[..., None, None] * G
    U, R = np.linalg.qr(U0)
    ph = np.diagonal(R, axis1=-2, axis2=-1)
    a = np.abs(ph)
    norm = np.where(a > 1e-30, ph / np.where(a > 0, a, 1.0), 1.0)
    return U * norm[..., None, :]


def cayley_retract(d, tau):
    """U = solve(I + tau d/2, I - tau d/2) (solver.py:122-138)."""
    n = d.shape[-1]
    eye = np.eye(n, dtype=d.dtype)
    A = 0.5 * np.asarray(tau)[..., None, None] * d
    return np.linalg.solve(eye + A, np.broadcast_to(eye - A, A.shape))


def cayley_spectral_setup(d):
    """eigh(herm(i d)) -> (V, lam) (solver.py:161-166)."""
    iA = herm(1j * d)
    lam, V = np.linalg.eigh(iA)
    return V, lam


def cayley_factor(lam, tau):
    """(1 + i tau lam/2) / (1 - i tau lam/2) (solver.py:169-175)."""
    iexp = 1j * (tau * lam * 0.5)
    return (1.0 + iexp) / (1.0 - iexp)


def cayley_unitary_from_spectrum(V, lam, tau):
    """U = V diag(c) V^H (solver.py:178-182)."""
    c = cayley_factor(lam, tau)
    return (V * c[..., None, :]) @ np.conj(np.swapaxes(V, -1, -2))


def diag_UFU_from_spectrum(V, Ft_eig, lam, tau):
    """diag(U^H Ft U) via V (cbar Ft_eig c) (solver.py:185-197)."""
    c = cayley_factor(lam, tau)
    M = np.conj(c)[..., :, None] * Ft_eig * c[..., None, :]
    A = V @ M
    return np.real(np.sum(A * np.conj(V), axis=-1))


# --------------------------------------------------------------------------
# Inner products (solver.py:205-233)
# --------------------------------------------------------------------------


def ip_matrix(X, Y, w):
    return float(np.sum(w * np.sum(np.real(np.conj(X) * Y), axis=(-2, -1))))


def ip_vec(x, y, w):
    return float(np.sum(w[..., None] * x * y))


def norm_matrix(X, w):
    return float(np.sqrt(max(0.0, ip_matrix(X, X, w))))


def project_occ(dp, w2d):
    nb = dp.shape[-1]
    return dp - np.sum(w2d[..., None] * dp) / (np.sum(w2d) * nb)


# --------------------------------------------------------------------------
# Direct-minimisation CG (solver.py:240-660)
# --------------------------------------------------------------------------


@dataclass(frozen=True)
class SolverConfig:
    """Field names and defaults of solver.py:240-286."""
    max_iter: int = 200
    tol_E: float = 1e-7
    tol_grad: float = 0.0
    denom_scale: float = 1e-3
    max_step: float = 0.6
    cg_restart: int = 10
    bt_shrink: float = 0.5
    bt_max: int = 8
    mu_maxiter: int = 25
    plateau_window: int = 5
    optimizer: str = "cg"
    tr_delta0: float = 0.5
    tr_cg_max: int = 20
    deflation_targets: Any = None
    deflation_sigma: float = 0.0
    deflation_length: float = 1.0
    block_sizes: Any = None
    project_fn: Any = None


def _fock_call(kernel_args, P, fock_build_fn, block_specs, project_fn=None, refP=None):
    a = kernel_args
    fn = fock_build_fn or build_fock
    return fn(P, h=a["h"], VR=a["VR"], refP=a["refP"] if refP is None else refP, HH=a["HH"],
              w2d=a["weights_b"][..., 0, 0], include_exchange=a["include_exchange"],
              include_hartree=a["include_hartree"],
              exchange_hermitian_channel_packing=a["exchange_hermitian_channel_packing"],
              contact_g=a["contact_g"], contact_Oi=a["contact_Oi"], contact_Oj=a["contact_Oj"],
              exchange_block_specs=block_specs, project_fn=project_fn)


def solve_cg(kernel, P0, n_electrons, config=None, fock_build_fn=None):
    """Preconditioned Riemannian CG (solver.py:307-660).  Returns a dict."""
    cfg = config or SolverConfig()
    validate_electron_count(kernel.w2d, kernel.h.shape[-1], n_electrons)
    a = kernel.as_args()
    h, weights_b = a["h"], a["weights_b"]
    tiny = 1e-30
    project = cfg.project_fn or (lambda A: A)
    specs = None if cfg.block_sizes is None else (("sizes", tuple(cfg.block_sizes)),)
    w2d = weights_b[..., 0, 0].real
    ws = float(a["weight_sum"])
    w_norm = w2d / max(ws, tiny)
    n_target_norm = float(n_electrons) / max(ws, tiny)
    T_r = max(float(a["T"]), 1e-12)
    nb = h.shape[-1]
    offdiag = (1.0 - np.eye(nb))[None, None]

    P0h = herm(np.asarray(P0, dtype=h.dtype))
    _, _, F0 = _fock_call(a, P0h, fock_build_fn, specs, cfg.project_fn)
    eps0, Q0 = np.linalg.eigh(F0)
    mu0 = solve_mu(eps0, w_norm, n_target_norm, 0.0, T_r, cfg.mu_maxiter)
    p0 = sigmoid((mu0 - eps0) / T_r)

    hist_E = np.zeros(cfg.max_iter)
    hist_G = np.zeros(cfg.max_iter)
    k, Q, p, mu = 0, Q0, p0, mu0
    dQ_prev = np.zeros_like(Q0)
    dp_prev = np.zeros_like(p0)
    GQ_prev = np.zeros_like(Q0)
    gp_prev = np.zeros_like(p0)
    grad_norm, E_prev, dE = np.inf, np.inf, np.inf
    n_builds = 1

    def cond():                                                   # solver.py:422-449
        if cfg.plateau_window > 0:
            e_now = hist_E[max(k - 1, 0)]
            e_past = hist_E[max(k - 1 - cfg.plateau_window, 0)]
            enc = (e_past - e_now) > cfg.tol_E if k > cfg.plateau_window else dE > cfg.tol_E
        else:
            enc = dE > cfg.tol_E
        nc = (grad_norm > cfg.tol_grad) if cfg.tol_grad > 0.0 else enc
        return k < cfg.max_iter and nc

    while cond():
        P_cur = herm(project(density_from_Qp(Q, p)))              # solver.py:462
        Sigma, Hh, F = _fock_call(a, P_cur, fock_build_fn, specs)
        n_builds += 1
        E = hf_energy(P_cur, h=h, Sigma=Sigma, H=Hh, weights_b=weights_b)
        Ft = fock_in_orbital_basis(Q, F)
        eps = np.real(np.diagonal(Ft, axis1=-2, axis2=-1))
        diff_p = p[..., None, :] - p[..., :, None]
        GQ = skew_hermitian(diff_p * Ft) * offdiag
        gp = eps + T_r * logit(p) - mu
        grad_norm = norm_matrix(GQ, w_norm)
        gap = eps[..., :, None] - eps[..., None, :]               # solver.py:495-504
        eps_scale = np.sqrt(np.mean(eps ** 2) + tiny)
        lam = max(T_r, cfg.denom_scale * eps_scale)
        HQ = GQ / np.sqrt(gap ** 2 + lam ** 2)
        ps = np.clip(p, 1e-8, 1.0 - 1e-8)
        hp = gp * (ps * (1.0 - ps) / T_r)
        pr_num = (ip_matrix(GQ, HQ, w_norm) - ip_matrix(GQ_prev, HQ, w_norm)
                  + ip_vec(gp, hp, w_norm) - ip_vec(gp_prev, hp, w_norm))
        pr_den = ip_matrix(GQ_prev, GQ_prev, w_norm) + ip_vec(gp_prev, gp_prev, w_norm)
        beta = max(0.0, pr_num / pr_den) if pr_den > tiny else 0.0
        beta = min(beta, 5.0)
        if k == 0 or k % cfg.cg_restart == 0:
            beta = 0.0
        dQ = HQ + beta * dQ_prev
        dp = hp + beta * dp_prev
        Vd, lamd = cayley_spectral_setup(dQ)                      # solver.py:543-547
        Ft_eig = np.conj(np.swapaxes(Vd, -2, -1)) @ Ft @ Vd
        dQn = norm_matrix(dQ, w_norm)
        tau0 = min(1.0, cfg.max_step / max(dQn, tiny))

        def frozen(tau):
            eps_t = diag_UFU_from_spectrum(Vd, Ft_eig, lamd, tau)
            pt = np.clip(p - tau * dp, 1e-8, 1.0 - 1e-8)
            return free_energy(np.sum(w_norm[..., None] * pt * eps_t), pt, w_norm, T_r)

        p0c = np.clip(p, 1e-8, 1.0 - 1e-8)
        Omega0 = free_energy(np.sum(w_norm[..., None] * p0c * eps), p0c, w_norm, T_r)
        tau, accepted, i = tau0, False, 0
        while i < cfg.bt_max and not accepted:                    # solver.py:563-577
            accepted = frozen(tau) < Omega0
            if not accepted:
                tau = tau * cfg.bt_shrink
            i += 1
        if not accepted:
            tau = tau0 * cfg.bt_shrink ** cfg.bt_max
        U = cayley_unitary_from_spectrum(Vd, lamd, tau)           # solver.py:586-592
        Q_new = Q @ U
        eps_new = diag_UFU_from_spectrum(Vd, Ft_eig, lamd, tau)
        mu_new = solve_mu(eps_new, w_norm, n_target_norm, mu, T_r, cfg.mu_maxiter)
        p_new = sigmoid((mu_new - eps_new) / T_r)
        hist_E[k] = E
        hist_G[k] = grad_norm
        dE = abs(E - E_prev)
        Q, p, mu = Q_new, p_new, mu_new
        dQ_prev, dp_prev, GQ_prev, gp_prev, E_prev = dQ, dp, GQ, gp, E
        k += 1

    P_pre = herm(project(density_from_Qp(Q, p)))                  # solver.py:613-638
    _, _, F_pre = _fock_call(a, P_pre, fock_build_fn, specs)
    Ft_fin = fock_in_orbital_basis(Q, F_pre)
    eps_fin, V_fin = np.linalg.eigh(Ft_fin)
    Q_fin = Q @ V_fin
    mu_fin = solve_mu(eps_fin, w_norm, n_target_norm, mu, T_r, cfg.mu_maxiter)
    p_fin = sigmoid((mu_fin - eps_fin) / T_r)
    P_fin = herm(project(density_from_Qp(Q_fin, p_fin)))
    Sigma_f, H_f, F_f = _fock_call(a, P_fin, fock_build_fn, specs)
    E_fin = hf_energy(P_fin, h=h, Sigma=Sigma_f, H=H_f, weights_b=weights_b)
    n_builds += 2
    converged = (grad_norm <= cfg.tol_grad) if cfg.tol_grad > 0.0 else (k < cfg.max_iter)
    return dict(Q=Q_fin, p=p_fin, mu=mu_fin, density=P_fin, fock=F_f, energy=E_fin, n_iter=k,
                converged=bool(converged), history=dict(E=hist_E, grad_norm=hist_G),
                n_builds=n_builds)


# --------------------------------------------------------------------------
# Trust-region Newton (solver.py:686-1078)
# --------------------------------------------------------------------------


def solve_newton(kernel, P0, n_electrons, config=None, fock_build_fn=None):
    """Steihaug truncated-CG trust-region Newton (solver.py:686-1078)."""
    cfg = config or SolverConfig(optimizer="newton")
    validate_electron_count(kernel.w2d, kernel.h.shape[-1], n_electrons)
    a = kernel.as_args()
    h, weights_b = a["h"], a["weights_b"]
    tiny = 1e-30
    project = cfg.project_fn or (lambda A: A)
    specs = None if cfg.block_sizes is None else (("sizes", tuple(cfg.block_sizes)),)
    w2d = weights_b[..., 0, 0].real
    ws = float(a["weight_sum"])
    w_norm = w2d / max(ws, tiny)
    ones_w = np.ones_like(w2d)
    n_target_norm = float(n_electrons) / max(ws, tiny)
    T_r = max(float(a["T"]), 1e-12)
    tol_g = float(cfg.tol_grad) if cfg.tol_grad > 0.0 else 1e-6     # solver.py:1191
    delta_min = 1e-10
    occ_clip = 1e-8
    noise_floor = max(1e-12, 4500.0 * np.finfo(np.float64).eps)
    nb = h.shape[-1]
    eye = np.eye(nb, dtype=h.dtype)
    offdiag = (1.0 - np.eye(nb))[None, None]
    has_defl = cfg.deflation_targets is not None and float(cfg.deflation_sigma) > 0.0
    if has_defl:
        targets = np.asarray(cfg.deflation_targets, dtype=h.dtype)
        if targets.ndim == 4:
            targets = targets[None]
        inv2L2 = 1.0 / (2.0 * max(float(cfg.deflation_length), 1e-12) ** 2)
        sig = float(cfg.deflation_sigma)
    n_builds = [0]

    def fock_full(P):
        n_builds[0] += 1
        return _fock_call(a, P, fock_build_fn, specs)

    def fock_response(dP):
        n_builds[0] += 1
        _, _, Fr = _fock_call(a, dP, fock_build_fn, specs, refP=np.zeros_like(a["refP"]))
        return Fr - h

    def jip(aX, ap, bX, bp):
        return ip_matrix(aX, bX, ones_w) + ip_vec(ap, bp, w2d)

    def jnorm(aX, ap):
        return np.sqrt(max(0.0, jip(aX, ap, aX, ap)))

    def defl_bias(P):                                             # solver.py:804-812
        diff = P[None] - targets
        d2 = np.sum(w2d[None] * np.sum(np.abs(diff) ** 2, axis=(-2, -1)), axis=(1, 2))
        phi = sig * np.exp(-d2 * inv2L2)
        phip = -phi * inv2L2
        S_pen = np.sum((2.0 * phip)[:, None, None, None, None] * diff, axis=0)
        return float(np.sum(phi)), S_pen, float(2.0 * np.sum(phip))

    def eval_state(Q, p):                                         # solver.py:814-837
        P = herm(project(density_from_Qp(Q, p)))
        Sg, Hh, F = fock_full(P)
        E = hf_energy(P, h=h, Sigma=Sg, H=Hh, weights_b=weights_b)
        pen = 0.0
        if has_defl:
            Phi, S_pen, pen = defl_bias(P)
            E, F = E + Phi, F + S_pen
        Ft = fock_in_orbital_basis(Q, F)
        diff_p = p[..., None, :] - p[..., :, None]
        G = skew_hermitian(diff_p * Ft) * offdiag
        return E, Ft, norm_matrix(G, w_norm), pen

    P0h = herm(np.asarray(P0, dtype=h.dtype))
    _, _, F0 = fock_full(P0h)
    eps0, Q0 = np.linalg.eigh(F0)
    mu0 = solve_mu(eps0, w_norm, n_target_norm, 0.0, T_r, cfg.mu_maxiter)
    p0 = sigmoid((mu0 - eps0) / T_r)
    E0, Ft0, g0, pen0 = eval_state(Q0, p0)
    if g0 <= tol_g:                                               # solver.py:858-877
        p_i, mu_i = p0, mu0
        for _ in range(30):
            P = herm(project(density_from_Qp(Q0, p_i)))
            _, _, F = fock_full(P)
            eps_i = np.real(np.diagonal(fock_in_orbital_basis(Q0, F), axis1=-2, axis2=-1))
            mu_i = solve_mu(eps_i, w_norm, n_target_norm, mu_i, T_r, cfg.mu_maxiter)
            p_i = sigmoid((mu_i - eps_i) / T_r)
        p0, mu0 = p_i, mu_i
        E0, Ft0, g0, pen0 = eval_state(Q0, p0)

    hist_E = np.zeros(cfg.max_iter)
    hist_G = np.zeros(cfg.max_iter)
    k, Q, p, mu, Ft, E, Delta, grad_norm, pen = 0, Q0, p0, mu0, Ft0, E0, float(cfg.tr_delta0), g0, pen0
    while k < cfg.max_iter and grad_norm > tol_g and Delta > delta_min:
        hist_E[k] = E
        hist_G[k] = grad_norm
        eps = np.real(np.diagonal(Ft, axis1=-2, axis2=-1))
        diff_p = p[..., None, :] - p[..., :, None]
        G = skew_hermitian(diff_p * Ft) * offdiag
        eps_scale = np.sqrt(np.mean(eps ** 2) + tiny)
        lam_pc = max(T_r, cfg.denom_scale * eps_scale)
        gap = eps[..., :, None] - eps[..., None, :]
        denomX = np.sqrt(gap ** 2 + lam_pc ** 2)
        pc = np.clip(p, occ_clip, 1.0 - occ_clip)
        fd_curv = pc * (1.0 - pc) / T_r

        def prec(aX, ap):
            return aX / denomX, project_occ(ap * fd_curv, w2d)

        def hvp(X, dp):                                           # solver.py:916-930
            M = X * diff_p + dp[..., :, None] * eye
            dP = herm(np.einsum("...in,...nm,...jm->...ij", Q, M, np.conj(Q)))
            resp = fock_response(dP)
            if has_defl:
                resp = resp + pen * dP
            St = fock_in_orbital_basis(Q, resp)
            A = Ft @ X - X @ Ft + St
            diff_dp = dp[..., None, :] - dp[..., :, None]
            C = diff_dp * Ft + diff_p * A
            HX = skew_hermitian(C) * offdiag
            Hp = np.real(np.diagonal(A, axis1=-2, axis2=-1)) + (T_r / (pc * (1.0 - pc))) * dp
            return HX, project_occ(Hp, w2d)

        rX, rp = -G, np.zeros_like(p)                             # solver.py:932-992
        zX, zp = prec(rX, rp)
        rz = jip(rX, rp, zX, zp)
        vX, vp = np.zeros_like(Q), np.zeros_like(p)
        HvX, Hvp = np.zeros_like(Q), np.zeros_like(p)
        dX, dp = zX, zp
        cg, done = 0, False
        while cg < cfg.tr_cg_max and not done:
            HdX, Hdp = hvp(dX, dp)
            dHd = jip(dX, dp, HdX, Hdp)
            dd = jip(dX, dp, dX, dp)
            neg = dHd <= 1e-14 * dd
            b = 2.0 * jip(vX, vp, dX, dp)
            cc = jip(vX, vp, vX, vp) - Delta * Delta
            disc = max(b ** 2 - 4.0 * dd * cc, 0.0)
            t_bd = (-b + np.sqrt(disc)) / (2.0 * dd + 1e-30)
            alpha = rz / (1.0 if neg else dHd)
            vXa, vpa = vX + alpha * dX, vp + alpha * dp
            cross = jnorm(vXa, vpa) >= Delta
            take_bd = neg or cross
            rXa, rpa = rX - alpha * HdX, rp - alpha * Hdp
            inner = jnorm(rXa, rpa) < 0.05 * grad_norm
            zXa, zpa = prec(rXa, rpa)
            rz_new = jip(rXa, rpa, zXa, zpa)
            beta = rz_new / (rz if abs(rz) > tiny else 1.0)
            stop = take_bd or inner
            if take_bd:
                vX, vp = vX + t_bd * dX, vp + t_bd * dp
                HvX, Hvp = HvX + t_bd * HdX, Hvp + t_bd * Hdp
            else:
                vX, vp = vXa, vpa
                HvX, Hvp = HvX + alpha * HdX, Hvp + alpha * Hdp
                rX, rp = rXa, rpa
            if not stop:
                dX, dp = zXa + beta * dX, zpa + beta * dp
                rz = rz_new
            cg += 1
            done = stop
        gv = ip_matrix(G, vX, w2d)                                # solver.py:998-1046
        vHv = ip_matrix(vX, HvX, w2d) + ip_vec(vp, Hvp, w2d)
        pred = -(gv + 0.5 * vHv)
        Vv, lamv = cayley_spectral_setup(vX)
        U = cayley_unitary_from_spectrum(Vv, lamv, -1.0)
        Qt = Q @ U
        eps_t = np.real(np.diagonal(fock_in_orbital_basis(U, Ft), axis1=-2, axis2=-1))
        mu_t = solve_mu(eps_t, w_norm, n_target_norm, mu, T_r, cfg.mu_maxiter)
        p_trial = sigmoid((mu_t - eps_t) / T_r)
        E_t, Ft_t, g_t, pen_t = eval_state(Qt, p_trial)
        noise = noise_floor * max(abs(E), 1.0)
        use_g = pred <= noise
        accept_g = g_t <= grad_norm and E_t <= E + noise
        Delta_g = Delta if accept_g else 0.5 * Delta
        ratio = (E - E_t) / (1.0 if use_g else pred)
        step_norm = jnorm(vX, vp)
        if ratio < 0.25:
            Delta_r = 0.25 * Delta
        elif ratio > 0.75 and step_norm > 0.9 * Delta:
            Delta_r = min(2.0 * Delta, 5.0)
        else:
            Delta_r = Delta
        accept = accept_g if use_g else ratio > 0.1
        Delta = Delta_g if use_g else Delta_r
        if accept:
            Q, p, Ft, E, mu, grad_norm, pen = Qt, p_trial, Ft_t, E_t, mu_t, g_t, pen_t
        k += 1
    P_fin = herm(project(density_from_Qp(Q, p)))
    Sg, Hf, Ff = fock_full(P_fin)
    E_fin = hf_energy(P_fin, h=h, Sigma=Sg, H=Hf, weights_b=weights_b)
    return dict(Q=Q, p=p, mu=mu, density=P_fin, fock=Ff, energy=E_fin, n_iter=k,
                converged=bool(grad_norm <= tol_g), history=dict(E=hist_E, grad_norm=hist_G),
                n_builds=n_builds[0])


def solve(kernel, P0, n_electrons, *, config=None, fock_build_fn=None):
    """Dispatch on optimizer (solver.py:1098-1247)."""
    cfg = config or SolverConfig()
    opt = str(cfg.optimizer).lower()
    if opt not in ("cg", "newton"):
        raise ValueError(f"Unknown optimizer {cfg.optimizer!r}; expected 'cg' or 'newton'.")
    if opt == "newton":
        return solve_newton(kernel, P0, n_electrons, cfg, fock_build_fn)
    return solve_cg(kernel, P0, n_electrons, cfg, fock_build_fn)


# --------------------------------------------------------------------------
# Reference SCF (reference_scf.py:31-365)
# --------------------------------------------------------------------------


@dataclass(frozen=True)
class SCFConfig:
    max_iter: int = 200
    density_tol: float = 1e-7
    comm_tol: float = 1e-6
    mixing: float = 0.5
    level_shift: float = 0.0
    acceleration: str = "linear"
    diis_size: int = 6
    diis_start: int = 2
    diis_damping: float = 1.0
    trust_radius: float = 0.0
    project_fn: Callable | None = None


def weighted_matrix_norm(M, w, ws):
    """reference_scf.py:82-84."""
    return float(np.sqrt(np.sum(w * np.sum(np.abs(M) ** 2, axis=(-2, -1))) / ws))


def density_from_fock(F, *, weights, n_electrons, temperature, level_shift):
    """reference_scf.py:87-96."""
    ev, orb = np.linalg.eigh(herm(F))
    mu_raw = find_chemical_potential(ev, weights, n_electrons, temperature)
    occ_raw = fermidirac(ev - mu_raw, temperature)
    shifted = ev + level_shift * (1.0 - occ_raw)
    mu = find_chemical_potential(shifted, weights, n_electrons, temperature)
    occ = fermidirac(shifted - mu, temperature)
    return herm(np.einsum("...in,...n,...jn->...ij", orb, occ, np.conj(orb))), mu


def diis_coefficients(R_hist, active, w2d):
    """Masked bordered Pulay system (reference_scf.py:99-121)."""
    N = R_hist.shape[0]
    B = np.real(np.einsum("iklab,jklab->ij", np.conj(R_hist), R_hist * w2d[None, :, :, None, None]))
    B = B / max(np.max(np.abs(B)), 1e-30)
    af = active.astype(np.float64)
    A = np.zeros((N + 1, N + 1))
    A[:N, :N] = B + np.diag(1.0 - af)
    A[:N, N] = -af
    A[N, :N] = -af
    rhs = np.zeros(N + 1)
    rhs[N] = -1.0
    try:
        sol = np.linalg.solve(A, rhs)
    except np.linalg.LinAlgError:
        sol = np.full(N + 1, np.nan)
    return sol[:N], bool(np.all(np.isfinite(sol)))


def solve_scf(kernel, P0, n_electrons, *, config=None, fock_build_fn=None):
    """Roothaan SCF with linear / DIIS / ODA (reference_scf.py:124-365).  Returns a dict."""
    cfg = config or SCFConfig()
    a = kernel.as_args()
    h, weights_b = a["h"], a["weights_b"]
    w2d = kernel.w2d
    ws = max(float(a["weight_sum"]), 1e-30)
    T = a["T"]
    project = cfg.project_fn or (lambda A: A)
    fn = fock_build_fn or build_fock

    def fock(dh):
        return fn(dh, h=h, VR=a["VR"], refP=a["refP"], HH=a["HH"], w2d=w2d,
                  include_exchange=a["include_exchange"], include_hartree=a["include_hartree"],
                  exchange_hermitian_channel_packing=a["exchange_hermitian_channel_packing"],
                  contact_g=a["contact_g"], contact_Oi=a["contact_Oi"], contact_Oj=a["contact_Oj"],
                  project_fn=cfg.project_fn)

    def build_and_occupy(dens):                                   # reference_scf.py:264-273
        dh = herm(np.asarray(project(dens), dtype=h.dtype))
        Sg, Hh, F = fock(dh)
        E = hf_energy(dh, h=h, Sigma=Sg, H=Hh, weights_b=weights_b)
        Pn, mu = density_from_fock(F, weights=w2d, n_electrons=n_electrons, temperature=T,
                                   level_shift=cfg.level_shift)
        return herm(np.asarray(project(Pn), dtype=h.dtype)), F, E, mu

    def linear(dens, delta):
        return herm(np.asarray(project(dens + cfg.mixing * delta), dtype=h.dtype))

    nh = cfg.diis_size if cfg.acceleration == "diis" else 0
    F_hist = np.zeros((nh,) + h.shape, h.dtype)
    R_hist = np.zeros((nh,) + h.shape, h.dtype)
    hE, hD, hC = np.zeros(cfg.max_iter), np.zeros(cfg.max_iter), np.zeros(cfg.max_iter)
    k, dens, converged = 0, np.asarray(P0, dtype=h.dtype), False
    while k < cfg.max_iter and not converged:
        Pn, F, E, mu = build_and_occupy(dens)
        delta = Pn - dens
        comm = F @ dens - dens @ F
        d_res = weighted_matrix_norm(delta, w2d, ws)
        c_res = weighted_matrix_norm(comm, w2d, ws)
        converged = d_res <= cfg.density_tol and c_res <= cfg.comm_tol
        if cfg.acceleration == "diis":
            idx = k % nh
            F_hist[idx] = F
            R_hist[idx] = comm
            count = min(k + 1, nh)
            active = np.arange(nh) < count
            coeffs, ok = diis_coefficients(R_hist, active, w2d)
            if ok:
                Fx = np.einsum("i,iklab->klab", coeffs.astype(h.dtype), F_hist)
            else:
                Fx = F
            damp = float(np.clip(cfg.diis_damping, 0.0, 1.0))
            Fx = damp * Fx + (1.0 - damp) * F
            engaged = count >= max(2, cfg.diis_start) and ok
            if engaged:
                Pd, _ = density_from_fock(herm(Fx), weights=w2d, n_electrons=n_electrons,
                                          temperature=T, level_shift=cfg.level_shift)
                updated = herm(np.asarray(project(Pd), dtype=h.dtype))
            else:
                updated = linear(dens, delta)
        elif cfg.acceleration == "oda":
            Sn, Hn, _ = fock(Pn)
            E_new = hf_energy(Pn, h=h, Sigma=Sn, H=Hn, weights_b=weights_b)
            c1 = float(np.sum(w2d * np.real(np.einsum("...ij,...ji->...", F, delta))))
            c2 = (E_new - E) - c1
            if c2 > 1e-12:
                lam = float(np.clip(-c1 / (2.0 * c2), 0.0, 1.0))
            else:
                lam = 1.0 if c1 < 0.0 else 0.0
            updated = herm(np.asarray(project(dens + lam * delta), dtype=h.dtype))
        else:
            updated = linear(dens, delta)
        step = updated - dens                                     # reference_scf.py:333-339
        sn = weighted_matrix_norm(step, w2d, ws)
        if cfg.trust_radius > 0.0 and sn > cfg.trust_radius:
            scale = cfg.trust_radius / max(sn, 1e-30)
            updated = herm(np.asarray(project(dens + scale * step), dtype=h.dtype))
        dens = Pn if converged else updated
        hE[k], hD[k], hC[k] = E, d_res, c_res
        k += 1
    _, F_fin, E_fin, mu_fin = build_and_occupy(dens)
    return dict(density_matrix=dens, fock_matrix=F_fin, energy=E_fin, chemical_potential=mu_fin,
                iterations=k, converged=bool(converged),
                history=dict(E=hE[:k], density_residual=hD[:k], commutator_residual=hC[:k]))


# ------------------------------------------------------------ gradients ---
# Partial derivatives of the objective at fixed density: what jax.grad of the
# reference returns for build_fock + hf_energy (fock.py:18-111) with the density
# held fixed; at a converged stationary point they are the total derivatives of
# the converged free energy (envelope theorem).

def coupling_gradient(kernel, P, dV):
    """1/2 sum_k w_k Re tr(Sigma_{dV}[P - refP] P): d hf_energy / d theta for V -> V + theta dV."""
    w = np.asarray(kernel.w2d, np.float64)
    VR = _fftn(w[..., None, None] * np.asarray(dV, np.complex128)) * shift_phase(P.shape[0], P.shape[1])
    dP = P - kernel.refP
    Sd = _selfenergy_fft_full(VR, dP)
    return float(0.5 * np.sum(w[..., None, None] * np.real(Sd * np.swapaxes(P, -1, -2))))


def fourier_coefficient_gradient(P, w2d, R):
    """sum_k w_k exp(-i k.R) P_k on the centred k grid: d E / d h_R for an independent h_R."""
    nk1, nk2 = P.shape[0], P.shape[1]
    k1 = 2.0 * np.pi * (np.arange(nk1) - nk1 // 2) / nk1
    k2 = 2.0 * np.pi * (np.arange(nk2) - nk2 // 2) / nk2
    K1, K2 = np.meshgrid(k1, k2, indexing="ij")
    w = np.asarray(w2d, np.float64)
    return np.stack([np.einsum("ij,ijab->ab", w * np.exp(-1j * (K1 * Rx + K2 * Ry)), P) for (Rx, Ry) in R])


# ---------------------------------------------------------------- continuation ----
def _resample_axis_periodic_linear(x, n_new, axis):
    """utils.py:477-509: periodic linear interpolation along one axis of a centered grid
    (k = 0 at index n // 2); positions and weights in the array's real precision."""
    x = np.asarray(x)
    n_old, n_new = int(x.shape[axis]), int(n_new)
    if n_new <= 0:
        raise ValueError("n_new must be a positive integer.")
    if n_old == n_new:
        return x
    rd = x.real.dtype
    j = np.arange(n_new, dtype=rd)
    u = (j - rd.type(n_new // 2)) * (rd.type(n_old) / rd.type(n_new)) + rd.type(n_old // 2)
    fl = np.floor(u)
    i0 = np.mod(fl.astype(np.int64), n_old)
    i1 = np.mod(i0 + 1, n_old)
    shape = [1] * x.ndim
    shape[axis] = n_new
    frac = (u - fl).reshape(shape).astype(rd)
    x0, x1 = np.take(x, i0, axis=axis), np.take(x, i1, axis=axis)
    return ((rd.type(1) - frac) * x0 + frac * x1).astype(x.dtype)


def resample_kgrid(values, nk, *, method="linear"):
    """utils.py:512-535: resample the two leading (centered, periodic) k axes to nk x nk."""
    nk = int(nk)
    x = np.asarray(values)
    if x.ndim < 2:
        raise ValueError("resample_kgrid expects an array with at least 2 dimensions (nk,nk,...).")
    if x.shape[0] == nk and x.shape[1] == nk:
        return x
    if str(method).lower() != "linear":
        raise ValueError(f"Unsupported resample method {method!r}. Only 'linear' is supported.")
    return _resample_axis_periodic_linear(_resample_axis_periodic_linear(x, nk, 0), nk, 1)


def resample_density(P, nk):
    """continuation.py:47-50: resampled density, hermitised."""
    Q = resample_kgrid(P, nk)
    return 0.5 * (Q + np.conj(np.swapaxes(Q, -1, -2)))


# ------------------------------------------------------------------ symmetry ----
def _flip_k(A, k_convention, flip_axes=(0, 1)):
    """symmetry.py:22-44."""
    if k_convention == "flip":
        return np.flip(A, axis=tuple(flip_axes))
    if k_convention == "mod":
        n1, n2 = A.shape[0], A.shape[1]
        i = (-np.arange(n1)) % n1 if 0 in flip_axes else np.arange(n1)
        j = (-np.arange(n2)) % n2 if 1 in flip_axes else np.arange(n2)
        return A[i[:, None], j[None, :], ...]
    raise ValueError(f"k_convention must be 'mod' or 'flip', got {k_convention!r}")


def _sum_conj(A, G):
    """symmetry.py:47-56: sum_i g_i A g_i^H."""
    acc = np.zeros_like(A)
    for g in G:
        acc = acc + (g @ A) @ np.conj(g.T)
    return acc


def make_project_fn(*, unitary_group=None, spatial_group=None, spatial_k_convention="mod",
                    spatial_k_flip_axes=(0, 1), spatial_k_index_maps=None, spatial_k_orbit_mask=None,
                    time_reversal_U=None, time_reversal_k_convention="mod", time_reversal_k_flip_axes=(0, 1),
                    time_reversal_k_index_map=None):
    """symmetry.py:153-281, NumPy restatement (same composition order and checks)."""
    G = None if unitary_group is None else np.asarray(unitary_group)
    S = None if spatial_group is None else np.asarray(spatial_group)
    U = None if time_reversal_U is None else np.asarray(time_reversal_U)
    if G is None and S is None and spatial_k_index_maps is None and U is None:
        return lambda A: A
    if spatial_k_index_maps is not None:
        si, sj = (np.asarray(m, dtype=np.int64) for m in spatial_k_index_maps)
        if si.shape != sj.shape:
            raise ValueError("spatial_k_index_maps[0] and [1] must have the same shape; "
                             f"got {si.shape} vs {sj.shape}.")
        if S is None:
            raise ValueError("spatial_k_index_maps requires spatial_group (the orbital unitaries to average over).")
        if S.shape[0] != si.shape[0]:
            raise ValueError("spatial_group and spatial_k_index_maps must have matching "
                             f"leading dim; got {S.shape[0]} and {si.shape[0]}.")
    else:
        si = sj = None
    omask = None if spatial_k_orbit_mask is None else np.asarray(spatial_k_orbit_mask, dtype=bool)
    if time_reversal_k_index_map is not None:
        if U is None:
            raise ValueError("time_reversal_k_index_map requires time_reversal_U.")
        ti, tj = (np.asarray(m, dtype=np.int64) for m in time_reversal_k_index_map[:2])
        tv = np.asarray(time_reversal_k_index_map[2], dtype=bool)
    else:
        ti = tj = tv = None
    sconv, saxes = str(spatial_k_convention), tuple(spatial_k_flip_axes)
    tconv, taxes = str(time_reversal_k_convention), tuple(time_reversal_k_flip_axes)

    def project(A):
        out = np.asarray(A)
        if si is not None:
            acc = np.zeros_like(out)
            for g in range(S.shape[0]):
                acc = acc + (S[g] @ out[si[g], sj[g]]) @ np.conj(S[g].T)
            avg = acc / S.shape[0]
            out = np.where(omask[..., None, None], avg, out) if omask is not None else avg
            if G is not None:
                out = _sum_conj(out, G) / G.shape[0]
        elif G is not None and S is not None:
            out = (_sum_conj(out, G) + _sum_conj(_flip_k(out, sconv, saxes), S)) / (G.shape[0] + S.shape[0])
        elif G is not None:
            out = _sum_conj(out, G) / G.shape[0]
        elif S is not None:
            eye = np.eye(S.shape[-1], dtype=S.dtype)[None]
            out = (_sum_conj(out, eye) + _sum_conj(_flip_k(out, sconv, saxes), S)) / (1 + S.shape[0])
        if U is not None:
            UH = np.conj(U.T)
            if ti is not None:
                Atr = U @ np.conj(out[ti, tj]) @ UH
                out = np.where(tv[..., None, None], 0.5 * (out + Atr), out)
            else:
                out = 0.5 * (out + U @ np.conj(_flip_k(out, tconv, taxes)) @ UH)
        return out

    return project


# -------------------------------------------------------------- superlattice ----
def sl_build_extended_layout(g_frac, B, nkx, nky, coulomb_V, w_scalar):
    """superlattice.py:72-164 restated with explicit loops; returns a dict of the tables."""
    g = np.asarray(g_frac, dtype=np.int64)
    nG = g.shape[0]
    pg = -g
    gx0, gx1, gy0, gy1 = pg[:, 0].min(), pg[:, 0].max(), pg[:, 1].min(), pg[:, 1].max()
    Nx, Ny = 2 * nkx * (gx1 - gx0 + 1), 2 * nky * (gy1 - gy0 + 1)
    off = np.stack([pg[:, 0] - gx0, pg[:, 1] - gy0], axis=1)
    dset, p2d = {}, np.empty((nG, nG), dtype=np.int64)
    for i in range(nG):
        for j in range(nG):
            key = (int(g[i, 0] - g[j, 0]), int(g[i, 1] - g[j, 1]))
            if key not in dset:
                dset[key] = len(dset)
            p2d[i, j] = dset[key]
    nd = len(dset)
    cnt = np.zeros(nd, dtype=np.int64)
    for i in range(nG):
        for j in range(nG):
            cnt[p2d[i, j]] += 1
    start = np.zeros(nd + 1, dtype=np.int64)
    start[1:] = np.cumsum(cnt)
    pi, pj, cur = np.empty(start[-1], np.int64), np.empty(start[-1], np.int64), start.copy()
    for i in range(nG):
        for j in range(nG):
            d = p2d[i, j]
            pi[cur[d]], pj[cur[d]] = i, j
            cur[d] += 1
    ix, iy = np.arange(Nx), np.arange(Ny)
    fx, fy = np.meshgrid(np.where(ix < Nx // 2, ix, ix - Nx) / float(nkx), np.where(iy < Ny // 2, iy, iy - Ny) / float(nky),
                         indexing="ij")
    B = np.asarray(B, dtype=float)
    q = np.sqrt((B[0, 0] * fx + B[0, 1] * fy) ** 2 + (B[1, 0] * fx + B[1, 1] * fy) ** 2)
    V = np.fft.fftn(float(w_scalar) * np.asarray(coulomb_V(q), dtype=float), axes=(0, 1))
    return dict(N_ext_x=Nx, N_ext_y=Ny, g_a_off=off, n_delta=nd, pair_to_delta=p2d, delta_pair_i=pi,
                delta_pair_j=pj, delta_pair_start=start, V_lag_fft=V)


def sl_streaming_fock(rho, L, nG, dorb, nkx, nky):
    """superlattice.py:202-229: per DG channel scatter, -IFFT2(FFT2 * V_lag_fft), gather."""
    rr = np.asarray(rho).reshape(nkx, nky, nG, dorb, nG, dorb)
    sig = np.empty_like(rr)
    for d in range(L["n_delta"]):
        buf = np.zeros((L["N_ext_x"], L["N_ext_y"], dorb, dorb), dtype=complex)
        ks = range(L["delta_pair_start"][d], L["delta_pair_start"][d + 1])
        for k in ks:
            i, j = L["delta_pair_i"][k], L["delta_pair_j"][k]
            ox, oy = nkx * L["g_a_off"][i, 0], nky * L["g_a_off"][i, 1]
            buf[ox:ox + nkx, oy:oy + nky] = rr[:, :, i, :, j, :]
        s = -np.fft.ifftn(np.fft.fftn(buf, axes=(0, 1)) * L["V_lag_fft"][:, :, None, None], axes=(0, 1))
        for k in ks:
            i, j = L["delta_pair_i"][k], L["delta_pair_j"][k]
            ox, oy = nkx * L["g_a_off"][i, 0], nky * L["g_a_off"][i, 1]
            sig[:, :, i, :, j, :] = s[ox:ox + nkx, oy:oy + nky]
    return sig.reshape(nkx, nky, nG * dorb, nG * dorb)
