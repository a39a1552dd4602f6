"""Pins the CPU oracle to the reference's golden vectors and known answers (CPU only)."""

from pathlib import Path

import numpy as np
import pytest

from oracle import hf_oracle as O

GOLD = Path(__file__).with_name("golden") / "meshgrid_v1.npz"


def _golden_kernel():
    d = np.load(GOLD)
    K = O.Kernel(d["weights"], d["hamiltonian"], d["coulomb_q"], float(d["T"]), include_hartree=True,
                 include_exchange=True, reference_density=d["reference_density"],
                 hartree_matrix=d["hartree_matrix"])
    return d, K


def test_golden_fock_and_energy():
    """tests/data/meshgrid_regression_case_v1.npz: F and E at the converged density."""
    d, K = _golden_kernel()
    a = K.as_args()
    P = d["P_expected"].astype(np.complex128)
    S, H, F = O.build_fock(P, h=a["h"], VR=a["VR"], refP=a["refP"], HH=a["HH"], w2d=K.w2d,
                           include_exchange=True, include_hartree=True,
                           exchange_hermitian_channel_packing=a["exchange_hermitian_channel_packing"],
                           contact_g=a["contact_g"], contact_Oi=a["contact_Oi"], contact_Oj=a["contact_Oj"])
    E = O.hf_energy(P, h=a["h"], Sigma=S, H=H, weights_b=a["weights_b"])
    assert np.abs(F - d["F_expected"]).max() < 2e-7   # complex64 fixture
    assert abs(E - float(d["E_expected"])) < 1e-6
    # the fixture density is self-consistent: P = density_from_fock(F[P]), mu matches
    P2, mu = O.density_from_fock(F, weights=K.w2d, n_electrons=float(d["electrondensity0"]),
                                 temperature=float(d["T"]), level_shift=0.0)
    assert abs(mu - float(d["mu_expected"])) < 1e-6
    assert np.abs(P2 - P).max() < 5e-6


def test_golden_needs_shift_phase():
    """Without the absorbed ifftshift phase the golden F is missed by ~1e-2 (convention check)."""
    d, K = _golden_kernel()
    a = K.as_args()
    P = d["P_expected"].astype(np.complex128)
    S, H, F = O.build_fock(P, h=a["h"], VR=K.VR, refP=a["refP"], HH=a["HH"], w2d=K.w2d,
                           include_exchange=True, include_hartree=True,
                           exchange_hermitian_channel_packing=True)
    assert np.abs(F - d["F_expected"]).max() > 1e-3


def test_single_k_identity():
    """tests/test_main.py:35-41: on a 1x1 mesh Sigma = -VR P."""
    VR = np.array([[[[0.3]]]], dtype=np.complex128)
    P = np.array([[[[1.0 + 0.5j, 0.2], [0.2, 0.8 - 0.1j]]]])
    S = O.selfenergy_fft(VR, P)
    np.testing.assert_allclose(S, -VR * P, atol=1e-15)


def test_packing_matches_full():
    """tests/test_linalg.py:77-98: packed == full for scalar real V and Hermitian P."""
    rng = np.random.default_rng(123)
    nk, nb = 8, 6
    raw = rng.normal(size=(nk, nk, nb, nb)) + 1j * rng.normal(size=(nk, nk, nb, nb))
    P = 0.5 * (raw + np.conj(np.swapaxes(raw, -1, -2)))
    VR = np.fft.fftn(rng.normal(size=(nk, nk, 1, 1)).astype(np.complex128), axes=(0, 1))
    np.testing.assert_allclose(O.selfenergy_fft(VR, P, hermitian_channel_packing=True),
                               O.selfenergy_fft(VR, P), atol=1e-12)


def test_block_specs_fallback_and_forced():
    """tests/test_linalg.py:140-174: coupled P falls back to full; forced block path differs."""
    nk, n0 = 4, 2
    nb = 2 * n0
    P = np.zeros((nk, nk, nb, nb), complex)
    P[:, :, 0, 0] = 1.0
    P[:, :, 2, 2] = 0.5
    P[:, :, 0, 2] = 0.1
    P[:, :, 2, 0] = 0.1
    VR = np.ones((nk, nk, 1, 1), complex)
    full = O.selfenergy_fft(VR, P)
    auto = O.selfenergy_fft(VR, P, block_specs=[{"block_sizes": [n0, n0]}], check_offdiag=True,
                            offdiag_atol=1e-6)
    np.testing.assert_allclose(auto, full, atol=1e-12)
    forced = O.selfenergy_fft(VR, P, block_specs=[{"block_sizes": [n0, n0]}], check_offdiag=False)
    assert np.abs(forced - full).max() > 1e-3


@pytest.mark.parametrize("method", ["bisection", "newton"])
def test_mu_hits_target(method):
    """tests/test_main.py:44-57."""
    rng = np.random.RandomState(42)
    bands = rng.randn(4, 4, 6)
    w = np.ones((4, 4)) / 16
    mu = O.find_chemical_potential(bands, w, 3.0, 0.05, method=method)
    assert abs(np.sum(w[..., None] * O.fermidirac(bands - mu, 0.05)) - 3.0) < 1e-4


def test_mu_cold_limit_and_unreachable():
    """tests/test_main.py:9-32,60-84."""
    bands = np.array([[[0.0, 1.0, 2.0]]])
    w = np.ones((1, 1))
    mu = O.find_chemical_potential(bands, w, 2.0, 1e-5)
    assert abs(np.sum(O.fermidirac(bands - mu, 1e-5)) - 2.0) < 1e-4
    with pytest.raises(ValueError, match="physically reachable range"):
        O.find_chemical_potential(np.array([[[0.0]]]), w, 2.0, 0.1)


def _skew(rng, shape):
    d = rng.normal(size=shape) + 1j * rng.normal(size=shape)
    return 0.5 * (d - np.conj(np.swapaxes(d, -1, -2)))


def test_cayley_spectral_matches_lu():
    """tests/test_solver.py:385-459."""
    rng = np.random.default_rng(0)
    d = _skew(rng, (3, 3, 6, 6))
    F = rng.normal(size=(3, 3, 6, 6)) + 1j * rng.normal(size=(3, 3, 6, 6))
    F = 0.5 * (F + np.conj(np.swapaxes(F, -1, -2)))
    V, lam = O.cayley_spectral_setup(d)
    Fe = np.conj(np.swapaxes(V, -2, -1)) @ F @ V
    for tau in [0.0, 0.1, 0.5, 1.0, -0.3]:
        U_lu = O.cayley_retract(d, tau)
        U_sp = O.cayley_unitary_from_spectrum(V, lam, tau)
        np.testing.assert_allclose(U_sp, U_lu, atol=1e-12)
        dg = O.diag_UFU_from_spectrum(V, Fe, lam, tau)
        np.testing.assert_allclose(dg, np.real(np.diagonal(np.conj(np.swapaxes(U_lu, -2, -1)) @ F @ U_lu,
                                                           axis1=-2, axis2=-1)), atol=1e-12)


def _bistable(nk=1, T=0.02, ex=1.0, delta=0.1):
    h = np.zeros((nk, nk, 2, 2), complex)
    h[..., 0, 0] = -delta
    h[..., 1, 1] = delta
    return O.Kernel(np.ones((nk, nk)), h, np.full((nk, nk, 1, 1), ex, complex), T)


def test_bistable_ground_state_energy():
    """tests/test_deflation.py:50-62,180-182: cold start lands on the E = -0.6 ground state."""
    K = _bistable()
    r = O.solve(K, np.zeros_like(K.h), 1.0, config=O.SolverConfig(optimizer="newton", tol_grad=1e-8,
                                                                    max_iter=100))
    assert abs(r["energy"] - (-0.6)) < 2e-2
    r2 = O.solve(K, np.zeros_like(K.h), 1.0, config=O.SolverConfig(max_iter=200, tol_E=1e-10))
    assert abs(r2["energy"] - (-0.6)) < 2e-2


def _dirac(nk=4, m=0.3, v=1.0, T=0.1, ex=0.7):
    ks = (np.arange(nk) - nk // 2) * (2 * np.pi / nk)
    KX, KY = np.meshgrid(ks, ks, indexing="ij")
    h = np.zeros((nk, nk, 2, 2), complex)
    h[..., 0, 0] = m
    h[..., 1, 1] = -m
    h[..., 0, 1] = v * (KX - 1j * KY)
    h[..., 1, 0] = v * (KX + 1j * KY)
    return O.Kernel(np.ones((nk, nk)), h, np.full((nk, nk, 1, 1), ex, complex), T)


def test_scf_schemes_agree_and_diis_faster():
    """tests/test_scf_acceleration.py:42-75."""
    K = _dirac()
    P0 = np.zeros_like(K.h)
    cfg = dict(max_iter=800, density_tol=1e-6, comm_tol=1e-5, mixing=0.5)
    res = {acc: O.solve_scf(K, P0, 16.0, config=O.SCFConfig(acceleration=acc, **cfg))
           for acc in ("linear", "diis", "oda")}
    E = [r["energy"] for r in res.values()]
    assert max(E) - min(E) < 1e-3
    assert res["linear"]["converged"] and res["diis"]["converged"]
    assert res["diis"]["iterations"] < res["linear"]["iterations"] // 3


def test_cg_and_scf_agree_on_two_band():
    """tests/test_solver.py (two-band model): DM and SCF reach the same self-consistent energy."""
    h = np.zeros((2, 2, 2, 2), complex)
    h[..., 0, 0] = -0.5
    h[..., 1, 1] = 0.5
    K = O.Kernel(np.ones((2, 2)), h, np.full((2, 2, 1, 1), 0.25, complex), 0.1)
    r = O.solve(K, np.zeros_like(K.h), 4.0, config=O.SolverConfig(max_iter=100, tol_E=1e-10))
    s = O.solve_scf(K, np.zeros_like(K.h), 4.0, config=O.SCFConfig(max_iter=300, acceleration="diis"))
    assert r["converged"] and s["converged"]
    assert abs(r["energy"] - s["energy"]) < 1e-6


def test_newton_hvp_matches_finite_difference():
    """tests/test_solver_newton.py:120-196 restated on the oracle (expm retraction, steps 1e-5/1e-6)."""
    from scipy.linalg import expm
    rng = np.random.default_rng(4)
    nk, nb, T, ex = 5, 5, 0.05, 0.4
    diag = np.linspace(-1.0, 1.0, nb)
    A = (rng.standard_normal((nb, nb)) + 1j * rng.standard_normal((nb, nb))) * 0.35
    A = 0.5 * (A + A.conj().T)
    h = np.zeros((nk, nk, nb, nb), complex)
    kx = np.arange(nk) / nk * 2 * np.pi
    for i in range(nk):
        for j in range(nk):
            hk = np.diag(diag) + A * (np.cos(kx[i]) + np.cos(kx[j]))
            h[i, j] = 0.5 * (hk + hk.conj().T)
    K = O.Kernel(np.ones((nk, nk)), h, np.full((nk, nk, 1, 1), ex, complex), T)
    a = K.as_args()
    w2 = K.w2d
    eye = np.eye(nb)
    off = 1.0 - eye

    def Fock(P):
        return O.build_fock(P, h=h, VR=a["VR"], refP=np.zeros_like(h), HH=a["HH"], w2d=w2,
                            include_exchange=True, include_hartree=False,
                            exchange_hermitian_channel_packing=True)[2]

    proj = lambda dp: dp - np.sum(w2[..., None] * dp) / (np.sum(w2) * nb)
    expm_b = lambda X: np.array([[expm(X[i, j]) for j in range(nk)] for i in range(nk)])
    rng2 = np.random.default_rng(1)
    eps, Q = np.linalg.eigh(Fock(np.zeros_like(h)))
    X0 = O.skew_hermitian(rng2.standard_normal(Q.shape) + 1j * rng2.standard_normal(Q.shape)) * off
    Q = Q @ expm_b(0.2 * X0)
    mu = float(np.median(eps))
    p = np.clip(O.sigmoid((mu - eps) / T), 0.05, 0.95)

    def grad(Q, p):
        Ft = O.fock_in_orbital_basis(Q, Fock(O.density_from_Qp(Q, p)))
        dpm = p[..., None, :] - p[..., :, None]
        G = O.skew_hermitian(dpm * Ft) * off
        gp = np.real(np.diagonal(Ft, axis1=-2, axis2=-1)) + T * np.log(p / (1 - p)) - mu
        return G, gp, Ft

    G0, gp0, Ft = grad(Q, p)
    X = O.skew_hermitian(rng2.standard_normal(Q.shape) + 1j * rng2.standard_normal(Q.shape)) * off
    dp = rng2.standard_normal(p.shape) * 0.1
    dpm = p[..., None, :] - p[..., :, None]
    M = X * dpm + dp[..., :, None] * eye
    dP = O.herm(np.einsum("...in,...nm,...jm->...ij", Q, M, np.conj(Q)))
    St = O.fock_in_orbital_basis(Q, Fock(dP) - h)
    Am = Ft @ X - X @ Ft + St
    C = (dp[..., None, :] - dp[..., :, None]) * Ft + dpm * Am
    HX = O.skew_hermitian(C) * off
    pc = np.clip(p, 1e-8, 1 - 1e-8)
    Hp = proj(np.real(np.diagonal(Am, axis1=-2, axis2=-1)) + T / (pc * (1 - pc)) * dp)
    errs = []
    for e in (1e-5, 1e-6):
        Ge, gpe, _ = grad(Q @ expm_b(e * X), p + e * dp)
        errs.append((np.abs((Ge - G0) / e - HX).max() / np.abs(HX).max(),
                     np.abs(proj((gpe - gp0) / e) - Hp).max() / np.abs(Hp).max()))
    assert errs[1][0] < 1e-4 and errs[1][1] < 1e-4
    assert errs[1][0] < 0.2 * errs[0][0] + 1e-12


def test_oracle_symmetry_projector_properties():
    """Restatement of make_project_fn (symmetry.py:153-281) on the reference's property tests."""
    rng = np.random.default_rng(4)
    A = rng.standard_normal((4, 4, 4, 4)) + 1j * rng.standard_normal((4, 4, 4, 4))
    G = np.stack([np.eye(4), np.diag([1, 1, -1, -1]).astype(complex)])
    p = O.make_project_fn(unitary_group=G)
    B = p(A)
    for g in G:
        np.testing.assert_allclose(g @ B @ np.conj(g.T), B, atol=1e-14)
    np.testing.assert_allclose(p(B), B, atol=1e-14)
    U = np.array([[0, -1j], [1j, 0]])
    A2 = A[..., :2, :2]
    for conv in ("flip", "mod"):
        q = O.make_project_fn(time_reversal_U=U, time_reversal_k_convention=conv)
        C = q(A2)
        Cneg = O._flip_k(C, conv)
        np.testing.assert_allclose(U @ np.conj(Cneg) @ np.conj(U.T), C, atol=1e-14)
    assert O.make_project_fn()(A) is A
