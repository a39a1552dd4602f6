"""GPU parity: CUDA Fock build / objective / per-k kernels against the CPU oracle.

Tolerances (relative to max|oracle|): complex128 1e-12 (plain FP64 target);
complex64 and the FP32-exchange mode 2e-5 (FP32 FFT round-off over <= 2*log2(N) stages).
"""

from pathlib import Path

import numpy as np
import pytest
import torch

from oracle import hf_oracle as O
from jax_hf_b200 import synthetic as S

pytestmark = pytest.mark.gpu

GOLD = Path(__file__).with_name("golden") / "meshgrid_v1.npz"
TOL64, TOL32 = 1e-12, 2e-5


def rel(a, b):
    a = a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
    b = np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _pair(prob, dtype=np.complex128, **kw):
    import jax_hf_b200 as G
    K = G.HartreeFockKernel(prob.weights, prob.hamiltonian.astype(dtype), prob.coulomb_q, prob.T, **kw)
    Ko = O.Kernel(prob.weights, prob.hamiltonian.astype(dtype), prob.coulomb_q, prob.T, **kw)
    return K, Ko


def _fock_both(K, Ko, P, **kw):
    import jax_hf_b200 as G
    a, ao = K.as_args(), Ko.as_args()
    Sg, H, F = G.build_fock(torch.as_tensor(P, device="cuda"), h=a["h"], VR=a["VR"], refP=a["refP"],
                            HH=a["HH"], w2d=K.w2d, include_exchange=a["include_exchange"],
                            include_hartree=a["include_hartree"],
                            exchange_hermitian_channel_packing=a["exchange_hermitian_channel_packing"],
                            contact_g=a["contact_g"], contact_Oi=a["contact_Oi"], contact_Oj=a["contact_Oj"], **kw)
    So, Ho, Fo = O.build_fock(P.astype(np.complex128), h=ao["h"].astype(np.complex128), VR=ao["VR"],
                              refP=ao["refP"], HH=ao["HH"], w2d=Ko.w2d,
                              include_exchange=ao["include_exchange"], include_hartree=ao["include_hartree"],
                              exchange_hermitian_channel_packing=ao["exchange_hermitian_channel_packing"],
                              contact_g=ao["contact_g"], contact_Oi=ao["contact_Oi"], contact_Oj=ao["contact_Oj"])
    return (Sg, H, F), (So, Ho, Fo)


def test_golden_fixture(cuda):
    import jax_hf_b200 as G
    d = np.load(GOLD)
    kw = dict(include_hartree=True, include_exchange=True, reference_density=d["reference_density"].astype(np.complex128),
              hartree_matrix=d["hartree_matrix"])
    h = d["hamiltonian"].astype(np.complex128)
    K = G.HartreeFockKernel(d["weights"], h, d["coulomb_q"], float(d["T"]), **kw)
    Ko = O.Kernel(d["weights"], h, d["coulomb_q"], float(d["T"]), **kw)
    P = d["P_expected"].astype(np.complex128)
    (Sg, H, F), (So, Ho, Fo) = _fock_both(K, Ko, P)
    assert rel(F, Fo) < TOL64
    assert rel(Sg, So) < TOL64
    assert np.abs(F.cpu().numpy() - d["F_expected"]).max() < 2e-7
    np.testing.assert_allclose(H.cpu().numpy()[0, 0], Ho[0, 0], atol=1e-14)
    E = G.hf_energy(torch.as_tensor(P, device="cuda"), h=K.h, Sigma=Sg, H=H, weights_b=K.weights_b)
    Eo = O.hf_energy(P, h=Ko.h, Sigma=So, H=Ho, weights_b=Ko.weights_b)
    assert abs(float(E) - Eo) <= 1e-12 * abs(Eo)
    assert abs(float(E) - float(d["E_expected"])) < 1e-6


def test_single_k_identity(cuda):
    """Sigma = -VR P on a 1x1 mesh (tests/test_main.py:35-41)."""
    import jax_hf_b200 as G
    P = np.array([[[[1.0 + 0.5j, 0.2], [0.2, 0.8 - 0.1j]]]])
    h = np.zeros_like(P)
    K = G.HartreeFockKernel(np.ones((1, 1)), h, np.full((1, 1, 1, 1), 0.3), 0.1)
    a = K.as_args()
    Sg, _, _ = G.build_fock(torch.as_tensor(P, device="cuda"), h=a["h"], VR=a["VR"], refP=a["refP"], HH=a["HH"],
                            w2d=K.w2d, include_exchange=True, include_hartree=False,
                            exchange_hermitian_channel_packing=False)
    np.testing.assert_allclose(Sg.cpu().numpy(), -0.3 * P, atol=1e-15)


CASES = [
    # nk1, nk2, nb, V, hartree/refP, contact
    (1, 1, 2, "scalar", False, False),
    (2, 3, 1, "scalar", False, False),
    (5, 7, 3, "layer", False, False),
    (12, 12, 4, "scalar", True, False),
    (24, 24, 4, "scalar", False, False),
    (36, 36, 6, "layer", False, True),
    (48, 40, 8, "layer", True, True),
    (7, 11, 5, "scalar", True, True),
    (16, 9, 8, "layer", False, False),
    (96, 96, 4, "scalar", False, False),
    (13, 26, 3, "layer", True, False),
    # band counts above the rows plan (tile slot groups / generic engine), up to the
    # largest supported nb = 32
    (10, 12, 9, "layer", True, False),
    (12, 8, 12, "scalar", False, True),
    (9, 6, 16, "layer", False, False),
    (4, 6, 32, "layer", True, False),
]


def _problem(nk1, nk2, nb, V, seed):
    rng = np.random.default_rng(seed)
    nkm = max(nk1, nk2)
    prob = S.fourier_problem(nkm, nb, 2.0, seed, V=V)
    h = prob.hamiltonian[:nk1, :nk2]
    Vq = prob.coulomb_q[:nk1, :nk2] if V == "scalar" else prob.coulomb_q[:nk1, :nk2]
    w = rng.uniform(0.5, 1.5, size=(nk1, nk2))
    w = w / w.sum()
    P = S.haar_density(nkm, nb, seed + 7)[:nk1, :nk2]
    return S.Problem("t", w, np.ascontiguousarray(h), np.ascontiguousarray(Vq), 0.1, 1.0, nkm, nb), P, rng


@pytest.mark.parametrize("nk1,nk2,nb,V,hartree,contact", CASES)
def test_fock_matches_oracle(cuda, nk1, nk2, nb, V, hartree, contact):
    prob, P, rng = _problem(nk1, nk2, nb, V, 11 + nk1 + 3 * nb)
    kw = {}
    if hartree:
        ref = S.haar_density(max(nk1, nk2), nb, 99)[:nk1, :nk2] * 0.5
        HH = rng.normal(size=(nb, nb))
        kw.update(include_hartree=True, reference_density=np.ascontiguousarray(ref), hartree_matrix=HH + HH.T)
    if contact:
        Oa = rng.normal(size=(nb, nb)) + 1j * rng.normal(size=(nb, nb))
        Ob = rng.normal(size=(nb, nb)) + 1j * rng.normal(size=(nb, nb))
        kw.update(contact_terms=[(0.3, Oa, Oa.conj().T), (-0.2, Ob, Ob)])
    K, Ko = _pair(prob, **kw)
    (Sg, H, F), (So, Ho, Fo) = _fock_both(K, Ko, P)
    assert rel(Sg, So) < TOL64, "Sigma"
    assert rel(F, Fo) < TOL64, "F"
    # F is exactly Hermitian
    Fn = F.cpu().numpy()
    assert np.abs(Fn - np.conj(np.swapaxes(Fn, -1, -2))).max() == 0.0


def test_fock_non_hermitian_input_full_channels(cuda):
    """Layer-resolved V computes all nb^2 channels: Sigma matches the reference for any P."""
    prob, P, rng = _problem(12, 10, 4, "layer", 5)
    P = P + 0.3 * (rng.normal(size=P.shape) + 1j * rng.normal(size=P.shape))
    K, Ko = _pair(prob)
    (Sg, H, F), (So, Ho, Fo) = _fock_both(K, Ko, P)
    assert rel(Sg, So) < TOL64 and rel(F, Fo) < TOL64


@pytest.mark.parametrize("mode", ["c64", "fp32fft"])
def test_fock_single_precision(cuda, mode):
    prob, P, _ = _problem(48, 48, 8, "layer", 3)
    if mode == "c64":
        K, Ko = _pair(prob, dtype=np.complex64)
        (Sg, H, F), (So, Ho, Fo) = _fock_both(K, Ko, P.astype(np.complex64))
    else:
        K, Ko = _pair(prob)
        (Sg, H, F), (So, Ho, Fo) = _fock_both(K, Ko, P, fft_precision="fp32")
        assert F.dtype == torch.complex128
    assert rel(Sg, So) < TOL32
    assert rel(F, Fo) < TOL32


def test_fock_full_size_192(cuda):
    """192x192, nb=8 layer-resolved V, Haar density: FP64 vs oracle at the benchmark size."""
    prob, P = S.fock_build_192()
    K, Ko = _pair(prob)
    (Sg, H, F), (So, Ho, Fo) = _fock_both(K, Ko, P)
    assert rel(Sg, So) < TOL64
    assert rel(F, Fo) < TOL64
    # size-independent properties: linearity of the exchange in P
    import jax_hf_b200 as G
    a = K.as_args()
    Pt = torch.as_tensor(P, device="cuda")
    kw = dict(h=a["h"], VR=a["VR"], refP=a["refP"], HH=a["HH"], w2d=K.w2d, include_exchange=True,
              include_hartree=False, exchange_hermitian_channel_packing=False)
    S2, _, _ = G.build_fock(2.0 * Pt, **kw)
    assert rel(S2, 2.0 * Sg.cpu().numpy()) < 1e-14


def test_energy_entropy_free_energy(cuda):
    import jax_hf_b200 as G
    prob, P, rng = _problem(24, 20, 6, "layer", 9)
    K, Ko = _pair(prob)
    (Sg, H, F), (So, Ho, Fo) = _fock_both(K, Ko, P)
    E = G.hf_energy(torch.as_tensor(P, device="cuda"), h=K.h, Sigma=Sg, H=H, weights_b=K.weights_b)
    Eo = O.hf_energy(P, h=Ko.h, Sigma=So, H=Ho, weights_b=Ko.weights_b)
    assert abs(float(E) - Eo) <= 1e-12 * max(abs(Eo), 1.0)
    p = rng.uniform(0, 1, size=(24, 20, 6))
    p[0, 0, 0] = 0.0
    p[0, 0, 1] = 1.0
    wn = K.w2d.cpu().numpy()
    Sent = G.occupation_entropy(torch.as_tensor(p, device="cuda"), K.w2d)
    assert abs(float(Sent) - O.occupation_entropy(p, wn)) < 1e-13
    Om = G.free_energy(E, torch.as_tensor(p, device="cuda"), K.w2d, 0.05)
    assert abs(float(Om) - O.free_energy(Eo, p, wn, 0.05)) < 1e-12 * max(1.0, abs(Eo))


@pytest.mark.parametrize("method", ["bisection", "newton"])
@pytest.mark.parametrize("T", [0.1, 0.01, 1e-5])
def test_find_mu(cuda, method, T):
    import jax_hf_b200 as G
    rng = np.random.default_rng(42)
    bands = rng.standard_normal((36, 36, 6)) * 2
    w = np.full((36, 36), 1 / 36 ** 2)
    mu = float(G.find_chemical_potential(torch.as_tensor(bands, device="cuda"), torch.as_tensor(w, device="cuda"),
                                         2.7, T, method=method))
    muo = O.find_chemical_potential(bands, w, 2.7, T, method=method)
    cnt = np.sum(w[..., None] * O.fermidirac(bands - mu, T))
    assert abs(cnt - 2.7) < 1e-9
    assert abs(mu - muo) < 1e-9 * max(1.0, abs(muo)) or T < 1e-3


@pytest.mark.parametrize("shape,T,kind", [((24, 24, 4), 0.1, "metal"), ((36, 36, 6), 0.05, "metal"),
                                          ((16, 16, 4), 0.01, "gapped"), ((12, 12, 3), 0.0, "metal"),
                                          ((96, 96, 4), 0.1, "metal")])
def test_bisection_hint_keeps_the_result(cuda, shape, T, kind):
    """hf_find_mu method 0 with a hint (mu0) decides the levels outside a certified
    bracket without evaluations; the result must be bit-identical to evaluating every
    level, for good, poor and useless hints, metals and a gapped spectrum."""
    from jax_hf_b200 import _lib
    rng = np.random.default_rng(7)
    nk1, nk2, nb = shape
    if kind == "gapped":
        lower = rng.uniform(-4, -1, (nk1, nk2, nb // 2))
        bands = np.concatenate([lower, rng.uniform(1, 4, (nk1, nk2, nb - nb // 2))], axis=-1)
        ne = float(nb // 2)
    else:
        bands = rng.standard_normal(shape) * 2
        ne = 0.4 * nb
    eps = torch.as_tensor(bands, device="cuda")
    w = torch.full((nk1, nk2), 1.0 / (nk1 * nk2), device="cuda", dtype=torch.float64)
    out = torch.zeros(1, device="cuda", dtype=torch.float64)
    L = _lib.lib()
    st = _lib.stream_ptr(eps.device)

    def run(hint):
        h = None
        if hint is not None:
            h = torch.tensor([hint], device="cuda", dtype=torch.float64)
        _lib.check(L.hf_find_mu(st, 0, 0, nk1, nk2, nb, eps.data_ptr(), w.data_ptr(), ne, T, 0,
                                None if h is None else h.data_ptr(), out.data_ptr()))
        return float(out.item())

    ref = run(None)
    if kind == "metal" and T >= 1e-3:
        # inside a gap the count is flat to rounding, and where the bisection stops there
        # depends on the summation order: only a metal's mu is compared with the oracle
        muo = O.find_chemical_potential(bands, w.cpu().numpy(), ne, T, method="bisection")
        assert abs(ref - muo) < 1e-9 * max(1.0, abs(muo))
    for hint in (ref, ref + 1e-9, ref - 1e-3, ref + 0.3, 0.0, 1e6, -50.0, float("nan")):
        assert run(hint) == ref, hint
    # the hint may alias the output (the SCF driver passes its previous mu in place)
    out.fill_(ref + 1e-6)
    _lib.check(L.hf_find_mu(st, 0, 0, nk1, nk2, nb, eps.data_ptr(), w.data_ptr(), ne, T, 0,
                            out.data_ptr(), out.data_ptr()))
    assert float(out.item()) == ref


def test_solve_mu_warm_start(cuda):
    from jax_hf_b200.utils import solve_mu
    rng = np.random.default_rng(1)
    eps = rng.standard_normal((144, 144, 8))
    w = np.full((144, 144), 1 / 144 ** 2)
    for mu0, T in ((0.0, 0.05), (0.7, 0.1), (-5.0, 0.02)):
        mu = float(solve_mu(torch.as_tensor(eps, device="cuda"), torch.as_tensor(w, device="cuda"), 3.0, mu0, T))
        muo = O.solve_mu(eps, w, 3.0, mu0, T)
        assert abs(mu - muo) < 1e-13 * max(1, abs(muo))


def test_unreachable_count_raises(cuda):
    import jax_hf_b200 as G
    with pytest.raises(ValueError, match="physically reachable range"):
        G.find_chemical_potential(torch.zeros((1, 1, 1), device="cuda", dtype=torch.float64),
                                  torch.ones((1, 1), device="cuda", dtype=torch.float64), 2.0, 0.1)


def _herm_batch(rng, shape):
    A = rng.normal(size=shape) + 1j * rng.normal(size=shape)
    return 0.5 * (A + np.conj(np.swapaxes(A, -1, -2)))


@pytest.mark.parametrize("nb", [1, 2, 3, 4, 5, 6, 8, 12, 16])
def test_eigh(cuda, nb):
    from jax_hf_b200 import linalg as L
    rng = np.random.default_rng(nb)
    A = _herm_batch(rng, (7, 5, nb, nb))
    A[0, 0] = np.diag(np.arange(nb, dtype=float))       # already diagonal
    A[0, 1] = np.eye(nb)                                  # fully degenerate
    w, V = L.eigh(torch.as_tensor(A, device="cuda"))
    w, V = w.cpu().numpy(), V.cpu().numpy()
    wo = np.linalg.eigvalsh(A)
    assert np.abs(w - wo).max() < 1e-13 * max(1, np.abs(wo).max())
    rec = np.einsum("...in,...n,...jn->...ij", V, w, np.conj(V))
    assert np.abs(rec - A).max() < 1e-13 * max(1, np.abs(A).max())
    VhV = np.conj(np.swapaxes(V, -1, -2)) @ V
    assert np.abs(VhV - np.eye(nb)).max() < 1e-13


def test_perk_kernels(cuda):
    from jax_hf_b200 import linalg as L
    rng = np.random.default_rng(0)
    nb = 6
    d = rng.normal(size=(3, 4, nb, nb)) + 1j * rng.normal(size=(3, 4, nb, nb))
    d = 0.5 * (d - np.conj(np.swapaxes(d, -1, -2)))
    F = _herm_batch(rng, (3, 4, nb, nb))
    Q = S.haar_unitaries((3, 4), nb, rng)
    p = rng.uniform(0, 1, size=(3, 4, nb))
    t = lambda x: torch.as_tensor(x, device="cuda")
    assert rel(L.density_from_Qp(t(Q), t(p)), O.herm(O.density_from_Qp(Q, p))) < 1e-14
    assert rel(L.fock_in_orbital_basis(t(Q), t(F)), O.fock_in_orbital_basis(Q, F)) < 1e-14
    V, lam = L.cayley_spectral_setup(t(d))
    Vo, lamo = O.cayley_spectral_setup(d)
    assert np.abs(lam.cpu().numpy() - lamo).max() < 1e-13
    Fe = O.fock_in_orbital_basis(V.cpu().numpy(), F)
    for tau in (0.0, 0.3, -0.7, 1.0):
        U_lu = L.cayley_retract(t(d), tau)
        assert rel(U_lu, O.cayley_retract(d, tau)) < 1e-13
        U_sp = L.cayley_unitary_from_spectrum(V, lam, tau)
        assert rel(U_sp, O.cayley_retract(d, tau)) < 1e-12
        dg = L.diag_UFU_from_spectrum(V, t(Fe), lam, tau)
        U = O.cayley_retract(d, tau)
        ref = np.real(np.diagonal(np.conj(np.swapaxes(U, -1, -2)) @ F @ U, axis1=-2, axis2=-1))
        assert np.abs(dg.cpu().numpy() - ref).max() < 1e-12
        assert rel(L.qr_retract(t(d), tau), O.qr_retract(d, tau)) < 1e-12


FAST_N = [12, 16, 24, 32, 36, 48, 64, 72, 96, 128, 144, 192]


@pytest.mark.parametrize("n1,n2", [(n, n) for n in FAST_N] + [(24, 48), (192, 144), (12, 36)])
@pytest.mark.parametrize("nb,V", [(1, "scalar"), (3, "layer"), (4, "scalar"), (8, "layer")])
def test_fast_engine_matches_generic(cuda, n1, n2, nb, V):
    """Register-FFT passes of the specialised mesh lengths == generic Stockham engine."""
    import jax_hf_b200 as G
    if n1 * n2 * nb * nb > 192 * 192 * 16 and nb == 8 and (n1, n2) != (192, 192):
        pytest.skip("size covered by the 192 case")
    prob, P, rng = _problem(n1, n2, nb, V, 31 + n1 + nb)
    K = G.HartreeFockKernel(prob.weights, prob.hamiltonian, prob.coulomb_q, prob.T)
    a = K.as_args()
    Pt = torch.as_tensor(P, device="cuda")
    kw = dict(h=a["h"], VR=a["VR"], refP=a["refP"], HH=a["HH"], w2d=K.w2d, include_exchange=True,
              include_hartree=False, exchange_hermitian_channel_packing=a["exchange_hermitian_channel_packing"])
    Sf, _, Ff = G.build_fock(Pt, **kw)
    Sg, _, Fg = G.build_fock(Pt, engine="generic", **kw)
    assert rel(Sf, Sg.cpu().numpy()) < TOL64
    assert rel(Ff, Fg.cpu().numpy()) < TOL64
    Sm, _, Fm = G.build_fock(Pt, fft_precision="fp32", **kw)
    assert rel(Sm, Sg.cpu().numpy()) < TOL32
    St, _, Ft = G.build_fock(Pt, engine="tile", **kw)  # 2x2-tile slot groups instead of the rows plan
    assert rel(St, Sg.cpu().numpy()) < TOL64
    assert rel(Ft, Fg.cpu().numpy()) < TOL64


@pytest.mark.parametrize("n1,n2,nb,V,hartree", [(48, 48, 8, "layer", False), (36, 36, 6, "layer", True),
                                                (24, 24, 4, "scalar", False), (30, 30, 8, "layer", False)])
def test_autotune_picks_a_schedule_that_matches(cuda, n1, n2, nb, V, hartree):
    """hf_fock_autotune: every candidate timed, outputs equal the default build, choice reused."""
    import jax_hf_b200 as G
    from jax_hf_b200 import fock as Fk
    prob, P, rng = _problem(n1, n2, nb, V, 7 + n1 + nb)
    hk = dict(include_hartree=True, hartree_matrix=0.2 + 0.5 * np.eye(nb),
              reference_density=0.3 * P) if hartree else {}
    K = G.HartreeFockKernel(prob.weights, prob.hamiltonian, prob.coulomb_q, prob.T, **hk)
    a = K.as_args()
    Pt = torch.as_tensor(P, device="cuda")
    kw = dict(h=a["h"], VR=a["VR"], refP=a["refP"], HH=a["HH"], w2d=K.w2d, include_exchange=True,
              include_hartree=hartree, exchange_hermitian_channel_packing=a["exchange_hermitian_channel_packing"])
    Fk.autotune_reset()
    S0, H0, F0 = G.build_fock(Pt, **kw)
    try:
        S1, H1, F1 = G.build_fock(Pt, autotune=True, autotune_reps=2, **kw)
        info = dict(Fk.last_autotune)
        assert info["shape"] == (n1, n2, nb)
        assert info["chosen"] in info["us"] and all(v > 0 for v in info["us"].values())
        assert "generic" in info["us"] and "default" in info["us"]
        assert rel(S1, S0.cpu().numpy()) < TOL64 and rel(F1, F0.cpu().numpy()) < TOL64
        assert rel(H1, H0.cpu().numpy()) < TOL64
        S2, _, F2 = G.build_fock(Pt, **kw)  # the stored choice
        assert rel(S2, S0.cpu().numpy()) < TOL64 and rel(F2, F0.cpu().numpy()) < TOL64
    finally:
        Fk.autotune_reset()


SYM_CASES = [
    (48, 48, 8, False, False, None),
    (24, 36, 6, True, True, None),
    (20, 14, 5, False, False, None),          # generic engine lengths
    (48, 48, 8, False, False, "fp32"),
    (48, 48, 8, False, False, "c64"),
    (36, 36, 4, False, False, "generic"),
]


@pytest.mark.parametrize("nk1,nk2,nb,hartree,contact,mode", SYM_CASES)
def test_fock_hermitian_density_packing_band_resolved(cuda, nk1, nk2, nb, hartree, contact, mode):
    """hermitian_density=True with a real, pair-symmetric band-resolved V transforms only the
    upper-triangle channels; for a Hermitian density the result equals the full reference build."""
    prob, P, rng = _problem(nk1, nk2, nb, "layer", 17 + nk1 + nb)
    kw = {}
    if hartree:
        ref = S.haar_density(max(nk1, nk2), nb, 98)[:nk1, :nk2] * 0.5
        HH = rng.normal(size=(nb, nb))
        kw.update(include_hartree=True, reference_density=np.ascontiguousarray(ref), hartree_matrix=HH + HH.T)
    if contact:
        Oa = rng.normal(size=(nb, nb)) + 1j * rng.normal(size=(nb, nb))
        kw.update(contact_terms=[(0.3, Oa, Oa.conj().T)])
    dtype = np.complex64 if mode == "c64" else np.complex128
    K, Ko = _pair(prob, dtype=dtype, **kw)
    assert K.v_pair_symmetric
    extra = {"hermitian_density": True}
    if mode == "fp32":
        extra["fft_precision"] = "fp32"
    if mode == "generic":
        extra["engine"] = "generic"
    (Sg, H, F), (So, Ho, Fo) = _fock_both(K, Ko, P.astype(dtype), **extra)
    tol = TOL32 if mode in ("fp32", "c64") else TOL64
    assert rel(Sg, So) < tol, "Sigma"
    assert rel(F, Fo) < tol, "F"
    Fn = F.cpu().numpy()
    assert np.abs(Fn - np.conj(np.swapaxes(Fn, -1, -2))).max() == 0.0


def test_fock_hermitian_density_packing_192(cuda):
    """The benchmark workload (192x192, nb=8, layer V, Haar density) through the packed path."""
    prob, P = S.fock_build_192()
    K, Ko = _pair(prob)
    (Sg, H, F), (So, Ho, Fo) = _fock_both(K, Ko, P, hermitian_density=True)
    assert rel(Sg, So) < TOL64
    assert rel(F, Fo) < TOL64



@pytest.mark.parametrize("streams", [1, 2, 3])
def test_build_fock_batch_matches_single_calls(cuda, streams):
    """Independent builds spread over internal streams (each with its own scratch) give
    exactly the single-call results; ``outs`` are filled in place."""
    import jax_hf_b200 as G
    prob, P, rng = _problem(48, 40, 8, "layer", 23)
    HH = rng.normal(size=(8, 8))
    ref = S.haar_density(48, 8, 5)[:48, :40] * 0.5
    K, _ = _pair(prob, include_hartree=True, reference_density=np.ascontiguousarray(ref), hartree_matrix=HH + HH.T)
    a = K.as_args()
    kw = dict(h=a["h"], VR=a["VR"], refP=a["refP"], HH=a["HH"], w2d=K.w2d, include_exchange=True,
              include_hartree=True, exchange_hermitian_channel_packing=a["exchange_hermitian_channel_packing"],
              contact_g=a["contact_g"], contact_Oi=a["contact_Oi"], contact_Oj=a["contact_Oj"])
    Ps = [torch.as_tensor(np.ascontiguousarray(S.haar_density(48, 8, 40 + i)[:48, :40]), device="cuda")
          for i in range(5)]
    single = [G.build_fock(Pi, **kw) for Pi in Ps]
    outs = [tuple(torch.full_like(x, float("nan")) for x in r) for r in single]
    got = G.build_fock_batch(Ps, outs=outs, streams=streams, **kw)
    torch.cuda.synchronize()
    for (s1, h1, f1), (s2, h2, f2), o in zip(single, got, outs):
        assert torch.equal(s1, s2) and torch.equal(h1, h2) and torch.equal(f1, f2)
        assert s2.data_ptr() == o[0].data_ptr() and f2.data_ptr() == o[2].data_ptr()
    # without outs, and numpy inputs
    got2 = G.build_fock_batch([Pi.cpu().numpy() for Pi in Ps], streams=streams, **kw)
    for (s1, _, f1), (s2, _, f2) in zip(single, got2):
        assert torch.equal(s1, s2) and torch.equal(f1, f2)
    with pytest.raises(ValueError, match="outs has"):
        G.build_fock_batch(Ps, outs=outs[:2], **kw)
