"""Hand-written adjoints: Fock-build / energy / free-energy VJPs against finite differences,
parameter gradients of the converged free energy against the oracle's formulas and against
central differences of re-converged solves (envelope theorem)."""

import numpy as np
import pytest
import torch

from oracle import hf_oracle as O
from jax_hf_b200 import synthetic as S

pytestmark = pytest.mark.gpu


def _herm_np(a):
    return 0.5 * (a + np.conj(np.swapaxes(a, -1, -2)))


def _kernel_kwargs(nk, nb, V, seed, hartree=False, complex_vr=False):
    p = S.fourier_problem(nk, nb, 2.0, seed, V=V, T=0.1)
    kw = p.kernel_kwargs()
    rng = np.random.default_rng(seed)
    if complex_vr:  # a V(q) that is not even in q makes the shifted VR complex
        kw["coulomb_q"] = kw["coulomb_q"] + 0.3 * rng.standard_normal(kw["coulomb_q"].shape)
    if hartree:
        kw["include_hartree"] = True
        kw["reference_density"] = 0.1 * S.haar_density(nk, nb, seed + 7)
        HH = rng.standard_normal((nb, nb))
        kw["hartree_matrix"] = 0.5 * (HH + HH.T)
    return kw


VJP_CASES = [
    ("scalar_packed", "scalar", False, False),
    ("layer", "layer", False, False),
    ("layer_complex_vr", "layer", False, True),
    ("scalar_hartree", "scalar", True, False),
]


@pytest.mark.parametrize("name,V,hartree,complex_vr", VJP_CASES, ids=[c[0] for c in VJP_CASES])
def test_fock_build_vjp_matches_finite_differences(cuda, name, V, hartree, complex_vr):
    import jax_hf_b200 as G
    from jax_hf_b200 import adjoint as A
    nk, nb = 6, 3
    K = G.HartreeFockKernel(**_kernel_kwargs(nk, nb, V, 11, hartree, complex_vr))
    rng = np.random.default_rng(5)
    shape = (nk, nk, nb, nb)

    def cplx():
        return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)

    C1, C2 = (torch.as_tensor(cplx(), device="cuda") for _ in range(2))
    C3 = torch.as_tensor(rng.standard_normal((1, 1, nb, nb)) + 0j, device="cuda")
    P = torch.as_tensor(S.haar_density(nk, nb, 3), device="cuda")
    h = K.h.to(torch.complex128).clone()

    def loss(P, h):
        Sg, H, F = A.fock_build(P, h, K)
        return (torch.real(torch.sum(C1.conj() * Sg)) + torch.real(torch.sum(C2.conj() * F))
                + torch.real(torch.sum(C3.conj() * H)))

    P1, h1 = P.clone().requires_grad_(True), h.clone().requires_grad_(True)
    loss(P1, h1).backward()
    # channel packing assumes a Hermitian density: probe along Hermitian directions there
    for trial in range(3):
        D = cplx()
        if V == "scalar":
            D = _herm_np(D)
        Dt, Dht = torch.as_tensor(D, device="cuda"), torch.as_tensor(cplx(), device="cuda")
        eps = 1e-3  # the loss is linear in P and h: central differences are exact up to rounding
        fd = (float(loss(P + eps * Dt, h)) - float(loss(P - eps * Dt, h))) / (2 * eps)
        an = float(torch.real(torch.sum(P1.grad.conj() * Dt)))
        assert abs(fd - an) <= 1e-9 * max(1.0, abs(fd)), (trial, fd, an)
        fdh = (float(loss(P, h + eps * Dht)) - float(loss(P, h - eps * Dht))) / (2 * eps)
        anh = float(torch.real(torch.sum(h1.grad.conj() * Dht)))
        assert abs(fdh - anh) <= 1e-9 * max(1.0, abs(fdh)), (trial, fdh, anh)


def test_objective_vjp_matches_finite_differences(cuda):
    """Omega(P, p) = hf_energy(P, h, Sigma[P], H[P]) - T S(p) differentiated in P and p."""
    import jax_hf_b200 as G
    from jax_hf_b200 import adjoint as A
    nk, nb = 6, 4
    K = G.HartreeFockKernel(**_kernel_kwargs(nk, nb, "scalar", 21, hartree=True))
    rng = np.random.default_rng(9)
    P = torch.as_tensor(S.haar_density(nk, nb, 4), device="cuda")
    p = torch.as_tensor(rng.uniform(0.05, 0.95, (nk, nk, nb)), device="cuda")
    P1, p1 = P.clone().requires_grad_(True), p.clone().requires_grad_(True)
    A.objective(P1, p1, K).backward()
    for _ in range(3):
        D = torch.as_tensor(_herm_np(rng.standard_normal((nk, nk, nb, nb))
                                     + 1j * rng.standard_normal((nk, nk, nb, nb))), device="cuda")
        dp = torch.as_tensor(rng.standard_normal((nk, nk, nb)), device="cuda")
        eps = 1e-5
        fd = (float(A.objective(P + eps * D, p, K)) - float(A.objective(P - eps * D, p, K))) / (2 * eps)
        an = float(torch.real(torch.sum(P1.grad.conj() * D)))
        assert abs(fd - an) <= 1e-8 * max(1.0, abs(fd))
        fdp = (float(A.objective(P, p + eps * dp, K)) - float(A.objective(P, p - eps * dp, K))) / (2 * eps)
        anp = float(torch.sum(p1.grad * dp))
        assert abs(fdp - anp) <= 1e-7 * max(1.0, abs(fdp))


def test_parameter_gradients_match_oracle(cuda):
    """Coupling and h_R gradients at a fixed density agree with the oracle's formulas."""
    import jax_hf_b200 as G
    from jax_hf_b200 import adjoint as A
    for V, nk, nb in (("scalar", 12, 4), ("layer", 10, 3)):
        prob = S.fourier_problem(nk, nb, 2.0, 31, V=V, T=0.1)
        K = G.HartreeFockKernel(**prob.kernel_kwargs())
        Ko = O.Kernel(**prob.kernel_kwargs())
        P = S.haar_density(nk, nb, 8)
        dV = S.coulomb_scalar_derivatives(nk) if V == "scalar" else S.coulomb_layer_derivatives(nk, nb)
        R = S.lattice_vectors(2.0)
        g = A.parameter_gradients(K, torch.as_tensor(P, device="cuda"), coupling_derivatives=dV,
                                  lattice_vectors=R)
        for name, d in dV.items():
            go = O.coupling_gradient(Ko, P, d)
            assert abs(g[name] - go) <= 1e-12 * max(1.0, abs(go)), (V, name, g[name], go)
        np.testing.assert_allclose(g["h_R"].cpu().numpy(), O.fourier_coefficient_gradient(P, Ko.w2d, R),
                                   rtol=0, atol=1e-13)


def _scf_omega(kw, ne):
    """Converged free energy Omega* = E - T S from a tight SCF-DIIS solve (its fixed point
    P = f(F[P] - mu) is a stationary point of Omega at fixed electron count)."""
    import jax_hf_b200 as G
    from jax_hf_b200.reference_scf import SCFConfig, solve_scf
    K = G.HartreeFockKernel(**kw)
    nk1, nk2, nb = K.shape
    P0 = torch.zeros((nk1, nk2, nb, nb), dtype=torch.complex128, device="cuda")
    r = solve_scf(K, P0, ne, config=SCFConfig(acceleration="diis", density_tol=1e-13, comm_tol=1e-12,
                                               max_iter=300))
    assert bool(r.converged)
    p = torch.linalg.eigvalsh(r.density_matrix).clamp(1e-14, 1 - 1e-14)
    wn = K.w2d / float(K.weight_sum)
    S_ = -torch.sum(wn[..., None] * (p * torch.log(p) + (1 - p) * torch.log1p(-p)))
    return float(r.energy) - K.T * float(S_), r, K


def test_envelope_gradients_match_resolved_finite_differences(cuda):
    """d Omega* / d(U, d, h_R) from the adjoint at the converged density vs central differences of
    re-converged solves (step 1e-5; SCF-DIIS to density_tol 1e-13, comm_tol 1e-12)."""
    from jax_hf_b200 import adjoint as A
    nk, nb, U, d = 8, 2, 1.0, 2.0
    coeffs = S.fourier_coeffs(nb, 1.0, 41)
    w = np.full((nk, nk), 1.0 / nk ** 2)
    base = dict(weights=w, hamiltonian=S.hamiltonian_from_coeffs(coeffs, nk),
                coulomb_q=S.coulomb_scalar(nk, U, d), T=0.1)
    ne = 0.8
    Om, r, K = _scf_omega(base, ne)
    R = [(1, 0), (-1, 0)]
    g = A.parameter_gradients(K, r.density_matrix, coupling_derivatives=S.coulomb_scalar_derivatives(nk, U, d),
                              lattice_vectors=R)
    step = 1e-5
    fd_U = (_scf_omega(dict(base, coulomb_q=S.coulomb_scalar(nk, U + step, d)), ne)[0]
            - _scf_omega(dict(base, coulomb_q=S.coulomb_scalar(nk, U - step, d)), ne)[0]) / (2 * step)
    fd_d = (_scf_omega(dict(base, coulomb_q=S.coulomb_scalar(nk, U, d + step)), ne)[0]
            - _scf_omega(dict(base, coulomb_q=S.coulomb_scalar(nk, U, d - step)), ne)[0]) / (2 * step)
    assert abs(fd_U - g["U"]) <= 1e-6 * max(abs(fd_U), 1e-3), (fd_U, g["U"])
    assert abs(fd_d - g["d"]) <= 1e-6 * max(abs(fd_d), 1e-3), (fd_d, g["d"])
    # h_R for R = (1, 0) with its tied partner h_{-R} = h_R^H: d/d Re and d/d Im of (h_R)_{01}
    B, Am = g["h_R"][0].cpu().numpy(), g["h_R"][1].cpu().numpy()
    i, j = 0, 1
    an_re = float(np.real(Am[j, i]) + np.real(B[i, j]))
    an_im = float(-np.imag(Am[j, i]) + np.imag(B[i, j]))

    def om_h(delta):
        c = {k: v.copy() for k, v in coeffs.items()}
        c[(1, 0)][i, j] += delta
        c[(-1, 0)] = c[(1, 0)].conj().T
        return _scf_omega(dict(base, hamiltonian=S.hamiltonian_from_coeffs(c, nk)), ne)[0]

    fd_re = (om_h(step) - om_h(-step)) / (2 * step)
    fd_im = (om_h(1j * step) - om_h(-1j * step)) / (2 * step)
    assert abs(fd_re - an_re) <= 1e-6 * max(abs(fd_re), 1e-3), (fd_re, an_re)
    assert abs(fd_im - an_im) <= 1e-6 * max(abs(fd_im), 1e-3), (fd_im, an_im)


def test_torch_library_ops(cuda):
    """torch.ops.hf_b200.fock_build / hf_energy: same values as the Python API, opcheck, gradients."""
    import jax_hf_b200 as G
    from jax_hf_b200 import torch_ops  # noqa: F401  (registers the ops)
    nk, nb = 6, 3
    K = G.HartreeFockKernel(**_kernel_kwargs(nk, nb, "layer", 51))
    a = K.as_args()
    P = torch.as_tensor(S.haar_density(nk, nb, 5), device="cuda")
    h = K.h.to(torch.complex128).contiguous()
    VR = a["VR"]
    Sg, H, F = torch.ops.hf_b200.fock_build(P, h, VR, True, False)
    S2, _, F2 = G.build_fock(P, h=h, VR=VR, refP=None, HH=None, w2d=None, include_exchange=True,
                             include_hartree=False, exchange_hermitian_channel_packing=False)
    assert torch.equal(Sg, S2) and torch.equal(F, F2)
    w = K.w2d.to(torch.float64)
    E = torch.ops.hf_b200.hf_energy(P, h, Sg, H, w)
    assert abs(float(E) - float(G.hf_energy(P, h=h, Sigma=Sg, H=H, weights_b=w[..., None, None]))) == 0.0
    torch.library.opcheck(torch.ops.hf_b200.fock_build.default, (P, h, VR, True, False),
                          test_utils=("test_schema", "test_faketensor", "test_autograd_registration"))
    torch.library.opcheck(torch.ops.hf_b200.hf_energy.default, (P, h, Sg, H, w),
                          test_utils=("test_schema", "test_faketensor", "test_autograd_registration"))
    # gradients through the ops against the autograd Functions of adjoint.py
    from jax_hf_b200 import adjoint as A
    P1, h1 = P.clone().requires_grad_(True), h.clone().requires_grad_(True)
    Sg1, H1, _ = torch.ops.hf_b200.fock_build(P1, h1, VR, True, False)
    torch.ops.hf_b200.hf_energy(P1, h1, Sg1, H1, w).backward()
    P2, h2 = P.clone().requires_grad_(True), h.clone().requires_grad_(True)
    Sg2, H2, _ = A.fock_build(P2, h2, K)
    A.hf_energy(P2, h2, Sg2, H2, K.w2d).backward()
    torch.testing.assert_close(P1.grad, P2.grad, rtol=0, atol=1e-13)
    torch.testing.assert_close(h1.grad, h2.grad, rtol=0, atol=1e-13)
