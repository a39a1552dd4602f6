"""Continuation: periodic-linear k-grid resampling (utils.py:477-535) and the coarse -> fine
driver (continuation.py:78-175).

CPU tests pin the oracle's resample on known answers; GPU tests compare the CUDA resample
with the oracle (float64 / complex128 bit-level 1e-15 relative, float32 / complex64 1e-6)
and the driver with a manual coarse-then-fine run and with the oracle's fine solve.
"""

import numpy as np
import pytest
import torch

from oracle import hf_oracle as O


def _dirac(nk, m=0.3, v=1.0, T=0.1, ex=0.7):
    ks = (np.arange(nk) - nk // 2) * (2 * np.pi / nk)
    KX, KY = np.meshgrid(ks, ks, indexing="ij")
    h = np.zeros((nk, nk, 2, 2), complex)
    h[..., 0, 0] = m
    h[..., 1, 1] = -m
    h[..., 0, 1] = v * (np.sin(KX) - 1j * np.sin(KY))
    h[..., 1, 0] = v * (np.sin(KX) + 1j * np.sin(KY))
    return dict(weights=np.full((nk, nk), 1.0 / nk ** 2), hamiltonian=h, coulomb_q=np.full((nk, nk, 1, 1), ex), T=T)


# ------------------------------------------------------------------ oracle (CPU) ----
def test_oracle_resample_known_answer_2_to_4():
    # u = (j - 2) * 0.5 + 1: j = 0..3 -> x0, (x0 + x1)/2, x1, (x1 + x0)/2 along each axis
    x = np.array([[1.0, 3.0], [5.0, 11.0]])
    line = lambda a, b: np.array([a, 0.5 * (a + b), b, 0.5 * (b + a)])
    rows = np.stack([line(x[0, 0], x[1, 0]), line(x[0, 1], x[1, 1])], axis=1)  # axis 0 first
    want = np.stack([line(rows[i, 0], rows[i, 1]) for i in range(4)], axis=0)
    np.testing.assert_allclose(O.resample_kgrid(x, 4), want, rtol=0, atol=0)


def test_oracle_resample_invariants():
    rng = np.random.default_rng(1)
    x = rng.standard_normal((6, 6, 3)) + 1j * rng.standard_normal((6, 6, 3))
    assert O.resample_kgrid(x, 6) is x
    np.testing.assert_array_equal(O.resample_kgrid(x, 12)[::2, ::2], x)  # even indices hit the coarse points
    c = np.full((5, 7, 2), 1.5 - 0.25j)
    np.testing.assert_allclose(O.resample_kgrid(c, 9), 1.5 - 0.25j, rtol=0, atol=1e-15)
    with pytest.raises(ValueError, match="at least 2 dimensions"):
        O.resample_kgrid(np.zeros(4), 8)
    with pytest.raises(ValueError, match="Only 'linear'"):
        O.resample_kgrid(x, 8, method="cubic")
    P = O.resample_density(x[..., None] * np.ones((1, 1, 1, 3)), 10)
    np.testing.assert_allclose(P, np.conj(np.swapaxes(P, -1, -2)), rtol=0, atol=0)


# --------------------------------------------------------------------------- GPU ----
@pytest.mark.gpu
@pytest.mark.parametrize("shape,nk", [((6, 6, 3), 12), ((12, 12, 2, 2), 5), ((7, 5), 9), ((24, 24, 4, 4), 36),
                                      ((36, 36, 8, 8), 24), ((3, 3, 2), 1)])
@pytest.mark.parametrize("dtype", [np.float64, np.complex128, np.float32, np.complex64])
def test_resample_matches_oracle(cuda, shape, nk, dtype):
    import jax_hf_b200 as G
    rng = np.random.default_rng(sum(shape) + nk)
    x = rng.standard_normal(shape)
    if np.iscomplexobj(np.zeros(1, dtype)):
        x = x + 1j * rng.standard_normal(shape)
    x = x.astype(dtype)
    y = G.resample_kgrid(torch.as_tensor(x, device="cuda"), nk)
    want = O.resample_kgrid(x, nk)
    assert tuple(y.shape) == (nk, nk) + shape[2:] and y.dtype == torch.as_tensor(x).dtype
    tol = 1e-15 if x.real.dtype == np.float64 else 1e-6
    assert np.abs(y.cpu().numpy() - want).max() <= tol * max(1.0, np.abs(want).max())


@pytest.mark.gpu
def test_resample_errors(cuda):
    import jax_hf_b200 as G
    x = torch.zeros((4, 4, 2), dtype=torch.float64, device="cuda")
    assert G.resample_kgrid(x, 4) is x
    with pytest.raises(ValueError, match="at least 2 dimensions"):
        G.resample_kgrid(torch.zeros(4, device="cuda"), 8)
    with pytest.raises(ValueError, match="Only 'linear'"):
        G.resample_kgrid(x, 8, method="nearest")
    with pytest.raises(ValueError, match="positive"):
        G.resample_kgrid(x, 0)


@pytest.mark.gpu
@pytest.mark.parametrize("n,m,nb,dt", [(4, 8, 2, np.complex128), (12, 18, 4, np.complex128), (10, 6, 3, np.complex64)])
def test_resample_density_matches_oracle(cuda, n, m, nb, dt):
    from jax_hf_b200.continuation import resample_density
    rng = np.random.default_rng(n + m + nb)
    P = (rng.standard_normal((n, n, nb, nb)) + 1j * rng.standard_normal((n, n, nb, nb))).astype(dt)
    out = resample_density(torch.as_tensor(P, device="cuda"), m).cpu().numpy()
    want = O.resample_density(P, m)
    tol = 1e-15 if dt == np.complex128 else 1e-6
    assert np.abs(out - want).max() <= tol * np.abs(want).max()
    np.testing.assert_allclose(out, np.conj(np.swapaxes(out, -1, -2)), rtol=0, atol=0)


@pytest.mark.gpu
def test_continuation_matches_manual_driver_and_oracle(cuda):
    import jax_hf_b200 as G
    from jax_hf_b200.continuation import ContinuationResult, solve_continuation
    from jax_hf_b200.solver import SolverConfig, solve
    kc, kf = G.HartreeFockKernel(**_dirac(4)), G.HartreeFockKernel(**_dirac(8))
    P0 = torch.zeros((4, 4, 2, 2), dtype=torch.complex128, device="cuda")
    cfg = SolverConfig(max_iter=200, tol_E=1e-10)
    res = solve_continuation(kc, kf, P0, 1.0, 1.0, coarse_config=cfg, fine_config=cfg)
    assert isinstance(res, ContinuationResult) and tuple(res.P0_fine.shape) == (8, 8, 2, 2)
    rc = solve(kc, P0, 1.0, config=cfg)
    Pf = G.resample_kgrid(rc.density, 8)
    Pf = 0.5 * (Pf + Pf.transpose(-1, -2).conj())
    assert torch.allclose(res.P0_fine, Pf, rtol=0, atol=1e-14)
    rf = solve(kf, Pf, 1.0, config=cfg)
    assert abs(float(res.fine.energy) - float(rf.energy)) <= 1e-12 * abs(float(rf.energy))
    # oracle: coarse solve, oracle resample, fine solve from that seed
    co = O.solve(O.Kernel(**_dirac(4)), np.zeros((4, 4, 2, 2), complex), 1.0, config=O.SolverConfig(max_iter=200, tol_E=1e-10))
    P0f = O.resample_density(co["density"], 8)
    assert np.abs(res.P0_fine.cpu().numpy() - P0f).max() < 1e-6
    fo = O.solve(O.Kernel(**_dirac(8)), P0f, 1.0, config=O.SolverConfig(max_iter=200, tol_E=1e-10))
    assert abs(float(res.fine.energy) - fo["energy"]) <= 1e-9 * abs(fo["energy"])
    # a cold fine solve lands at the same fixed point (reference test_continuation.py:141-160)
    cold = solve(kf, torch.zeros((8, 8, 2, 2), dtype=torch.complex128, device="cuda"), 1.0, config=cfg)
    assert abs(float(cold.energy) - float(res.fine.energy)) < 1e-6


@pytest.mark.gpu
def test_continuation_scf_stage_and_validation(cuda):
    import jax_hf_b200 as G
    from jax_hf_b200.continuation import solve_continuation
    from jax_hf_b200.reference_scf import SCFConfig, SCFResult
    from jax_hf_b200.solver import SolveResult, SolverConfig
    kc, kf = G.HartreeFockKernel(**_dirac(4)), G.HartreeFockKernel(**_dirac(8))
    P0 = torch.zeros((4, 4, 2, 2), dtype=torch.complex128, device="cuda")
    res = solve_continuation(kc, kf, P0, 1.0, 1.0, coarse_config=SCFConfig(max_iter=60, mixing=0.5),
                             fine_config=SolverConfig(max_iter=100, tol_E=1e-8))
    assert isinstance(res.coarse, SCFResult) and isinstance(res.fine, SolveResult)
    k3 = G.HartreeFockKernel(**dict(_dirac(8), hamiltonian=np.zeros((8, 8, 3, 3), complex)))
    with pytest.raises(ValueError, match="share orbital dimensions"):
        solve_continuation(kc, k3, P0, 1.0, 1.0)
    with pytest.raises(ValueError, match="does not match"):
        solve_continuation(kc, kf, torch.zeros((5, 5, 2, 2), dtype=torch.complex128), 1.0, 1.0)
    with pytest.raises(TypeError, match="coarse_config must be"):
        solve_continuation(kc, kf, P0, 1.0, 1.0, coarse_config=3)
