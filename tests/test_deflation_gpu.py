"""solve_deflated (deflation.py:56-183) on the device Newton solver: the reference's end-to-end
test (tests/test_deflation.py:160-182) on its bistable two-band model, whose two self-consistent
solutions have the analytic energies -0.6 (ground) and -0.4 (metastable)."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _bistable(T=0.02, ex=1.0, delta=0.1):
    h = np.zeros((1, 1, 2, 2), complex)
    h[..., 0, 0] = -delta
    h[..., 1, 1] = +delta
    return dict(weights=np.ones((1, 1)), hamiltonian=h, coulomb_q=np.full((1, 1, 1, 1), ex), T=T)


def _comm_rms(F, P, w2d):
    F, P, w2d = (x.cpu().numpy() if isinstance(x, torch.Tensor) else np.asarray(x) for x in (F, P, w2d))
    c = F @ P - P @ F
    return float(np.sqrt(np.sum(w2d * np.sum(np.abs(c) ** 2, axis=(-2, -1))) / max(float(np.sum(w2d)), 1e-30)))


def test_deflation_finds_the_metastable_solution(cuda):
    import jax_hf_b200 as G
    from jax_hf_b200.deflation import DeflatedResult, solve_deflated
    from jax_hf_b200.solver import SolverConfig, solve
    K = G.HartreeFockKernel(**_bistable())
    P0 = torch.zeros((1, 1, 2, 2), dtype=torch.complex128, device="cuda")
    base = SolverConfig(optimizer="newton", tol_grad=1e-6, max_iter=300)
    res = solve_deflated(K, P0, 1.0, base_config=base, n_solutions=2, seed=0)
    assert isinstance(res, DeflatedResult) and res.n_found >= 2
    for s in res.solutions:
        assert _comm_rms(s.fock, s.density, K.w2d) < 1e-3
    d = res.solutions[0].density.cpu().numpy() - res.solutions[1].density.cpu().numpy()
    assert float(np.max(np.abs(d))) > 1e-2
    cold = solve(K, P0, 1.0, config=base)
    assert float(res.best.energy) <= float(cold.energy) + 1e-7
    np.testing.assert_allclose(float(res.best.energy), -0.6, atol=2e-2)
    np.testing.assert_allclose(sorted(res.energies)[:2], [-0.6, -0.4], atol=3e-2)
    assert list(res.energies) == sorted(res.energies)


def test_deflation_single_solution_is_the_plain_newton_solve(cuda):
    import jax_hf_b200 as G
    from jax_hf_b200.deflation import solve_deflated
    from jax_hf_b200.solver import SolverConfig, solve
    K = G.HartreeFockKernel(**_bistable())
    P0 = torch.zeros((1, 1, 2, 2), dtype=torch.complex128, device="cuda")
    base = SolverConfig(optimizer="newton", tol_grad=1e-6, max_iter=300)
    res = solve_deflated(K, P0, 1.0, base_config=base, n_solutions=1)
    r = solve(K, P0, 1.0, config=base)
    assert res.n_found == 1 and abs(float(res.best.energy) - float(r.energy)) < 1e-12
