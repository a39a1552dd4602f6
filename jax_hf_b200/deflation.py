"""Deflated basin search (drop-in for jax_hf.deflation, deflation.py:1-183).

``solve_deflated`` runs the device trust-region Newton solver (whose deflation
bias, solver.py:799-812, is implemented in ``newton.py``) repeatedly: an
unbiased solve from P0, then biased re-solves against every solution found so
far with an escalating bias height and a growing Hermitian perturbation of the
seed, each biased result re-polished unbiased and kept if it is converged and
farther than ``distinct_tol`` (weighted Frobenius distance) from all others.
Same arguments, defaults, random stream (NumPy ``default_rng(seed)``) and
result tuple as the reference; solutions are sorted by energy.
"""

from __future__ import annotations

from dataclasses import replace
from typing import NamedTuple

import numpy as np
import torch

from .solver import SolveResult, SolverConfig, solve_direct_minimization


class DeflatedResult(NamedTuple):
    solutions: list          # distinct minima, ascending energy
    energies: np.ndarray     # their physical energies, ascending
    best: SolveResult        # lowest-energy solution
    n_found: int


def _np(x) -> np.ndarray:
    return x.detach().cpu().numpy() if isinstance(x, torch.Tensor) else np.asarray(x)


def _wnorm2(M, w2d) -> float:
    """sum_k w_k ||M_k||_F^2 (deflation.py:37-40)."""
    return float(np.sum(np.asarray(w2d) * np.sum(np.abs(M) ** 2, axis=(-2, -1))))


def _wdist(A, B, w2d) -> float:
    return float(np.sqrt(max(_wnorm2(_np(A) - _np(B), w2d), 0.0)))


def _hermitian_perturbation(shape, scale: float, rng) -> np.ndarray:
    A = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex128)
    return scale * 0.5 * (A + np.conj(np.swapaxes(A, -1, -2)))


def solve_deflated(kernel, P0, n_electrons: float, *, base_config: SolverConfig | None = None, n_solutions: int = 4,
                   sigma: float | None = None, length: float | None = None, distinct_tol: float | None = None,
                   max_retries: int = 4, sigma_growth: float = 3.0, perturb: float = 1e-2, repolish: bool = True,
                   seed: int = 0) -> DeflatedResult:
    """Distinct HF solutions by deflated trust-region Newton (deflation.py:56-183)."""
    w2d = _np(kernel.w2d)
    rng = np.random.default_rng(seed)
    base = base_config if base_config is not None else SolverConfig()
    newton_cfg = replace(base, optimizer="newton", deflation_targets=None, deflation_sigma=0.0)
    dev = kernel.device
    P0 = np.ascontiguousarray(_np(P0), dtype=np.complex128)

    def run(P, cfg):
        return solve_direct_minimization(kernel, torch.as_tensor(P, device=dev), float(n_electrons), config=cfg)

    r0 = run(P0, newton_cfg)
    solutions = [r0]
    if length is None:
        d0 = float(np.sqrt(max(_wnorm2(_np(r0.density), w2d), 0.0)))
        length = 0.5 * d0 if d0 > 0.0 else 1.0
    if sigma is None:
        sigma = max(abs(float(r0.energy)), 1.0)
    if distinct_tol is None:
        distinct_tol = 0.25 * length
    while len(solutions) < n_solutions:
        found_new = False
        cur_sigma = float(sigma)
        for attempt in range(max_retries):
            targets = np.stack([_np(s.density) for s in solutions])
            biased = replace(newton_cfg, deflation_targets=targets, deflation_sigma=cur_sigma,
                             deflation_length=float(length))
            seed_P = np.ascontiguousarray(P0 + _hermitian_perturbation(P0.shape, perturb * (attempt + 1), rng))
            rb = run(seed_P, biased)
            cand = run(np.ascontiguousarray(_np(rb.density), dtype=np.complex128), newton_cfg) if repolish else rb
            if bool(cand.converged) and all(_wdist(cand.density, s.density, w2d) > distinct_tol for s in solutions):
                solutions.append(cand)
                found_new = True
                break
            cur_sigma *= sigma_growth
        if not found_new:
            break
    order = np.argsort([float(s.energy) for s in solutions])
    solutions = [solutions[i] for i in order]
    energies = np.array([float(s.energy) for s in solutions])
    return DeflatedResult(solutions=solutions, energies=energies, best=solutions[0], n_found=len(solutions))


__all__ = ["DeflatedResult", "solve_deflated"]
