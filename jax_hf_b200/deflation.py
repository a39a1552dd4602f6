"""Deflated basin search (drop-in for jax_hf.deflation.solve_deflated, deflation.py:56-183).

Hartree-Fock has several self-consistent solutions; a local solver lands in the
basin of its seed.  ``solve_deflated`` collects distinct ones with the device
trust-region Newton solver, whose objective can carry a repulsive Gaussian bias
around known densities (``SolverConfig.deflation_targets``; the bias term of
solver.py:799-812 is evaluated on the GPU in ``newton.py``).

Design: a :class:`_BasinSearch` object owns the search state (the unbiased
solver configuration, the basins found so far as device densities, the bias
height / width, the distinctness radius and the random stream).  A *round*
looks for one new basin: up to ``max_retries`` biased solves from a perturbed
copy of the seed, the bias height multiplied by ``sigma_growth`` after each
failure; a biased result is re-solved without bias (``repolish``) so that every
kept density is a stationary point of the physical free energy, and it is kept
when it converged and lies farther than the distinctness radius from every
known basin.  The search ends after ``n_solutions`` basins or after a round
that finds none.  Distances are the weighted Frobenius metric of the bias,
d(A, B)^2 = sum_k w_k ||A_k - B_k||_F^2, computed on the device.

Public contract kept from the reference: arguments and defaults, the automatic
bias scale from the first solution (width = half its weighted norm, or 1 for a
zero density; height = max(|E_0|, 1); radius = width / 4), the result tuple
(solutions sorted by physical energy) and the random stream, so that the same
``seed`` perturbs the seeds identically.  Random draw order: one draw per biased
attempt, in the order the attempts run; a draw is the real part then the
imaginary part of a standard normal array of the density's shape from
``numpy.random.default_rng(seed)``, Hermitian-symmetrised and scaled by
``perturb * (attempt index within the round, from 1)``.
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


class _BasinSearch:
    """State of one deflated search over the basins of a HartreeFockKernel."""

    def __init__(self, kernel, n_electrons: float, base_config: SolverConfig | None, seed: int):
        self.kernel = kernel
        self.n_electrons = float(n_electrons)
        base = base_config if base_config is not None else SolverConfig()
        # the unbiased Newton configuration every solve starts from
        self.plain = replace(base, optimizer="newton", deflation_targets=None, deflation_sigma=0.0)
        self.device = kernel.device
        self.w = torch.as_tensor(kernel.w2d).to(self.device, torch.float64)
        self.rng = np.random.default_rng(seed)
        self.basins: list[SolveResult] = []
        self.height = self.width = self.radius = None

    # -- metric on the device ------------------------------------------------
    def norm(self, A: torch.Tensor) -> float:
        per_k = (A.abs() ** 2).sum(dim=(-2, -1))
        return float(torch.sqrt(torch.clamp((self.w * per_k).sum(), min=0.0)))

    def is_new(self, cand: SolveResult) -> bool:
        D = cand.density
        return bool(cand.converged) and all(self.norm(D - b.density) > self.radius for b in self.basins)

    # -- solves ---------------------------------------------------------------
    def _solve(self, P, cfg) -> SolveResult:
        P = torch.as_tensor(P).to(self.device, torch.complex128).contiguous()
        return solve_direct_minimization(self.kernel, P, self.n_electrons, config=cfg)

    def start(self, P0, sigma, length, distinct_tol) -> None:
        first = self._solve(P0, self.plain)
        self.basins.append(first)
        if length is None:
            n0 = self.norm(first.density)
            length = 0.5 * n0 if n0 > 0.0 else 1.0
        self.width = float(length)
        self.height = float(sigma) if sigma is not None else max(abs(float(first.energy)), 1.0)
        self.radius = float(distinct_tol) if distinct_tol is not None else 0.25 * self.width

    def perturbation(self, shape, scale: float) -> np.ndarray:
        re = self.rng.standard_normal(shape)
        im = self.rng.standard_normal(shape)
        A = re + 1j * im
        return (0.5 * scale) * (A + np.conj(np.swapaxes(A, -1, -2)))

    def round(self, P0: np.ndarray, max_retries: int, growth: float, perturb: float, repolish: bool) -> bool:
        """Looks for one new basin; returns whether one was added."""
        height = self.height
        targets = np.stack([b.density.detach().cpu().numpy() for b in self.basins])
        for k in range(1, max_retries + 1):
            biased = replace(self.plain, deflation_targets=targets, deflation_sigma=height,
                             deflation_length=self.width)
            seed_P = P0 + self.perturbation(P0.shape, perturb * k)
            res = self._solve(seed_P, biased)
            cand = self._solve(res.density, self.plain) if repolish else res
            if self.is_new(cand):
                self.basins.append(cand)
                return True
            height *= growth
        return False

    def result(self) -> DeflatedResult:
        ranked = sorted(self.basins, key=lambda r: float(r.energy))
        energies = np.array([float(r.energy) for r in ranked])
        return DeflatedResult(solutions=ranked, energies=energies, best=ranked[0], n_found=len(ranked))


def solve_deflated(kernel, P0, n_electrons: float, *, base_config: SolverConfig | None = None, n_solutions: int = 4,
                   sigma: float | None = None, length: float | None = None, distinct_tol: float | None = None,
                   max_retries: int = 4, sigma_growth: float = 3.0, perturb: float = 1e-2, repolish: bool = True,
                   seed: int = 0) -> DeflatedResult:
    """Distinct HF solutions by deflated trust-region Newton, sorted by energy (deflation.py:56-183)."""
    P0n = P0.detach().cpu().numpy() if isinstance(P0, torch.Tensor) else np.asarray(P0)
    P0n = np.ascontiguousarray(P0n, dtype=np.complex128)
    search = _BasinSearch(kernel, n_electrons, base_config, seed)
    search.start(P0n, sigma, length, distinct_tol)
    while len(search.basins) < n_solutions:
        if not search.round(P0n, max_retries, sigma_growth, perturb, repolish):
            break  # a round without a new basin ends the search
    return search.result()


__all__ = ["DeflatedResult", "solve_deflated"]
