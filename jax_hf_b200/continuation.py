"""Coarse-to-fine continuation (drop-in for jax_hf.continuation, continuation.py:1-178).

``solve_continuation`` runs ``solve`` (or ``solve_scf`` when given an
``SCFConfig``) on a coarse kernel, resamples the converged density onto the
fine k-grid with the hermitised periodic-linear resample of the reference
(``hf_resample_density``, one CUDA kernel) and runs the fine solve from that
seed.  Same arguments, validation messages and result tuple as the reference.
"""

from __future__ import annotations

from typing import Any, NamedTuple

import torch

from . import _lib
from .problem import HartreeFockKernel
from .reference_scf import SCFConfig, SCFResult, solve_scf
from .solver import SolverConfig, solve


class ContinuationResult(NamedTuple):
    """(coarse, fine) stage results and the fine-grid seed P0_fine (continuation.py:30-44)."""

    coarse: Any
    fine: Any
    P0_fine: torch.Tensor


def resample_density(density: torch.Tensor, nk_fine: int) -> torch.Tensor:
    """(Q + Q^H) / 2 with Q = resample_kgrid(density, nk_fine) (continuation.py:47-50)."""
    P = density.contiguous()
    n1, n2, nb = int(P.shape[0]), int(P.shape[1]), int(P.shape[-1])
    if n1 == nk_fine and n2 == nk_fine:
        return 0.5 * (P + P.transpose(-1, -2).conj())
    out = torch.empty((nk_fine, nk_fine, nb, nb), dtype=P.dtype, device=P.device)
    _lib.check(_lib.lib().hf_resample_density(_lib.stream_ptr(P.device), _lib.dtype_code(P), n1, n2, int(nk_fine),
                                              int(nk_fine), nb, P.data_ptr(), out.data_ptr()))
    return out


def _run_stage(kernel, P0, n_electrons, config, *, stage_name):
    if isinstance(config, SCFConfig):
        return solve_scf(kernel, P0, float(n_electrons), config=config)
    if isinstance(config, SolverConfig) or config is None:
        return solve(kernel, P0, float(n_electrons), config=config)
    raise TypeError(f"{stage_name}_config must be SolverConfig, SCFConfig, or None; got {type(config).__name__}.")


def _density_of(result):
    return result.density_matrix if isinstance(result, SCFResult) else result.density


def _validate_kernels(coarse: HartreeFockKernel, fine: HartreeFockKernel) -> None:
    """continuation.py:148-175, same messages."""
    if tuple(coarse.h.shape[-2:]) != tuple(fine.h.shape[-2:]):
        raise ValueError("coarse_kernel and fine_kernel must share orbital dimensions "
                         f"(..., nb, nb); got {tuple(coarse.h.shape[-2:])} vs {tuple(fine.h.shape[-2:])}.")
    if coarse.include_hartree != fine.include_hartree:
        raise ValueError("coarse_kernel and fine_kernel must agree on include_hartree.")
    if coarse.include_exchange != fine.include_exchange:
        raise ValueError("coarse_kernel and fine_kernel must agree on include_exchange.")
    if coarse.h.shape[0] != coarse.h.shape[1]:
        raise ValueError(f"coarse_kernel must have a square k-mesh, got shape {tuple(coarse.h.shape[:2])}.")
    if fine.h.shape[0] != fine.h.shape[1]:
        raise ValueError(f"fine_kernel must have a square k-mesh, got shape {tuple(fine.h.shape[:2])}.")


def solve_continuation(coarse_kernel: HartreeFockKernel, fine_kernel: HartreeFockKernel, P0_coarse,
                       n_electrons_coarse: float, n_electrons_fine: float, *, coarse_config=None,
                       fine_config=None) -> ContinuationResult:
    """Coarse solve, resampled hermitised density as the fine seed, fine solve (continuation.py:78-145)."""
    _validate_kernels(coarse_kernel, fine_kernel)
    P0c = torch.as_tensor(P0_coarse).to(coarse_kernel.h.device, coarse_kernel.h.dtype)
    if tuple(P0c.shape) != tuple(coarse_kernel.h.shape):
        raise ValueError(f"P0_coarse shape {tuple(P0c.shape)} does not match "
                         f"coarse_kernel hamiltonian shape {tuple(coarse_kernel.h.shape)}.")
    coarse = _run_stage(coarse_kernel, P0c, n_electrons_coarse, coarse_config, stage_name="coarse")
    nk_fine = int(fine_kernel.h.shape[0])
    P0_fine = resample_density(torch.as_tensor(_density_of(coarse)), nk_fine).to(fine_kernel.h.dtype)
    fine = _run_stage(fine_kernel, P0_fine, n_electrons_fine, fine_config, stage_name="fine")
    return ContinuationResult(coarse=coarse, fine=fine, P0_fine=P0_fine)


__all__ = ["ContinuationResult", "solve_continuation", "resample_density"]
