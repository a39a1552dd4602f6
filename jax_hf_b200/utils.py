"""Occupations, chemical potential and validation (drop-in for jax_hf.utils).

``find_chemical_potential`` runs the cluster-wide mu root find on the GPU
(``hf_find_mu``); ``validate_electron_count`` is the reference's host check
(utils.py:21-43) with the same ValueError text; ``resample_kgrid`` (utils.py:477-535)
resamples a centered periodic k-grid array on the GPU (``hf_resample_kgrid``).
"""

from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .fock import _as_dev


def validate_electron_count(weights, nbands: int, n_electrons, *, context: str = "n_electrons") -> None:
    """utils.py:21-43."""
    if isinstance(weights, torch.Tensor):
        total_weight = float(weights.real.sum().item()) if weights.is_complex() else float(weights.sum().item())
    else:
        total_weight = float(np.real(np.asarray(weights)).sum())
    target = float(n_electrons.item() if isinstance(n_electrons, torch.Tensor) else np.asarray(n_electrons))
    max_electrons = total_weight * int(nbands)
    tol = max(1e-8, 1e-6 * max(1.0, abs(max_electrons)))
    if not np.isfinite(target):
        raise ValueError(f"{context} must be finite, got {target!r}.")
    if target < -tol or target > max_electrons + tol:
        raise ValueError(
            f"{context}={target} is outside the physically reachable range "
            f"[0, {max_electrons}] for {int(nbands)} bands and weights.sum()={total_weight}.")


def hermitize(X: torch.Tensor) -> torch.Tensor:
    return 0.5 * (X + X.transpose(-1, -2).conj())


def fermidirac(x, T: float):
    """1/(1 + exp(x/T)) as expit(-x/(T + 1e-12)) (utils.py:51-53)."""
    x = _as_dev(x)
    return torch.sigmoid(-x / (T + 1e-12))


_METHODS = {"bisection": 0, "newton": 1}


def find_chemical_potential(bands, weights, n_electrons: float, T: float, *, maxiter: int | None = None,
                            method: str = "bisection"):
    """mu with sum_k w_k sum_j f(eps_kj - mu) = n_electrons (utils.py:314-350)."""
    bands = _as_dev(bands)
    if bands.is_complex():
        bands = bands.real.contiguous()
    dev = bands.device
    validate_electron_count(weights, bands.shape[-1], n_electrons, context="n_electrons")
    m = str(method).lower()
    if m not in _METHODS:
        raise ValueError(f"method must be 'bisection' or 'newton', got {method!r}")
    w = _as_dev(weights, dev, bands.dtype)
    nb = int(bands.shape[-1])
    nk = bands.numel() // nb
    mu = torch.empty((), dtype=torch.float64, device=dev)
    _lib.check(_lib.lib().hf_find_mu(_lib.stream_ptr(dev), _lib.dtype_code(bands), _METHODS[m], nk, 1, nb,
                                     bands.data_ptr(), w.data_ptr(), float(n_electrons), float(T),
                                     int(maxiter or 0), None, mu.data_ptr()))
    return mu


def solve_mu(eps, w_norm, n_target_norm: float, mu0, T: float, maxiter: int = 25, out=None):
    """Newton-bracket mu of the direct-minimisation solver (solver.py:62-101)."""
    eps = _as_dev(eps)
    dev = eps.device
    w = _as_dev(w_norm, dev, eps.dtype)
    nb = int(eps.shape[-1])
    nk = eps.numel() // nb
    m0 = mu0 if isinstance(mu0, torch.Tensor) else torch.tensor(float(mu0), dtype=torch.float64, device=dev)
    m0 = m0.to(dev, torch.float64).reshape(()).contiguous()
    mu = out if out is not None else torch.empty((), dtype=torch.float64, device=dev)
    _lib.check(_lib.lib().hf_find_mu(_lib.stream_ptr(dev), _lib.dtype_code(eps), 2, nk, 1, nb, eps.data_ptr(),
                                     w.data_ptr(), float(n_target_norm), float(T), int(maxiter), m0.data_ptr(),
                                     mu.data_ptr()))
    return mu


def resample_kgrid(values, nk: int, *, method: str = "linear") -> torch.Tensor:
    """Resamples a centered, periodic (nk1, nk2, ...) k-grid array to (nk, nk, ...) (utils.py:512-535).

    Periodic linear interpolation along axis 0 and then axis 1 on the centered grid
    (k = 0 at index n // 2), on the GPU (``hf_resample_kgrid``); float32/64 and
    complex64/128 arrays.  Returns the input unchanged when it already is nk x nk.
    """
    nk = int(nk)
    x = values if isinstance(values, torch.Tensor) else torch.as_tensor(np.asarray(values))
    if x.dim() < 2:
        raise ValueError("resample_kgrid expects an array with at least 2 dimensions (nk,nk,...).")
    if x.shape[0] == nk and x.shape[1] == nk:
        return x
    if str(method).lower() != "linear":
        raise ValueError(f"Unsupported resample method {method!r}. Only 'linear' is supported.")
    if nk <= 0:
        raise ValueError("n_new must be a positive integer.")
    if x.dtype not in (torch.float64, torch.float32, torch.complex128, torch.complex64):
        raise TypeError(f"resample_kgrid: unsupported dtype {x.dtype}")
    if x.device.type != "cuda":
        x = x.to(torch.device("cuda", torch.cuda.current_device()))
    _lib.require_cuda(x)
    x = x.contiguous()
    inner = 1
    for d in x.shape[2:]:
        inner *= int(d)
    ncomp = inner * (2 if x.is_complex() else 1)
    y = torch.empty((nk, nk) + tuple(x.shape[2:]), dtype=x.dtype, device=x.device)
    _lib.check(_lib.lib().hf_resample_kgrid(_lib.stream_ptr(x.device), _lib.dtype_code(x), int(x.shape[0]),
                                            int(x.shape[1]), nk, nk, ncomp, x.data_ptr(), y.data_ptr()))
    return y
