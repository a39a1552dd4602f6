"""Superlattice (plane-wave basis) Fock exchange on the GPU (drop-in for jax_hf.superlattice).

For a Hamiltonian in a reciprocal-vector basis g_basis, the Fock self-energy
Sigma[(a, alpha), (b, beta)](k) = -sum_{q, G0} V(|k - q + G0|) rho[(a+G0, alpha), (b+G0, beta)](q)
is a 2D convolution in absolute momentum, independent per (alpha, beta,
DG = G_a - G_b) channel (superlattice.py:1-17).  ``build_extended_layout`` is
the host-side index planning of the reference (superlattice.py:72-164);
``make_superlattice_fock_fn`` returns a callable that runs the convolution
through ``hf_sl_fock`` (tile scatter, the library's exchange FFT over chunks of
DG channels, tile gather); ``make_superlattice_build_fock_fn`` is the
``fock_build_fn`` adapter with the superlattice Hartree shift
(superlattice.py:232-385).  complex128.
"""

from __future__ import annotations

import ctypes as C
import warnings
from dataclasses import dataclass
from typing import Callable

import numpy as np
import torch

from . import _lib


@dataclass(frozen=True)
class ExtendedGridLayout:
    """Index tables of the extended-grid superlattice Fock (superlattice.py:31-69)."""

    N_ext_x: int
    N_ext_y: int
    n_supp_x: int
    n_supp_y: int
    g_a_off: np.ndarray
    n_delta: int
    pair_to_delta: np.ndarray
    V_lag_fft: np.ndarray
    delta_pair_count: np.ndarray
    delta_pair_i: np.ndarray
    delta_pair_j: np.ndarray
    delta_pair_start: np.ndarray


def build_extended_layout(g_basis_fractional, g_basis_B, nkx: int, nky: int, coulomb_V: Callable, w_scalar: float):
    """Index tables and the lag-grid Coulomb FFT (superlattice.py:72-164).

    Tiles: G with fractional coordinates g sits at tile offset (-g) - min(-g) of a grid of
    2 x (nk x G_dim) points per axis; DG values are numbered in first-seen (i, j) row-major
    order and the pairs of each DG are listed CSR-style; the lag grid holds V(|B f|) at
    fractional lags f = (FFT-natural index) / nk, scaled by w_scalar, transformed by FFT2.
    """
    g = np.asarray(g_basis_fractional, dtype=np.int64)
    nG = int(g.shape[0])
    pg = -g
    lo, hi = pg.min(axis=0), pg.max(axis=0)
    gdim = hi - lo + 1
    n_supp_x, n_supp_y = int(nkx * gdim[0]), int(nky * gdim[1])
    Nx, Ny = 2 * n_supp_x, 2 * n_supp_y
    g_a_off = (pg - lo).astype(np.int64)
    index: dict = {}
    pair_to_delta = np.empty((nG, nG), dtype=np.int64)
    for i in range(nG):
        for j in range(nG):
            pair_to_delta[i, j] = index.setdefault((int(g[i, 0] - g[j, 0]), int(g[i, 1] - g[j, 1])), len(index))
    n_delta = len(index)
    count = np.bincount(pair_to_delta.ravel(), minlength=n_delta).astype(np.int64)
    start = np.zeros(n_delta + 1, dtype=np.int64)
    start[1:] = np.cumsum(count)
    order = np.argsort(pair_to_delta.ravel(), kind="stable")  # row-major (i, j) within each DG
    dpi, dpj = (order // nG).astype(np.int64), (order % nG).astype(np.int64)
    lagx = np.where(np.arange(Nx) < Nx // 2, np.arange(Nx), np.arange(Nx) - Nx).astype(float) / float(nkx)
    lagy = np.where(np.arange(Ny) < Ny // 2, np.arange(Ny), np.arange(Ny) - Ny).astype(float) / float(nky)
    fx, fy = np.meshgrid(lagx, lagy, indexing="ij")
    B = np.asarray(g_basis_B, dtype=float)
    qmag = np.hypot(B[0, 0] * fx + B[0, 1] * fy, B[1, 0] * fx + B[1, 1] * fy)
    V_lag_fft = np.fft.fftn(float(w_scalar) * np.asarray(coulomb_V(qmag), dtype=float), axes=(0, 1))
    return ExtendedGridLayout(Nx, Ny, n_supp_x, n_supp_y, g_a_off, n_delta, pair_to_delta,
                              np.ascontiguousarray(V_lag_fft, dtype=np.complex128), count, dpi, dpj, start)


def _tile_owner(layout: ExtendedGridLayout, nG: int, nkx: int, nky: int) -> np.ndarray:
    TX, TY = layout.N_ext_x // nkx, layout.N_ext_y // nky
    own = np.full((layout.n_delta, TX, TY), -1, dtype=np.int32)
    for d in range(layout.n_delta):
        for k in range(int(layout.delta_pair_start[d]), int(layout.delta_pair_start[d + 1])):
            i, j = int(layout.delta_pair_i[k]), int(layout.delta_pair_j[k])
            own[d, int(layout.g_a_off[i, 0]), int(layout.g_a_off[i, 1])] = i * nG + j
    return own


def make_superlattice_fock_fn(layout: ExtendedGridLayout, n_G: int, dim_orb: int, nkx: int, nky: int):
    """rho (nkx, nky, n_G dim_orb, n_G dim_orb) -> Sigma_F, same shape (superlattice.py:167-229)."""
    nG, do = int(n_G), int(dim_orb)
    D = nG * do
    tables: dict = {}

    def dev_tables(device):
        if device not in tables:
            tables[device] = dict(
                owner=torch.as_tensor(_tile_owner(layout, nG, nkx, nky), device=device),
                off=torch.as_tensor(np.ascontiguousarray(layout.g_a_off, dtype=np.int32), device=device),
                p2d=torch.as_tensor(np.ascontiguousarray(layout.pair_to_delta, dtype=np.int32), device=device),
                V=torch.as_tensor(layout.V_lag_fft, device=device).reshape(layout.N_ext_x, layout.N_ext_y, 1, 1)
                .contiguous())
        return tables[device]

    def fock_fn(rho) -> torch.Tensor:
        rho = torch.as_tensor(rho)
        if rho.device.type != "cuda":
            rho = rho.to(torch.device("cuda", torch.cuda.current_device()))
        _lib.require_cuda(rho)
        rho = rho.to(torch.complex128).contiguous()
        if tuple(rho.shape) != (nkx, nky, D, D):
            raise ValueError(f"rho must have shape {(nkx, nky, D, D)}, got {tuple(rho.shape)}")
        t = dev_tables(rho.device)
        need = C.c_size_t(0)
        _lib.check(_lib.lib().hf_sl_fock_workspace_size(nkx, nky, nG, do, layout.N_ext_x, layout.N_ext_y,
                                                        layout.n_delta, C.byref(need)))
        ws = _lib.workspace(need.value, rho.device, "superlattice")
        sigma = torch.empty_like(rho)
        _lib.check(_lib.lib().hf_sl_fock(_lib.stream_ptr(rho.device), nkx, nky, nG, do, layout.N_ext_x,
                                         layout.N_ext_y, layout.n_delta, t["owner"].data_ptr(), t["off"].data_ptr(),
                                         t["p2d"].data_ptr(), t["V"].data_ptr(), rho.data_ptr(), sigma.data_ptr(),
                                         ws.data_ptr(), ws.numel()))
        return sigma

    return fock_fn


def make_superlattice_build_fock_fn(layout: ExtendedGridLayout, n_G: int, dim_orb: int, nkx: int, nky: int,
                                    HH_GG, hartree_degeneracy: float, HH_GG_orbital=None):
    """``fock_build_fn`` adapter (superlattice.py:232-385): Sigma = Sigma_F + Hartree shift, H = 0,
    F = herm(h + Sigma) (then project_fn and herm)."""
    fock_fn = make_superlattice_fock_fn(layout, n_G, dim_orb, nkx, nky)
    nG, do = int(n_G), int(dim_orb)
    D = nG * do
    n_delta = int(layout.n_delta)
    p2d = np.asarray(layout.pair_to_delta, dtype=np.int64)
    deg = float(hartree_degeneracy)
    HHgg = np.asarray(HH_GG, dtype=np.float64)
    orbital = HH_GG_orbital is not None
    if orbital:
        HHo = np.asarray(HH_GG_orbital, dtype=np.float64)
        if HHo.shape != (nG, nG, do, do):
            raise ValueError(f"HH_GG_orbital must have shape {(nG, nG, do, do)}; got {HHo.shape}")
        if float(np.max(np.abs(HHo[np.arange(nG), np.arange(nG)]))) > 1e-12:
            warnings.warn("HH_GG_orbital has nonzero diagonal-G blocks; the q=0 layer Hartree will be included.  "
                          "This is intended for a layer-resolved system at finite displacement field; for the "
                          "moire/TBG convention pass HH_GG_orbital[i, i, :, :] = 0.", stacklevel=2)

    def herm(X):
        return 0.5 * (X + X.transpose(-1, -2).conj())

    def build_fock_sl(P, *, h, VR, refP, HH, w2d, include_exchange, include_hartree,
                      exchange_hermitian_channel_packing, contact_g, contact_Oi, contact_Oj, project_fn=None,
                      exchange_block_specs=None, exchange_check_offdiag=None, exchange_offdiag_atol=1e-12,
                      exchange_offdiag_rtol=0.0):
        P = torch.as_tensor(P)
        dev = P.device if P.device.type == "cuda" else torch.device("cuda", torch.cuda.current_device())
        P = P.to(dev, torch.complex128)
        ref = torch.zeros_like(P) if refP is None else torch.as_tensor(refP).to(dev, torch.complex128)
        rho = P - ref
        Sigma = fock_fn(rho) if include_exchange else torch.zeros_like(P)
        if include_hartree:
            w = torch.as_tensor(w2d).to(dev, torch.float64).reshape(P.shape[0], P.shape[1])
            rb = torch.einsum("ij,ijab->ab", w.to(rho.dtype), rho).reshape(nG, do, nG, do).cpu().numpy()
            blocks = np.zeros((nG, do, nG, do), dtype=np.complex128)
            if orbital:
                per = np.einsum("AxBx->ABx", rb)
                acc = np.zeros((n_delta, do), dtype=np.complex128)
                np.add.at(acc, p2d.ravel(), per.reshape(nG * nG, do))
                s = deg * np.einsum("ABag,ABg->ABa", HHo.astype(np.complex128), acc[p2d])
                for a in range(do):
                    blocks[:, a, :, a] = s[:, :, a]
            else:
                rgg = np.einsum("AxBx->AB", rb)
                acc = np.zeros(n_delta, dtype=np.complex128)
                np.add.at(acc, p2d.ravel(), rgg.ravel())
                s = deg * HHgg * acc[p2d]
                for a in range(do):
                    blocks[:, a, :, a] = s
            Sigma = Sigma + torch.as_tensor(blocks.reshape(D, D), device=dev)[None, None]
        F = herm(torch.as_tensor(h).to(dev, torch.complex128) + Sigma)
        if project_fn is not None:
            F = herm(torch.as_tensor(project_fn(F)).to(dev, torch.complex128))
        return Sigma, torch.zeros_like(P), F

    return build_fock_sl


__all__ = ["ExtendedGridLayout", "build_extended_layout", "make_superlattice_fock_fn",
           "make_superlattice_build_fock_fn"]
