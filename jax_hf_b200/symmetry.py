"""Symmetry projectors on the GPU (drop-in for jax_hf.symmetry, symmetry.py:153-281).

``make_project_fn`` takes the reference's arguments and checks and returns a
callable A -> projected A for (nk1, nk2, nb, nb) complex arrays, usable as
``project_fn`` of ``build_fock`` / ``solve`` / ``solve_scf``.  Each averaging
stage is one CUDA kernel (``hf_sym_group_average``, ``hf_sym_time_reversal``):
per k-point the group elements' U A(k_g) U^H are formed in shared memory and
summed in registers.  The stages are composed in the reference's order:
spatial average (index maps or convention), orbital-only average, time reversal.
"""

from __future__ import annotations

from typing import Callable

import numpy as np
import torch

from . import _lib

ProjectFn = Callable[[torch.Tensor], torch.Tensor]

HF_K_FLIP, HF_K_MOD, HF_K_INDEX_MAP = 0, 1, 2


def _conv(conv: str) -> int:
    c = str(conv)
    if c == "flip":
        return HF_K_FLIP
    if c == "mod":
        return HF_K_MOD
    raise ValueError(f"k_convention must be 'mod' or 'flip', got {c!r}")


def _axes_bits(axes) -> int:
    axes = tuple(int(a) for a in axes)
    return (1 if 0 in axes else 0) | (2 if 1 in axes else 0)


def make_project_fn(*, unitary_group=None, spatial_group=None, spatial_k_convention: str = "mod",
                    spatial_k_flip_axes=(0, 1), spatial_k_index_maps=None, spatial_k_orbit_mask=None,
                    time_reversal_U=None, time_reversal_k_convention: str = "mod",
                    time_reversal_k_flip_axes=(0, 1), time_reversal_k_index_map=None) -> ProjectFn:
    """Symmetry-averaging projection (symmetry.py:153-281); same arguments, checks and composition."""
    has_group = unitary_group is not None or spatial_group is not None or spatial_k_index_maps is not None
    if not has_group and time_reversal_U is None:
        return lambda A: A
    G = None if unitary_group is None else np.asarray(unitary_group)
    S = None if spatial_group is None else np.asarray(spatial_group)
    U = None if time_reversal_U is None else np.asarray(time_reversal_U)
    if spatial_k_index_maps is not None:
        si = np.asarray(spatial_k_index_maps[0], dtype=np.int32)
        sj = np.asarray(spatial_k_index_maps[1], dtype=np.int32)
        if si.shape != sj.shape:
            raise ValueError("spatial_k_index_maps[0] and [1] must have the same shape; "
                             f"got {si.shape} vs {sj.shape}.")
        if S is None:
            raise ValueError("spatial_k_index_maps requires spatial_group (the orbital unitaries to average over).")
        if S.shape[0] != si.shape[0]:
            raise ValueError("spatial_group and spatial_k_index_maps must have matching "
                             f"leading dim; got {S.shape[0]} and {si.shape[0]}.")
    else:
        si = sj = None
    omask = None if spatial_k_orbit_mask is None else np.asarray(spatial_k_orbit_mask, dtype=bool)
    if time_reversal_k_index_map is not None:
        if U is None:
            raise ValueError("time_reversal_k_index_map requires time_reversal_U.")
        ti = np.asarray(time_reversal_k_index_map[0], dtype=np.int32)
        tj = np.asarray(time_reversal_k_index_map[1], dtype=np.int32)
        tv = np.asarray(time_reversal_k_index_map[2], dtype=bool)
    else:
        ti = tj = tv = None
    s_conv, s_bits = _conv(spatial_k_convention), _axes_bits(spatial_k_flip_axes)
    t_conv, t_bits = _conv(time_reversal_k_convention), _axes_bits(time_reversal_k_flip_axes)
    cache: dict = {}

    def dev_arrays(A: torch.Tensor):
        key = (A.device, A.dtype, tuple(A.shape))
        if key in cache:
            return cache[key]
        nk1, nk2 = int(A.shape[0]), int(A.shape[1])
        to_c = lambda M: None if M is None else torch.as_tensor(np.ascontiguousarray(M)).to(A.device, A.dtype).contiguous()
        def to_i(M):
            if M is None:
                return None
            M = np.ascontiguousarray(M)
            if M.shape[-2:] != (nk1, nk2):
                raise ValueError(f"k-index maps must end in the k-grid shape {(nk1, nk2)}, got {M.shape}")
            if M.size and (M.min() < 0):
                raise ValueError("k-index maps must hold indices in [0, nk)")
            return torch.as_tensor(M, dtype=torch.int32, device=A.device).contiguous()
        def to_m(M):
            return None if M is None else torch.as_tensor(np.ascontiguousarray(M, dtype=np.uint8), device=A.device)
        for M, n in ((si, nk1), (ti, nk1)):
            if M is not None and M.size and M.max() >= n:
                raise ValueError("k-index maps must hold indices in [0, nk)")
        for M, n in ((sj, nk2), (tj, nk2)):
            if M is not None and M.size and M.max() >= n:
                raise ValueError("k-index maps must hold indices in [0, nk)")
        eye = None if S is None else np.eye(S.shape[-1], dtype=np.complex128)[None]
        d = dict(G=to_c(G), S=to_c(S), U=to_c(U), I=to_c(eye), si=to_i(si), sj=to_i(sj), om=to_m(omask),
                 ti=to_i(ti), tj=to_i(tj), tv=to_m(tv))
        cache[key] = d
        return d

    def group(A, n_same, Gs, n_map, Gm, mode, bits, ii, jj, mask):
        out = torch.empty_like(A)
        nk1, nk2, nb = int(A.shape[0]), int(A.shape[1]), int(A.shape[-1])
        _lib.check(_lib.lib().hf_sym_group_average(
            _lib.stream_ptr(A.device), _lib.dtype_code(A), nk1, nk2, nb, A.data_ptr(), out.data_ptr(), n_same,
            _lib.ptr(Gs), n_map, _lib.ptr(Gm), mode, bits, _lib.ptr(ii), _lib.ptr(jj), _lib.ptr(mask)))
        return out

    def project(A) -> torch.Tensor:
        A = torch.as_tensor(A)
        if A.device.type != "cuda":
            A = A.to(torch.device("cuda", torch.cuda.current_device()))
        _lib.require_cuda(A)
        if not A.is_complex():
            A = A.to(torch.complex128)
        out = A.contiguous()
        d = dev_arrays(out)
        if si is not None:
            out = group(out, 0, None, S.shape[0], d["S"], HF_K_INDEX_MAP, 0, d["si"], d["sj"], d["om"])
            if G is not None:
                out = group(out, G.shape[0], d["G"], 0, None, HF_K_MOD, 0, None, None, None)
        elif G is not None and S is not None:
            out = group(out, G.shape[0], d["G"], S.shape[0], d["S"], s_conv, s_bits, None, None, None)
        elif G is not None:
            out = group(out, G.shape[0], d["G"], 0, None, HF_K_MOD, 0, None, None, None)
        elif S is not None:
            out = group(out, 1, d["I"], S.shape[0], d["S"], s_conv, s_bits, None, None, None)
        if U is not None:
            res = torch.empty_like(out)
            nk1, nk2, nb = int(out.shape[0]), int(out.shape[1]), int(out.shape[-1])
            mode = HF_K_INDEX_MAP if ti is not None else t_conv
            _lib.check(_lib.lib().hf_sym_time_reversal(
                _lib.stream_ptr(out.device), _lib.dtype_code(out), nk1, nk2, nb, out.data_ptr(), res.data_ptr(),
                d["U"].data_ptr(), mode, t_bits, _lib.ptr(d["ti"]), _lib.ptr(d["tj"]), _lib.ptr(d["tv"])))
            out = res
        return out

    return project


__all__ = ["ProjectFn", "make_project_fn"]
