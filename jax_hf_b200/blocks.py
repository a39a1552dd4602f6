"""Block-diagonal exchange specs on the GPU (utils.py:176-311, linalg.py:19-91).

Semantics of the reference: with ``block_specs`` the exchange is computed block by
block for the first spec whose off-block entries satisfy
``max|P - refP| * mask <= atol + rtol * max|P - refP|`` (or unconditionally with
``check_offdiag=False``); off-block channels of Sigma's exchange part are then
zero, while the Hartree and contact terms still see the whole density.

On the GPU (``hf_fock_build_block_specs``): one kernel evaluates the off-block
maxima of every spec in a single pass over P - refP, a one-thread kernel picks the
first compatible spec and sets a device flag, and the masked build of every spec
plus the full build are queued behind it; only the flagged candidate's kernels do
any work, so the host never waits.  A masked build (``hf_fock_build_blocks``)
transforms only the in-block channels, one slot group per block (two 4x4 blocks
of nb = 8: half of the channels), and writes the off-block channels in a separate
pass.  ``choose_spec`` is the host-side form of the same choice (one read).
"""

from __future__ import annotations

from typing import Any, Sequence

import numpy as np
import torch

from .problem import is_marked_zero


def _as_sequence(obj: Any) -> Sequence[Any]:
    if isinstance(obj, (list, tuple)):
        return obj
    if hasattr(obj, "tolist"):
        out = obj.tolist()
        if isinstance(out, list):
            return out
    raise TypeError(f"Expected a sequence; got {type(obj)}.")


def normalize_block_specs(block_specs):
    """Canonical (("sizes", ...), ("indices", ...)) form (linalg.py:19-91)."""
    if block_specs is None:
        return None
    items = (block_specs,) if isinstance(block_specs, dict) else block_specs
    if not isinstance(items, (list, tuple)):
        raise TypeError("block_specs must be a sequence of specs or a single spec dict; "
                        f"got {type(block_specs)}.")
    out = []
    for spec in items:
        if spec is None:
            raise TypeError("block_specs entries must be non-None.")
        if isinstance(spec, tuple) and len(spec) == 2 and isinstance(spec[0], str) and \
                spec[0].strip().lower() in ("sizes", "indices"):
            kind = spec[0].strip().lower()
            if kind == "sizes":
                out.append(("sizes", tuple(int(x) for x in _as_sequence(spec[1]))))
            else:
                out.append(("indices", tuple(tuple(int(i) for i in _as_sequence(b)) for b in _as_sequence(spec[1]))))
        elif isinstance(spec, dict):
            if "block_sizes" in spec:
                out.append(("sizes", tuple(int(x) for x in _as_sequence(spec["block_sizes"]))))
            elif "block_indices" in spec:
                out.append(("indices", tuple(tuple(int(i) for i in _as_sequence(b))
                                             for b in _as_sequence(spec["block_indices"]))))
            else:
                raise TypeError("Spec dict must contain 'block_sizes' or 'block_indices'.")
        else:
            seq = _as_sequence(spec)
            if len(seq) == 0:
                raise TypeError("Spec sequences must be non-empty.")
            if all(isinstance(x, (int, np.integer)) for x in seq):
                out.append(("sizes", tuple(int(x) for x in seq)))
            else:
                out.append(("indices", tuple(tuple(int(i) for i in _as_sequence(b)) for b in seq)))
    return tuple(out)


def inblock_mask(kind, data, n):
    """True on in-block channels (complement of utils.py:176-191)."""
    m = np.zeros((n, n), bool)
    if kind == "sizes":
        if sum(int(s) for s in data) != n:
            raise ValueError(f"block_sizes must sum to {n}.")
        start = 0
        for s in data:
            m[start:start + s, start:start + s] = True
            start += s
    else:
        for idx in data:
            idx = np.asarray(idx, int)
            m[np.ix_(idx, idx)] = True
    return m


_MASKS: dict = {}


def spec_masks(specs, n):
    """In-block masks (uint8, (len(specs), n, n)) of normalised specs; cached per (specs, n)."""
    key = (specs, int(n))
    m = _MASKS.get(key)
    if m is None:
        m = np.stack([inblock_mask(kind, data, n) for kind, data in specs]).astype(np.uint8)
        m = np.ascontiguousarray(m)
        _MASKS[key] = m
    return m


def choose_spec(P, refP, specs, masks, *, check, atol, rtol):
    """Index of the first spec whose off-block |P - refP| is within tolerance (utils.py:263-309),
    or None for the full build.  One device pass and one host read for all specs."""
    from . import _lib
    if not check:
        return 0
    n = int(P.shape[-1])
    nk = int(P.shape[0]) * int(P.shape[1])
    refPt = None if refP is None or is_marked_zero(refP) else refP
    out = torch.empty(len(specs) + 1, dtype=torch.float64, device=P.device)
    _lib.check(_lib.lib().hf_block_offdiag_max(
        _lib.stream_ptr(P.device), _lib.dtype_code(P), nk, n, P.data_ptr(), _lib.ptr(refPt), len(specs),
        masks.ctypes.data_as(_lib.C.c_void_p), out.data_ptr()))
    vals = out.cpu().numpy()
    tol = float(atol) + float(rtol) * float(vals[0])
    for i in range(len(specs)):
        if vals[i + 1] <= tol:
            return i
    return None


def build_fock_block_specs(P, *, h, VR, refP, HH, w2d, include_exchange, include_hartree,
                           exchange_hermitian_channel_packing, contact_g=None, contact_Oi=None, contact_Oj=None,
                           exchange_block_specs=None, exchange_check_offdiag=None, exchange_offdiag_atol=1e-12,
                           exchange_offdiag_rtol=0.0, project_fn=None, fft_precision=None):
    from .fock import build_fock
    specs = normalize_block_specs(exchange_block_specs)
    common = dict(h=h, VR=VR, refP=refP, HH=HH, w2d=w2d, include_hartree=include_hartree,
                  exchange_hermitian_channel_packing=exchange_hermitian_channel_packing, contact_g=contact_g,
                  contact_Oi=contact_Oi, contact_Oj=contact_Oj, project_fn=project_fn, fft_precision=fft_precision)
    if not specs or not include_exchange:
        return build_fock(P, include_exchange=include_exchange, **common)
    if len(specs) > 8:
        raise ValueError("at most 8 block specs are supported")
    n = int(P.shape[-1])
    masks = spec_masks(specs, n)
    check = bool(exchange_check_offdiag) if exchange_check_offdiag is not None else True
    if not check:                                                # the first spec, unconditionally
        return build_fock(P, include_exchange=True, _inblock=masks[0], **common)
    # the device picks the spec (or the full build): no host round trip
    return build_fock(P, include_exchange=True, _inblock=masks,
                      _spec_check=(float(exchange_offdiag_atol), float(exchange_offdiag_rtol)), **common)
