"""Block-diagonal exchange specs on the GPU (utils.py:176-311, linalg.py:19-91).

Semantics of the reference: with ``block_specs`` the exchange is computed block by
block for the first spec whose off-block entries satisfy
``max|P| * mask <= atol + rtol * max|P|`` (or unconditionally with
``check_offdiag=False``); off-block channels of Sigma are then zero, while the
contact and Hartree terms still see the whole density.  Because exchange
channels are independent, the block result is the CUDA exchange of the
in-block channels of P - refP; off-block channels contribute nothing.  The
contact term is added from the full density afterwards.
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


def build_fock_block_specs(P, *, h, VR, refP, HH, w2d, include_exchange, include_hartree,
                           exchange_hermitian_channel_packing, contact_g=None, contact_Oi=None, contact_Oj=None,
                           exchange_block_specs=None, exchange_check_offdiag=None, exchange_offdiag_atol=1e-12,
                           exchange_offdiag_rtol=0.0, project_fn=None, fft_precision=None):
    from .fock import build_fock, _herm
    specs = normalize_block_specs(exchange_block_specs)
    common = dict(h=h, VR=VR, HH=HH, w2d=w2d, include_hartree=include_hartree,
                  exchange_hermitian_channel_packing=exchange_hermitian_channel_packing,
                  fft_precision=fft_precision)
    if not specs or not include_exchange:
        return build_fock(P, refP=refP, include_exchange=include_exchange, contact_g=contact_g,
                          contact_Oi=contact_Oi, contact_Oj=contact_Oj, project_fn=project_fn, **common)
    n = int(P.shape[-1])
    check = bool(exchange_check_offdiag) if exchange_check_offdiag is not None else True
    chosen = None
    if check:
        absP = P.abs()
        tol = float(exchange_offdiag_atol) + float(exchange_offdiag_rtol) * float(absP.max())
        for kind, data in specs:
            off = torch.as_tensor(~inblock_mask(kind, data, n), device=P.device)
            if float((absP * off).max()) <= tol:
                chosen = (kind, data)
                break
    else:
        chosen = specs[0]
    if chosen is None:                                           # no compatible spec: full path
        return build_fock(P, refP=refP, include_exchange=True, contact_g=contact_g, contact_Oi=contact_Oi,
                          contact_Oj=contact_Oj, project_fn=project_fn, **common)
    mask = torch.as_tensor(inblock_mask(*chosen, n), device=P.device).to(P.dtype)
    Pm = P * mask
    refm = None if refP is None or is_marked_zero(refP) else refP * mask
    Sg, H, F = build_fock(Pm, refP=refm, include_exchange=True, **common)
    if include_hartree and refm is not None:
        pass  # the Hartree term only reads diagonal channels, which are in-block
    has_contact = contact_g is not None and contact_Oi is not None and contact_Oj is not None and \
        not is_marked_zero(contact_g)
    if has_contact:
        dP = P if refP is None or is_marked_zero(refP) else P - refP
        rho = torch.einsum("ij,ijab->ab", w2d.to(P.dtype), dP)
        tr = torch.einsum("tij,ji->t", contact_Oj, rho)
        s_h = torch.einsum("t,tij->ij", contact_g.to(P.dtype) * tr, contact_Oi)
        s_f = torch.einsum("t,tij->ij", -contact_g.to(P.dtype),
                           torch.einsum("tik,tkl->til", torch.einsum("tij,jk->tik", contact_Oi, rho), contact_Oj))
        sc = (s_h + s_f)[None, None]
        Sg = Sg + sc
        F = F + _herm(sc.expand_as(F))
    if project_fn is not None:
        F = _herm(torch.as_tensor(project_fn(F)).to(P.dtype))
    return Sg, H, F
