"""Fock build and HF objective on the GPU (drop-in for jax_hf.fock).

``build_fock``, ``hf_energy``, ``occupation_entropy`` and ``free_energy`` keep
the reference signatures (fock.py:18-129) and run the hand-written CUDA
kernels of ``lib/libhf_b200.so`` through the C ABI.  Inputs are CUDA torch
tensors (NumPy arrays are copied to the current device); scalars come back as
0-d float64 device tensors (FP64 accumulation).  There is no CPU fallback.

Differences in form, not in value:
* ``H`` is returned as an (1, 1, nb, nb) array that broadcasts over k (the
  reference returns that shape with Hartree on and a zero (nk1, nk2, nb, nb)
  array with it off).
* ``fft_precision="fp32"`` (extension) runs the exchange FFT of complex128
  inputs in FP32; everything else stays FP64.
* ``engine="generic"`` (extension, for testing) forces the shared-memory
  Stockham engine instead of the register FFT of the specialised mesh lengths;
  ``engine="tile"`` forces the 2x2-tile slot groups in the register engine;
  ``engine="pipe"`` runs the bulk-copy pipelined passes (nb in {4, 8} on
  register lengths; the default schedule elsewhere).
* ``autotune=True`` (extension) times the schedules that apply to this shape
  (``hf_fock_autotune``), keeps the fastest for every later build of the same
  shape and flags (solver drivers included) and records the timings in
  ``last_autotune``.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .problem import is_marked_zero


def _as_dev(x, device=None, dtype=None):
    if isinstance(x, torch.Tensor):
        t = x
        if device is not None and t.device != device:
            t = t.to(device)
    else:
        t = torch.as_tensor(np.asarray(x), device=device or torch.device("cuda", torch.cuda.current_device()))
    if dtype is not None and t.dtype != dtype:
        t = t.to(dtype)
    return t.contiguous()


# timings of the last build_fock(autotune=True): shape, flags, chosen schedule, us per candidate
last_autotune: dict = {}


def autotune_reset() -> None:
    """Forgets every schedule stored by build_fock(autotune=True)."""
    _lib.check(_lib.lib().hf_fock_autotune_reset())


def _herm(X: torch.Tensor) -> torch.Tensor:
    return 0.5 * (X + X.transpose(-1, -2).conj())


def _real_of(dt: torch.dtype) -> torch.dtype:
    return torch.float64 if dt in (torch.complex128, torch.float64) else torch.float32


_block_ws: dict = {}  # workspace sizes of block-spec builds, per (dtype, flags, shape, masks)


def build_fock(P, *, h, VR, refP, HH, w2d, include_exchange: bool, include_hartree: bool,
               exchange_hermitian_channel_packing: bool, contact_g=None, contact_Oi=None,
               contact_Oj=None, exchange_block_specs=None, exchange_check_offdiag=None,
               exchange_offdiag_atol: float = 1e-12, exchange_offdiag_rtol: float = 0.0,
               project_fn=None, fft_precision=None, engine=None, hermitian_density: bool = False, out=None,
               autotune: bool = False, autotune_reps: int = 5, _inblock=None, _spec_check=None):
    """Returns (Sigma, H, F) with F = herm(h + Sigma[P - refP] + H[P - refP]) (fock.py:18-97).

    Extensions (keyword-only, defaults keep the reference behaviour): ``fft_precision="fp32"``
    runs the exchange FFT in FP32; ``engine="generic"`` forces the shared-memory FFT engine;
    ``hermitian_density=True`` states that P (and refP) are Hermitian, which lets a kernel
    whose V(q) is real and symmetric in the band pair use the Hermitian channel packing
    (upper-triangle channels only) for a band-resolved V as well; ``out`` = (Sigma, H, F).
    ``_inblock`` (internal, set by the block-spec path) is an (nb, nb) uint8 in-block mask:
    the exchange is formed on those channels only (hf_fock_build_blocks); with
    ``_spec_check = (atol, rtol)`` it is a stack of masks, one per spec, and the device
    picks the first compatible one (hf_fock_build_block_specs).
    """
    h = _as_dev(h)
    dev = h.device
    _lib.require_cuda(h)
    cdt = h.dtype
    rdt = _real_of(cdt)
    P = _as_dev(P, dev, cdt)
    if P.shape != h.shape:
        raise ValueError(f"P must have shape {tuple(h.shape)}, got {tuple(P.shape)}")
    nk1, nk2, nb = int(h.shape[0]), int(h.shape[1]), int(h.shape[-1])
    if exchange_block_specs is not None:
        from .blocks import build_fock_block_specs
        return build_fock_block_specs(
            P, h=h, VR=VR, refP=refP, HH=HH, w2d=w2d, include_exchange=include_exchange,
            include_hartree=include_hartree,
            exchange_hermitian_channel_packing=exchange_hermitian_channel_packing,
            contact_g=contact_g, contact_Oi=contact_Oi, contact_Oj=contact_Oj,
            exchange_block_specs=exchange_block_specs, exchange_check_offdiag=exchange_check_offdiag,
            exchange_offdiag_atol=exchange_offdiag_atol, exchange_offdiag_rtol=exchange_offdiag_rtol,
            project_fn=project_fn, fft_precision=fft_precision)

    flags = 0
    sym_v = bool(getattr(VR, "_hf_v_pair_symmetric", False))
    if include_exchange:
        flags |= _lib.FOCK_EXCHANGE
    if include_hartree:
        flags |= _lib.FOCK_HARTREE
    VRt = None
    if include_exchange:
        VRt = VR if isinstance(VR, torch.Tensor) else torch.as_tensor(np.asarray(VR))
        VRt = VRt.to(dev)
        if VRt.is_complex():
            VRt = VRt.to(cdt).contiguous()
        else:
            VRt = VRt.to(rdt).contiguous()
            flags |= _lib.FOCK_VR_REAL
        if tuple(VRt.shape[-2:]) == (1, 1):
            flags |= _lib.FOCK_VR_SCALAR
        elif tuple(VRt.shape[-2:]) != (nb, nb):
            raise ValueError(f"VR must have shape (nk1, nk2, 1, 1) or (nk1, nk2, nb, nb), got {tuple(VRt.shape)}")
    if exchange_hermitian_channel_packing:
        if VRt is not None and tuple(VRt.shape[-2:]) != (1, 1):
            raise ValueError("hermitian_channel_packing requires a scalar interaction kernel with shape (..., 1, 1).")
        flags |= _lib.FOCK_PACKING
    elif hermitian_density and include_exchange and sym_v and exchange_block_specs is None:
        flags |= _lib.FOCK_PACKING | _lib.FOCK_SYM_V
    refPt = None
    if refP is not None and not is_marked_zero(refP):
        refPt = _as_dev(refP, dev, cdt)
        flags |= _lib.FOCK_HAS_REFP
    if engine is not None and str(engine).lower() == "generic":
        flags |= _lib.FOCK_GENERIC_FFT
    elif engine is not None and str(engine).lower() == "tile":
        flags |= _lib.FOCK_TILE_PLAN
    elif engine is not None and str(engine).lower() == "pipe":
        flags |= _lib.FOCK_PIPE
    if fft_precision is not None and str(fft_precision).lower() in ("fp32", "float32", "single"):
        if cdt == torch.complex128:
            flags |= _lib.FOCK_FFT_FP32
    HHt = _as_dev(HH, dev, rdt) if HH is not None else None
    w2dt = _as_dev(w2d, dev, rdt) if w2d is not None else None
    n_contact = 0
    cg = cOi = cOj = None
    if contact_g is not None and contact_Oi is not None and contact_Oj is not None and not is_marked_zero(contact_g):
        cg = _as_dev(contact_g, dev, rdt)
        cOi = _as_dev(contact_Oi, dev, cdt)
        cOj = _as_dev(contact_Oj, dev, cdt)
        n_contact = int(cg.shape[0])

    if out is not None:
        Sigma, H, F = out
    else:
        Sigma = torch.empty_like(P)
        F = torch.empty_like(P)
        H = torch.empty((1, 1, nb, nb), dtype=cdt, device=dev)
    dt = _lib.dtype_code(P)
    need = _lib.C.c_size_t(0)
    if _inblock is not None and _spec_check is not None:
        masks = np.ascontiguousarray(np.asarray(_inblock, dtype=np.uint8).reshape(-1, nb, nb))
        mptr = masks.ctypes.data_as(_lib.C.c_void_p)
        ns = int(masks.shape[0])
        key = ("specs", dt, flags, nk1, nk2, nb, masks.tobytes())
        if key not in _block_ws:
            _lib.check(_lib.lib().hf_fock_block_specs_workspace_size(dt, flags, nk1, nk2, nb, ns, mptr,
                                                                     _lib.C.byref(need)))
            _block_ws[key] = int(need.value)
        ws = _lib.workspace(_block_ws[key], dev, "fock")
        _lib.check(_lib.lib().hf_fock_build_block_specs(
            _lib.stream_ptr(dev), dt, flags, nk1, nk2, nb, ns, mptr, float(_spec_check[0]), float(_spec_check[1]),
            P.data_ptr(), h.data_ptr(), _lib.ptr(VRt), _lib.ptr(refPt), _lib.ptr(HHt), _lib.ptr(w2dt), n_contact,
            _lib.ptr(cg), _lib.ptr(cOi), _lib.ptr(cOj), Sigma.data_ptr(), H.data_ptr(), F.data_ptr(), ws.data_ptr(),
            ws.numel(), None))
        if project_fn is not None:
            F = _herm(torch.as_tensor(project_fn(F)).to(cdt))
        return Sigma, H, F
    if _inblock is not None:
        mask = np.ascontiguousarray(np.asarray(_inblock, dtype=np.uint8).reshape(nb, nb))
        mptr = mask.ctypes.data_as(_lib.C.c_void_p)
        key = ("mask", dt, flags, nk1, nk2, nb, mask.tobytes())
        if key not in _block_ws:
            _lib.check(_lib.lib().hf_fock_blocks_workspace_size(dt, flags, nk1, nk2, nb, mptr, _lib.C.byref(need)))
            _block_ws[key] = int(need.value)
        ws = _lib.workspace(_block_ws[key], dev, "fock")
        _lib.check(_lib.lib().hf_fock_build_blocks(
            _lib.stream_ptr(dev), dt, flags, nk1, nk2, nb, mptr, P.data_ptr(), h.data_ptr(), _lib.ptr(VRt),
            _lib.ptr(refPt), _lib.ptr(HHt), _lib.ptr(w2dt), n_contact, _lib.ptr(cg), _lib.ptr(cOi), _lib.ptr(cOj),
            Sigma.data_ptr(), H.data_ptr(), F.data_ptr(), ws.data_ptr(), ws.numel()))
        if project_fn is not None:
            F = _herm(torch.as_tensor(project_fn(F)).to(cdt))
        return Sigma, H, F
    _lib.check(_lib.lib().hf_fock_workspace_size(dt, flags, nk1, nk2, nb, _lib.C.byref(need)))
    ws = _lib.workspace(need.value, dev, "fock")
    args = (_lib.stream_ptr(dev), dt, flags, nk1, nk2, nb, P.data_ptr(), h.data_ptr(), _lib.ptr(VRt),
            _lib.ptr(refPt), _lib.ptr(HHt), _lib.ptr(w2dt), n_contact, _lib.ptr(cg), _lib.ptr(cOi),
            _lib.ptr(cOj), Sigma.data_ptr(), H.data_ptr(), F.data_ptr(), ws.data_ptr(), ws.numel())
    if autotune:
        chosen = _lib.C.c_uint(0)
        us = (_lib.C.c_float * 4)()
        _lib.check(_lib.lib().hf_fock_autotune(*args, int(autotune_reps), _lib.C.byref(chosen), us))
        names = ("default", "tile", "generic", "pipe")
        pick = {0: "default", _lib.FOCK_TILE_PLAN: "tile", _lib.FOCK_GENERIC_FFT: "generic",
                _lib.FOCK_PIPE: "pipe"}[chosen.value]
        last_autotune.clear()
        last_autotune.update(shape=(nk1, nk2, nb), flags=flags, chosen=pick,
                             us={n: float(v) for n, v in zip(names, us) if v >= 0})
    else:
        _lib.check(_lib.lib().hf_fock_build(*args))
    if project_fn is not None:
        F = _herm(torch.as_tensor(project_fn(F)).to(cdt))
    return Sigma, H, F


_batch_streams: dict = {}


def build_fock_batch(Ps, *, h, VR, refP, HH, w2d, include_exchange: bool, include_hartree: bool,
                     exchange_hermitian_channel_packing: bool, contact_g=None, contact_Oi=None,
                     contact_Oj=None, fft_precision=None, outs=None, streams: int = 3):
    """Fock builds of several independent densities that share one kernel (no reference counterpart).

    Returns ``[build_fock(P, ...) for P in Ps]`` (each result bit-identical to the single
    call).  The builds are spread over ``streams`` internal CUDA streams forked from and
    joined back into the caller's current stream, so the passes of one build fill the
    SMs that another build's passes leave idle (the last round of a pass, its memory-
    or FP64-bound phases): a density scan or any batch of independent builds runs at a
    higher rate than the same builds one after another (192x192, nb = 8, complex128 on a
    B200: 81.4 us per build on one stream, 68.0 on two, 65.5 on three, 66.6 on four).
    Each stream has its own workspace.  ``outs``: optional list of (Sigma, H, F) per
    density; build i uses stream i % streams, so an output set shared by builds i and
    i + k * streams is written in order.
    """
    Ps = list(Ps)
    if outs is not None and len(outs) != len(Ps):
        raise ValueError(f"outs has {len(outs)} entries for {len(Ps)} densities")
    h = _as_dev(h)
    dev = h.device
    _lib.require_cuda(h)
    n = max(1, min(int(streams), len(Ps)))
    pool = _batch_streams.setdefault(str(dev), [])
    while len(pool) < n:
        pool.append(torch.cuda.Stream(dev))
    kw = dict(h=h, VR=VR, refP=refP, HH=HH, w2d=w2d, include_exchange=include_exchange,
              include_hartree=include_hartree,
              exchange_hermitian_channel_packing=exchange_hermitian_channel_packing, contact_g=contact_g,
              contact_Oi=contact_Oi, contact_Oj=contact_Oj, fft_precision=fft_precision)
    caller = torch.cuda.current_stream(dev)
    if outs is None:
        cdt = h.dtype
        nb = int(h.shape[-1])
        outs = [(torch.empty_like(h), torch.empty((1, 1, nb, nb), dtype=cdt, device=dev), torch.empty_like(h))
                for _ in Ps]
    Pd = [_as_dev(P, dev, h.dtype) for P in Ps]  # copies (if any) are made on the caller's stream
    for s in pool[:n]:
        s.wait_stream(caller)
    results = []
    for i, P in enumerate(Pd):
        with torch.cuda.stream(pool[i % n]):
            results.append(build_fock(P, out=outs[i], **kw))
    for s in pool[:n]:
        caller.wait_stream(s)  # inputs, outputs and results are ordered on the caller's stream again
    return results


def _reduce_ws(dev):
    need = _lib.C.c_size_t(0)
    _lib.check(_lib.lib().hf_reduce_workspace_size(1, 1, 1, _lib.C.byref(need)))
    return _lib.workspace(need.value, dev, "reduce")


def hf_energy(P, *, h, Sigma, H, weights_b, out=None):
    """E = sum_k w_k Re Tr[(h + (Sigma + H)/2) P] in FP64 (fock.py:100-111)."""
    h = _as_dev(h)
    dev = h.device
    cdt = h.dtype
    P = _as_dev(P, dev, cdt)
    Sigma = _as_dev(Sigma, dev, cdt)
    nk1, nk2, nb = int(h.shape[0]), int(h.shape[1]), int(h.shape[-1])
    H_mode, Ht = 0, None
    if H is not None and not is_marked_zero(H):
        Ht = _as_dev(H, dev, cdt)
        if Ht.numel() == nb * nb:
            H_mode = 1
        elif tuple(Ht.shape) == tuple(h.shape):
            H_mode = 2
        else:
            Ht = Ht.expand(h.shape).contiguous()
            H_mode = 2
    w = _as_dev(weights_b, dev, _real_of(cdt)).reshape(nk1, nk2).contiguous()
    E = out if out is not None else torch.empty((), dtype=torch.float64, device=dev)
    ws = _reduce_ws(dev)
    _lib.check(_lib.lib().hf_energy(_lib.stream_ptr(dev), _lib.dtype_code(P), nk1, nk2, nb, P.data_ptr(),
                                    h.data_ptr(), Sigma.data_ptr(), _lib.ptr(Ht), H_mode, w.data_ptr(),
                                    E.data_ptr(), ws.data_ptr(), ws.numel()))
    return E


def occupation_entropy(p, w_norm, out=None):
    """S = -sum w [p log p + (1-p) log1p(-p)] with p clipped to [1e-14, 1-1e-14] (fock.py:114-118)."""
    p = _as_dev(p)
    dev = p.device
    w = _as_dev(w_norm, dev, p.dtype)
    nb = int(p.shape[-1])
    nk = p.numel() // nb
    S = out if out is not None else torch.empty((), dtype=torch.float64, device=dev)
    ws = _reduce_ws(dev)
    _lib.check(_lib.lib().hf_occupation_entropy(_lib.stream_ptr(dev), _lib.dtype_code(p), nk, 1, nb,
                                                p.data_ptr(), w.data_ptr(), S.data_ptr(), ws.data_ptr(),
                                                ws.numel()))
    return S


def free_energy(E, p, w_norm, T, out=None):
    """Omega = E - max(T, 1e-14) S(p) (fock.py:121-129)."""
    p = _as_dev(p)
    dev = p.device
    w = _as_dev(w_norm, dev, p.dtype)
    nb = int(p.shape[-1])
    nk = p.numel() // nb
    Et = E if isinstance(E, torch.Tensor) else torch.tensor(float(E), dtype=torch.float64, device=dev)
    Et = Et.to(dev, torch.float64).reshape(()).contiguous()
    Om = out if out is not None else torch.empty((), dtype=torch.float64, device=dev)
    ws = _reduce_ws(dev)
    _lib.check(_lib.lib().hf_free_energy(_lib.stream_ptr(dev), _lib.dtype_code(p), nk, 1, nb, Et.data_ptr(),
                                         p.data_ptr(), w.data_ptr(), float(T), Om.data_ptr(), ws.data_ptr(),
                                         ws.numel()))
    return Om
