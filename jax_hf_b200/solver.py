"""Direct-minimisation solver on the GPU (drop-in for jax_hf.solver).

``solve(kernel, P0, n_electrons, config=SolverConfig())`` keeps the reference
signature and result type (solver.py:240-298, 1098-1251).  With
``optimizer="cg"`` the whole Riemannian-CG loop runs on the device through
``hf_cg_solve`` (one C-ABI call per solve); ``optimizer="newton"`` runs the
trust-region Newton loop of ``newton.py``.

Extensions (keyword-only, default off): ``SolverConfig.fp32_exchange`` turns on
the mixed-precision mode (FP32 exchange FFT, FP64 defect-correction builds at
the end); ``SolverConfig.chunk`` is the number of iterations queued between
host checks of the device stop flag.
"""

from __future__ import annotations

import ctypes as C
import warnings
from dataclasses import dataclass
from typing import Any, NamedTuple

import numpy as np
import torch

from . import _lib
from .problem import is_marked_zero
from .utils import validate_electron_count


@dataclass(frozen=True)
class SolverConfig:
    """solver.py:240-286 (same fields and defaults) + mixed-precision knobs."""
    max_iter: int = 200
    tol_E: float = 1e-7
    tol_grad: float = 0.0
    denom_scale: float = 1e-3
    max_step: float = 0.6
    cg_restart: int = 10
    bt_shrink: float = 0.5
    bt_max: int = 8
    mu_maxiter: int = 25
    plateau_window: int = 5
    optimizer: str = "cg"
    tr_delta0: float = 0.5
    tr_cg_max: int = 20
    deflation_targets: Any = None
    deflation_sigma: float = 0.0
    deflation_length: float = 1.0
    block_sizes: tuple | None = None
    project_fn: Any = None
    fp32_exchange: bool = False
    fp32_switch_rel: float = 3e-7
    chunk: int = 4
    # polish="scf": after the CG loop, an FP64 SCF-DIIS run from its density to the
    # self-consistent fixed point (density residual <= polish_density_tol); the CG's
    # plateau stop ends 1e-9 .. 1e-6 (relative) above that point in energy
    polish: str = "none"
    polish_density_tol: float = 1e-8
    polish_comm_tol: float = 1e-7
    polish_max_iter: int = 100
    # an FP64 reference solution (energy, and optionally density) to report errors against
    reference_energy: float | None = None
    reference_density: Any = None


class SolveResult(NamedTuple):
    Q: torch.Tensor
    p: torch.Tensor
    mu: torch.Tensor
    density: torch.Tensor
    fock: torch.Tensor
    energy: torch.Tensor
    n_iter: torch.Tensor
    converged: torch.Tensor
    history: dict


class _CgProblem(C.Structure):
    _fields_ = [("nk1", C.c_int), ("nk2", C.c_int), ("nb", C.c_int), ("fock_flags", C.c_uint),
                ("T", C.c_double), ("n_electrons", C.c_double), ("weight_sum", C.c_double),
                ("h", C.c_void_p), ("VR", C.c_void_p), ("refP", C.c_void_p), ("HH", C.c_void_p),
                ("w2d", C.c_void_p), ("n_contact", C.c_int), ("contact_g", C.c_void_p),
                ("contact_Oi", C.c_void_p), ("contact_Oj", C.c_void_p), ("sigma_buf", C.c_void_p),
                ("h_buf", C.c_void_p)]


FOCK_CB = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p)
PROJECT_CB = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_void_p)


class _CgConfig(C.Structure):
    _fields_ = [("max_iter", C.c_int), ("tol_E", C.c_double), ("tol_grad", C.c_double),
                ("denom_scale", C.c_double), ("max_step", C.c_double), ("cg_restart", C.c_int),
                ("bt_shrink", C.c_double), ("bt_max", C.c_int), ("mu_maxiter", C.c_int),
                ("plateau_window", C.c_int), ("fp32_exchange", C.c_int), ("fp32_switch_rel", C.c_double),
                ("chunk", C.c_int), ("fock_cb", FOCK_CB), ("project_cb", PROJECT_CB), ("cb_user", C.c_void_p)]


def _bind():
    L = _lib.lib()
    if not getattr(L, "_cg_bound", False):
        L.hf_cg_workspace_size.argtypes = [C.POINTER(_CgProblem), C.POINTER(_CgConfig), C.POINTER(C.c_size_t)]
        L.hf_cg_workspace_size.restype = C.c_int
        L.hf_cg_solve.argtypes = [C.c_void_p, C.POINTER(_CgProblem), C.POINTER(_CgConfig), C.c_void_p, C.c_void_p,
                                  C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.c_void_p, C.c_size_t]
        L.hf_cg_solve.restype = C.c_int
        L._cg_bound = True
    return L


class KernelC128:
    """complex128 views of a kernel's arrays for the device solvers (kept alive with the problem)."""

    def __init__(self, kernel):
        self.kernel = kernel
        up = kernel.dtype != torch.complex128
        cd, rd = torch.complex128, torch.float64
        self.h = kernel.h.to(cd).contiguous() if up else kernel.h
        VR = kernel._VR_shifted
        self.VR = (VR.to(rd) if not VR.is_complex() else VR.to(cd)).contiguous() if up else VR
        self.refP = None if is_marked_zero(kernel.refP) else kernel.refP.to(cd).contiguous()
        self.HH = kernel.HH.to(rd).contiguous()
        self.w2d = kernel.w2d.to(rd).contiguous()
        self.has_contact = kernel.has_contact
        self.cg = kernel.contact_g.to(rd).contiguous()
        self.cOi = kernel.contact_Oi.to(cd).contiguous()
        self.cOj = kernel.contact_Oj.to(cd).contiguous()

    def flags(self):
        k = self.kernel
        f = 0
        if k.include_exchange:
            f |= _lib.FOCK_EXCHANGE
            if not self.VR.is_complex():
                f |= _lib.FOCK_VR_REAL
            if tuple(self.VR.shape[-2:]) == (1, 1):
                f |= _lib.FOCK_VR_SCALAR
        if k.include_hartree:
            f |= _lib.FOCK_HARTREE
        if k.exchange_hermitian_channel_packing:
            f |= _lib.FOCK_PACKING
        if self.refP is not None:
            f |= _lib.FOCK_HAS_REFP
        return f

    def problem(self, n_electrons):
        k = self.kernel
        nk1, nk2, nb = k.shape
        return _CgProblem(nk1, nk2, nb, self.flags(), float(k.T), float(n_electrons), float(k.weight_sum),
                          self.h.data_ptr(), self.VR.data_ptr(), _lib.ptr(self.refP), self.HH.data_ptr(),
                          self.w2d.data_ptr(), int(self.cg.shape[0]) if self.has_contact else 0,
                          self.cg.data_ptr(), self.cOi.data_ptr(), self.cOj.data_ptr(), None, None)

    def autotune(self, P, fp32: bool = False, reps: int = 5) -> int:
        """Runs hf_fock_autotune for this kernel's Fock flags (the ones the CG driver uses) on P
        (nk1, nk2, nb, nb) complex128; returns the chosen engine flags."""
        k = self.kernel
        nk1, nk2, nb = k.shape
        dev = self.h.device
        P = torch.as_tensor(P).to(dev, torch.complex128).contiguous()
        flags = self.flags() | (_lib.FOCK_FFT_FP32 if fp32 else 0)
        S, F = torch.empty_like(P), torch.empty_like(P)
        H = torch.empty((nb, nb), dtype=torch.complex128, device=dev)
        need = C.c_size_t(0)
        _lib.check(_lib.lib().hf_fock_workspace_size(_lib.HF_C128, flags, nk1, nk2, nb, C.byref(need)))
        ws = torch.empty(max(int(need.value), 256), dtype=torch.uint8, device=dev)
        chosen = C.c_uint(0)
        _lib.check(_lib.lib().hf_fock_autotune(
            _lib.stream_ptr(dev), _lib.HF_C128, flags, nk1, nk2, nb, P.data_ptr(), self.h.data_ptr(),
            self.VR.data_ptr(), _lib.ptr(self.refP), self.HH.data_ptr(), self.w2d.data_ptr(),
            int(self.cg.shape[0]) if self.has_contact else 0, self.cg.data_ptr(), self.cOi.data_ptr(),
            self.cOj.data_ptr(), S.data_ptr(), H.data_ptr(), F.data_ptr(), ws.data_ptr(), ws.numel(), int(reps),
            C.byref(chosen), None))
        return int(chosen.value)

    def fock_kwargs(self):
        k = self.kernel
        return dict(h=self.h, VR=self.VR, refP=k.refP if self.refP is None else self.refP, HH=self.HH, w2d=self.w2d,
                    include_exchange=k.include_exchange, include_hartree=k.include_hartree,
                    exchange_hermitian_channel_packing=k.exchange_hermitian_channel_packing,
                    contact_g=k.contact_g if not self.has_contact else self.cg,
                    contact_Oi=self.cOi, contact_Oj=self.cOj)


def _solve_cg(kernel, P0, n_electrons, cfg: SolverConfig, fock_build_fn=None):
    L = _bind()
    dev = kernel.device
    nk1, nk2, nb = kernel.shape
    kc = KernelC128(kernel)
    prob = kc.problem(n_electrons)
    conf = _CgConfig(int(cfg.max_iter), float(cfg.tol_E), float(cfg.tol_grad), float(cfg.denom_scale),
                     float(cfg.max_step), int(cfg.cg_restart), float(cfg.bt_shrink), int(cfg.bt_max),
                     int(cfg.mu_maxiter), int(cfg.plateau_window), int(bool(cfg.fp32_exchange)),
                     float(cfg.fp32_switch_rel), int(cfg.chunk), FOCK_CB(), PROJECT_CB(), None)
    need = C.c_size_t(0)
    _lib.check(L.hf_cg_workspace_size(C.byref(prob), C.byref(conf), C.byref(need)))
    ws = _lib.workspace(need.value, dev, "cg")
    P0t = torch.as_tensor(P0).to(dev, torch.complex128).contiguous() if not (
        isinstance(P0, torch.Tensor) and P0.dtype == torch.complex128 and P0.device == dev) else P0.contiguous()
    Q = torch.empty((nk1, nk2, nb, nb), dtype=torch.complex128, device=dev)
    p = torch.empty((nk1, nk2, nb), dtype=torch.float64, device=dev)
    P = torch.empty_like(Q)
    F = torch.empty_like(Q)
    hE = torch.zeros(max(cfg.max_iter, 1), dtype=torch.float64, device=dev)
    hG = torch.zeros(max(cfg.max_iter, 1), dtype=torch.float64, device=dev)
    sc = torch.zeros(8, dtype=torch.float64, device=dev)
    errors = []
    if cfg.project_fn is not None or cfg.block_sizes is not None or fock_build_fn is not None:
        # Python hooks: the loop stays on the device, the callbacks enqueue their work on the same stream
        Sg_t = torch.empty_like(Q)
        H_t = torch.zeros((nb, nb), dtype=torch.complex128, device=dev)
        prob.sigma_buf, prob.h_buf = Sg_t.data_ptr(), H_t.data_ptr()
        fn = fock_build_fn
        if fn is None:
            from .fock import build_fock as fn
        specs = None if cfg.block_sizes is None else (("sizes", tuple(int(s) for s in cfg.block_sizes)),)
        fkw = kc.fock_kwargs()
        calls = [0]

        def fock_cb(user, stream, Pp, Sp, Hp, Fp):
            try:
                first = calls[0] == 0
                calls[0] += 1
                Sg, Hh, Fn = fn(P, exchange_block_specs=specs, project_fn=cfg.project_fn if first else None, **fkw)
                Sg_t.copy_(Sg)
                Hh = torch.as_tensor(Hh).to(dev, torch.complex128)
                H_t.copy_(Hh.reshape(-1, nb, nb)[0] if Hh.numel() >= nb * nb else Hh.expand(nb, nb))
                F.copy_(Fn)
                return 0
            except Exception as exc:  # re-raised after the C call returns
                errors.append(exc)
                return _lib.HF_ERR_ABORTED

        def project_cb(user, stream, Pp):
            try:
                X = torch.as_tensor(cfg.project_fn(P)).to(dev, torch.complex128)
                P.copy_(0.5 * (X + X.transpose(-1, -2).conj()))
                return 0
            except Exception as exc:
                errors.append(exc)
                return _lib.HF_ERR_ABORTED

        conf.fock_cb = FOCK_CB(fock_cb)
        if cfg.project_fn is not None:
            conf.project_cb = PROJECT_CB(project_cb)
        _keep = (conf.fock_cb, conf.project_cb)
    st = L.hf_cg_solve(_lib.stream_ptr(dev), C.byref(prob), C.byref(conf), P0t.data_ptr(), Q.data_ptr(),
                             p.data_ptr(), P.data_ptr(), F.data_ptr(), hE.data_ptr(), hG.data_ptr(), sc.data_ptr(),
                             ws.data_ptr(), ws.numel())
    if errors:
        raise errors[0]
    _lib.check(st)
    out_c = kernel.dtype
    out_r = kernel.real_dtype
    s = sc.cpu().numpy()
    hist = dict(E=hE[:cfg.max_iter].to(out_r), grad_norm=hG[:cfg.max_iter].to(out_r))
    res = SolveResult(Q=Q.to(out_c), p=p.to(out_r), mu=sc[0].to(out_r), density=P.to(out_c), fock=F.to(out_c),
                      energy=sc[1].clone(), n_iter=torch.tensor(int(s[2]), dtype=torch.int32),
                      converged=torch.tensor(bool(s[3])), history=hist)
    res.history["fp32_switch_iter"] = int(s[5])
    return _finish(kernel, res, n_electrons, cfg)


def _polish(kernel, res: SolveResult, n_electrons, cfg: SolverConfig) -> SolveResult:
    """FP64 SCF-DIIS from the CG density to the fixed point (the library's SCF driver, Newton
    mu warm-started from the previous iteration); orbitals and occupations from eigh(F)."""
    from .reference_scf import SCFConfig, solve_scf
    r = solve_scf(kernel, res.density, n_electrons,
                  config=SCFConfig(acceleration="diis", density_tol=float(cfg.polish_density_tol),
                                   comm_tol=float(cfg.polish_comm_tol), max_iter=int(cfg.polish_max_iter),
                                   mu_method="newton", warm_eigh=True))
    return _from_scf(kernel, r, res.n_iter, res.history, float(res.energy))


def _from_scf(kernel, r, n_iter, history, cg_energy):
    from .linalg import eigh
    eps, Q = eigh(r.fock_matrix)
    T = max(float(kernel.T), 1e-12)
    mu = torch.as_tensor(r.chemical_potential, dtype=torch.float64, device=eps.device)
    p = torch.sigmoid((mu - eps.to(torch.float64)) / T)
    hist = dict(history)
    hist.update(polish_iterations=int(r.iterations), polish_converged=bool(r.converged), cg_energy=cg_energy)
    return SolveResult(Q=Q.to(kernel.dtype), p=p.to(kernel.real_dtype), mu=mu.to(kernel.real_dtype),
                       density=r.density_matrix.to(kernel.dtype), fock=r.fock_matrix.to(kernel.dtype),
                       energy=torch.as_tensor(r.energy, dtype=torch.float64), n_iter=n_iter,
                       converged=torch.tensor(bool(r.converged)), history=hist)


def _report(res: SolveResult, cfg: SolverConfig) -> SolveResult:
    """Errors against a supplied FP64 reference solution, in the history."""
    if cfg.reference_energy is not None:
        Eref = float(cfg.reference_energy)
        res.history["rel_dE_vs_reference"] = abs(float(res.energy) - Eref) / max(abs(Eref), 1e-300)
    if cfg.reference_density is not None:
        D = torch.as_tensor(cfg.reference_density).to(res.density.device, res.density.dtype)
        res.history["max_abs_dP_vs_reference"] = float((res.density - D).abs().max())
    return res


def _finish(kernel, res, n_electrons, cfg):
    if str(cfg.polish).lower() == "scf":
        res = _polish(kernel, res, n_electrons, cfg)
    elif str(cfg.polish).lower() != "none":
        raise ValueError(f"SolverConfig.polish must be 'none' or 'scf'; got {cfg.polish!r}")
    return _report(res, cfg)


def solve_direct_minimization(kernel, P0, n_electrons: float, *, config: SolverConfig | None = None,
                              fock_build_fn=None) -> SolveResult:
    """Direct-minimisation HF solver (solver.py:1098-1247)."""
    if config is None:
        config = SolverConfig()
    validate_electron_count(kernel.w2d, kernel.h.shape[-1], n_electrons, context="n_electrons")
    optimizer = str(config.optimizer).lower()
    if optimizer not in ("cg", "newton"):
        raise ValueError(f"Unknown optimizer {config.optimizer!r}; expected 'cg' or 'newton'.")
    deflation_on = config.deflation_targets is not None and float(config.deflation_sigma) > 0.0
    if deflation_on and optimizer != "newton":
        raise ValueError("deflation is only supported with optimizer='newton' "
                         f"(got optimizer={config.optimizer!r}).")
    if optimizer == "newton":
        if kernel.real_dtype != torch.float64:
            warnings.warn(
                "optimizer='newton' needs float64 precision to converge reliably; the kernel is float32. "
                "Build the kernel in complex128. The CG optimizer works in float32.", stacklevel=2)
        from .newton import solve_newton
        return solve_newton(kernel, P0, n_electrons, config, fock_build_fn)
    return _solve_cg(kernel, P0, n_electrons, config, fock_build_fn)


solve = solve_direct_minimization


class _CgBatchItem(C.Structure):
    _fields_ = [("problem", _CgProblem), ("P0", C.c_void_p), ("Q", C.c_void_p), ("p", C.c_void_p),
                ("density", C.c_void_p), ("fock", C.c_void_p), ("hist_E", C.c_void_p), ("hist_grad", C.c_void_p),
                ("scalars_out", C.c_void_p)]


def solve_batch(kernels, P0s, n_electrons, *, config: SolverConfig | None = None, lanes: int = 8,
                return_times: bool = False, autotune: bool = False, graph: bool = False):
    """Many independent CG solves in one native call (density scans).

    ``kernels``, ``P0s`` and ``n_electrons`` are equal-length sequences; each
    solve has the semantics of ``solve(kernel, P0, n, config=config)`` with
    ``optimizer="cg"`` and no hooks.  The C driver runs ``lanes`` solves at a
    time, each on its own stream with CUDA-graph iterations, longest first.
    Returns the list of ``SolveResult`` (and, with ``return_times``, each
    solve's device time in ms from its start to its final scalars).
    ``autotune=True`` first runs the Fock-schedule autotuner (``hf_fock_autotune``) once for
    every distinct (mesh, nb, Fock flags) of the scan, on that solve's P0; the stored choices
    then apply to every build of the batch.
    ``graph=True`` runs the whole batch as one CUDA graph launched once
    (``hf_cg_solve_batch_graph``): every solve a branch whose iteration loop is a
    device-side conditional node, all solves at once with a workspace each (``lanes``
    is then unused); the results are those of the stream driver.
    """
    cfg = config or SolverConfig()
    if str(cfg.optimizer).lower() != "cg":
        raise ValueError("solve_batch runs the CG optimizer only.")
    if cfg.project_fn is not None or cfg.block_sizes is not None or cfg.deflation_targets is not None:
        raise ValueError("solve_batch takes no project_fn, block_sizes or deflation hooks.")
    n = len(kernels)
    if n == 0 or len(P0s) != n or len(n_electrons) != n:
        raise ValueError("kernels, P0s and n_electrons must be non-empty and of equal length.")
    L = _lib.lib()
    dev = kernels[0].device
    if autotune:
        _autotune_scan(kernels, P0s, cfg)
    items, outs, keep, scs, conf, per_lane = _batch_items(kernels, P0s, n_electrons, cfg)
    lanes = max(1, min(int(lanes), n))
    times = (C.c_double * n)()
    if graph:
        # one workspace per solve, released on return (not kept in the workspace cache)
        ws = torch.empty(max(n * per_lane, 256), dtype=torch.uint8, device=dev)
        _lib.check(L.hf_cg_solve_batch_graph(_lib.stream_ptr(dev), items, n, C.byref(conf), ws.data_ptr(),
                                             per_lane, times))
    else:
        ws = _lib.workspace(lanes * per_lane, dev, "cg_batch")
        _lib.check(L.hf_cg_solve_batch(_lib.stream_ptr(dev), items, n, C.byref(conf), lanes, ws.data_ptr(),
                                       per_lane, times))
    results = _batch_results(outs, scs, cfg)
    del keep
    times = list(times)
    if str(cfg.polish).lower() == "scf":
        # the FP64 polish of every solve, on concurrent streams (one host thread each)
        from .reference_scf import SCFConfig, solve_scf_batch
        pol = solve_scf_batch(kernels, [r.density for r in results], list(n_electrons),
                              config=SCFConfig(acceleration="diis", density_tol=float(cfg.polish_density_tol),
                                               comm_tol=float(cfg.polish_comm_tol),
                                               max_iter=int(cfg.polish_max_iter), mu_method="newton",
                                               warm_eigh=True),
                              workers=lanes, return_times=True)
        results = [_from_scf(k, r, res.n_iter, res.history, float(res.energy))
                   for k, r, res in zip(kernels, pol[0], results)]
        times = [a + b for a, b in zip(times, pol[1])]
    return (results, times) if return_times else results


def _autotune_scan(kernels, P0s, cfg):
    seen = set()
    for kern, P0 in zip(kernels, P0s):
        kc = KernelC128(kern)
        for fp32 in ((False, True) if cfg.fp32_exchange else (False,)):
            key = (tuple(kern.shape), kc.flags(), fp32)
            if key not in seen:
                seen.add(key)
                kc.autotune(P0, fp32=fp32)


def _batch_items(kernels, P0s, n_electrons, cfg):
    """The C batch items of a scan: every output a view of one allocation (one allocator call per
    batch instead of seven per solve; the block lives as long as any returned tensor does)."""
    L = _lib.lib()
    n = len(kernels)
    dev = kernels[0].device
    conf = _CgConfig(int(cfg.max_iter), float(cfg.tol_E), float(cfg.tol_grad), float(cfg.denom_scale),
                     float(cfg.max_step), int(cfg.cg_restart), float(cfg.bt_shrink), int(cfg.bt_max),
                     int(cfg.mu_maxiter), int(cfg.plateau_window), int(bool(cfg.fp32_exchange)),
                     float(cfg.fp32_switch_rel), int(cfg.chunk), FOCK_CB(), PROJECT_CB(), None)
    items = (_CgBatchItem * n)()
    keep, outs = [], []
    nh = max(cfg.max_iter, 1)
    shapes = [tuple(k.shape) for k in kernels]
    al = lambda b: (b + 255) // 256 * 256
    per = [3 * al(a * b * c * c * 16) + al(a * b * c * 8) + 2 * al(nh * 8) for (a, b, c) in shapes]
    block = torch.empty(sum(per) + al(n * 64), dtype=torch.uint8, device=dev)
    cursor = [0]

    def take(count, dtype, shape):
        o = cursor[0]
        nbytes = count * torch.empty((), dtype=dtype).element_size()
        cursor[0] = o + al(nbytes)
        return block[o:o + nbytes].view(dtype).view(shape)

    scs = take(n * 8, torch.float64, (n, 8))  # every solve's scalars, read back in one copy
    scs.zero_()
    for i, (kern, P0, ne) in enumerate(zip(kernels, P0s, n_electrons)):
        validate_electron_count(kern.w2d, kern.h.shape[-1], ne, context="n_electrons")
        nk1, nk2, nb = kern.shape
        kc = KernelC128(kern)
        P0t = torch.as_tensor(P0).to(dev, torch.complex128).contiguous()
        Q = take(nk1 * nk2 * nb * nb, torch.complex128, (nk1, nk2, nb, nb))
        p = take(nk1 * nk2 * nb, torch.float64, (nk1, nk2, nb))
        P = take(nk1 * nk2 * nb * nb, torch.complex128, (nk1, nk2, nb, nb))
        F = take(nk1 * nk2 * nb * nb, torch.complex128, (nk1, nk2, nb, nb))
        hE = take(nh, torch.float64, (nh,))
        hG = take(nh, torch.float64, (nh,))
        hE.zero_()
        hG.zero_()
        sc = scs[i]
        items[i] = _CgBatchItem(kc.problem(ne), P0t.data_ptr(), Q.data_ptr(), p.data_ptr(), P.data_ptr(),
                                F.data_ptr(), hE.data_ptr(), hG.data_ptr(), sc.data_ptr())
        keep += [kc, P0t]
        outs.append((kern, Q, p, P, F, hE, hG, sc))
    per_lane = C.c_size_t(0)
    _lib.check(L.hf_cg_batch_workspace_size(items, n, C.byref(conf), C.byref(per_lane)))
    return items, outs, keep, scs, conf, per_lane.value


def _batch_results(outs, scs, cfg, copy=False):
    results = []
    host = scs.cpu().numpy()
    cp = (lambda t: t.clone()) if copy else (lambda t: t)
    for i, (kern, Q, p, P, F, hE, hG, sc) in enumerate(outs):
        s = host[i]
        hist = dict(E=cp(hE[:cfg.max_iter].to(kern.real_dtype)), grad_norm=cp(hG[:cfg.max_iter].to(kern.real_dtype)),
                    fp32_switch_iter=int(s[5]))
        results.append(SolveResult(Q=cp(Q.to(kern.dtype)), p=cp(p.to(kern.real_dtype)), mu=sc[0].to(kern.real_dtype).clone(),
                                   density=cp(P.to(kern.dtype)), fock=cp(F.to(kern.dtype)), energy=sc[1].clone(),
                                   n_iter=torch.tensor(int(s[2]), dtype=torch.int32),
                                   converged=torch.tensor(bool(s[3])), history=hist))
    return results


class ScanGraph:
    """A batch of CG solves captured once as ONE CUDA graph (``hf_cg_batch_graph_create``) and
    launched any number of times (no reference counterpart; the reference loops ``solve``).

    Every solve is a branch of the graph whose iteration loop is a device-side conditional
    node, so a launch runs the whole scan without a host round trip.  ``run(P0s=None)``
    writes new starting densities (same shapes) into the graph's P0 buffers, launches and
    returns fresh ``SolveResult``s (and each solve's device time with ``return_times``).
    ``launch()`` only enqueues the graph on the current stream.  Hooks are not supported
    (``optimizer="cg"`` without project_fn / block_sizes)."""

    def __init__(self, kernels, P0s, n_electrons, *, config: SolverConfig | None = None, autotune: bool = False):
        cfg = config or SolverConfig()
        if str(cfg.optimizer).lower() != "cg" or cfg.project_fn is not None or cfg.block_sizes is not None:
            raise ValueError("ScanGraph runs the CG optimizer without hooks.")
        n = len(kernels)
        if n == 0 or len(P0s) != n or len(n_electrons) != n:
            raise ValueError("kernels, P0s and n_electrons must be non-empty and of equal length.")
        if autotune:
            _autotune_scan(kernels, P0s, cfg)
        self.cfg = cfg
        self.L = _lib.lib()
        self.dev = kernels[0].device
        self.items, self.outs, self.keep, self.scs, self.conf, per = _batch_items(kernels, P0s, n_electrons, cfg)
        self.P0 = [k for k in self.keep if isinstance(k, torch.Tensor)]
        self.ws = torch.empty(max(n * per, 256), dtype=torch.uint8, device=self.dev)
        h = C.c_void_p(None)
        _lib.check(self.L.hf_cg_batch_graph_create(self.items, n, C.byref(self.conf), self.ws.data_ptr(), per,
                                                   C.byref(h)))
        self.handle = h
        self.n = n

    def launch(self, times=None):
        _lib.check(self.L.hf_cg_batch_graph_launch(self.handle, _lib.stream_ptr(self.dev), times))

    def run(self, P0s=None, return_times: bool = False):
        if P0s is not None:
            if len(P0s) != self.n:
                raise ValueError(f"expected {self.n} starting densities, got {len(P0s)}")
            for dst, src in zip(self.P0, P0s):
                dst.copy_(torch.as_tensor(src).to(self.dev, torch.complex128).reshape(dst.shape))
        times = (C.c_double * self.n)()
        self.launch(times)
        res = _batch_results(self.outs, self.scs, self.cfg, copy=True)
        return (res, list(times)) if return_times else res

    def close(self):
        if getattr(self, "handle", None) is not None and self.handle.value:
            self.L.hf_cg_batch_graph_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
