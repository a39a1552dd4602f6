"""Reference SCF solver on the GPU (drop-in for jax_hf.reference_scf).

Roothaan iteration with linear mixing, Pulay C-DIIS or ODA, optional level
shift and trust-radius clip (reference_scf.py:31-365).  Every array operation
runs in the CUDA library (Fock build, energy, Jacobi eigh, bisection mu,
occupations, residuals/commutators, DIIS Gram matrix, extrapolation); the
loop's scalar decisions are taken on the host from a few float64 reductions per
iteration, as the reference does in its traced loop.  The (N+1)^2 bordered DIIS
system is solved on the host with LAPACK (numpy), like jnp.linalg.solve on CPU.

solve_scf runs the same loop in the library's C++ driver (hf_scf_solve), which
issues the same device operations and reads the loop's scalars once per
iteration; a project_fn or a custom fock_build_fn runs there as a host callback
on the same stream.  The Python loop below is the same loop step for step
(USE_NATIVE = False, or a DIIS history longer than 16).
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Any, Callable

import numpy as np
import torch

from . import _lib
from .fock import build_fock, hf_energy
from .linalg import eigh, density_from_Qp
from .utils import validate_electron_count


# solve_scf runs the library's SCF driver (hf_scf_solve; hooks as host callbacks);
# False keeps every call on the Python loop below.
USE_NATIVE = True


@dataclass(frozen=True)
class SCFConfig:
    """reference_scf.py:31-63 (same fields, defaults and validation)."""
    max_iter: int = 200
    density_tol: float = 1e-7
    comm_tol: float = 1e-6
    mixing: float = 0.5
    level_shift: float = 0.0
    acceleration: str = "linear"
    diis_size: int = 6
    diis_start: int = 2
    diis_damping: float = 1.0
    trust_radius: float = 0.0
    project_fn: Callable[[Any], Any] | None = None
    # extensions (the library's SCF driver only; defaults keep the reference behaviour):
    # fp32_exchange runs the exchange FFT in FP32 while the density residual is above
    # fp32_switch_density, then FP64 to convergence (the FP64 fixed point);
    # mu_method="newton" takes each iteration's mu from the Newton-bracket solver
    # started at the previous mu instead of the 54-step bisection (same root to rounding);
    # warm_eigh starts each eigendecomposition (nb <= 8) from the previous eigenvectors
    fp32_exchange: bool = False
    fp32_switch_density: float = 1e-5
    mu_method: str = "bisection"
    warm_eigh: bool = False
    # an FP64 reference solution (energy, and optionally density) to report the result's
    # error against: history["rel_dE_vs_reference"], history["max_abs_dP_vs_reference"]
    reference_energy: float | None = None
    reference_density: Any = None

    def __post_init__(self) -> None:
        if self.max_iter <= 0:
            raise ValueError("max_iter must be positive")
        if self.acceleration not in ("linear", "diis", "oda"):
            raise ValueError("SCFConfig.acceleration must be 'linear', 'diis', or 'oda'; "
                             f"got {self.acceleration!r}")
        if self.diis_size <= 0:
            raise ValueError("diis_size must be positive")
        if self.mu_method not in ("bisection", "newton"):
            raise ValueError(f"SCFConfig.mu_method must be 'bisection' or 'newton'; got {self.mu_method!r}")


@dataclass(frozen=True)
class SCFResult:
    density_matrix: Any
    fock_matrix: Any
    energy: Any
    chemical_potential: Any
    iterations: int
    converged: bool
    message: str
    history: dict[str, Any] = field(default_factory=dict)


class _Ops:
    """Thin wrappers of the C-ABI operations on complex128 / float64 tensors."""

    def __init__(self, device, nk1, nk2, nb):
        self.dev = device
        self.nk = nk1 * nk2
        self.nk1, self.nk2, self.nb = nk1, nk2, nb
        L = _lib.lib()
        self.L = L
        n = C.c_size_t(0)
        _lib.check(L.hf_ops_workspace_size(C.byref(n)))
        self.ws = torch.empty(n.value, dtype=torch.uint8, device=device)
        self.red = torch.empty(64, dtype=torch.float64, device=device)
        self.s = _lib.stream_ptr(device)

    def herm(self, X, out=None, a=1.0, Y=None, b=0.0):
        out = torch.empty_like(X) if out is None else out
        _lib.check(self.L.hf_axpby(self.s, self.nk, self.nb, a, X.data_ptr(), b, _lib.ptr(Y), 1, out.data_ptr()))
        return out

    def fermi(self, eps, mu, T, mode, shift=0.0, out=None):
        out = torch.empty_like(eps) if out is None else out
        _lib.check(self.L.hf_fermi(self.s, eps.numel(), eps.data_ptr(), mu.data_ptr(), float(T), mode, float(shift),
                                   out.data_ptr()))
        return out

    def find_mu(self, eps, w, n_electrons, T, method=0, mu0=None, out=None):
        out = torch.empty((), dtype=torch.float64, device=self.dev) if out is None else out
        _lib.check(self.L.hf_find_mu(self.s, _lib.HF_C128, method, self.nk, 1, self.nb, eps.data_ptr(), w.data_ptr(),
                                     float(n_electrons), float(T), 0, _lib.ptr(mu0), out.data_ptr()))
        return out


def solve_scf(kernel, P0, n_electrons: float, *, config: SCFConfig | None = None,
              fock_build_fn: Callable | None = None) -> SCFResult:
    """Reference SCF solver (reference_scf.py:124-219)."""
    cfg = config if config is not None else SCFConfig()
    return _reference_errors(_solve_scf_impl(kernel, P0, n_electrons, cfg, fock_build_fn), cfg)


def _reference_errors(r: SCFResult, cfg: SCFConfig) -> SCFResult:
    """Adds the result's error against a supplied FP64 reference to its history."""
    if cfg.reference_energy is not None:
        Er = float(cfg.reference_energy)
        r.history["rel_dE_vs_reference"] = abs(float(r.energy) - Er) / max(abs(Er), 1e-300)
    if cfg.reference_density is not None:
        Pr = torch.as_tensor(cfg.reference_density).to(r.density_matrix.device, r.density_matrix.dtype)
        r.history["max_abs_dP_vs_reference"] = float((r.density_matrix - Pr).abs().max())
    return r


def _solve_scf_impl(kernel, P0, n_electrons, cfg, fock_build_fn):
    dev = kernel.device
    nk1, nk2, nb = kernel.shape
    cd = torch.complex128
    h = kernel.h.to(cd)
    w2d = kernel.w2d.to(torch.float64).contiguous()
    ws = max(float(kernel.weight_sum), 1e-30)
    T = float(kernel.T)
    ops = _Ops(dev, nk1, nk2, nb)
    project = cfg.project_fn
    validate_electron_count(w2d, nb, n_electrons, context="n_electrons")
    if USE_NATIVE and (cfg.acceleration != "diis" or cfg.diis_size <= 16):
        return _solve_scf_native(kernel, P0, n_electrons, cfg, fock_build_fn)
    if cfg.fp32_exchange or cfg.mu_method != "bisection" or cfg.warm_eigh:
        raise ValueError("SCFConfig.fp32_exchange, mu_method='newton' and warm_eigh run in the library's SCF driver "
                         "(diis_size <= 16).")
    a = kernel.as_args()
    VR = a["VR"] if kernel.dtype == cd else (a["VR"].to(cd) if a["VR"].is_complex() else a["VR"].to(torch.float64))
    fock_kw = dict(h=h, VR=VR, refP=kernel.refP if kernel.dtype == cd else kernel.refP.to(cd), HH=kernel.HH.double(),
                   w2d=w2d, include_exchange=kernel.include_exchange, include_hartree=kernel.include_hartree,
                   exchange_hermitian_channel_packing=kernel.exchange_hermitian_channel_packing,
                   contact_g=kernel.contact_g.double(), contact_Oi=kernel.contact_Oi.to(cd),
                   contact_Oj=kernel.contact_Oj.to(cd))
    if kernel.dtype == cd:
        fock_kw["refP"] = kernel.refP
        fock_kw["contact_g"] = kernel.contact_g
        fock_kw["contact_Oi"] = kernel.contact_Oi
        fock_kw["contact_Oj"] = kernel.contact_Oj
    fn = fock_build_fn or build_fock

    def proj_herm(X):
        if project is None:
            return ops.herm(X)
        return ops.herm(torch.as_tensor(project(X)).to(cd).contiguous())

    def fock(P):
        return fn(P, project_fn=project, **fock_kw)

    def density_from_fock(F):
        """reference_scf.py:87-96: eigh, bisection mu, level shift, occupations."""
        ev, orb = eigh(F)
        mu_raw = ops.find_mu(ev, w2d, n_electrons, T, method=0)
        if cfg.level_shift != 0.0:
            shifted = ops.fermi(ev, mu_raw, T, 2, cfg.level_shift)
            mu = ops.find_mu(shifted, w2d, n_electrons, T, method=0)
        else:
            shifted, mu = ev, mu_raw
        occ = ops.fermi(shifted, mu, T, 0)
        return density_from_Qp(orb, occ), mu

    def build_and_occupy(dens):
        dh = proj_herm(dens)
        Sg, Hh, F = fock(dh)
        E = hf_energy(dh, h=h, Sigma=Sg, H=Hh, weights_b=w2d)
        Pn, mu = density_from_fock(F)
        if project is not None:
            Pn = proj_herm(Pn)
        return Pn, F, E, mu

    use_diis = cfg.acceleration == "diis"
    n_hist = cfg.diis_size if use_diis else 0
    if use_diis:
        F_hist = torch.zeros((n_hist, nk1, nk2, nb, nb), dtype=cd, device=dev)
        R_hist = torch.zeros_like(F_hist)
        stride = nk1 * nk2 * nb * nb
    comm_buf = torch.empty((nk1, nk2, nb, nb), dtype=cd, device=dev)
    delta = torch.empty_like(comm_buf)
    sums = torch.empty(3, dtype=torch.float64, device=dev)
    gram = torch.empty(256, dtype=torch.float64, device=dev)
    coeff_dev = torch.empty(max(n_hist, 1), dtype=torch.float64, device=dev)
    hE, hD, hC = [], [], []
    density = torch.as_tensor(P0).to(dev, cd).contiguous() if not (
        isinstance(P0, torch.Tensor) and P0.dtype == cd) else P0.to(dev).contiguous()
    k, converged = 0, False
    while k < cfg.max_iter and not converged:
        P_new, F, E, mu = build_and_occupy(density)
        R_out = R_hist[k % n_hist] if use_diis else comm_buf
        _lib.check(ops.L.hf_scf_residuals(ops.s, ops.nk, nb, F.data_ptr(), density.data_ptr(), P_new.data_ptr(),
                                          w2d.data_ptr(), R_out.data_ptr(), delta.data_ptr(), sums.data_ptr(),
                                          ops.ws.data_ptr()))
        s_host = sums.cpu().numpy()
        E_host = float(E)
        d_res = float(np.sqrt(s_host[0] / ws))
        c_res = float(np.sqrt(s_host[1] / ws))
        converged = d_res <= cfg.density_tol and c_res <= cfg.comm_tol
        if use_diis:
            idx = k % n_hist
            F_hist[idx].copy_(F)
            count = min(k + 1, n_hist)
            active = (np.arange(n_hist) < count).astype(np.float64)
            B = _gram_matrix(ops, R_hist, n_hist, stride, w2d, gram)
            B = B / max(np.max(np.abs(B)), 1e-30)
            A = np.zeros((n_hist + 1, n_hist + 1))
            A[:n_hist, :n_hist] = B + np.diag(1.0 - active)
            A[:n_hist, n_hist] = -active
            A[n_hist, :n_hist] = -active
            rhs = np.zeros(n_hist + 1)
            rhs[n_hist] = -1.0
            try:
                sol = np.linalg.solve(A, rhs)
            except np.linalg.LinAlgError:
                sol = np.full(n_hist + 1, np.nan)
            coeffs = sol[:n_hist]
            ok = bool(np.all(np.isfinite(sol)))
            engaged = count >= max(2, cfg.diis_start) and ok
            if engaged:
                coeff_dev.copy_(torch.from_numpy(coeffs))
                Fx = torch.empty_like(F)
                _lib.check(ops.L.hf_lincomb(ops.s, n_hist, stride, stride, F_hist.data_ptr(), coeff_dev.data_ptr(),
                                            Fx.data_ptr()))
                damp = float(np.clip(cfg.diis_damping, 0.0, 1.0))
                if damp != 1.0:
                    Fd = torch.empty_like(F)
                    _lib.check(ops.L.hf_axpby(ops.s, ops.nk, nb, damp, Fx.data_ptr(), 1.0 - damp, F.data_ptr(), 0,
                                              Fd.data_ptr()))
                    Fx = Fd
                Pd, _ = density_from_fock(ops.herm(Fx))
                updated = proj_herm(Pd) if project is not None else Pd
            else:
                updated = _linear(ops, density, delta, cfg.mixing, project, proj_herm)
        elif cfg.acceleration == "oda":
            Sn, Hn, _ = fock(P_new)
            E_new = float(hf_energy(P_new, h=h, Sigma=Sn, H=Hn, weights_b=w2d))
            c1 = float(s_host[2])
            c2 = (E_new - E_host) - c1
            if c2 > 1e-12:
                lam = float(np.clip(-c1 / (2.0 * c2), 0.0, 1.0))
            else:
                lam = 1.0 if c1 < 0.0 else 0.0
            updated = proj_herm_axpy(ops, density, delta, lam, project, proj_herm)
        else:
            updated = _linear(ops, density, delta, cfg.mixing, project, proj_herm)
        if cfg.trust_radius > 0.0:                              # reference_scf.py:333-339
            step = torch.empty_like(density)
            _lib.check(ops.L.hf_axpby(ops.s, ops.nk, nb, 1.0, updated.data_ptr(), -1.0, density.data_ptr(), 0,
                                      step.data_ptr()))
            _lib.check(ops.L.hf_jdot(ops.s, ops.nk, nb, step.data_ptr(), step.data_ptr(), w2d.data_ptr(), None, None,
                                     None, ops.red.data_ptr(), ops.ws.data_ptr()))
            sn = float(np.sqrt(float(ops.red[0]) / ws))
            if sn > cfg.trust_radius:
                scale = cfg.trust_radius / max(sn, 1e-30)
                updated = proj_herm_axpy(ops, density, step, scale, project, proj_herm)
        density = P_new if converged else updated
        hE.append(E_host)
        hD.append(d_res)
        hC.append(c_res)
        k += 1
    _, F_fin, E_fin, mu_fin = build_and_occupy(density)
    n_iter = k
    if converged:
        message = f"converged in {n_iter} iterations"
    else:
        dr = hD[-1] if n_iter > 0 else float("nan")
        cr = hC[-1] if n_iter > 0 else float("nan")
        message = f"stopped after {n_iter} iterations (density_res={dr:.3e}, comm_res={cr:.3e})"
    out_c = kernel.dtype
    return SCFResult(density_matrix=density.to(out_c), fock_matrix=F_fin.to(out_c), energy=E_fin,
                     chemical_potential=mu_fin, iterations=n_iter, converged=bool(converged), message=message,
                     history={"E": np.asarray(hE), "density_residual": np.asarray(hD),
                              "commutator_residual": np.asarray(hC)})


class _ScfConfig(C.Structure):
    pass


def _scf_config_type():
    from .solver import FOCK_CB, PROJECT_CB
    if not getattr(_ScfConfig, "_fields_", None):
        _ScfConfig._fields_ = [("max_iter", C.c_int), ("density_tol", C.c_double), ("comm_tol", C.c_double),
                               ("mixing", C.c_double), ("level_shift", C.c_double), ("acceleration", C.c_int),
                               ("diis_size", C.c_int), ("diis_start", C.c_int), ("diis_damping", C.c_double),
                               ("trust_radius", C.c_double), ("fp32_exchange", C.c_int),
                               ("fp32_switch_density", C.c_double), ("mu_method", C.c_int), ("warm_eigh", C.c_int),
                               ("fock_cb", FOCK_CB), ("project_cb", PROJECT_CB), ("cb_user", C.c_void_p)]
    return _ScfConfig


def _buffer_views(*tensors):
    """Maps a device pointer inside one of ``tensors`` to a tensor view of the given shape (the
    driver hands its callbacks pointers into the workspace and the output buffers)."""
    bases = [(t.data_ptr(), t.numel() * t.element_size(), t.view(-1).view(torch.uint8)) for t in tensors]

    def view(ptr, shape):
        nbytes = int(np.prod(shape)) * 16
        for b, n, flat in bases:
            if b <= ptr and ptr + nbytes <= b + n:
                return flat[ptr - b:ptr - b + nbytes].view(torch.complex128).view(shape)
        raise RuntimeError("callback buffer outside the driver's allocations")

    return view


def _solve_scf_native(kernel, P0, n_electrons, cfg, fock_build_fn=None):
    """solve_scf through the library's SCF driver (hf_scf_solve): the same steps as the
    loop above, sequenced in C++ with one small device->host read per iteration.  A
    project_fn or a custom fock_build_fn runs as a host callback of the driver on the
    same stream."""
    from .solver import FOCK_CB, PROJECT_CB, KernelC128, _CgProblem

    L = _lib.lib()
    if not getattr(L, "_scf_bound", False):
        L.hf_scf_workspace_size.argtypes = [C.POINTER(_CgProblem), C.POINTER(_ScfConfig), C.POINTER(C.c_size_t)]
        L.hf_scf_workspace_size.restype = C.c_int
        L.hf_scf_solve.argtypes = [C.c_void_p, C.POINTER(_CgProblem), C.POINTER(_ScfConfig), C.c_void_p,
                                   C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_size_t]
        L.hf_scf_solve.restype = C.c_int
        L._scf_bound = True
    dev = kernel.device
    cd = torch.complex128
    kc = KernelC128(kernel)
    pb = kc.problem(n_electrons)
    project = cfg.project_fn
    if cfg.fp32_exchange and fock_build_fn is not None:
        raise ValueError("SCFConfig.fp32_exchange applies to the built-in Fock build, not to a fock_build_fn.")
    sc = _scf_config_struct(cfg)
    need = C.c_size_t(0)
    _lib.check(L.hf_scf_workspace_size(C.byref(pb), C.byref(sc), C.byref(need)))
    ws = _lib.workspace(need.value, dev, "scf")
    P0d = torch.as_tensor(P0).to(dev, cd).contiguous()
    density = torch.empty_like(P0d)
    fock = torch.empty_like(P0d)
    errors = []
    if fock_build_fn is not None or project is not None:
        nk1, nk2, nb = kernel.shape
        shape = (nk1, nk2, nb, nb)
        view = _buffer_views(ws, density, fock)
        fkw = kc.fock_kwargs()
        ops_L, s_ptr = _lib.lib(), _lib.stream_ptr(dev)

        def fock_cb(user, stream, Pp, Sp, Hp, Fp):
            try:
                Sg, Hh, Fn = fock_build_fn(view(Pp, shape), project_fn=None, **fkw)
                view(Sp, shape).copy_(Sg)
                Hh = torch.as_tensor(Hh).to(dev, cd)
                view(Hp, (nb, nb)).copy_(Hh.reshape(-1, nb, nb)[0] if Hh.numel() >= nb * nb else Hh.expand(nb, nb))
                view(Fp, shape).copy_(Fn)
                return 0
            except Exception as exc:  # re-raised after the C call returns
                errors.append(exc)
                return _lib.HF_ERR_ABORTED

        def project_cb(user, stream, Xp):
            try:
                X = view(Xp, shape)
                Y = torch.as_tensor(project(X)).to(dev, cd).contiguous()
                _lib.check(ops_L.hf_axpby(s_ptr, nk1 * nk2, nb, 1.0, Y.data_ptr(), 0.0, None, 1, X.data_ptr()))
                return 0
            except Exception as exc:
                errors.append(exc)
                return _lib.HF_ERR_ABORTED

        sc.fock_cb = FOCK_CB(fock_cb) if fock_build_fn is not None else FOCK_CB()
        sc.project_cb = PROJECT_CB(project_cb) if project is not None else PROJECT_CB()
    m = int(cfg.max_iter)
    hist = np.zeros((3, m))
    out = np.full(5, -1.0)
    dp = lambda a: a.ctypes.data_as(C.c_void_p)
    st = L.hf_scf_solve(_lib.stream_ptr(dev), C.byref(pb), C.byref(sc), P0d.data_ptr(), density.data_ptr(),
                        fock.data_ptr(), dp(hist[0]), dp(hist[1]), dp(hist[2]), dp(out), ws.data_ptr(), ws.numel())
    if errors:
        raise errors[0]
    _lib.check(st)
    n_iter = int(out[2])
    converged = bool(out[3] != 0.0)
    hE, hD, hC = hist[0, :n_iter].copy(), hist[1, :n_iter].copy(), hist[2, :n_iter].copy()
    if converged:
        message = f"converged in {n_iter} iterations"
    else:
        dr = hD[-1] if n_iter > 0 else float("nan")
        cr = hC[-1] if n_iter > 0 else float("nan")
        message = f"stopped after {n_iter} iterations (density_res={dr:.3e}, comm_res={cr:.3e})"
    out_c = kernel.dtype
    return SCFResult(density_matrix=density.to(out_c), fock_matrix=fock.to(out_c),
                     energy=torch.tensor(float(out[0]), dtype=torch.float64, device=dev),
                     chemical_potential=torch.tensor(float(out[1]), dtype=torch.float64, device=dev),
                     iterations=n_iter, converged=converged, message=message,
                     history={"E": hE, "density_residual": hD, "commutator_residual": hC,
                              "fp32_switch_iter": int(out[4]) if cfg.fp32_exchange else -1})


_STREAMS: dict = {}


def _worker_streams(dev, n):
    """The first n streams of a per-device pool that lives as long as the process: the
    solvers' workspaces are cached per stream, so reusing the streams reuses them."""
    pool = _STREAMS.setdefault(str(dev), [])
    while len(pool) < n:
        pool.append(torch.cuda.Stream(dev))
    return pool[:n]


class _ScfBatchItem(C.Structure):
    pass


def _scf_batch_item_type():
    from .solver import _CgProblem
    if not getattr(_ScfBatchItem, "_fields_", None):
        _ScfBatchItem._fields_ = [("problem", _CgProblem), ("P0", C.c_void_p), ("density", C.c_void_p),
                                  ("fock", C.c_void_p), ("hist_E", C.c_void_p), ("hist_D", C.c_void_p),
                                  ("hist_C", C.c_void_p), ("scalars_out", C.c_void_p)]
    return _ScfBatchItem


def _scf_config_struct(cfg):
    acc = {"linear": 0, "diis": 1, "oda": 2}[cfg.acceleration]
    return _scf_config_type()(int(cfg.max_iter), float(cfg.density_tol), float(cfg.comm_tol), float(cfg.mixing),
                      float(cfg.level_shift), acc, int(cfg.diis_size), int(cfg.diis_start), float(cfg.diis_damping),
                      float(cfg.trust_radius), int(bool(cfg.fp32_exchange)), float(cfg.fp32_switch_density),
                      2 if cfg.mu_method == "newton" else 0, int(bool(cfg.warm_eigh)))


class ScfScanGraph:
    """A batch of SCF solves captured once as ONE CUDA graph (``hf_scf_batch_graph_create``)
    and launched any number of times (extension; no reference counterpart).

    The loop of ``solve_scf`` runs with its decisions on the device: every solve is a
    branch of the graph whose iterations are device-side conditional loops, and the
    DIIS system is solved on the device, so a launch runs the whole batch without a
    host round trip.  Each result equals the library's SCF driver's (``solve_scf``)
    to the rounding of the DIIS solve.  ``run(P0s=None)`` writes new starting densities
    (same shapes), launches and returns fresh ``SCFResult``s; ``launch()`` only enqueues.
    ODA, the trust-radius clip and ``project_fn`` are not supported."""

    def __init__(self, kernels, P0s, n_electrons, *, config: SCFConfig | None = None):
        from .solver import KernelC128
        cfg = config or SCFConfig()
        n = len(kernels)
        if n == 0 or len(P0s) != n or len(n_electrons) != n:
            raise ValueError("kernels, P0s and n_electrons must be non-empty and of equal length.")
        if cfg.project_fn is not None or cfg.acceleration == "oda" or cfg.trust_radius > 0.0:
            raise ValueError("ScfScanGraph runs DIIS or linear mixing without project_fn or trust radius.")
        if cfg.acceleration == "diis" and cfg.diis_size > 16:
            raise ValueError("ScfScanGraph: diis_size <= 16")
        Item = _scf_batch_item_type()
        self.L = _lib.lib()
        self.cfg = cfg
        self.dev = kernels[0].device
        self.sc = _scf_config_struct(cfg)
        cd = torch.complex128
        m = max(int(cfg.max_iter), 1)
        self.items = (Item * n)()
        self.keep, self.outs = [], []
        for i, (kern, P0, ne) in enumerate(zip(kernels, P0s, n_electrons)):
            validate_electron_count(kern.w2d, kern.h.shape[-1], ne, context="n_electrons")
            kc = KernelC128(kern)
            P0d = torch.as_tensor(P0).to(self.dev, cd).contiguous().clone()
            dens, fock = torch.empty_like(P0d), torch.empty_like(P0d)
            hist = torch.zeros((3, m), dtype=torch.float64, device=self.dev)
            out = torch.full((5,), -1.0, dtype=torch.float64, device=self.dev)
            self.items[i] = Item(kc.problem(ne), P0d.data_ptr(), dens.data_ptr(), fock.data_ptr(), hist[0].data_ptr(),
                                 hist[1].data_ptr(), hist[2].data_ptr(), out.data_ptr())
            self.keep += [kc, P0d]
            self.outs.append((kern, P0d, dens, fock, hist, out))
        per = C.c_size_t(0)
        _lib.check(self.L.hf_scf_batch_workspace_size(self.items, n, C.byref(self.sc), C.byref(per)))
        self.ws = torch.empty(max(n * per.value, 256), dtype=torch.uint8, device=self.dev)
        h = C.c_void_p(None)
        _lib.check(self.L.hf_scf_batch_graph_create(self.items, n, C.byref(self.sc), self.ws.data_ptr(), per.value,
                                                    C.byref(h)))
        self.handle = h
        self.n = n

    def launch(self, times=None):
        _lib.check(self.L.hf_scf_batch_graph_launch(self.handle, _lib.stream_ptr(self.dev), times))

    def run(self, P0s=None, return_times: bool = False):
        if P0s is not None:
            if len(P0s) != self.n:
                raise ValueError(f"expected {self.n} starting densities, got {len(P0s)}")
            for (_, dst, *_), src in zip(self.outs, P0s):
                dst.copy_(torch.as_tensor(src).to(self.dev, torch.complex128).reshape(dst.shape))
        times = (C.c_double * self.n)()
        self.launch(times)
        results = []
        for kern, _, dens, fock, hist, out in self.outs:
            o = out.cpu().numpy()
            n_iter = int(o[2])
            converged = bool(o[3] != 0.0)
            h = hist[:, :n_iter].cpu().numpy()
            if converged:
                message = f"converged in {n_iter} iterations"
            else:
                dr = h[1, -1] if n_iter > 0 else float("nan")
                cr = h[2, -1] if n_iter > 0 else float("nan")
                message = f"stopped after {n_iter} iterations (density_res={dr:.3e}, comm_res={cr:.3e})"
            results.append(SCFResult(
                density_matrix=dens.to(kern.dtype).clone(), fock_matrix=fock.to(kern.dtype).clone(),
                energy=torch.tensor(float(o[0]), dtype=torch.float64, device=self.dev),
                chemical_potential=torch.tensor(float(o[1]), dtype=torch.float64, device=self.dev),
                iterations=n_iter, converged=converged, message=message,
                history={"E": h[0].copy(), "density_residual": h[1].copy(), "commutator_residual": h[2].copy(),
                         "fp32_switch_iter": int(o[4]) if self.cfg.fp32_exchange else -1}))
        results = [_reference_errors(r, self.cfg) for r in results]
        return (results, list(times)) if return_times else results

    def close(self):
        if getattr(self, "handle", None) is not None and self.handle.value:
            self.L.hf_scf_batch_graph_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def solve_scf_batch(kernels, P0s, n_electrons, *, config: SCFConfig | None = None, workers: int = 16,
                    return_times: bool = False, graph: bool = False):
    """Many independent SCF solves at once (extension; density scans).

    Each solve has the semantics of ``solve_scf(kernel, P0, n, config=config)``
    through the library's SCF driver.  ``workers`` host threads each own a CUDA
    stream and take the next solve (longest first, by nk1 nk2 nb^2) until none
    is left; the driver's once-per-iteration scalar read blocks only its own
    thread, so the solves of the other streams keep the GPU busy.  Returns the
    list of ``SCFResult`` (and, with ``return_times``, each solve's wall time
    in ms, from its start on its stream to its final scalars).
    ``graph=True`` runs the batch as one CUDA graph with the loops on the device
    (``ScfScanGraph``, built and launched once; DIIS or linear mixing only).
    """
    import threading
    import time
    cfg = config or SCFConfig()
    if graph:
        sg = ScfScanGraph(kernels, P0s, n_electrons, config=cfg)
        try:
            return sg.run(return_times=return_times)
        finally:
            sg.close()
    n = len(kernels)
    if n == 0 or len(P0s) != n or len(n_electrons) != n:
        raise ValueError("kernels, P0s and n_electrons must be non-empty and of equal length.")
    if cfg.project_fn is not None:
        raise ValueError("solve_scf_batch takes no project_fn.")
    dev = kernels[0].device
    order = sorted(range(n), key=lambda i: -int(np.prod(kernels[i].shape)) * int(kernels[i].shape[-1]))
    nxt = iter(order)
    lock = threading.Lock()
    results, times, errors = [None] * n, [0.0] * n, []
    main = torch.cuda.current_stream(dev)
    ready = torch.cuda.Event()
    ready.record(main)
    streams = _worker_streams(dev, max(1, min(int(workers), n)))

    def work(stream):
        try:
            stream.wait_event(ready)
            with torch.cuda.device(dev), torch.cuda.stream(stream):
                while True:
                    with lock:
                        i = next(nxt, None)
                    if i is None or errors:
                        return
                    t0 = time.perf_counter()
                    results[i] = solve_scf(kernels[i], P0s[i], n_electrons[i], config=cfg)
                    times[i] = 1e3 * (time.perf_counter() - t0)
        except Exception as exc:  # re-raised on the calling thread
            errors.append(exc)

    threads = [threading.Thread(target=work, args=(st,)) for st in streams]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    for st in streams:
        main.wait_stream(st)
    if errors:
        raise errors[0]
    return (results, times) if return_times else results


def _linear(ops, density, delta, mixing, project, proj_herm):
    """herm(project(density + mixing * delta)) (reference_scf.py:275-276)."""
    return proj_herm_axpy(ops, density, delta, mixing, project, proj_herm)


def proj_herm_axpy(ops, X, Y, b, project, proj_herm):
    if project is None:
        return ops.herm(X, a=1.0, Y=Y, b=b)
    tmp = torch.empty_like(X)
    _lib.check(ops.L.hf_axpby(ops.s, ops.nk, ops.nb, 1.0, X.data_ptr(), b, Y.data_ptr(), 0, tmp.data_ptr()))
    return proj_herm(tmp)


def _gram_matrix(ops, R_hist, n, stride, w2d, gram):
    """B_ij = sum_k w Re tr(R_i^H R_j) over all n history slots (reference_scf.py:110-111)."""
    B = np.zeros((n, n))
    if n <= 6:
        _lib.check(ops.L.hf_gram(ops.s, n, stride, ops.nk, ops.nb, R_hist.data_ptr(), w2d.data_ptr(),
                                 gram.data_ptr(), ops.ws.data_ptr()))
        g = gram[: n * (n + 1) // 2].cpu().numpy()
        q = 0
        for i in range(n):
            for j in range(i, n):
                B[i, j] = B[j, i] = g[q]
                q += 1
        return B
    if n > 16:
        for i in range(n):
            for j in range(i, n):
                _lib.check(ops.L.hf_jdot(ops.s, ops.nk, ops.nb, R_hist[i].data_ptr(), R_hist[j].data_ptr(),
                                         w2d.data_ptr(), None, None, None, gram.data_ptr(), ops.ws.data_ptr()))
                B[i, j] = B[j, i] = float(gram[0])
        return B
    # n = 7 .. 16: one row per launch, all rows read back at once
    for i in range(n):
        _lib.check(ops.L.hf_gram_row(ops.s, n, i, stride, ops.nk, ops.nb, R_hist.data_ptr(), w2d.data_ptr(),
                                     gram[i * n:].data_ptr(), ops.ws.data_ptr()))
    g = gram[: n * n].cpu().numpy().reshape(n, n)
    return np.triu(g) + np.triu(g, 1).T
