"""Trust-region Newton solver on the GPU (solver.py:686-1078, optimizer="newton").

Steihaug truncated CG on the joint (Q, p) Hessian; every Hessian-vector product
is one Fock build of the linear response (refP = 0) plus two per-k kernels
(`hf_newton_dP`, `hf_newton_hvp`).  Vectors, products and reductions run in the
CUDA library in float64.  Deflation (the Gaussian bias of solver.py:799-812) is
supported.

Two drivers issue the same device operations in the same order:

* the library's C++ driver ``hf_newton_solve`` (the default without hooks:
  project_fn, block_sizes and fock_build_fn all None, nb <= 16), which reads
  the loop's reductions in small batches (two reads per inner CG step);
* the Python loop below (with hooks, or ``USE_NATIVE = False``), which reads
  every reduction as it comes and runs the branch logic line for line with the
  reference loop body.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from .fock import build_fock, hf_energy
from .linalg import (cayley_spectral_setup, cayley_unitary_from_spectrum, density_from_Qp, eigh,
                     fock_in_orbital_basis)


class _V:
    """Device vector algebra over the joint space (X complex (nk,nb,nb), p real (nk,nb))."""

    def __init__(self, dev, nk1, nk2, nb, w2d):
        self.L = _lib.lib()
        self.dev = dev
        self.nk = nk1 * nk2
        self.nb = nb
        self.shape = (nk1, nk2, nb, nb)
        self.w2d = w2d
        n = C.c_size_t(0)
        _lib.check(self.L.hf_ops_workspace_size(C.byref(n)))
        self.ws = torch.empty(n.value, dtype=torch.uint8, device=dev)
        self.red = torch.zeros(8, dtype=torch.float64, device=dev)
        self.s = _lib.stream_ptr(dev)
        self.ones = torch.ones_like(w2d)

    def zX(self):
        return torch.zeros(self.shape, dtype=torch.complex128, device=self.dev)

    def zp(self):
        return torch.zeros(self.shape[:-1], dtype=torch.float64, device=self.dev)

    def axpy(self, a, X, b, Y, out=None):
        out = torch.empty_like(X) if out is None else out
        if X.is_complex():
            _lib.check(self.L.hf_axpby(self.s, self.nk, self.nb, float(a), X.data_ptr(), float(b), _lib.ptr(Y), 0,
                                       out.data_ptr()))
        else:
            _lib.check(self.L.hf_axpby_real(self.s, X.numel(), float(a), X.data_ptr(), float(b), _lib.ptr(Y),
                                            out.data_ptr()))
        return out

    def dot(self, aX=None, bX=None, wX=None, ap=None, bp=None, wp=None):
        _lib.check(self.L.hf_jdot(self.s, self.nk, self.nb, _lib.ptr(aX), _lib.ptr(bX), _lib.ptr(wX), _lib.ptr(ap),
                                  _lib.ptr(bp), _lib.ptr(wp), self.red.data_ptr(), self.ws.data_ptr()))
        return float(self.red[0])

    def jip(self, aX, ap, bX, bp):
        """ip_matrix(aX, bX, ones) + ip_vec(ap, bp, w2d) (solver.py:783-784)."""
        return self.dot(aX, bX, None, ap, bp, self.w2d)

    def project_occ(self, x, wsum_dev):
        """x -= sum w2d x / (sum w2d * nb) (solver.py:224-233); wsum on device."""
        den = float(self.w2d_sum) * self.nb
        _lib.check(self.L.hf_sub_scalar(self.s, x.numel(), x.data_ptr(), wsum_dev.data_ptr(), 1.0 / den))


# solve_newton runs the library's Newton driver (hf_newton_solve) when no hook is given;
# tests switch this off to compare it with the Python loop over the same device operations.
USE_NATIVE = True


class _NewtonConfig(C.Structure):
    _fields_ = [("max_iter", C.c_int), ("tol_grad", C.c_double), ("denom_scale", C.c_double),
                ("mu_maxiter", C.c_int), ("tr_delta0", C.c_double), ("tr_cg_max", C.c_int),
                ("n_deflation", C.c_int), ("deflation_targets", C.c_void_p), ("deflation_sigma", C.c_double),
                ("deflation_length", C.c_double)]


def _deflation_targets(cfg, dev, shape):
    targets = torch.as_tensor(cfg.deflation_targets).to(dev, torch.complex128)
    if targets.ndim == 4:
        targets = targets[None]
    if targets.ndim != 5 or tuple(targets.shape[1:]) != tuple(shape):
        raise ValueError("deflation_targets must have shape (n_solutions, nk1, nk2, nb, nb) matching the kernel; "
                         f"got {tuple(targets.shape)}.")
    return targets.contiguous()


def _solve_newton_native(kernel, P0, n_electrons, cfg):
    from .solver import KernelC128, SolveResult, _CgProblem
    L = _lib.lib()
    if not getattr(L, "_newton_bound", False):
        L.hf_newton_workspace_size.argtypes = [C.POINTER(_CgProblem), C.POINTER(_NewtonConfig),
                                               C.POINTER(C.c_size_t)]
        L.hf_newton_workspace_size.restype = C.c_int
        L.hf_newton_solve.argtypes = [C.c_void_p, C.POINTER(_CgProblem), C.POINTER(_NewtonConfig)] + \
            [C.c_void_p] * 9 + [C.c_size_t]
        L.hf_newton_solve.restype = C.c_int
        L._newton_bound = True
    dev = kernel.device
    nk1, nk2, nb = kernel.shape
    cd, rd = torch.complex128, torch.float64
    kc = KernelC128(kernel)
    pb = kc.problem(n_electrons)
    has_defl = cfg.deflation_targets is not None and float(cfg.deflation_sigma) > 0.0
    targets = _deflation_targets(cfg, dev, (nk1, nk2, nb, nb)) if has_defl else None
    nc = _NewtonConfig(int(cfg.max_iter), float(cfg.tol_grad), float(cfg.denom_scale), int(cfg.mu_maxiter),
                       float(cfg.tr_delta0), int(cfg.tr_cg_max), int(targets.shape[0]) if has_defl else 0,
                       targets.data_ptr() if has_defl else None, float(cfg.deflation_sigma),
                       float(cfg.deflation_length))
    need = C.c_size_t(0)
    _lib.check(L.hf_newton_workspace_size(C.byref(pb), C.byref(nc), C.byref(need)))
    ws = _lib.workspace(need.value, dev, "newton")
    P0d = torch.as_tensor(P0).to(dev, cd).contiguous()
    Q = torch.empty((nk1, nk2, nb, nb), dtype=cd, device=dev)
    p = torch.empty((nk1, nk2, nb), dtype=rd, device=dev)
    density, fock = torch.empty_like(Q), torch.empty_like(Q)
    m = max(int(cfg.max_iter), 1)
    hist = np.zeros((2, m))
    out = np.zeros(6)
    dp = lambda a: a.ctypes.data_as(C.c_void_p)
    _lib.check(L.hf_newton_solve(_lib.stream_ptr(dev), C.byref(pb), C.byref(nc), P0d.data_ptr(), Q.data_ptr(),
                                 p.data_ptr(), density.data_ptr(), fock.data_ptr(), dp(hist[0]), dp(hist[1]), dp(out),
                                 ws.data_ptr(), ws.numel()))
    out_c, out_r = kernel.dtype, kernel.real_dtype
    hE, hG = hist[0, :int(cfg.max_iter)], hist[1, :int(cfg.max_iter)]
    history = dict(E=torch.as_tensor(hE, dtype=out_r), grad_norm=torch.as_tensor(hG, dtype=out_r),
                   n_builds=int(out[5]))
    return SolveResult(Q=Q.to(out_c), p=p.to(out_r), mu=torch.tensor(float(out[0]), dtype=out_r),
                       density=density.to(out_c), fock=fock.to(out_c),
                       energy=torch.tensor(float(out[1]), dtype=torch.float64, device=dev),
                       n_iter=torch.tensor(int(out[2]), dtype=torch.int32), converged=torch.tensor(out[3] != 0.0),
                       history=history)


def solve_newton(kernel, P0, n_electrons, cfg, fock_build_fn=None):
    from .solver import SolveResult
    dev = kernel.device
    nk1, nk2, nb = kernel.shape
    if USE_NATIVE and fock_build_fn is None and cfg.project_fn is None and cfg.block_sizes is None and nb <= 16:
        return _solve_newton_native(kernel, P0, n_electrons, cfg)
    cd, rd = torch.complex128, torch.float64
    h = kernel.h.to(cd).contiguous()
    w2d = kernel.w2d.to(rd).contiguous()
    ws_sum = float(kernel.weight_sum)
    tiny = 1e-30
    w_norm = (w2d / max(ws_sum, tiny)).contiguous()
    n_target_norm = float(n_electrons) / max(ws_sum, tiny)
    T_r = max(float(kernel.T), 1e-12)
    tol_g = float(cfg.tol_grad) if cfg.tol_grad > 0.0 else 1e-6       # solver.py:1191
    delta_min, occ_clip = 1e-10, 1e-8
    noise_floor = max(1e-12, 4500.0 * float(np.finfo(np.float64).eps))
    project = cfg.project_fn
    V = _V(dev, nk1, nk2, nb, w2d)
    V.w2d_sum = float(w2d.sum().item())
    a = kernel.as_args()
    VR = a["VR"] if kernel.dtype == cd else (a["VR"].to(cd) if a["VR"].is_complex() else a["VR"].to(rd))
    specs = None if cfg.block_sizes is None else (("sizes", tuple(int(s) for s in cfg.block_sizes)),)
    fkw = dict(h=h, VR=VR, HH=kernel.HH.to(rd), w2d=w2d, include_exchange=kernel.include_exchange,
               include_hartree=kernel.include_hartree,
               exchange_hermitian_channel_packing=kernel.exchange_hermitian_channel_packing,
               contact_g=kernel.contact_g if kernel.dtype == cd else kernel.contact_g.to(rd),
               contact_Oi=kernel.contact_Oi.to(cd), contact_Oj=kernel.contact_Oj.to(cd),
               exchange_block_specs=specs)
    refP = kernel.refP if kernel.dtype == cd else kernel.refP.to(cd)
    from .problem import _mark_zero
    refP_zero = _mark_zero(torch.zeros_like(h))
    fn = fock_build_fn or build_fock
    mu_buf = torch.zeros((), dtype=rd, device=dev)
    n_builds = [0]

    def herm_project(P):
        if project is None:
            return P
        X = torch.as_tensor(project(P)).to(cd)
        return 0.5 * (X + X.transpose(-1, -2).conj())

    def fock_full(P):
        n_builds[0] += 1
        return fn(P, refP=refP, project_fn=None, **fkw)

    def fock_response(dP):
        n_builds[0] += 1
        _, _, Fr = fn(dP, refP=refP_zero, project_fn=None, **fkw)
        return Fr

    def solve_mu(eps, mu0):
        m0 = torch.tensor(float(mu0), dtype=rd, device=dev)
        _lib.check(V.L.hf_find_mu(V.s, _lib.HF_C128, 2, V.nk, 1, nb, eps.data_ptr(), w_norm.data_ptr(), n_target_norm,
                                  T_r, int(cfg.mu_maxiter), m0.data_ptr(), mu_buf.data_ptr()))
        return float(mu_buf)

    def occupations(eps, mu):
        m = torch.tensor(float(mu), dtype=rd, device=dev)
        out = torch.empty_like(eps)
        _lib.check(V.L.hf_fermi(V.s, eps.numel(), eps.data_ptr(), m.data_ptr(), T_r, 1, 0.0, out.data_ptr()))
        return out

    has_defl = cfg.deflation_targets is not None and float(cfg.deflation_sigma) > 0.0
    if has_defl:
        targets = _deflation_targets(cfg, dev, (nk1, nk2, nb, nb))
        inv2L2 = 1.0 / (2.0 * max(float(cfg.deflation_length), 1e-12) ** 2)
        dsig = float(cfg.deflation_sigma)

    def deflation_bias(P):                                       # solver.py:804-812
        Phi, pen = 0.0, 0.0
        S_pen = torch.zeros_like(P)
        for i in range(targets.shape[0]):
            diff = V.axpy(1.0, P, -1.0, targets[i])
            d2 = V.dot(diff, diff, w2d)
            phi = dsig * np.exp(-d2 * inv2L2)
            phip = -phi * inv2L2
            V.axpy(2.0 * phip, diff, 1.0, S_pen, out=S_pen)
            Phi += phi
            pen += 2.0 * phip
        return Phi, S_pen, pen

    def eval_state(Q, p):                                        # solver.py:814-837
        P = herm_project(density_from_Qp(Q, p))
        Sg, Hh, F = fock_full(P)
        E = float(hf_energy(P, h=h, Sigma=Sg, H=Hh, weights_b=w2d))
        pen = 0.0
        if has_defl:
            Phi, S_pen, pen = deflation_bias(P)
            E = E + Phi
            F = V.axpy(1.0, F, 1.0, S_pen)
        Ft = fock_in_orbital_basis(Q, F)
        G = torch.empty_like(Ft)
        _lib.check(V.L.hf_orbital_grad(V.s, V.nk, nb, Ft.data_ptr(), p.data_ptr(), G.data_ptr(), None))
        g = float(np.sqrt(max(0.0, V.dot(G, G, w_norm))))
        return E, Ft, g, pen

    # ---- init (solver.py:840-877) ----
    P0t = torch.as_tensor(P0).to(dev, cd)
    P0h = 0.5 * (P0t + P0t.transpose(-1, -2).conj())
    _, _, F0 = fock_full(P0h.contiguous())
    eps0, Q0 = eigh(F0)
    mu0 = solve_mu(eps0, 0.0)
    p0 = occupations(eps0, mu0)
    E0, Ft0, g0, pen0 = eval_state(Q0, p0)
    if g0 <= tol_g:
        p_i, mu_i = p0, mu0
        for _ in range(30):
            P = herm_project(density_from_Qp(Q0, p_i))
            _, _, F = fock_full(P)
            eps_i = torch.empty_like(p_i)
            Ftt = fock_in_orbital_basis(Q0, F)
            _lib.check(V.L.hf_real_diag(V.s, V.nk, nb, Ftt.data_ptr(), eps_i.data_ptr()))
            mu_i = solve_mu(eps_i, mu_i)
            p_i = occupations(eps_i, mu_i)
        p0, mu0 = p_i, mu_i
        E0, Ft0, g0, pen0 = eval_state(Q0, p0)

    hist_E = np.zeros(cfg.max_iter)
    hist_G = np.zeros(cfg.max_iter)
    k, Q, p, mu, Ft, E, Delta, grad_norm, pen = 0, Q0, p0, mu0, Ft0, E0, float(cfg.tr_delta0), g0, pen0
    wsum = torch.zeros((), dtype=rd, device=dev)
    while k < cfg.max_iter and grad_norm > tol_g and Delta > delta_min:
        hist_E[k] = E
        hist_G[k] = grad_norm
        G = torch.empty_like(Ft)
        eps = torch.empty_like(p)
        _lib.check(V.L.hf_orbital_grad(V.s, V.nk, nb, Ft.data_ptr(), p.data_ptr(), G.data_ptr(), eps.data_ptr()))
        eps_scale = float(np.sqrt(V.dot(ap=eps, bp=eps) / (V.nk * nb) + tiny))
        lam_pc = max(T_r, cfg.denom_scale * eps_scale)

        def prec(aX, ap):
            zX, zp = torch.empty_like(aX), torch.empty_like(ap)
            _lib.check(V.L.hf_newton_prec(V.s, V.nk, nb, aX.data_ptr(), ap.data_ptr(), eps.data_ptr(), p.data_ptr(),
                                          lam_pc, T_r, occ_clip, w2d.data_ptr(), zX.data_ptr(), zp.data_ptr(),
                                          wsum.data_ptr(), V.ws.data_ptr()))
            V.project_occ(zp, wsum)
            return zX, zp

        def hvp(X, dp):                                          # solver.py:916-930
            dP = torch.empty_like(X)
            _lib.check(V.L.hf_newton_dP(V.s, V.nk, nb, Q.data_ptr(), X.data_ptr(), dp.data_ptr(), p.data_ptr(),
                                        dP.data_ptr()))
            Fr = fock_response(dP)
            HX, Hp = torch.empty_like(X), torch.empty_like(dp)
            _lib.check(V.L.hf_newton_hvp(V.s, V.nk, nb, Q.data_ptr(), Ft.data_ptr(), X.data_ptr(), dp.data_ptr(),
                                         p.data_ptr(), Fr.data_ptr(), h.data_ptr(), T_r, occ_clip,
                                         float(pen) if has_defl else 0.0, dP.data_ptr() if has_defl else None,
                                         HX.data_ptr(), Hp.data_ptr(), w2d.data_ptr(), wsum.data_ptr(),
                                         V.ws.data_ptr()))
            V.project_occ(Hp, wsum)
            return HX, Hp

        # ---- Steihaug truncated CG (solver.py:932-992) ----
        rX = V.axpy(-1.0, G, 0.0, None)
        rp = V.zp()
        zX, zp = prec(rX, rp)
        rz = V.jip(rX, rp, zX, zp)
        vX, vp, HvX, Hvp = V.zX(), V.zp(), V.zX(), V.zp()
        dX, dp = zX, zp
        cg, done = 0, False
        while cg < cfg.tr_cg_max and not done:
            HdX, Hdp = hvp(dX, dp)
            dHd = V.jip(dX, dp, HdX, Hdp)
            dd = V.jip(dX, dp, dX, dp)
            neg = dHd <= 1e-14 * dd
            b = 2.0 * V.jip(vX, vp, dX, dp)
            cc = V.jip(vX, vp, vX, vp) - Delta * Delta
            disc = max(b ** 2 - 4.0 * dd * cc, 0.0)
            t_bd = (-b + np.sqrt(disc)) / (2.0 * dd + 1e-30)
            alpha = rz / (1.0 if neg else dHd)
            vXa, vpa = V.axpy(1.0, vX, alpha, dX), V.axpy(1.0, vp, alpha, dp)
            cross = np.sqrt(max(0.0, V.jip(vXa, vpa, vXa, vpa))) >= Delta
            take_bd = neg or cross
            rXa, rpa = V.axpy(1.0, rX, -alpha, HdX), V.axpy(1.0, rp, -alpha, Hdp)
            rn = np.sqrt(max(0.0, V.jip(rXa, rpa, rXa, rpa)))
            inner = rn < 0.05 * grad_norm
            zXa, zpa = prec(rXa, rpa)
            rz_new = V.jip(rXa, rpa, zXa, zpa)
            beta = rz_new / (rz if abs(rz) > tiny else 1.0)
            stop = take_bd or inner
            if take_bd:
                vX, vp = V.axpy(1.0, vX, t_bd, dX), V.axpy(1.0, vp, t_bd, dp)
                HvX, Hvp = V.axpy(1.0, HvX, t_bd, HdX), V.axpy(1.0, Hvp, t_bd, Hdp)
            else:
                vX, vp = vXa, vpa
                HvX, Hvp = V.axpy(1.0, HvX, alpha, HdX), V.axpy(1.0, Hvp, alpha, Hdp)
                rX, rp = rXa, rpa
            if not stop:
                dX, dp = V.axpy(1.0, zXa, beta, dX), V.axpy(1.0, zpa, beta, dp)
                rz = rz_new
            cg += 1
            done = stop

        # ---- predicted reduction and trial step (solver.py:998-1046) ----
        gv = V.dot(G, vX, w2d)
        vHv = V.dot(vX, HvX, w2d, vp, Hvp, w2d)
        pred = -(gv + 0.5 * vHv)
        Vv, lamv = cayley_spectral_setup(vX)
        U = cayley_unitary_from_spectrum(Vv, lamv, -1.0)
        Qt = torch.empty_like(Q)
        _lib.check(V.L.hf_matmul(V.s, V.nk, nb, Q.data_ptr(), U.data_ptr(), Qt.data_ptr()))
        Ftf = fock_in_orbital_basis(U, Ft)
        eps_t = torch.empty_like(p)
        _lib.check(V.L.hf_real_diag(V.s, V.nk, nb, Ftf.data_ptr(), eps_t.data_ptr()))
        mu_t = solve_mu(eps_t, mu)
        p_trial = occupations(eps_t, mu_t)
        E_t, Ft_t, g_t, pen_t = eval_state(Qt, p_trial)
        noise = noise_floor * max(abs(E), 1.0)
        use_g = pred <= noise
        accept_g = g_t <= grad_norm and E_t <= E + noise
        Delta_g = Delta if accept_g else 0.5 * Delta
        ratio = (E - E_t) / (1.0 if use_g else pred)
        step_norm = np.sqrt(max(0.0, V.jip(vX, vp, vX, vp)))
        if ratio < 0.25:
            Delta_r = 0.25 * Delta
        elif ratio > 0.75 and step_norm > 0.9 * Delta:
            Delta_r = min(2.0 * Delta, 5.0)
        else:
            Delta_r = Delta
        accept = accept_g if use_g else ratio > 0.1
        Delta = Delta_g if use_g else Delta_r
        if accept:
            Q, p, Ft, E, mu, grad_norm, pen = Qt, p_trial, Ft_t, E_t, mu_t, g_t, pen_t
        k += 1

    P_fin = herm_project(density_from_Qp(Q, p))                  # solver.py:1062-1066
    Sg, Hf, Ff = fock_full(P_fin)
    E_fin = hf_energy(P_fin, h=h, Sigma=Sg, H=Hf, weights_b=w2d)
    out_c, out_r = kernel.dtype, kernel.real_dtype
    hist = dict(E=torch.as_tensor(hist_E, dtype=out_r), grad_norm=torch.as_tensor(hist_G, dtype=out_r),
                n_builds=n_builds[0])
    return SolveResult(Q=Q.to(out_c), p=p.to(out_r), mu=torch.tensor(mu, dtype=out_r), density=P_fin.to(out_c),
                       fock=Ff.to(out_c), energy=E_fin, n_iter=torch.tensor(k, dtype=torch.int32),
                       converged=torch.tensor(bool(grad_norm <= tol_g)), history=hist)
