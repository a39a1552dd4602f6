"""Hand-written reverse mode of the Fock build and the HF objective.

The reference obtains gradients by ``jax.grad`` through ``build_fock`` /
``hf_energy`` / ``free_energy`` (fock.py:18-129).  Here the adjoints are
explicit CUDA kernels behind ``torch.autograd.Function``:

* ``fock_build(P, h, kernel)`` -> (Sigma, H, F), differentiable in P and h.  The
  exchange self-energy is the C-linear map ``A(dP) = -IFFT2(VR . FFT2(dP))``; its
  VJP is ``A^H`` = the same Fock-build kernels run on the cotangent with
  ``conj(VR)`` (``hf_fock_build_vjp``).  The Hartree and contact terms are
  linear maps of the k-summed density ``rho = sum_k w_k dP_k`` (fock.py:66-92)
  and are differentiated through a small nb x nb torch graph.
* ``hf_energy`` / ``free_energy``: ``hf_energy_vjp`` / ``hf_free_energy_vjp``.
* ``parameter_gradients``: derivatives of the converged free energy with respect
  to interaction parameters (through dV/dtheta) and to Fourier coefficients h_R
  of the Hamiltonian.  At a converged stationary point of Omega over the density
  at fixed electron count, the occupation / mu implicit terms vanish (envelope
  theorem), so dOmega*/dtheta is the partial derivative at fixed P:
  ``1/2 sum_k w_k Re tr(Sigma_{dV/dtheta}[dP] P)`` for the coupling (one Fock
  build with dV/dtheta) and ``sum_k w_k exp(-i k.R) P_k`` for h_R.
"""

from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np
import torch

from . import _lib
from .problem import is_marked_zero, shift_phase


def _flags(kernel, VR):
    f = 0
    if kernel.include_exchange:
        f |= _lib.FOCK_EXCHANGE
        if not VR.is_complex():
            f |= _lib.FOCK_VR_REAL
        if tuple(VR.shape[-2:]) == (1, 1):
            f |= _lib.FOCK_VR_SCALAR
    return f


def _k_sum(X, w2d):
    """sum_k w_k X_k (nb x nb) with the CUDA Fourier-coefficient reduction at R = 0."""
    nk1, nk2, nb = X.shape[0], X.shape[1], X.shape[-1]
    out = torch.empty((1, nb, nb), dtype=torch.complex128, device=X.device)
    R = torch.zeros(2, dtype=torch.int32, device=X.device)
    Xc = X.to(torch.complex128).contiguous()
    w = w2d.to(torch.float64).contiguous()
    _lib.check(_lib.lib().hf_fourier_coeffs(_lib.stream_ptr(X.device), nk1, nk2, nb, Xc.data_ptr(),
                                            w.data_ptr(), 1, R.data_ptr(), out.data_ptr()))
    return out[0]


def _consts(rho, kernel):
    """Hartree matrix and contact self-energy from rho = sum_k w dP (fock.py:66-92), torch ops on nb x nb."""
    nb = rho.shape[-1]
    H = torch.zeros((nb, nb), dtype=rho.dtype, device=rho.device)
    if kernel.include_hartree:
        n = torch.real(torch.diagonal(rho))
        H = torch.diag((kernel.HH.to(torch.float64) @ n).to(rho.dtype))
    sc = torch.zeros_like(H)
    if kernel.has_contact:
        g = kernel.contact_g.to(torch.float64).to(rho.dtype)
        Oi, Oj = kernel.contact_Oi.to(rho.dtype), kernel.contact_Oj.to(rho.dtype)
        tr = torch.einsum("tij,ji->t", Oj, rho)
        sc = torch.einsum("t,tij->ij", g * tr, Oi) - torch.einsum("t,tij,jk,tkl->il", g, Oi, rho, Oj)
    return H, sc


class _FockBuildFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, P, h, kernel):
        from .fock import build_fock
        a = kernel.as_args()
        Sg, H, F = build_fock(P, h=h, VR=a["VR"], refP=a["refP"], HH=a["HH"], w2d=kernel.w2d,
                              include_exchange=kernel.include_exchange, include_hartree=kernel.include_hartree,
                              exchange_hermitian_channel_packing=a["exchange_hermitian_channel_packing"],
                              contact_g=a["contact_g"], contact_Oi=a["contact_Oi"], contact_Oj=a["contact_Oj"])
        ctx.kernel = kernel
        ctx.save_for_backward(P)
        return Sg, H, F

    @staticmethod
    def backward(ctx, gS, gH, gF):
        kernel = ctx.kernel
        (P,) = ctx.saved_tensors
        nk1, nk2, nb = kernel.shape
        dev = P.device
        VR = kernel._VR_shifted
        VR_adj = VR.conj().resolve_conj().contiguous() if VR.is_complex() else VR
        flags = _flags(kernel, VR)
        gS = torch.zeros_like(P) if gS is None else gS.to(torch.complex128).contiguous()
        gF = torch.zeros_like(P) if gF is None else gF.to(torch.complex128).contiguous()
        Pb = torch.empty_like(P)
        hb = torch.empty_like(P)
        need = C.c_size_t(0)
        _lib.check(_lib.lib().hf_fock_vjp_workspace_size(_lib.HF_C128, flags, nk1, nk2, nb, C.byref(need)))
        ws = _lib.workspace(need.value, dev, "fock_vjp")
        _lib.check(_lib.lib().hf_fock_build_vjp(_lib.stream_ptr(dev), _lib.HF_C128, flags, nk1, nk2, nb,
                                                gS.data_ptr(), gF.data_ptr(), _lib.ptr(VR_adj), Pb.data_ptr(),
                                                hb.data_ptr(), ws.data_ptr(), ws.numel()))
        if kernel.include_hartree or kernel.has_contact:
            # the k-independent terms: H enters F at every k; the contact term enters Sigma and F
            w2d = kernel.w2d.to(torch.float64).contiguous()
            ones = torch.ones_like(w2d)
            Fh = 0.5 * (gF + gF.transpose(-1, -2).conj())
            terms, cots = [], []
            refP = kernel.refP
            dP = P if is_marked_zero(refP) else P - refP.to(torch.complex128)
            rho = _k_sum(dP, w2d).detach().requires_grad_(True)
            with torch.enable_grad():
                Hm, sc = _consts(rho, kernel)
                if kernel.include_hartree:
                    cH = _k_sum(Fh, ones)
                    if gH is not None:
                        cH = cH + gH.reshape(nb, nb).to(torch.complex128)
                    terms.append(Hm)
                    cots.append(cH)
                if kernel.has_contact:
                    terms.append(sc)
                    cots.append(_k_sum(Fh + gS, ones))
                (grho,) = torch.autograd.grad(terms, [rho], cots, allow_unused=True)
            if grho is not None:
                Pb = Pb + w2d[..., None, None].to(torch.complex128) * grho
        return Pb, hb, None


def fock_build(P, h, kernel):
    """Differentiable (Sigma, H, F) = build_fock(P) for a complex128 kernel (gradients in P and h)."""
    if kernel.dtype != torch.complex128:
        raise ValueError("the hand-written adjoint runs in complex128; build the kernel in complex128")
    return _FockBuildFn.apply(P, h, kernel)


class _EnergyFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, P, h, Sigma, H, w2d):
        from .fock import hf_energy
        E = hf_energy(P, h=h, Sigma=Sigma, H=H, weights_b=w2d[..., None, None])
        ctx.save_for_backward(P, h, Sigma, H, w2d)
        return E

    @staticmethod
    def backward(ctx, gE):
        P, h, Sigma, H, w2d = ctx.saved_tensors
        nk1, nk2, nb = P.shape[0], P.shape[1], P.shape[-1]
        Ht = H.reshape(nb, nb).to(torch.complex128).contiguous()
        Pb, hb, Sb = torch.empty_like(P), torch.empty_like(P), torch.empty_like(P)
        Eb = float(gE)
        _lib.check(_lib.lib().hf_energy_vjp(_lib.stream_ptr(P.device), nk1, nk2, nb, P.data_ptr(), h.data_ptr(),
                                            Sigma.data_ptr(), Ht.data_ptr(), 1, w2d.data_ptr(), Eb, Pb.data_ptr(),
                                            hb.data_ptr(), Sb.data_ptr()))
        Hb = (0.5 * Eb) * _k_sum(P.transpose(-1, -2).conj(), w2d).reshape(H.shape)
        return Pb, hb, Sb, Hb, None


def hf_energy(P, h, Sigma, H, w2d):
    """Differentiable E = sum_k w_k Re tr((h + (Sigma + H)/2) P) (fock.py:100-111); H is (1, 1, nb, nb)."""
    return _EnergyFn.apply(P.contiguous(), h.contiguous(), Sigma.contiguous(), H.contiguous(),
                           w2d.to(torch.float64).contiguous())


class _FreeEnergyFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, E, p, w_norm, T):
        from .fock import free_energy
        ctx.save_for_backward(p, w_norm)
        ctx.T = float(T)
        return free_energy(E, p, w_norm, T)

    @staticmethod
    def backward(ctx, gO):
        p, w_norm = ctx.saved_tensors
        nb = p.shape[-1]
        nk = p.numel() // nb
        pb = torch.empty_like(p)
        _lib.check(_lib.lib().hf_free_energy_vjp(_lib.stream_ptr(p.device), nk, 1, nb, p.data_ptr(),
                                                 w_norm.data_ptr(), ctx.T, float(gO), pb.data_ptr()))
        return gO, pb, None, None


def free_energy(E, p, w_norm, T):
    """Differentiable Omega = E - max(T, 1e-14) S(p) (fock.py:121-129)."""
    return _FreeEnergyFn.apply(E, p.to(torch.float64).contiguous(), w_norm.to(torch.float64).contiguous(), T)


def objective(P, p, kernel, h=None):
    """Omega(P, p) = hf_energy(P, h, Sigma[P], H[P]) - T S(p), differentiable in P, p and h."""
    h = kernel.h.to(torch.complex128) if h is None else h
    Sg, H, _ = fock_build(P, h, kernel)
    E = hf_energy(P, h, Sg, H.reshape(1, 1, *H.shape[-2:]), kernel.w2d)
    wn = kernel.w2d.to(torch.float64) / max(float(kernel.weight_sum), 1e-30)
    return free_energy(E, p, wn, kernel.T)


def shifted_vr(dV, weights):
    """VR of an interaction array dV (nk1, nk2, a, b) as HartreeFockKernel builds it (problem.py:88-98)."""
    dV = np.asarray(dV)
    w = np.asarray(weights, dtype=np.float64)[..., None, None]
    VR = np.fft.fftn(w * dV.astype(np.complex128), axes=(0, 1)) * shift_phase(dV.shape[0], dV.shape[1])
    if float(np.max(np.abs(VR.imag))) <= 1e-14 * max(float(np.max(np.abs(VR))), 1e-300):
        return np.ascontiguousarray(VR.real)
    return np.ascontiguousarray(VR)


def coupling_gradient(kernel, P, dV):
    """1/2 sum_k w_k Re tr(Sigma_{dV}[P - refP] P): d hf_energy / d theta at fixed P for V -> V + theta dV."""
    from .fock import build_fock, hf_energy as _hf_energy
    dev = P.device
    VRd = torch.as_tensor(shifted_vr(dV, kernel.w2d.cpu().numpy()), device=dev)
    if not VRd.is_complex():
        VRd = VRd.to(torch.float64)
    packing = bool(tuple(VRd.shape[-2:]) == (1, 1) and not VRd.is_complex())
    zero_h = torch.zeros_like(P)
    a = kernel.as_args()
    Sd, _, _ = build_fock(P, h=zero_h, VR=VRd, refP=a["refP"], HH=None, w2d=kernel.w2d, include_exchange=True,
                          include_hartree=False, exchange_hermitian_channel_packing=packing)
    return _hf_energy(P, h=zero_h, Sigma=Sd, H=None, weights_b=kernel.w2d[..., None, None])


def fourier_coefficient_gradient(P, w2d, R: Sequence[tuple[int, int]]):
    """sum_k w_k exp(-i k.R) P_k for every R (k on the centred grid): d E / d h_R for independent h_R."""
    nk1, nk2, nb = P.shape[0], P.shape[1], P.shape[-1]
    Rt = torch.as_tensor(np.asarray(R, dtype=np.int32).reshape(-1), device=P.device)
    out = torch.empty((len(R), nb, nb), dtype=torch.complex128, device=P.device)
    w = w2d.to(torch.float64).contiguous()
    Pc = P.to(torch.complex128).contiguous()
    _lib.check(_lib.lib().hf_fourier_coeffs(_lib.stream_ptr(P.device), nk1, nk2, nb, Pc.data_ptr(), w.data_ptr(),
                                            len(R), Rt.data_ptr(), out.data_ptr()))
    return out


def parameter_gradients(kernel, density, *, coupling_derivatives=None, lattice_vectors=None):
    """Gradients of the converged free energy (envelope theorem, see the module docstring).

    coupling_derivatives: {name: dV/dtheta array shaped like the kernel's V(q)};
    lattice_vectors: the R for which d Omega / d h_R (independent h_R) is returned under "h_R".
    """
    P = density.to(torch.complex128).contiguous()
    out = {}
    for name, dV in (coupling_derivatives or {}).items():
        out[name] = float(coupling_gradient(kernel, P, dV))
    if lattice_vectors:
        out["h_R"] = fourier_coefficient_gradient(P, kernel.w2d, lattice_vectors)
    return out
