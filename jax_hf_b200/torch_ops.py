"""PyTorch operator registrations (``torch.ops.hf_b200.*``).

The Fock build and the HF energy as ``torch.library`` custom ops, so PyTorch
programs (FX graphs, ``torch.compile`` regions that keep them as opaque calls,
other frameworks' dispatchers) can call the CUDA kernels by name.  Each op has a
fake (meta) implementation for shape propagation and an autograd formula that
runs the hand-written adjoints of ``adjoint.py`` / ``csrc/adjoint.cu``:

* ``hf_b200::fock_build(P, h, VR, include_exchange, packing)``
  -> (Sigma, H, F), the interface of build_fock (fock.py:18-97) without refP,
  Hartree matrix or contact terms (use ``jax_hf_b200.build_fock`` for those);
  differentiable in P and h.
* ``hf_b200::hf_energy(P, h, Sigma, H, w2d)`` -> E (fock.py:100-111); differentiable in
  P, h, Sigma and H.
"""

from __future__ import annotations

import ctypes as C

import torch

from . import _lib


@torch.library.custom_op("hf_b200::fock_build", mutates_args=())
def fock_build(P: torch.Tensor, h: torch.Tensor, VR: torch.Tensor, include_exchange: bool,
               packing: bool) -> tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
    from .fock import build_fock
    nb = int(P.shape[-1])
    Sg, H, F = build_fock(P, h=h, VR=VR, refP=None, HH=None, w2d=None, include_exchange=include_exchange,
                          include_hartree=False, exchange_hermitian_channel_packing=packing)
    return Sg, H.reshape(1, 1, nb, nb).clone(), F


@fock_build.register_fake
def _fock_build_fake(P, h, VR, include_exchange, packing):
    nb = P.shape[-1]
    return torch.empty_like(P), P.new_empty((1, 1, nb, nb)), torch.empty_like(P)


def _fock_setup(ctx, inputs, output):
    P, h, VR, include_exchange, packing = inputs
    ctx.save_for_backward(VR)
    ctx.include_exchange = include_exchange
    ctx.shape = tuple(P.shape)


def _fock_backward(ctx, gS, gH, gF):
    (VR,) = ctx.saved_tensors
    nk1, nk2, nb = ctx.shape[0], ctx.shape[1], ctx.shape[-1]
    dev = VR.device
    flags = 0
    if ctx.include_exchange:
        flags |= _lib.FOCK_EXCHANGE
        if not VR.is_complex():
            flags |= _lib.FOCK_VR_REAL
        if tuple(VR.shape[-2:]) == (1, 1):
            flags |= _lib.FOCK_VR_SCALAR
    VR_adj = VR.conj().resolve_conj().contiguous() if VR.is_complex() else VR.contiguous()
    zeros = torch.zeros(ctx.shape, dtype=torch.complex128, device=dev)
    gS = zeros if gS is None else gS.to(torch.complex128).contiguous()
    gF = zeros if gF is None else gF.to(torch.complex128).contiguous()
    Pb, hb = torch.empty_like(zeros), torch.empty_like(zeros)
    need = C.c_size_t(0)
    _lib.check(_lib.lib().hf_fock_vjp_workspace_size(_lib.HF_C128, flags, nk1, nk2, nb, C.byref(need)))
    ws = torch.empty(max(need.value, 256), dtype=torch.uint8, device=dev)
    _lib.check(_lib.lib().hf_fock_build_vjp(_lib.stream_ptr(dev), _lib.HF_C128, flags, nk1, nk2, nb, gS.data_ptr(),
                                            gF.data_ptr(), _lib.ptr(VR_adj), Pb.data_ptr(), hb.data_ptr(),
                                            ws.data_ptr(), ws.numel()))
    # H is zero without Hartree: its cotangent does not reach P or h
    return Pb, hb, None, None, None


fock_build.register_autograd(_fock_backward, setup_context=_fock_setup)


@torch.library.custom_op("hf_b200::hf_energy", mutates_args=())
def hf_energy(P: torch.Tensor, h: torch.Tensor, Sigma: torch.Tensor, H: torch.Tensor,
              w2d: torch.Tensor) -> torch.Tensor:
    from .fock import hf_energy as _energy
    return _energy(P, h=h, Sigma=Sigma, H=H, weights_b=w2d[..., None, None]).clone()


@hf_energy.register_fake
def _hf_energy_fake(P, h, Sigma, H, w2d):
    return P.new_empty((), dtype=torch.float64)


def _energy_setup(ctx, inputs, output):
    P, h, Sigma, H, w2d = inputs
    ctx.save_for_backward(P, h, Sigma, H, w2d)


def _energy_backward(ctx, gE):
    P, h, Sigma, H, w2d = ctx.saved_tensors
    nk1, nk2, nb = P.shape[0], P.shape[1], P.shape[-1]
    Ht = H.reshape(nb, nb).to(torch.complex128).contiguous()
    w = w2d.to(torch.float64).contiguous()
    Pb, hb, Sb = torch.empty_like(P), torch.empty_like(P), torch.empty_like(P)
    Eb = float(gE)
    _lib.check(_lib.lib().hf_energy_vjp(_lib.stream_ptr(P.device), nk1, nk2, nb, P.data_ptr(), h.data_ptr(),
                                        Sigma.data_ptr(), Ht.data_ptr(), 1, w.data_ptr(), Eb, Pb.data_ptr(),
                                        hb.data_ptr(), Sb.data_ptr()))
    from .adjoint import _k_sum
    Hb = (0.5 * Eb) * _k_sum(P.transpose(-1, -2).conj(), w).reshape(H.shape)
    return Pb, hb, Sb, Hb, None


hf_energy.register_autograd(_energy_backward, setup_context=_energy_setup)

__all__ = ["fock_build", "hf_energy"]
