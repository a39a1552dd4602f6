"""Per-k small-matrix operations on the GPU (one warp per k-point).

Wrappers of the C ABI for the nb x nb kernels used by the solvers
(solver.py:42-49, 108-197; linalg.eigh).  Leading axes are flattened into a
batch; tau is a Python float.
"""

from __future__ import annotations

import torch

from . import _lib
from .fock import _as_dev


def _batch(A: torch.Tensor):
    nb = int(A.shape[-1])
    return A.numel() // (nb * nb), nb


def _real(dt):
    return torch.float64 if dt == torch.complex128 else torch.float32


def eigh(A):
    """Hermitian eigendecomposition (input hermitised), ascending eigenvalues; A = V diag(w) V^H."""
    A = _as_dev(A)
    if not A.is_complex():
        A = A.to(torch.complex128 if A.dtype == torch.float64 else torch.complex64)
    batch, nb = _batch(A)
    w = torch.empty(A.shape[:-1], dtype=_real(A.dtype), device=A.device)
    V = torch.empty_like(A)
    _lib.check(_lib.lib().hf_eigh(_lib.stream_ptr(A.device), _lib.dtype_code(A), batch, nb, A.data_ptr(),
                                  w.data_ptr(), V.data_ptr()))
    return w, V


def density_from_Qp(Q, p):
    """P = herm(Q diag(p) Q^H)."""
    Q = _as_dev(Q)
    batch, nb = _batch(Q)
    p = _as_dev(p, Q.device, _real(Q.dtype))
    P = torch.empty_like(Q)
    _lib.check(_lib.lib().hf_density_from_Qp(_lib.stream_ptr(Q.device), _lib.dtype_code(Q), batch, nb,
                                             Q.data_ptr(), p.data_ptr(), P.data_ptr()))
    return P


def fock_in_orbital_basis(Q, F):
    """Ft = Q^H F Q."""
    Q = _as_dev(Q)
    F = _as_dev(F, Q.device, Q.dtype)
    batch, nb = _batch(Q)
    Ft = torch.empty_like(Q)
    _lib.check(_lib.lib().hf_fock_orbital(_lib.stream_ptr(Q.device), _lib.dtype_code(Q), batch, nb,
                                          Q.data_ptr(), F.data_ptr(), Ft.data_ptr()))
    return Ft


def cayley_retract(d, tau: float):
    """U = (I + tau d/2)^-1 (I - tau d/2) by LU with partial pivoting (solver.py:122-138)."""
    d = _as_dev(d)
    batch, nb = _batch(d)
    U = torch.empty_like(d)
    _lib.check(_lib.lib().hf_cayley_retract(_lib.stream_ptr(d.device), _lib.dtype_code(d), batch, nb,
                                            d.data_ptr(), float(tau), U.data_ptr()))
    return U


def cayley_spectral_setup(d):
    """(V, lam) = eigh(herm(i d)) (solver.py:161-166)."""
    d = _as_dev(d)
    batch, nb = _batch(d)
    V = torch.empty_like(d)
    lam = torch.empty(d.shape[:-1], dtype=_real(d.dtype), device=d.device)
    _lib.check(_lib.lib().hf_cayley_spectral(_lib.stream_ptr(d.device), _lib.dtype_code(d), batch, nb,
                                             d.data_ptr(), V.data_ptr(), lam.data_ptr()))
    return V, lam


def cayley_unitary_from_spectrum(V, lam, tau: float):
    """U = V diag(c(tau, lam)) V^H (solver.py:178-182)."""
    V = _as_dev(V)
    lam = _as_dev(lam, V.device, _real(V.dtype))
    batch, nb = _batch(V)
    U = torch.empty_like(V)
    _lib.check(_lib.lib().hf_cayley_unitary(_lib.stream_ptr(V.device), _lib.dtype_code(V), batch, nb,
                                            V.data_ptr(), lam.data_ptr(), float(tau), U.data_ptr()))
    return U


def diag_UFU_from_spectrum(V, Ft_eig, lam, tau: float):
    """diag(U(tau)^H Ft U(tau)) from Ft_eig = V^H Ft V (solver.py:185-197)."""
    V = _as_dev(V)
    Fe = _as_dev(Ft_eig, V.device, V.dtype)
    lam = _as_dev(lam, V.device, _real(V.dtype))
    batch, nb = _batch(V)
    out = torch.empty(V.shape[:-1], dtype=_real(V.dtype), device=V.device)
    _lib.check(_lib.lib().hf_diag_UFU(_lib.stream_ptr(V.device), _lib.dtype_code(V), batch, nb, V.data_ptr(),
                                      Fe.data_ptr(), lam.data_ptr(), float(tau), out.data_ptr()))
    return out


def qr_retract(G, tau: float):
    """U = QR(I - tau G) with the diag(R) phase normalised (solver.py:108-119)."""
    G = _as_dev(G)
    batch, nb = _batch(G)
    U = torch.empty_like(G)
    _lib.check(_lib.lib().hf_qr_retract(_lib.stream_ptr(G.device), _lib.dtype_code(G), batch, nb, G.data_ptr(),
                                        float(tau), U.data_ptr()))
    return U
