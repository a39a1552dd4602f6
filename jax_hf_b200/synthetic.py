"""Seeded synthetic Hartree-Fock problems on square k-meshes (NumPy only).

Conventions follow the reference's grid convention (problem.py:90-98,
utils.py:490): square reciprocal lattice b1=(2pi,0), b2=(0,2pi); centered
storage k_m = 2 pi (m - nk//2)/nk (k=0 at index nk//2); the momentum transfer q
uses the same centered grid, which is already the minimal image in [-pi, pi);
uniform weights 1/nk^2 (so the electron count is sum_k w_k sum_i p_i and
"2 electrons per k" means ``n_electrons = 2.0``).

Workloads (the reference publishes no dataset; these stand in for its shapes):

* ``fourier_model``  H(k) = sum_{|R|<=rmax} h_R e^{i k.R}, h_{-R} = h_R^H, entries of
  h_R complex N(0,1)/(1+|R|^2) from ``numpy.random.default_rng(seed)``.
* ``coulomb_scalar`` V(q) = U 2pi tanh(|q| d)/|q|, V(0) = 0, shape (nk,nk,1,1).
* ``coulomb_layer``  V_ab(q) = U 2pi tanh(|q| d_ab)/|q|, d_ab = d0 + |a-b|/2, V(0)=0.
* ``haar_density``   P(k) = U(k) diag(f) U(k)^H, U Haar (QR of a complex Ginibre
  matrix with the diag(R) phase fix), f ~ Uniform(0,1).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


def lattice_vectors(rmax: float):
    """Integer R with |R|^2 <= rmax^2, in a fixed order."""
    r = int(np.floor(rmax))
    out = []
    for rx in range(-r, r + 1):
        for ry in range(-r, r + 1):
            if rx * rx + ry * ry <= rmax * rmax + 1e-9:
                out.append((rx, ry))
    return out


def half_space(R):
    return R[0] > 0 or (R[0] == 0 and R[1] > 0)


def kgrid(nk: int):
    return 2.0 * np.pi * (np.arange(nk) - nk // 2) / nk


def fourier_coeffs(nb: int, rmax: float, seed: int):
    """h_R for every R with |R| <= rmax; h_{-R} = h_R^H and h_0 Hermitian."""
    rng = np.random.default_rng(seed)
    coeffs = {}
    for R in lattice_vectors(rmax):
        if R == (0, 0):
            a = rng.standard_normal((nb, nb)) + 1j * rng.standard_normal((nb, nb))
            coeffs[R] = 0.5 * (a + a.conj().T)
        elif half_space(R):
            a = (rng.standard_normal((nb, nb)) + 1j * rng.standard_normal((nb, nb)))
            a = a / (1.0 + R[0] ** 2 + R[1] ** 2)
            coeffs[R] = a
            coeffs[(-R[0], -R[1])] = a.conj().T
    return coeffs


def hamiltonian_from_coeffs(coeffs, nk: int):
    ks = kgrid(nk)
    kx, ky = np.meshgrid(ks, ks, indexing="ij")
    nb = next(iter(coeffs.values())).shape[0]
    H = np.zeros((nk, nk, nb, nb), np.complex128)
    for R, hR in coeffs.items():
        H += np.exp(1j * (kx * R[0] + ky * R[1]))[..., None, None] * hR[None, None]
    return np.ascontiguousarray(0.5 * (H + np.conj(np.swapaxes(H, -1, -2))))


def _qabs(nk: int):
    qs = kgrid(nk)
    qx, qy = np.meshgrid(qs, qs, indexing="ij")
    return np.sqrt(qx * qx + qy * qy)


def _screened(q, d, U):
    out = np.zeros_like(q)
    nz = q > 0
    out[nz] = U * 2.0 * np.pi * np.tanh(q[nz] * d) / q[nz]
    return out


def coulomb_scalar(nk: int, U: float = 1.0, d: float = 2.0):
    return _screened(_qabs(nk), d, U)[..., None, None]


def coulomb_layer(nk: int, nb: int, U: float = 1.0, d0: float = 1.0):
    q = _qabs(nk)
    V = np.zeros((nk, nk, nb, nb))
    for a in range(nb):
        for b in range(nb):
            V[..., a, b] = _screened(q, d0 + abs(a - b) / 2.0, U)
    return V


def haar_unitaries(shape, nb: int, rng):
    Z = (rng.standard_normal(shape + (nb, nb)) + 1j * rng.standard_normal(shape + (nb, nb))) / np.sqrt(2)
    Qm, R = np.linalg.qr(Z)
    d = np.diagonal(R, axis1=-2, axis2=-1)
    return Qm * (d / np.abs(d))[..., None, :]


def haar_density(nk: int, nb: int, seed: int):
    rng = np.random.default_rng(seed)
    U = haar_unitaries((nk, nk), nb, rng)
    f = rng.uniform(0.0, 1.0, size=(nk, nk, nb))
    P = np.einsum("...in,...n,...jn->...ij", U, f, np.conj(U))
    return np.ascontiguousarray(0.5 * (P + np.conj(np.swapaxes(P, -1, -2))))


@dataclass
class Problem:
    """Inputs of a ``HartreeFockKernel`` plus the solve parameters."""
    name: str
    weights: np.ndarray
    hamiltonian: np.ndarray
    coulomb_q: np.ndarray
    T: float
    n_electrons: float
    nk: int
    nb: int

    def kernel_kwargs(self):
        return dict(weights=self.weights, hamiltonian=self.hamiltonian,
                    coulomb_q=self.coulomb_q, T=self.T)


def fourier_problem(nk, nb, rmax, seed, *, V="scalar", U=1.0, d=2.0, T=0.1, n_electrons=None,
                    name="fourier"):
    h = hamiltonian_from_coeffs(fourier_coeffs(nb, rmax, seed), nk)
    if V == "scalar":
        Vq = coulomb_scalar(nk, U, d)
    else:
        Vq = coulomb_layer(nk, nb, U)
    w = np.full((nk, nk), 1.0 / (nk * nk))
    ne = 0.5 * nb if n_electrons is None else float(n_electrons)
    return Problem(name, w, h, Vq, float(T), ne, nk, nb)


def scf_diis_24():
    """4 bands, 24x24 mesh, |R|<=2, scalar gate-screened V (U=1, d=2), T=0.1, half filling."""
    return fourier_problem(24, 4, 2.0, seed=0, V="scalar", U=1.0, d=2.0, T=0.1,
                           n_electrons=2.0, name="scf_diis_24x24_nb4")


def fock_build_192(seed: int = 1):
    """192x192 mesh, nb=8, layer-resolved V; returns (problem, P)."""
    prob = fourier_problem(192, 8, 3.0, seed=seed, V="layer", T=0.05, n_electrons=3.0,
                           name="fock_build_192x192_nb8")
    return prob, haar_density(192, 8, seed + 1000)


def cg_144(seed: int = 2):
    """144x144 mesh, nb=8, |R|<=3, layer-resolved V, T=0.05, filling 3/8."""
    return fourier_problem(144, 8, 3.0, seed=seed, V="layer", T=0.05, n_electrons=3.0,
                           name="cg_144x144_nb8")


def newton_96(seed: int = 3):
    """96x96 mesh, nb=4, the scalar-V Fourier model of ``scf_diis_24``."""
    return fourier_problem(96, 4, 2.0, seed=seed, V="scalar", U=1.0, d=2.0, T=0.1,
                           n_electrons=2.0, name="newton_96x96_nb4")


def density_scan(n: int = 64, seed: int = 4):
    """n independent solves: mesh from {36,48,72,96,120}, nb from {4,6,8}, filling in (0.1, 0.9)."""
    rng = np.random.default_rng(seed)
    meshes = rng.choice([36, 48, 72, 96, 120], size=n)
    nbs = rng.choice([4, 6, 8], size=n)
    out = []
    for i in range(n):
        filling = 0.1 + 0.8 * (i + 0.5) / n
        nb = int(nbs[i])
        out.append(fourier_problem(int(meshes[i]), nb, 2.0, seed=seed * 1000 + i,
                                   V="scalar" if i % 2 == 0 else "layer", T=0.1,
                                   n_electrons=filling * nb, name=f"scan_{i}"))
    return out


def coulomb_scalar_derivatives(nk: int, U: float = 1.0, d: float = 2.0):
    """dV/dU and dV/dd of the gate-screened V(q) = U 2 pi tanh(|q| d) / |q| (V(0) = 0)."""
    q = _qabs(nk)
    dU = np.zeros_like(q)
    dd = np.zeros_like(q)
    nz = q > 0
    dU[nz] = 2.0 * np.pi * np.tanh(q[nz] * d) / q[nz]
    dd[nz] = U * 2.0 * np.pi / np.cosh(q[nz] * d) ** 2
    return {"U": dU[..., None, None], "d": dd[..., None, None]}


def coulomb_layer_derivatives(nk: int, nb: int, U: float = 1.0, d0: float = 1.0):
    """dV/dU and dV/dd0 of the layer-resolved V_ab(q) with d_ab = d0 + |a - b| / 2."""
    q = _qabs(nk)
    nz = q > 0
    dU = np.zeros((nk, nk, nb, nb))
    dd = np.zeros((nk, nk, nb, nb))
    for a in range(nb):
        for b in range(nb):
            dab = d0 + abs(a - b) / 2.0
            t = np.zeros_like(q)
            t[nz] = 2.0 * np.pi * np.tanh(q[nz] * dab) / q[nz]
            dU[..., a, b] = t
            s = np.zeros_like(q)
            s[nz] = U * 2.0 * np.pi / np.cosh(q[nz] * dab) ** 2
            dd[..., a, b] = s
    return {"U": dU, "d": dd}
