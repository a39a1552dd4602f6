"""HartreeFockKernel: precomputed device arrays for the Fock build and solvers.

Mirrors jax_hf.problem.HartreeFockKernel (problem.py:22-217): same constructor
arguments, validation messages, attributes and ``as_args()`` keys.  The
one-off precompute (VR = FFT2(w V) with the ifftshift phase absorbed,
problem.py:88-98) runs on the host in float64; the arrays then live on the GPU
as torch tensors.  When the phase-shifted VR is real to round-off (any V that is
even in q on the centered grid, e.g. |q|-dependent V), it is stored as a real
array so the exchange pass reads half the bytes; the imaginary round-off it
drops is below 1e-14 of max|VR|.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _lib


def _to_numpy(x):
    if isinstance(x, torch.Tensor):
        return x.detach().cpu().numpy()
    return np.asarray(x)


def _mark_zero(t: torch.Tensor) -> torch.Tensor:
    """Tags a tensor that is all zeros so the Fock build can skip reading it."""
    t._hf_is_zero = True
    return t


def is_marked_zero(t) -> bool:
    return t is None or bool(getattr(t, "_hf_is_zero", False))


def shift_phase(n0: int, n1: int) -> np.ndarray:
    s0, s1 = n0 // 2, n1 // 2
    ph0 = np.exp(2j * np.pi * np.arange(n0) * s0 / n0)
    ph1 = np.exp(2j * np.pi * np.arange(n1) * s1 / n1)
    return (ph0[:, None] * ph1[None, :])[..., None, None]


def _selfenergy_host(VRs: np.ndarray, P: np.ndarray, packing: bool) -> np.ndarray:
    """Host float64 exchange used once at construction for the embedded mode."""
    if packing:
        n = P.shape[-1]
        ti, tj = np.triu_indices(n)
        off = ti != tj
        Pf = P.reshape(P.shape[:-2] + (n * n,))
        sig = -np.fft.ifftn(np.fft.fftn(Pf[..., ti * n + tj], axes=(0, 1)) * VRs[..., 0, 0][..., None], axes=(0, 1))
        out = np.zeros_like(Pf)
        out[..., ti * n + tj] = sig
        out[..., tj[off] * n + ti[off]] = np.conj(sig[..., off])
        return out.reshape(P.shape)
    return -np.fft.ifftn(np.fft.fftn(P, axes=(0, 1)) * VRs, axes=(0, 1))


class HartreeFockKernel:
    """Precomputed arrays for the device solver loop (problem.py:14-217)."""

    def __init__(self, weights, hamiltonian, coulomb_q, T: float, include_hartree: bool = False,
                 include_exchange: bool = True, reference_density=None, hartree_matrix=None,
                 contact_terms=None, embed_reference_potential: bool = False,
                 center_embedded_hartree: bool = True, device=None):
        if not torch.cuda.is_available():
            raise RuntimeError("jax_hf_b200 needs a CUDA device (no CPU fallback)")
        _lib.lib()
        dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        h_np = _to_numpy(hamiltonian)
        if not np.iscomplexobj(h_np):
            h_np = h_np.astype(np.complex128)
        cdt = h_np.dtype
        rdt = np.zeros((), cdt).real.dtype
        self.dtype = torch.complex128 if cdt == np.complex128 else torch.complex64
        self.real_dtype = torch.float64 if rdt == np.float64 else torch.float32
        nk1, nk2, nb = h_np.shape[0], h_np.shape[1], h_np.shape[-1]
        self.shape = (nk1, nk2, nb)

        w_np = _to_numpy(weights).astype(rdt)
        Vq = _to_numpy(coulomb_q)
        if np.iscomplexobj(Vq):                                   # problem.py:79-84
            if float(np.max(np.abs(np.imag(Vq)))) <= 1e-8:
                Vq = np.real(Vq)
        else:
            Vq = Vq.astype(rdt)
        self.exchange_hermitian_channel_packing = bool(Vq.shape[-2:] == (1, 1) and not np.iscomplexobj(Vq))
        # VR = FFT2(w V), ifftshift phase absorbed (problem.py:88-98), float64 on host
        wb64 = w_np.astype(np.float64)[..., None, None]
        VR64 = np.fft.fftn(wb64 * np.asarray(Vq).astype(np.complex128), axes=(0, 1))
        VRs64 = VR64 * shift_phase(nk1, nk2)
        scale = float(np.max(np.abs(VRs64))) if VRs64.size else 0.0
        self.vr_real = bool(float(np.max(np.abs(VRs64.imag))) <= 1e-14 * max(scale, 1e-300))
        self.vr_scalar = VRs64.shape[-2:] == (1, 1)
        if self.vr_real:
            VRdev = torch.as_tensor(np.ascontiguousarray(VRs64.real.astype(rdt)), device=dev)
        else:
            VRdev = torch.as_tensor(np.ascontiguousarray(VRs64.astype(cdt)), device=dev)
        self._VR_shifted = VRdev
        # V(q) real and V_ab = V_ba: Hermitian channel packing is exact for Hermitian densities
        # with a band-resolved V too (used by the solvers and build_fock(hermitian_density=True))
        Vr = np.asarray(Vq)
        self.v_pair_symmetric = bool(not np.iscomplexobj(Vr) and (
            Vr.shape[-2:] == (1, 1) or np.array_equal(Vr, np.swapaxes(Vr, -1, -2))))
        if self.v_pair_symmetric:
            VRdev._hf_v_pair_symmetric = True
        self.VR = torch.as_tensor(VR64.astype(cdt), device=dev)

        self.T = float(T)
        self.include_hartree = bool(include_hartree)
        self.include_exchange = bool(include_exchange)
        if (not self.include_hartree) and (not self.include_exchange):
            raise ValueError("HartreeFockKernel must include at least one of Hartree or exchange.")

        if reference_density is not None:
            ref = _to_numpy(reference_density).astype(cdt)
            if ref.shape != h_np.shape:
                raise ValueError(f"reference_density must have shape {h_np.shape}, got {ref.shape}")
            ref_np = ref
            self.refP = torch.as_tensor(ref, device=dev)
            if not np.any(ref):
                _mark_zero(self.refP)
        else:
            ref_np = np.zeros_like(h_np)
            self.refP = _mark_zero(torch.zeros(h_np.shape, dtype=self.dtype, device=dev))

        if self.include_hartree:
            if hartree_matrix is None:
                raise ValueError("include_hartree=True requires hartree_matrix to be provided")
            if reference_density is None:
                raise ValueError("include_hartree=True requires reference_density to be provided")
            HH = _to_numpy(hartree_matrix).astype(rdt)
            if HH.shape != h_np.shape[-2:]:
                raise ValueError(f"hartree_matrix must have shape {h_np.shape[-2:]}, got {HH.shape}")
        else:
            HH = np.zeros(h_np.shape[-2:], dtype=rdt)
        HH_np = HH
        self.HH = torch.as_tensor(np.ascontiguousarray(HH), device=dev)

        n_orb = nb                                                # problem.py:125-158
        if contact_terms is None or len(contact_terms) == 0:
            g_np = np.zeros((1,), rdt)
            Oi_np = np.zeros((1, n_orb, n_orb), cdt)
            Oj_np = np.zeros((1, n_orb, n_orb), cdt)
            self.has_contact = False
        else:
            gs, Ois, Ojs = [], [], []
            for k, term in enumerate(contact_terms):
                if len(term) != 3:
                    raise ValueError(f"contact_terms[{k}] must be (g, O_i, O_j); got len={len(term)}")
                g_t, Oi_t, Oj_t = term
                Oi_arr = _to_numpy(Oi_t).astype(cdt)
                Oj_arr = _to_numpy(Oj_t).astype(cdt)
                if Oi_arr.shape != (n_orb, n_orb):
                    raise ValueError(f"contact_terms[{k}].O_i must have shape {(n_orb, n_orb)}, got {Oi_arr.shape}")
                if Oj_arr.shape != (n_orb, n_orb):
                    raise ValueError(f"contact_terms[{k}].O_j must have shape {(n_orb, n_orb)}, got {Oj_arr.shape}")
                gs.append(np.asarray(g_t).astype(rdt))
                Ois.append(Oi_arr)
                Ojs.append(Oj_arr)
            g_np, Oi_np, Oj_np = np.stack(gs), np.stack(Ois), np.stack(Ojs)
            self.has_contact = True
        self.contact_g = torch.as_tensor(g_np, device=dev)
        self.contact_Oi = torch.as_tensor(Oi_np, device=dev)
        self.contact_Oj = torch.as_tensor(Oj_np, device=dev)
        if not self.has_contact:
            for t in (self.contact_g, self.contact_Oi, self.contact_Oj):
                _mark_zero(t)

        # Embedded reference potential (problem.py:160-199), host float64 once.
        self.embed_reference_potential = bool(embed_reference_potential)
        self.center_embedded_hartree = bool(center_embedded_hartree)
        self.embedded_energy_offset = 0.0
        h_eff = h_np
        if self.embed_reference_potential:
            if reference_density is None:
                raise ValueError("embed_reference_potential=True requires reference_density.")
            ref = ref_np.astype(np.complex128)
            const_J = 0.0
            J_ref_diag = np.zeros(n_orb)
            if self.include_hartree:
                diag_R = np.einsum("ij,ijaa->a", w_np.astype(np.float64), ref).real
                J_ref_diag = HH_np.astype(np.float64) @ diag_R
                if self.center_embedded_hartree:
                    J_ref_diag = J_ref_diag - np.mean(J_ref_diag)
                const_J = float(np.sum(J_ref_diag * diag_R))
            const_S = 0.0
            Sigma_ref = None
            if self.include_exchange:
                Sigma_ref = _selfenergy_host(VRs64, ref, self.exchange_hermitian_channel_packing)
                const_S = float(np.einsum("ij,ijab,ijba->", w_np.astype(np.float64), Sigma_ref, ref).real)
            h64 = h_np.astype(np.complex128)
            if Sigma_ref is not None:
                h64 = h64 + Sigma_ref
            h64 = h64 + np.diag(J_ref_diag.astype(np.complex128))[None, None]
            h_eff = h64.astype(cdt)
            self.embedded_energy_offset = 0.5 * (const_J + const_S)
        self.h = torch.as_tensor(np.ascontiguousarray(h_eff), device=dev)
        self.w2d = torch.as_tensor(np.ascontiguousarray(w_np), device=dev)
        self.weights_b = self.w2d[..., None, None]
        self.weight_sum = float(np.sum(w_np))

    def as_args(self):
        """Dynamic inputs for the solvers (problem.py:201-217)."""
        return dict(h=self.h, weights_b=self.weights_b, weight_sum=self.weight_sum, VR=self._VR_shifted,
                    T=self.T, refP=self.refP, HH=self.HH, include_hartree=self.include_hartree,
                    include_exchange=self.include_exchange,
                    exchange_hermitian_channel_packing=self.exchange_hermitian_channel_packing,
                    contact_g=self.contact_g, contact_Oi=self.contact_Oi, contact_Oj=self.contact_Oj)
