"""Embedded reference potential mode of HartreeFockKernel (problem.py:160-199).

With ``embed_reference_potential=True`` the kernel folds the Hartree-Fock
potential of the reference density into h once (h_eff = h + Sigma[refP] +
J[refP]) and records the constant 0.5 (Tr J refP + Tr Sigma refP) as
``embedded_energy_offset``.  The identities checked here are the ones the
reference pins in tests/test_embedded_reference_potential.py:65-149:

* at P = refP the embedded build returns h_eff (the density deviation is zero);
* F_embed[P] - F_plain[P] = h_eff - h for every P (the embedding is a constant shift);
* a zero reference density leaves h unchanged and the offset zero;
* E_embed[refP] - E_plain[refP] = 2 * embedded_energy_offset.

The GPU kernel's h_eff and offset are also compared with the oracle's.
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NK, NO = 6, 3


def _model(scalar_v: bool, seed: int = 3):
    rng = np.random.default_rng(seed)
    w = np.full((NK, NK), 1.0 / (NK * NK))
    k = 2 * np.pi * (np.arange(NK) - NK // 2) / NK
    h = np.zeros((NK, NK, NO, NO), np.complex128)
    onsite = np.array([-0.6, 0.1, 0.7])
    for a in range(NO):
        h[..., a, a] = onsite[a] - 0.4 * (np.cos(k)[:, None] + np.cos(k)[None, :])
    hop = 0.2 * (rng.standard_normal((NO, NO)) + 1j * rng.standard_normal((NO, NO)))
    hop = 0.5 * (hop + hop.conj().T)
    h += np.sin(k)[:, None, None, None] * hop[None, None]
    q = np.sqrt(k[:, None] ** 2 + k[None, :] ** 2)
    with np.errstate(divide="ignore", invalid="ignore"):
        base = np.where(q > 0, 2 * np.pi * np.tanh(q) / q, 0.0)
    if scalar_v:
        V = (0.25 * base)[..., None, None].astype(np.complex128)
    else:
        d = 1.0 + 0.5 * np.abs(np.arange(NO)[:, None] - np.arange(NO)[None, :])
        with np.errstate(divide="ignore", invalid="ignore"):
            V = np.where(q[..., None, None] > 0, 2 * np.pi * np.tanh(q[..., None, None] * d) / q[..., None, None],
                         0.0)
        V = (0.25 * V).astype(np.complex128)
    HH = np.array([[0.5, -0.1, 0.05], [-0.1, 0.4, -0.1], [0.05, -0.1, 0.6]])
    refP = np.zeros((NK, NK, NO, NO), np.complex128)
    refP[..., np.arange(NO), np.arange(NO)] = [0.3, 0.5, 0.2]
    return w, h, V, HH, refP


def _kernels(scalar_v: bool, hartree: bool, refP=None):
    import jax_hf_b200 as G

    w, h, V, HH, ref = _model(scalar_v)
    if refP is not None:
        ref = refP
    common = dict(weights=w, hamiltonian=h, coulomb_q=V, T=0.05, include_exchange=True,
                  include_hartree=hartree, hartree_matrix=HH if hartree else None, reference_density=ref)
    plain = G.HartreeFockKernel(**common)
    embed = G.HartreeFockKernel(**common, embed_reference_potential=True, center_embedded_hartree=False)
    return plain, embed


def _build(kernel, P):
    import torch
    import jax_hf_b200 as G

    a = kernel.as_args()
    Pd = torch.as_tensor(np.ascontiguousarray(P), device=kernel.h.device)
    S, H, F = G.build_fock(Pd, h=a["h"], VR=a["VR"], refP=a["refP"], HH=a["HH"], w2d=kernel.w2d,
                           include_exchange=a["include_exchange"], include_hartree=a["include_hartree"],
                           exchange_hermitian_channel_packing=a["exchange_hermitian_channel_packing"],
                           contact_g=a["contact_g"], contact_Oi=a["contact_Oi"], contact_Oj=a["contact_Oj"])
    return S, H, F


CASES = [(sv, hh) for sv in (True, False) for hh in (True, False)]


@pytest.mark.parametrize("scalar_v,hartree", CASES)
def test_embedded_build_at_reference_density_returns_h_eff(scalar_v, hartree):
    plain, embed = _kernels(scalar_v, hartree)
    ref = plain.refP.cpu().numpy()
    _, _, Fp = _build(plain, ref)
    _, _, Fe = _build(embed, ref)
    h = plain.h.cpu().numpy()
    h_eff = embed.h.cpu().numpy()
    np.testing.assert_allclose(Fp.cpu().numpy(), h, atol=1e-13)
    np.testing.assert_allclose(Fe.cpu().numpy(), h_eff, atol=1e-13)
    assert np.max(np.abs(h_eff - h)) > 1e-3  # the embedding is not trivial here


@pytest.mark.parametrize("scalar_v,hartree", CASES)
def test_embedding_is_a_density_independent_shift(scalar_v, hartree):
    plain, embed = _kernels(scalar_v, hartree)
    rng = np.random.default_rng(11)
    P = rng.standard_normal((NK, NK, NO, NO)) + 1j * rng.standard_normal((NK, NK, NO, NO))
    P = 0.5 * (P + np.conj(np.swapaxes(P, -1, -2)))
    _, _, Fp = _build(plain, P)
    _, _, Fe = _build(embed, P)
    shift = (embed.h - plain.h).cpu().numpy()
    np.testing.assert_allclose((Fe - Fp).cpu().numpy(), shift, atol=1e-12)


@pytest.mark.parametrize("hartree", [True, False])
def test_zero_reference_density_is_a_no_op(hartree):
    w, h, V, HH, ref = _model(True)
    plain, embed = _kernels(True, hartree, refP=np.zeros_like(ref))
    np.testing.assert_allclose(embed.h.cpu().numpy(), h, atol=1e-15)
    assert embed.embedded_energy_offset == 0.0


@pytest.mark.parametrize("scalar_v", [True, False])
def test_embedded_energy_offset(scalar_v):
    import jax_hf_b200 as G

    plain, embed = _kernels(scalar_v, True)
    ref = plain.refP
    Sp, Hp, _ = _build(plain, ref.cpu().numpy())
    Se, He, _ = _build(embed, ref.cpu().numpy())
    Ep = float(G.hf_energy(ref, h=plain.h, Sigma=Sp, H=Hp, weights_b=plain.weights_b))
    Ee = float(G.hf_energy(ref, h=embed.h, Sigma=Se, H=He, weights_b=embed.weights_b))
    assert abs(embed.embedded_energy_offset) > 1e-3
    np.testing.assert_allclose(Ee - Ep, 2.0 * embed.embedded_energy_offset, rtol=1e-12, atol=1e-13)


@pytest.mark.parametrize("scalar_v,hartree", CASES)
@pytest.mark.parametrize("center", [True, False])
def test_embedded_kernel_matches_oracle(scalar_v, hartree, center):
    import jax_hf_b200 as G
    from oracle import hf_oracle as O

    w, h, V, HH, ref = _model(scalar_v)
    kw = dict(weights=w, hamiltonian=h, coulomb_q=V, T=0.05, include_exchange=True, include_hartree=hartree,
              hartree_matrix=HH if hartree else None, reference_density=ref, embed_reference_potential=True,
              center_embedded_hartree=center)
    K = G.HartreeFockKernel(**kw)
    KO = O.Kernel(**kw)
    np.testing.assert_allclose(K.h.cpu().numpy(), KO.h, atol=1e-13)
    np.testing.assert_allclose(K.embedded_energy_offset, KO.embedded_energy_offset, rtol=1e-12, atol=1e-15)
