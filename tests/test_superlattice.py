"""Superlattice Fock (superlattice.py): layout tables against the oracle's loop restatement (CPU),
the CUDA streaming exchange against the oracle's per-DG NumPy FFT (GPU, 1e-12 relative, the
reference's own bar in tests/test_superlattice.py:106-122), and the fock_build_fn adapter."""

import warnings

import numpy as np
import pytest
import torch

from oracle import hf_oracle as O


def _hex_g_basis(g_cut):
    b0 = 4 * np.pi / np.sqrt(3)
    B = np.stack([np.array([np.sqrt(3) / 2, -0.5]) * b0, np.array([0.0, 1.0]) * b0], axis=1)
    fr, cn = [], []
    for n1 in range(-g_cut - 1, g_cut + 2):
        for n2 in range(-g_cut - 1, g_cut + 2):
            fr.append((n1, n2))
            cn.append(np.linalg.norm(B @ np.array([n1, n2])))
    cn, fr = np.array(cn), np.array(fr, dtype=np.int64)
    u = np.sort(np.unique(np.round(cn, 6)))
    return fr[cn <= u[min(g_cut, len(u) - 1)] + 1e-3], B


V = lambda q: 1.0 / np.sqrt(q ** 2 + 0.25)


@pytest.mark.parametrize("g_cut,nk", [(1, 6), (2, 4), (0, 5)])
def test_layout_matches_oracle(g_cut, nk):
    from jax_hf_b200.superlattice import build_extended_layout
    g, B = _hex_g_basis(g_cut)
    L = build_extended_layout(g, B, nk, nk, V, 1.0 / nk ** 2)
    Lo = O.sl_build_extended_layout(g, B, nk, nk, V, 1.0 / nk ** 2)
    for k in ("N_ext_x", "N_ext_y", "n_delta"):
        assert getattr(L, k) == Lo[k]
    for k in ("g_a_off", "pair_to_delta", "delta_pair_i", "delta_pair_j", "delta_pair_start"):
        np.testing.assert_array_equal(getattr(L, k), Lo[k])
    np.testing.assert_allclose(L.V_lag_fft, Lo["V_lag_fft"], rtol=0, atol=1e-14 * np.abs(Lo["V_lag_fft"]).max())
    assert L.delta_pair_count.sum() == len(g) ** 2


@pytest.mark.gpu
@pytest.mark.parametrize("g_cut,nk,dorb", [(1, 6, 3), (1, 6, 2), (2, 4, 2), (0, 5, 1), (1, 8, 4)])
def test_streaming_fock_matches_oracle(cuda, g_cut, nk, dorb):
    from jax_hf_b200.superlattice import build_extended_layout, make_superlattice_fock_fn
    g, B = _hex_g_basis(g_cut)
    nG = len(g)
    L = build_extended_layout(g, B, nk, nk, V, 1.0 / nk ** 2)
    D = nG * dorb
    rng = np.random.default_rng(nk + dorb)
    rho = (rng.standard_normal((nk, nk, D, D)) + 1j * rng.standard_normal((nk, nk, D, D))) * 1e-3
    sig = make_superlattice_fock_fn(L, nG, dorb, nk, nk)(torch.as_tensor(rho, device="cuda")).cpu().numpy()
    ref = O.sl_streaming_fock(rho, O.sl_build_extended_layout(g, B, nk, nk, V, 1.0 / nk ** 2), nG, dorb, nk, nk)
    assert np.abs(sig - ref).max() / np.abs(ref).max() < 1e-12
    z = make_superlattice_fock_fn(L, nG, dorb, nk, nk)(torch.zeros((nk, nk, D, D), dtype=torch.complex128))
    assert float(z.abs().max()) < 1e-12


@pytest.mark.gpu
def test_build_fock_adapter_hartree_paths(cuda):
    """Orbital Hartree with HH_orb[A, B, a, c] = HH[A, B] reproduces the scalar path
    (reference test_superlattice.py:125-...), and F = herm(h + Sigma)."""
    from jax_hf_b200.superlattice import build_extended_layout, make_superlattice_build_fock_fn
    g, B = _hex_g_basis(1)
    nG, nk, do = len(g), 6, 2
    D = nG * do
    L = build_extended_layout(g, B, nk, nk, V, 1.0 / nk ** 2)
    rng = np.random.default_rng(3)
    HH = rng.standard_normal((nG, nG))
    HH = 0.5 * (HH + HH.T)
    np.fill_diagonal(HH, 0.0)
    HHo = np.broadcast_to(HH[:, :, None, None], (nG, nG, do, do)).copy()
    P = (rng.standard_normal((nk, nk, D, D)) + 1j * rng.standard_normal((nk, nk, D, D))) * 1e-2
    P = 0.5 * (P + np.conj(np.swapaxes(P, -1, -2)))
    h = np.zeros((nk, nk, D, D), complex)
    kw = dict(h=torch.as_tensor(h, device="cuda"), VR=None, refP=None, HH=None, w2d=np.full((nk, nk), 1.0 / nk ** 2),
              include_exchange=True, include_hartree=True, exchange_hermitian_channel_packing=False,
              contact_g=None, contact_Oi=None, contact_Oj=None)
    fs = make_superlattice_build_fock_fn(L, nG, do, nk, nk, HH, 2.0)
    fo = make_superlattice_build_fock_fn(L, nG, do, nk, nk, HH, 2.0, HH_GG_orbital=HHo)
    S1, H1, F1 = fs(torch.as_tensor(P, device="cuda"), **kw)
    S2, _, F2 = fo(torch.as_tensor(P, device="cuda"), **kw)
    assert float((S1 - S2).abs().max()) < 1e-12 and float(H1.abs().max()) == 0.0
    Fh = 0.5 * (S1 + S1.transpose(-1, -2).conj())
    assert float((F1 - Fh).abs().max()) < 1e-14
    bad = HHo.copy()
    bad[0, 0] = 1.0
    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter("always")
        make_superlattice_build_fock_fn(L, nG, do, nk, nk, HH, 2.0, HH_GG_orbital=bad)
    assert any("diagonal-G" in str(x.message) for x in w)
    with pytest.raises(ValueError, match="HH_GG_orbital must have shape"):
        make_superlattice_build_fock_fn(L, nG, do, nk, nk, HH, 2.0, HH_GG_orbital=HHo[:, :, :1])
