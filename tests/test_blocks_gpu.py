"""Block-diagonal exchange specs on the GPU against the oracle (utils.py:206-309).

hf_fock_build_blocks transforms only the in-block channels and writes the
off-block channels in a separate pass; hf_block_offdiag_max checks every spec in
one pass over P - refP.  The oracle is the NumPy restatement of the reference's
block path (per-block FFTs, lax.cond chain over the specs).  Tolerances: 1e-12
relative for complex128, 2e-5 for complex64 and the FP32 exchange FFT.
"""

import numpy as np
import pytest
import torch

from oracle import hf_oracle as O
from jax_hf_b200 import synthetic as S

pytestmark = pytest.mark.gpu


def _problem(nk, nb, seed, V="layer", hartree=True, contact=True, refp=True):
    rng = np.random.default_rng(seed)
    prob = S.fourier_problem(nk, nb, 2.0, seed, V=V)
    P = S.haar_density(nk, nb, seed + 1)
    kw = dict(weights=prob.weights, hamiltonian=prob.hamiltonian, coulomb_q=prob.coulomb_q, T=0.1,
              include_hartree=hartree)
    if refp:
        kw["reference_density"] = 0.3 * S.haar_density(nk, nb, seed + 2)
    if hartree:
        HH = rng.normal(size=(nb, nb))
        kw["hartree_matrix"] = HH + HH.T
    if contact:
        Oa = rng.normal(size=(nb, nb)) + 1j * rng.normal(size=(nb, nb))
        kw["contact_terms"] = [(0.25, Oa, Oa.conj().T)]
    return kw, P


def _builds(kw, P, dtype=torch.complex128, **bkw):
    import jax_hf_b200 as G
    K = G.HartreeFockKernel(**kw) if dtype == torch.complex128 else G.HartreeFockKernel(
        **dict(kw, hamiltonian=np.asarray(kw["hamiltonian"]).astype(np.complex64)))
    Ko = O.Kernel(**kw)
    a, ao = K.as_args(), Ko.as_args()
    fk = dict(h=a["h"], VR=a["VR"], refP=a["refP"], HH=a["HH"], w2d=K.w2d, include_exchange=True,
              include_hartree=kw.get("include_hartree", True),
              exchange_hermitian_channel_packing=a["exchange_hermitian_channel_packing"],
              contact_g=a["contact_g"], contact_Oi=a["contact_Oi"], contact_Oj=a["contact_Oj"])
    fo = dict(h=ao["h"], VR=ao["VR"], refP=ao["refP"], HH=ao["HH"], w2d=Ko.w2d, include_exchange=True,
              include_hartree=kw.get("include_hartree", True),
              exchange_hermitian_channel_packing=ao["exchange_hermitian_channel_packing"],
              contact_g=ao["contact_g"], contact_Oi=ao["contact_Oi"], contact_Oj=ao["contact_Oj"])
    fft = bkw.pop("fft_precision", None)
    Pt = torch.as_tensor(P, device="cuda").to(dtype)
    out = G.build_fock(Pt, fft_precision=fft, **fk, **bkw)
    ref = O.build_fock(P, **fo, **bkw)
    return [o.cpu().numpy() for o in out], ref


def _rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-300))


CASES = [
    # (name, nk, nb, V, spec, forced)
    ("sizes_4_4_fast24", 24, 8, "layer", [{"block_sizes": [4, 4]}], True),
    ("sizes_4_4_fast48", 48, 8, "layer", [{"block_sizes": [4, 4]}], True),
    ("sizes_2_3_1_generic20", 20, 6, "layer", [{"block_sizes": [2, 3, 1]}], True),
    ("indices_band_left_out", 24, 6, "layer", [{"block_indices": [[0, 1, 2], [4, 5]]}], True),
    ("indices_scattered", 16, 5, "scalar", [{"block_indices": [[0, 3], [1, 4]]}], True),
    ("sizes_scalar_packing", 24, 8, "scalar", [{"block_sizes": [4, 4]}], True),
]


@pytest.mark.parametrize("name,nk,nb,V,spec,forced", CASES, ids=[c[0] for c in CASES])
def test_block_build_matches_oracle(cuda, name, nk, nb, V, spec, forced):
    kw, P = _problem(nk, nb, 11 + nk + nb, V=V)
    (Sg, H, F), (So, Ho, Fo) = _builds(kw, P, exchange_block_specs=spec, exchange_check_offdiag=not forced)
    assert _rel(Sg, So) <= 1e-12
    assert _rel(F, Fo) <= 1e-12
    assert _rel(H.reshape(-1, nb, nb)[0], np.asarray(Ho).reshape(-1, nb, nb)[0]) <= 1e-12


@pytest.mark.parametrize("dtype,fft,tol", [(torch.complex64, None, 2e-5), (torch.complex128, "fp32", 2e-5)],
                         ids=["c64", "fp32fft"])
def test_block_build_reduced_precision(cuda, dtype, fft, tol):
    kw, P = _problem(24, 8, 5)
    spec = [{"block_sizes": [4, 4]}]
    (Sg, _, F), (So, _, Fo) = _builds(kw, P, dtype=dtype, exchange_block_specs=spec, exchange_check_offdiag=False,
                                      fft_precision=fft)
    assert _rel(Sg, So) <= tol and _rel(F, Fo) <= tol


def test_block_spec_choice_matches_oracle(cuda):
    """The first compatible spec wins; a coupled density falls back to the full build; the
    check is on |P - refP|; NaN in P selects the full build (as jnp.max propagates NaN)."""
    nk, nb = 16, 6
    kw, P = _problem(nk, nb, 3, refp=True)
    refP = np.asarray(kw["reference_density"])
    specs = [{"block_sizes": [3, 3]}, {"block_indices": [[0, 1, 2, 3], [4, 5]]}, {"block_sizes": [2, 2, 2]}]
    mask33 = np.zeros((nb, nb), bool)
    mask33[:3, :3] = mask33[3:, 3:] = True
    mask42 = np.zeros((nb, nb), bool)
    mask42[:4, :4] = mask42[4:, 4:] = True
    # P - refP is block-diagonal under the second spec only
    Pb = refP + np.where(mask42, P - refP, 0.0)
    for Pc, atol in ((Pb, 1e-9), (P, 1e-9), (P, 10.0)):
        (Sg, _, F), (So, _, Fo) = _builds(kw, Pc, exchange_block_specs=specs, exchange_check_offdiag=True,
                                          exchange_offdiag_atol=atol)
        assert _rel(Sg, So) <= 1e-12 and _rel(F, Fo) <= 1e-12
    # which spec was taken: the exchange vanishes exactly on its off-block channels
    (Sg, _, _), _ = _builds(dict(kw, contact_terms=None), Pb, exchange_block_specs=specs,
                            exchange_check_offdiag=True, exchange_offdiag_atol=1e-9)
    assert np.all(Sg[..., ~mask42] == 0) and not np.all(Sg[..., ~mask33] == 0)


def test_offdiag_max_kernel(cuda):
    from jax_hf_b200 import _lib
    from jax_hf_b200.blocks import normalize_block_specs, spec_masks
    g = torch.Generator(device="cpu").manual_seed(9)
    nk, nb = 300, 7
    P = torch.randn(nk, nb, nb, dtype=torch.complex128, generator=g).cuda()
    R = torch.randn(nk, nb, nb, dtype=torch.complex128, generator=g).cuda()
    specs = normalize_block_specs([{"block_sizes": [3, 4]}, {"block_indices": [[0, 6], [2, 3, 5]]}])
    masks = spec_masks(specs, nb)
    out = torch.empty(3, dtype=torch.float64, device="cuda")
    _lib.check(_lib.lib().hf_block_offdiag_max(_lib.stream_ptr(P.device), _lib.HF_C128, nk, nb, P.data_ptr(),
                                               R.data_ptr(), 2, masks.ctypes.data_as(_lib.C.c_void_p),
                                               out.data_ptr()))
    A = (P - R).abs().cpu().numpy()
    want = [A.max()] + [A[:, ~masks[i].astype(bool)].max() for i in range(2)]
    np.testing.assert_array_equal(out.cpu().numpy(), np.asarray(want))
    P[5, 0, 6] = float("nan")
    _lib.check(_lib.lib().hf_block_offdiag_max(_lib.stream_ptr(P.device), _lib.HF_C128, nk, nb, P.data_ptr(),
                                               None, 2, masks.ctypes.data_as(_lib.C.c_void_p), out.data_ptr()))
    v = out.cpu().numpy()
    assert np.isnan(v[0]) and np.isnan(v[1]) and not np.isnan(v[2])   # (0, 6) is off-block in spec 0 only


def test_block_mask_must_be_symmetric(cuda):
    from jax_hf_b200 import _lib
    nb = 4
    m = np.ones((nb, nb), np.uint8)
    m[0, 1] = 0
    need = _lib.C.c_size_t(0)
    st = _lib.lib().hf_fock_blocks_workspace_size(_lib.HF_C128, _lib.FOCK_EXCHANGE | _lib.FOCK_VR_REAL, 8, 8, nb,
                                                  m.ctypes.data_as(_lib.C.c_void_p), _lib.C.byref(need))
    assert st == _lib.HF_ERR_INVALID


def test_device_spec_choice_index(cuda):
    """hf_fock_build_block_specs reports the spec its device check picked: the first compatible
    one, -1 (full build) when none is, and -1 when P holds a NaN."""
    import jax_hf_b200 as G
    from jax_hf_b200 import _lib
    from jax_hf_b200.blocks import normalize_block_specs, spec_masks
    nk, nb = 16, 6
    kw, P = _problem(nk, nb, 4, hartree=False, contact=False, refp=False)
    K = G.HartreeFockKernel(**kw)
    a = K.as_args()
    specs = normalize_block_specs([{"block_sizes": [3, 3]}, {"block_indices": [[0, 1, 2, 3], [4, 5]]}])
    masks = spec_masks(specs, nb)
    m42 = masks[1].astype(bool)
    flags = _lib.FOCK_EXCHANGE | _lib.FOCK_VR_REAL
    need = _lib.C.c_size_t(0)
    mptr = masks.ctypes.data_as(_lib.C.c_void_p)
    _lib.check(_lib.lib().hf_fock_block_specs_workspace_size(_lib.HF_C128, flags, nk, nk, nb, 2, mptr,
                                                             _lib.C.byref(need)))
    ws = torch.empty(need.value, dtype=torch.uint8, device="cuda")
    chosen = torch.full((1,), 99, dtype=torch.int32, device="cuda")
    VR = a["VR"].to(torch.float64).contiguous()
    assert not a["VR"].is_complex()

    def pick(Pn, atol):
        Pt = torch.as_tensor(Pn, device="cuda").contiguous()
        S_, F_ = torch.empty_like(Pt), torch.empty_like(Pt)
        _lib.check(_lib.lib().hf_fock_build_block_specs(
            _lib.stream_ptr(Pt.device), _lib.HF_C128, flags, nk, nk, nb, 2, mptr, atol, 0.0, Pt.data_ptr(),
            K.h.data_ptr(), VR.data_ptr(), None, None, K.w2d.data_ptr(), 0, None, None, None, S_.data_ptr(), None,
            F_.data_ptr(), ws.data_ptr(), ws.numel(), chosen.data_ptr()))
        return int(chosen.item())

    Pb = np.where(m42, P, 0.0)
    assert pick(Pb, 1e-9) == 1
    assert pick(P, 1e-9) == -1
    assert pick(P, 10.0) == 0
    Pn = Pb.copy()
    Pn[3, 2, 1, 1] = np.nan
    assert pick(Pn, 1e9) == -1
