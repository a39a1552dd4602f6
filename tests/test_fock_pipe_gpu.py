"""GPU parity of the bulk-copy pipelined Fock passes (rows plan, nb in {4, 8}).

Every case runs the pipeline (engine="pipe") and the default register passes
and checks both against the CPU oracle:
Sigma and F within 1e-12 of max|oracle| in complex128, 2e-5 for complex64 and
the FP32 exchange.  Sigma of the two schedules must agree to rounding (same
FFT arithmetic); F may differ in the last bits (h + Sigma is summed before the
hermitisation in the pipeline).  The device fault word of the pipelined
passes must stay zero.
"""

import ctypes

import numpy as np
import pytest
import torch

from oracle import hf_oracle as O
from jax_hf_b200 import synthetic as S

pytestmark = pytest.mark.gpu

TOL64, TOL32 = 1e-12, 2e-5


def rel(a, b):
    a = a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
    b = b.detach().cpu().numpy() if isinstance(b, torch.Tensor) else np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def fault_word():
    from jax_hf_b200 import _lib
    code = ctypes.c_int(-1)
    _lib.check(_lib.lib().hf_fock_fault_status(ctypes.byref(code), 1))
    return code.value


CASES = [
    # nk1, nk2, nb, V ("layer" / "scalar" / "complex"), hartree + refP, contact, precision
    (192, 192, 8, "layer", False, False, "c128"),
    (144, 144, 8, "layer", False, False, "c128"),
    (96, 144, 4, "layer", False, False, "c128"),
    (64, 48, 8, "layer", True, True, "c128"),
    (128, 32, 4, "layer", True, False, "c128"),
    (48, 48, 4, "scalar", False, False, "c128"),
    (32, 64, 8, "complex", False, True, "c128"),
    (16, 16, 8, "layer", False, False, "c128"),
    (192, 192, 8, "layer", False, False, "c64"),
    (96, 48, 4, "layer", True, False, "c64"),
    (144, 72, 8, "layer", False, False, "c64"),
    (192, 192, 8, "layer", False, False, "fp32"),
    (144, 144, 4, "complex", False, False, "fp32"),
]


def _problem(nk1, nk2, nb, V, seed):
    rng = np.random.default_rng(seed)
    nkm = max(nk1, nk2)
    prob = S.fourier_problem(nkm, nb, 2.0, seed, V="scalar" if V == "scalar" else "layer")
    h = np.ascontiguousarray(prob.hamiltonian[:nk1, :nk2])
    Vq = np.ascontiguousarray(prob.coulomb_q[:nk1, :nk2])
    if V == "complex":
        Vq = Vq * (1.0 + 0.25j)
    w = rng.uniform(0.5, 1.5, size=(nk1, nk2))
    w = w / w.sum()
    P = np.ascontiguousarray(S.haar_density(nkm, nb, seed + 7)[:nk1, :nk2])
    return w, h, Vq, P, rng


@pytest.mark.parametrize("nk1,nk2,nb,V,hartree,contact,prec", CASES)
def test_pipe_matches_oracle_and_register_passes(cuda, nk1, nk2, nb, V, hartree, contact, prec):
    import jax_hf_b200 as G
    w, h, Vq, P, rng = _problem(nk1, nk2, nb, V, 5 + nk1 + 7 * nk2 + nb)
    kw = {}
    if hartree:
        ref = 0.5 * S.haar_density(max(nk1, nk2), nb, 41)[:nk1, :nk2]
        HH = rng.normal(size=(nb, nb))
        kw.update(include_hartree=True, reference_density=np.ascontiguousarray(ref), hartree_matrix=HH + HH.T)
    if contact:
        Oa = rng.normal(size=(nb, nb)) + 1j * rng.normal(size=(nb, nb))
        kw.update(contact_terms=[(0.3, Oa, Oa.conj().T)])
    cdt = np.complex64 if prec == "c64" else np.complex128
    K = G.HartreeFockKernel(w, h.astype(cdt), Vq, 0.1, **kw)
    Ko = O.Kernel(w, h.astype(cdt), Vq, 0.1, **kw)
    a, ao = K.as_args(), Ko.as_args()
    Pt = torch.as_tensor(P.astype(cdt), device="cuda")
    args = dict(h=a["h"], VR=a["VR"], refP=a["refP"], HH=a["HH"], w2d=K.w2d,
                include_exchange=True, include_hartree=a["include_hartree"],
                exchange_hermitian_channel_packing=False,
                contact_g=a["contact_g"], contact_Oi=a["contact_Oi"], contact_Oj=a["contact_Oj"])
    extra = dict(fft_precision="fp32") if prec == "fp32" else {}
    fault_word()
    Sp, Hp, Fp = G.build_fock(Pt, engine="pipe", **args, **extra)
    Sr, Hr, Fr = G.build_fock(Pt, **args, **extra)
    assert fault_word() == 0
    So, Ho, Fo = O.build_fock(P.astype(cdt).astype(np.complex128), h=ao["h"].astype(np.complex128), VR=ao["VR"],
                              refP=ao["refP"], HH=ao["HH"], w2d=Ko.w2d, include_exchange=True,
                              include_hartree=ao["include_hartree"], exchange_hermitian_channel_packing=False,
                              contact_g=ao["contact_g"], contact_Oi=ao["contact_Oi"], contact_Oj=ao["contact_Oj"])
    tol = TOL64 if prec == "c128" else TOL32
    assert rel(Sp, So) < tol, "Sigma (pipeline)"
    assert rel(Fp, Fo) < tol, "F (pipeline)"
    assert rel(Sr, So) < tol and rel(Fr, Fo) < tol, "register passes"
    assert rel(Sp, Sr) < (1e-15 if prec == "c128" else 1e-6), "Sigma of the two schedules"
    assert torch.equal(Hp, Hr)
    Fn = Fp.cpu().numpy()
    assert np.array_equal(Fn, np.conj(np.swapaxes(Fn, -1, -2))), "F exactly Hermitian"


def test_pipe_repeated_builds_and_stream_order(cuda):
    """Back-to-back builds on one stream into the same outputs (the stages' barrier
    phases restart at every launch); each equals the single build."""
    import jax_hf_b200 as G
    w, h, Vq, P, _ = _problem(96, 96, 8, "layer", 3)
    K = G.HartreeFockKernel(w, h, Vq, 0.1)
    a = K.as_args()
    Ps = [torch.as_tensor(np.roll(P, 5 * r, axis=0), device="cuda") for r in range(3)]
    args = dict(h=a["h"], VR=a["VR"], refP=a["refP"], HH=a["HH"], w2d=K.w2d, include_exchange=True,
                include_hartree=False, exchange_hermitian_channel_packing=False)
    ref = [G.build_fock(Pi, engine="pipe", **args) for Pi in Ps]
    torch.cuda.synchronize()
    S = torch.empty_like(Ps[0])
    F = torch.empty_like(Ps[0])
    H = torch.empty((1, 1, 8, 8), dtype=Ps[0].dtype, device="cuda")
    for it in range(12):
        G.build_fock(Ps[it % 3], out=(S, H, F), engine="pipe", **args)
        if it % 3 == 2:
            torch.cuda.synchronize()
            assert torch.equal(S, ref[2][0]) and torch.equal(F, ref[2][2])
    assert fault_word() == 0
