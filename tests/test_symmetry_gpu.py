"""Symmetry projectors (symmetry.py:153-281): CUDA kernels against the NumPy restatement and the
reference's own property tests (tests/test_symmetry.py: invariance, idempotence, Hermiticity,
masked index maps).  Tolerances: complex128 1e-13 relative to max|A|, complex64 2e-6."""

import numpy as np
import pytest
import torch

from oracle import hf_oracle as O

pytestmark = pytest.mark.gpu


def _rand(shape, seed, dt=np.complex128):
    r = np.random.default_rng(seed)
    return (r.standard_normal(shape) + 1j * r.standard_normal(shape)).astype(dt)


def _gpu(kw):
    from jax_hf_b200.symmetry import make_project_fn
    return make_project_fn(**kw)


def _close(a, b, dt=np.complex128):
    a = a.cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
    tol = 1e-13 if dt == np.complex128 else 2e-6
    assert np.abs(a - b).max() <= tol * max(1.0, np.abs(b).max()), np.abs(a - b).max()


def _c4_maps(n):
    """C4 rotation maps on an n x n centered periodic grid: k -> R^g k (g = 0..3)."""
    i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    x, y = i - n // 2, j - n // 2
    mi, mj = [], []
    for g in range(4):
        for _ in range(g):
            x, y = -y, x
        mi.append((x + n // 2) % n)
        mj.append((y + n // 2) % n)
        x, y = i - n // 2, j - n // 2
    return np.stack(mi).astype(np.int32), np.stack(mj).astype(np.int32)


def _c4_unitaries(nb):
    # a cyclic permutation of the first 4 orbitals, identity on the rest
    P = np.eye(nb, dtype=complex)
    if nb >= 4:
        P[:4, :4] = np.roll(np.eye(4), 1, axis=0)
    return np.stack([np.linalg.matrix_power(P, g) for g in range(4)])


ZN = np.diag([1, 1, -1, -1]).astype(complex)
PERM3 = np.roll(np.eye(3), 1, axis=0).astype(complex)
TRU = np.array([[0, -1j], [1j, 0]])
CONFIGS = [
    ("unitary", (3, 3, 4), dict(unitary_group=np.stack([np.eye(4), ZN]))),
    ("perm3", (2, 2, 3), dict(unitary_group=np.stack([np.eye(3), PERM3, PERM3 @ PERM3]))),
    ("tr_flip", (4, 4, 2), dict(time_reversal_U=TRU, time_reversal_k_convention="flip")),
    ("tr_mod", (5, 4, 2), dict(time_reversal_U=TRU, time_reversal_k_convention="mod")),
    ("unitary_tr", (4, 4, 2), dict(unitary_group=np.stack([np.eye(2), np.diag([1, -1]).astype(complex)]),
                                   time_reversal_U=TRU)),
    ("spatial_flip", (4, 6, 2), dict(spatial_group=np.stack([np.eye(2)[::-1].astype(complex)]),
                                     spatial_k_convention="flip")),
    ("same_and_flip", (6, 6, 4), dict(unitary_group=np.stack([np.eye(4), ZN]),
                                      spatial_group=np.stack([np.eye(4)[::-1].astype(complex)]),
                                      spatial_k_convention="mod")),
    ("kx_flip", (6, 5, 3), dict(spatial_group=np.stack([np.eye(3, dtype=complex)]), spatial_k_convention="mod",
                                spatial_k_flip_axes=(0,))),
    ("large_nb", (3, 2, 20), dict(unitary_group=np.stack([np.eye(20), np.diag(np.exp(1j * np.arange(20)))]),
                                  time_reversal_U=np.eye(20)[::-1].astype(complex))),
]


@pytest.mark.parametrize("name,shape,kw", CONFIGS, ids=[c[0] for c in CONFIGS])
@pytest.mark.parametrize("dt", [np.complex128, np.complex64])
def test_projector_matches_oracle(cuda, name, shape, kw, dt):
    nk1, nk2, nb = shape
    A = _rand((nk1, nk2, nb, nb), nk1 * 7 + nb, dt)
    out = _gpu(kw)(torch.as_tensor(A, device="cuda"))
    assert out.dtype == torch.as_tensor(A).dtype
    _close(out, O.make_project_fn(**kw)(A.astype(np.complex128)), dt)


def test_identity_when_no_args(cuda):
    A = torch.ones((2, 2, 3, 3), dtype=torch.complex64, device="cuda")
    assert _gpu({})(A) is A


def test_unitary_average_invariant_idempotent_hermitian(cuda):
    G = np.stack([np.eye(3), PERM3, PERM3 @ PERM3])
    proj = _gpu(dict(unitary_group=G))
    A = _rand((3, 3, 3, 3), 5)
    A = 0.5 * (A + np.conj(np.swapaxes(A, -1, -2)))
    once = proj(torch.as_tensor(A, device="cuda"))
    twice = proj(once)
    _close(twice, once.cpu().numpy())
    B = once.cpu().numpy()
    for g in G:
        _close(g @ B @ np.conj(g.T), B)
    _close(once, np.conj(np.swapaxes(B, -1, -2)))


def test_spatial_index_maps_with_orbit_mask_and_unitary(cuda):
    n, nb = 6, 4
    mi, mj = _c4_maps(n)
    S = _c4_unitaries(nb)
    mask = np.ones((n, n), bool)
    mask[0, :] = False
    kw = dict(spatial_group=S, spatial_k_index_maps=(mi, mj), spatial_k_orbit_mask=mask,
              unitary_group=np.stack([np.eye(nb), ZN]))
    A = _rand((n, n, nb, nb), 11)
    once = _gpu(kw)(torch.as_tensor(A, device="cuda"))
    _close(once, O.make_project_fn(**kw)(A))
    kw2 = dict(spatial_group=S, spatial_k_index_maps=(mi, mj))
    p2 = _gpu(kw2)
    o1 = p2(torch.as_tensor(A, device="cuda"))
    _close(p2(o1), o1.cpu().numpy())  # idempotent without a mask


def test_time_reversal_index_map_with_invalid_mask(cuda):
    n, nb = 4, 2
    i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    ti, tj = ((-i) % n).astype(np.int32), ((-j) % n).astype(np.int32)
    valid = np.ones((n, n), bool)
    valid[0, 0] = False
    kw = dict(time_reversal_U=TRU, time_reversal_k_index_map=(ti, tj, valid))
    A = _rand((n, n, nb, nb), 3)
    out = _gpu(kw)(torch.as_tensor(A, device="cuda")).cpu().numpy()
    np.testing.assert_allclose(out[0, 0], A[0, 0], atol=1e-15)
    _close(out, O.make_project_fn(**kw)(A))


def test_argument_errors(cuda):
    S = np.stack([np.eye(2, dtype=complex)] * 2)
    mi = np.zeros((2, 3, 3), np.int32)
    with pytest.raises(ValueError, match="requires spatial_group"):
        _gpu(dict(spatial_k_index_maps=(mi, mi)))
    with pytest.raises(ValueError, match="matching"):
        _gpu(dict(spatial_group=S[:1], spatial_k_index_maps=(mi, mi)))
    with pytest.raises(ValueError, match="same shape"):
        _gpu(dict(spatial_group=S, spatial_k_index_maps=(mi, mi[:, :2])))
    with pytest.raises(ValueError, match="requires time_reversal_U"):
        _gpu(dict(unitary_group=S, time_reversal_k_index_map=(mi[0], mi[0], np.ones((3, 3), bool))))
    with pytest.raises(ValueError, match="'mod' or 'flip'"):
        _gpu(dict(time_reversal_U=TRU, time_reversal_k_convention="wrap"))
    bad = np.full((2, 3, 3), 7, np.int32)
    with pytest.raises(ValueError, match="indices"):
        _gpu(dict(spatial_group=S, spatial_k_index_maps=(bad, bad)))(torch.zeros((3, 3, 2, 2), dtype=torch.complex128))


def test_projector_in_cg_solve_matches_oracle(cuda):
    """The projector as SolverConfig.project_fn of the CG solver, against the oracle's CG with its own."""
    import jax_hf_b200 as G
    from jax_hf_b200.solver import SolverConfig, solve
    from jax_hf_b200 import synthetic as Sy
    prob = Sy.fourier_problem(8, 4, 2.0, seed=5, V="scalar", T=0.1, n_electrons=2.0)
    Gz = np.stack([np.eye(4), ZN])
    kw = dict(unitary_group=Gz, time_reversal_U=np.eye(4, dtype=complex))
    cfg = dict(max_iter=150, tol_E=1e-10)
    P0 = np.zeros((8, 8, 4, 4), complex)
    r = solve(G.HartreeFockKernel(**prob.kernel_kwargs()), torch.as_tensor(P0, device="cuda"), 2.0,
              config=SolverConfig(project_fn=_gpu(kw), **cfg))
    ro = O.solve(O.Kernel(**prob.kernel_kwargs()), P0, 2.0,
                 config=O.SolverConfig(project_fn=O.make_project_fn(**kw), **cfg))
    assert abs(float(r.energy) - ro["energy"]) <= 1e-9 * max(1.0, abs(ro["energy"]))
    D = r.density.cpu().numpy()
    for g in Gz:
        np.testing.assert_allclose(g @ D @ np.conj(g.T), D, atol=1e-10)
