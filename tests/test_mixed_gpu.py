"""GPU tests of the mixed-precision solvers against the FP64 oracle's fixed point.

The reference CG stops on an energy plateau that lies 1e-9 .. 4e-6 (relative)
above the self-consistent fixed point (tests/golden/scan64_oracle.json), so the
FP64 oracle energy these tests use is the fixed point itself: the oracle's
SCF-DIIS run to a density residual of 1e-11.  Bars: |dE/E| <= 1e-9 and a
density within 1e-6 of the oracle's (max abs entry).
"""

import ctypes
import json
from pathlib import Path

import numpy as np
import pytest
import torch

from oracle import hf_oracle as O
from jax_hf_b200 import synthetic as S

pytestmark = pytest.mark.gpu

FIXTURE = Path(__file__).with_name("golden") / "scan64_oracle.json"
TOL_E, TOL_P = 1e-9, 1e-6


def _oracle_fixed_point(kw, ne):
    Ko = O.Kernel(**kw)
    P0 = np.zeros_like(np.asarray(kw["hamiltonian"], complex))
    return O.solve_scf(Ko, P0, ne, config=O.SCFConfig(acceleration="diis", density_tol=1e-11, comm_tol=1e-10,
                                                      max_iter=400))


def _fourier(nk, nb, V, T, seed):
    p = S.fourier_problem(nk, nb, 2.0, seed, V=V, T=T)
    return dict(weights=p.weights, hamiltonian=p.hamiltonian, coulomb_q=p.coulomb_q, T=T)


FAST = dict(acceleration="diis", density_tol=1e-8, comm_tol=1e-7, max_iter=300, mu_method="newton",
            warm_eigh=True)
CASES = [
    ("fourier_16_nb4_scalar", _fourier(16, 4, "scalar", 0.1, 3), 2.0),
    ("fourier_24_nb8_layer", _fourier(24, 8, "layer", 0.05, 5), 3.0),
    ("fourier_12_nb6_layer", _fourier(12, 6, "layer", 0.1, 7), 2.4),
]


@pytest.mark.parametrize("name,kw,ne", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("fp32", [False, True], ids=["fp64", "mixed"])
def test_fast_scf_reaches_the_oracle_fixed_point(cuda, name, kw, ne, fp32):
    import jax_hf_b200 as G
    from jax_hf_b200.reference_scf import SCFConfig, solve_scf
    K = G.HartreeFockKernel(**kw)
    P0 = torch.zeros(np.asarray(kw["hamiltonian"]).shape, dtype=torch.complex128, device="cuda")
    r = solve_scf(K, P0, ne, config=SCFConfig(**FAST, fp32_exchange=fp32))
    ro = _oracle_fixed_point(kw, ne)
    assert r.converged
    Eo = ro["energy"]
    assert abs(float(r.energy) - Eo) <= TOL_E * abs(Eo)
    assert float(np.abs(r.density_matrix.cpu().numpy() - ro["density_matrix"]).max()) < TOL_P
    if fp32:
        # an FP32 phase ran, then the FP64 builds that decided convergence
        assert r.history["fp32_switch_iter"] >= 1
    else:
        assert r.history["fp32_switch_iter"] == -1
    # the same solve reporting its error against the oracle's fixed point
    r2 = solve_scf(K, P0, ne, config=SCFConfig(**FAST, fp32_exchange=fp32, reference_energy=Eo,
                                               reference_density=ro["density_matrix"]))
    assert r2.history["rel_dE_vs_reference"] <= TOL_E
    assert r2.history["max_abs_dP_vs_reference"] < TOL_P


@pytest.mark.parametrize("name,kw,ne", CASES[:2], ids=[c[0] for c in CASES[:2]])
def test_cg_polish_reaches_the_fixed_point_and_reports_errors(cuda, name, kw, ne):
    import jax_hf_b200 as G
    from jax_hf_b200.solver import SolverConfig, solve
    K = G.HartreeFockKernel(**kw)
    P0 = torch.zeros(np.asarray(kw["hamiltonian"]).shape, dtype=torch.complex128, device="cuda")
    ro = _oracle_fixed_point(kw, ne)
    cfg = SolverConfig(max_iter=400, tol_E=1e-6, fp32_exchange=True, fp32_switch_rel=1e-6, polish="scf",
                       reference_energy=ro["energy"], reference_density=ro["density_matrix"])
    r = solve(K, P0, ne, config=cfg)
    assert bool(r.converged)
    assert r.history["rel_dE_vs_reference"] <= TOL_E
    assert r.history["max_abs_dP_vs_reference"] < TOL_P
    assert r.history["polish_iterations"] >= 1
    # the orbitals and occupations describe the returned Fock matrix
    Q, p, F = r.Q, r.p, r.fock
    D = torch.diagonal(Q.conj().transpose(-1, -2) @ F @ Q, dim1=-2, dim2=-1).real
    eps = torch.linalg.eigvalsh(F)
    assert float((torch.sort(D, dim=-1).values - eps).abs().max()) < 1e-10
    assert float(p.min()) >= 0.0 and float(p.max()) <= 1.0


def test_scf_batch_equals_single_solves(cuda):
    """solve_scf_batch: every result bit-identical to the same solve run alone."""
    import jax_hf_b200 as G
    from jax_hf_b200.reference_scf import SCFConfig, solve_scf, solve_scf_batch
    probs = [(_fourier(12 + 4 * i, 4 + 2 * (i % 2), "layer" if i % 2 else "scalar", 0.1, 20 + i), 1.5 + 0.3 * i)
             for i in range(5)]
    Ks = [G.HartreeFockKernel(**kw) for kw, _ in probs]
    P0s = [torch.zeros(np.asarray(kw["hamiltonian"]).shape, dtype=torch.complex128, device="cuda") for kw, _ in probs]
    nes = [ne for _, ne in probs]
    cfg = SCFConfig(**FAST, fp32_exchange=True)
    single = [solve_scf(K, P0, ne, config=cfg) for K, P0, ne in zip(Ks, P0s, nes)]
    batch, times = solve_scf_batch(Ks, P0s, nes, config=cfg, workers=3, return_times=True)
    assert len(times) == 5 and all(t > 0 for t in times)
    for a, b in zip(single, batch):
        assert a.iterations == b.iterations
        assert torch.equal(a.density_matrix, b.density_matrix)
        assert float(a.energy) == float(b.energy)


GRAPH_CFGS = [
    ("mixed_fast", dict(FAST, fp32_exchange=True)),
    ("fp64_fast", dict(FAST)),
    ("reference_steps", dict(acceleration="diis", density_tol=1e-8, comm_tol=1e-7, max_iter=300)),
    ("linear", dict(acceleration="linear", mixing=0.5, density_tol=1e-7, comm_tol=1e-6, max_iter=300)),
    ("diis10_damped_shift", dict(acceleration="diis", diis_size=10, diis_damping=0.8, level_shift=0.2,
                                 density_tol=1e-8, comm_tol=1e-7, max_iter=300)),
]


@pytest.mark.parametrize("name,cfg", GRAPH_CFGS, ids=[c[0] for c in GRAPH_CFGS])
def test_scf_graph_batch_matches_single_solves(cuda, name, cfg):
    """ScfScanGraph (the SCF loop on the device, the batch as one CUDA graph): every solve
    takes the host driver's steps (iteration count, switch point, histories) and ends at its
    energy and density."""
    import jax_hf_b200 as G
    from jax_hf_b200.reference_scf import SCFConfig, ScfScanGraph, solve_scf
    probs = [(_fourier(12 + 4 * i, 4 + 2 * (i % 2), "layer" if i % 2 else "scalar", 0.1, 40 + i), 1.5 + 0.3 * i)
             for i in range(4)]
    Ks = [G.HartreeFockKernel(**kw) for kw, _ in probs]
    P0s = [torch.zeros(np.asarray(kw["hamiltonian"]).shape, dtype=torch.complex128, device="cuda") for kw, _ in probs]
    nes = [ne for _, ne in probs]
    c = SCFConfig(**cfg)
    sg = ScfScanGraph(Ks, P0s, nes, config=c)
    res, times = sg.run(return_times=True)
    res2 = sg.run()  # a second launch of the same graph
    sg.close()
    assert all(t > 0 for t in times)
    for K, P0, ne, a, a2 in zip(Ks, P0s, nes, res, res2):
        b = solve_scf(K, P0, ne, config=c)
        assert a.iterations == b.iterations and a.converged == b.converged
        assert a.history["fp32_switch_iter"] == b.history["fp32_switch_iter"]
        np.testing.assert_allclose(a.history["E"], b.history["E"], rtol=1e-12, atol=1e-13)
        np.testing.assert_allclose(a.history["density_residual"], b.history["density_residual"], rtol=1e-9,
                                   atol=1e-15)
        assert abs(float(a.energy) - float(b.energy)) <= 1e-12 * max(1.0, abs(float(b.energy)))
        assert float((a.density_matrix - b.density_matrix).abs().max()) < 1e-10
        assert float(a2.energy) == float(a.energy) and torch.equal(a2.density_matrix, a.density_matrix)


@pytest.mark.parametrize("index", [3, 10, 17])
def test_scan_fixture_problems(cuda, index):
    """Problems of the 64-solve density scan: the mixed SCF matches the committed oracle fixed
    point, and the FP64 CG (the reference algorithm) matches the oracle's own CG result."""
    import jax_hf_b200 as G
    from jax_hf_b200.reference_scf import SCFConfig, solve_scf
    from jax_hf_b200.solver import SolverConfig, solve
    row = json.loads(FIXTURE.read_text())["rows"][index]
    p = S.density_scan(64)[index]
    assert (p.nk, p.nb) == (row["nk"], row["nb"])
    K = G.HartreeFockKernel(**p.kernel_kwargs())
    P0 = torch.zeros((p.nk, p.nk, p.nb, p.nb), dtype=torch.complex128, device="cuda")
    r = solve_scf(K, P0, p.n_electrons, config=SCFConfig(**FAST, fp32_exchange=True))
    assert r.converged and abs(float(r.energy) - row["energy"]) <= TOL_E * abs(row["energy"])
    rc = solve(K, P0, p.n_electrons, config=SolverConfig(max_iter=400, tol_E=1e-9))
    assert abs(float(rc.energy) - row["cg_energy"]) <= 1e-9 * abs(row["cg_energy"])
    assert int(rc.n_iter) == row["cg_n_iter"]


@pytest.mark.parametrize("nb", [3, 4, 8])
def test_eigh_warm_matches_eigh(cuda, nb):
    """hf_eigh_warm, cold and from a nearby basis, against hf_eigh: eigenvalues, and
    A = V diag(w) V^H with unitary V."""
    from jax_hf_b200 import _lib
    L = _lib.lib()
    g = torch.Generator(device="cpu").manual_seed(nb)
    nk = 777
    X = torch.randn(nk, nb, nb, dtype=torch.complex128, generator=g)
    A = (X + X.conj().transpose(-1, -2)).cuda().contiguous()
    w0 = torch.empty(nk, nb, dtype=torch.float64, device="cuda")
    V0 = torch.empty_like(A)
    _lib.check(L.hf_eigh(_lib.stream_ptr(A.device), _lib.HF_C128, nk, nb, A.data_ptr(), w0.data_ptr(), V0.data_ptr()))
    w1, V1 = torch.empty_like(w0), torch.empty_like(A)
    _lib.check(L.hf_eigh_warm(_lib.stream_ptr(A.device), nk, nb, A.data_ptr(), None, V1.data_ptr(), w1.data_ptr()))
    Y = torch.randn(nk, nb, nb, dtype=torch.complex128, generator=g).cuda()
    A2 = (A + 1e-3 * (Y + Y.conj().transpose(-1, -2))).contiguous()
    w2 = torch.empty_like(w0)
    V2 = V1.clone()  # start from the eigenvectors of the nearby matrix A, in place
    _lib.check(L.hf_eigh_warm(_lib.stream_ptr(A.device), nk, nb, A2.data_ptr(), V2.data_ptr(), V2.data_ptr(),
                              w2.data_ptr()))
    torch.cuda.synchronize()
    ref2 = torch.linalg.eigvalsh(A2)
    assert float((w1 - w0).abs().max()) < 1e-12 * float(w0.abs().max())
    assert float((w2 - ref2).abs().max()) < 1e-12 * float(ref2.abs().max())
    eye = torch.eye(nb, dtype=torch.complex128, device="cuda")
    for Am, w, V in ((A, w1, V1), (A2, w2, V2)):
        R = V @ torch.diag_embed(w.to(torch.complex128)) @ V.conj().transpose(-1, -2)
        assert float((R - Am).abs().max()) < 1e-12 * float(Am.abs().max())
        assert float((V.conj().transpose(-1, -2) @ V - eye).abs().max()) < 1e-12
        assert bool((w[:, 1:] >= w[:, :-1]).all())
