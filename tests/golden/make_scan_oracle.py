"""Converged FP64 oracle energies of the 64-solve density scan (seeded synthetic problems).

Each problem of ``jax_hf_b200.synthetic.density_scan(64)`` (meshes 36-120, nb 4/6/8,
fillings in (0.1, 0.9), T = 0.1, scalar V for even and layer-resolved V for odd
indices) is solved by the CPU oracle's SCF-DIIS (reference_scf.py:124-365 restated)
from P0 = 0 to a density residual of 1e-11 and a commutator residual of 1e-10: the
self-consistent fixed point, which no stopping rule can move.  The energies pin the
|dE/E| of every GPU solve of the scan against the FP64 oracle.  Also stored: the
reference CG's own result (solver.py:307-660, plateau stop tol_E = 1e-9) for the same
problems, to show where that stopping rule ends.

Run from the repo root: ``python tests/golden/make_scan_oracle.py [n_workers]``
(about ten minutes on eight cores).  Writes ``tests/golden/scan64_oracle.json``.
"""

import json
import multiprocessing as mp
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))


def _one(i):
    from jax_hf_b200 import synthetic as S
    from oracle import hf_oracle as O
    p = S.density_scan(64)[i]
    K = O.Kernel(**p.kernel_kwargs())
    P0 = np.zeros((p.nk, p.nk, p.nb, p.nb), complex)
    t = time.time()
    rs = O.solve_scf(K, P0, p.n_electrons,
                     config=O.SCFConfig(acceleration="diis", density_tol=1e-11, comm_tol=1e-10, max_iter=400))
    rc = O.solve_cg(K, P0, p.n_electrons, config=O.SolverConfig(max_iter=400, tol_E=1e-9))
    return {"index": i, "nk": int(p.nk), "nb": int(p.nb), "n_electrons": float(p.n_electrons),
            "energy": float(rs["energy"]), "scf_iterations": int(rs["iterations"]),
            "scf_converged": bool(rs["converged"]), "mu": float(rs["chemical_potential"]),
            "cg_energy": float(rc["energy"]), "cg_n_iter": int(rc["n_iter"]), "seconds": round(time.time() - t, 1)}


def main(workers: int) -> None:
    with mp.get_context("spawn").Pool(workers) as pool:
        rows = pool.map(_one, range(64))
    rows.sort(key=lambda r: r["index"])
    out = Path(__file__).with_name("scan64_oracle.json")
    out.write_text(json.dumps({"problems": "jax_hf_b200.synthetic.density_scan(64)",
                               "scf": "oracle SCF-DIIS from P0 = 0, density_tol 1e-11, comm_tol 1e-10",
                               "cg": "oracle CG, tol_E 1e-9 (reference plateau rule)", "rows": rows}, indent=1))
    print("wrote", out, "max |E_cg - E|/|E| =", max(abs(r["cg_energy"] - r["energy"]) / abs(r["energy"]) for r in rows))


if __name__ == "__main__":
    main(int(sys.argv[1]) if len(sys.argv) > 1 else 8)
