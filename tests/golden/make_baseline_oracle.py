"""Oracle results for the whole-solve workloads of the benchmark (seeded synthetic problems).

For ``synthetic.scf_diis_24()`` (24x24, nb 4), ``synthetic.cg_144()`` (144x144, nb 8,
T 0.05, filling 3/8) and ``synthetic.newton_96()`` (96x96, nb 4) the CPU oracle
(the NumPy restatement of the reference) computes:

* the self-consistent fixed point: SCF-DIIS from P0 = 0 to a density residual of
  1e-11 and a commutator residual of 1e-10 (its energy is what a solve must reach
  for |dE/E| <= 1e-9 against the FP64 oracle);
* the reference algorithm's own result for the benchmark's settings: SCF-DIIS with
  default tolerances (24x24), CG with tol_E = 1e-9 (144x144), trust-region Newton
  with tol_grad = 1e-6 (96x96).

Run from the repo root: ``python tests/golden/make_baseline_oracle.py`` (about a
minute).  Writes ``tests/golden/baseline_oracle.json``.
"""

import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))


def main() -> None:
    from jax_hf_b200 import synthetic as S
    from oracle import hf_oracle as O
    out = {}
    tight = O.SCFConfig(acceleration="diis", density_tol=1e-11, comm_tol=1e-10, max_iter=400)
    for name, p, algo in (("scf_diis_24x24_nb4", S.scf_diis_24(), "scf"), ("cg_144x144_nb8", S.cg_144(), "cg"),
                          ("newton_96x96_nb4", S.newton_96(), "newton")):
        K = O.Kernel(**p.kernel_kwargs())
        P0 = np.zeros((p.nk, p.nk, p.nb, p.nb), complex)
        t = time.time()
        fp = O.solve_scf(K, P0, p.n_electrons, config=tight)
        if algo == "scf":
            r = O.solve_scf(K, P0, p.n_electrons, config=O.SCFConfig(acceleration="diis"))
            ref = {"energy": float(r["energy"]), "iterations": int(r["iterations"]), "converged": bool(r["converged"])}
        elif algo == "cg":
            r = O.solve(K, P0, p.n_electrons, config=O.SolverConfig(max_iter=400, tol_E=1e-9))
            ref = {"energy": float(r["energy"]), "n_iter": int(r["n_iter"]), "converged": bool(r["converged"])}
        else:
            r = O.solve(K, P0, p.n_electrons, config=O.SolverConfig(optimizer="newton", tol_grad=1e-6, max_iter=200))
            ref = {"energy": float(r["energy"]), "n_iter": int(r["n_iter"]), "converged": bool(r["converged"])}
        out[name] = {"fixed_point_energy": float(fp["energy"]), "fixed_point_iterations": int(fp["iterations"]),
                     "fixed_point_converged": bool(fp["converged"]), "reference_algorithm": ref,
                     "seconds": round(time.time() - t, 1)}
        print(name, out[name], flush=True)
    dst = Path(__file__).with_name("baseline_oracle.json")
    dst.write_text(json.dumps(out, indent=1))
    print("wrote", dst)


if __name__ == "__main__":
    main()
