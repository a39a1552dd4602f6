"""Extract the golden vectors that pin the oracle from the reference's test data.

Reads ``tests/data/meshgrid_regression_case_v1.npz`` of the reference (jax_hf)
and keeps the fields that pin ``build_fock`` + ``hf_energy`` (12x12 mesh, 4
bands, complex64, exchange + Hartree + reference density).  Run from the repo
root with the reference checkout's root directory as the one required argument:
``python tests/golden/make_golden.py <reference-root>``.
"""

import argparse
from pathlib import Path

import numpy as np

KEEP = ("nk", "T", "weights", "hamiltonian", "coulomb_q", "hartree_matrix",
        "reference_density", "P_expected", "F_expected", "E_expected", "mu_expected",
        "electrondensity0")


def main(ref_root: str) -> None:
    src = Path(ref_root) / "tests" / "data" / "meshgrid_regression_case_v1.npz"
    d = np.load(src)
    out = {k: d[k] for k in KEEP}
    dst = Path(__file__).with_name("meshgrid_v1.npz")
    np.savez_compressed(dst, **out)
    print("wrote", dst, sorted(out))


if __name__ == "__main__":
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("reference_root", help="root directory of the jax_hf checkout (holds tests/data/)")
    main(ap.parse_args().reference_root)
