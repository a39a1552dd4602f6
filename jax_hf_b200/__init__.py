"""jax_hf_b200 — B200-native (sm_100a) Fock build and HF objective.

Drop-in for the hot path of jax_hf: ``HartreeFockKernel``, ``build_fock``,
``hf_energy``, ``free_energy``, ``occupation_entropy`` and the solvers that
call them, running hand-written CUDA kernels through the C ABI in
``include/hf_b200.h`` (library ``lib/libhf_b200.so``, built in-tree).
"""

from .problem import HartreeFockKernel  # noqa: F401
from .fock import build_fock, build_fock_batch, hf_energy, free_energy, occupation_entropy  # noqa: F401
from .utils import find_chemical_potential, fermidirac, validate_electron_count, resample_kgrid  # noqa: F401
from . import linalg  # noqa: F401

__all__ = [
    "HartreeFockKernel",
    "build_fock",
    "build_fock_batch",
    "hf_energy",
    "free_energy",
    "occupation_entropy",
    "find_chemical_potential",
    "fermidirac",
    "validate_electron_count",
    "resample_kgrid",
    "linalg",
]
