"""ctypes binding of the in-tree CUDA library (``lib/libhf_b200.so``).

The product path has no CPU fallback: if the library is missing or CUDA is
unavailable, every operation raises.  Status codes map to exceptions; the
reference's validation errors (ValueError) keep their type and message.
"""

from __future__ import annotations

import ctypes as C
import threading
from pathlib import Path

import torch

_LIB_PATH = Path(__file__).resolve().parent / "lib" / "libhf_b200.so"
_lock = threading.Lock()
_lib = None

HF_OK, HF_ERR_INVALID, HF_ERR_UNSUPPORTED, HF_ERR_CUDA = 0, 1, 2, 3
HF_ERR_WORKSPACE, HF_ERR_NONFINITE, HF_ERR_MAXITER, HF_ERR_ABORTED = 4, 5, 6, 7
HF_C128, HF_C64 = 0, 1

FOCK_EXCHANGE = 1 << 0
FOCK_HARTREE = 1 << 1
FOCK_PACKING = 1 << 2
FOCK_VR_SCALAR = 1 << 3
FOCK_VR_REAL = 1 << 4
FOCK_FFT_FP32 = 1 << 5
FOCK_HAS_REFP = 1 << 6
FOCK_GENERIC_FFT = 1 << 7
FOCK_SYM_V = 1 << 8
FOCK_TILE_PLAN = 1 << 9
FOCK_PIPE = 1 << 10

vp, i32, u32, f64, sz = C.c_void_p, C.c_int, C.c_uint, C.c_double, C.c_size_t
pf64 = C.POINTER(C.c_double)
psz = C.POINTER(C.c_size_t)

_SIGS = {
    "hf_last_error": ([], C.c_char_p),
    "hf_status_string": ([i32], C.c_char_p),
    "hf_version": ([], i32),
    "hf_fock_workspace_size": ([i32, u32, i32, i32, i32, psz], i32),
    "hf_fock_build": ([vp, i32, u32, i32, i32, i32, vp, vp, vp, vp, vp, vp, i32, vp, vp, vp,
                       vp, vp, vp, vp, sz], i32),
    "hf_fock_blocks_workspace_size": ([i32, u32, i32, i32, i32, vp, psz], i32),
    "hf_fock_build_blocks": ([vp, i32, u32, i32, i32, i32, vp, vp, vp, vp, vp, vp, vp, i32, vp, vp, vp, vp, vp, vp,
                              vp, sz], i32),
    "hf_block_offdiag_max": ([vp, i32, sz, i32, vp, vp, i32, vp, vp], i32),
    "hf_fock_block_specs_workspace_size": ([i32, u32, i32, i32, i32, i32, vp, psz], i32),
    "hf_fock_build_block_specs": ([vp, i32, u32, i32, i32, i32, i32, vp, f64, f64, vp, vp, vp, vp, vp, vp, i32, vp,
                                   vp, vp, vp, vp, vp, vp, sz, vp], i32),
    "hf_fock_autotune": ([vp, i32, u32, i32, i32, i32, vp, vp, vp, vp, vp, vp, i32, vp, vp, vp,
                          vp, vp, vp, vp, sz, i32, C.POINTER(C.c_uint), C.POINTER(C.c_float)], i32),
    "hf_fock_autotune_reset": ([], i32),
    "hf_fock_fault_status": ([C.POINTER(C.c_int), i32], i32),
    "hf_resample_kgrid": ([vp, i32, i32, i32, i32, i32, C.c_longlong, vp, vp], i32),
    "hf_resample_density": ([vp, i32, i32, i32, i32, i32, i32, vp, vp], i32),
    "hf_sym_group_average": ([vp, i32, i32, i32, i32, vp, vp, i32, vp, i32, vp, i32, i32, vp, vp, vp], i32),
    "hf_sym_time_reversal": ([vp, i32, i32, i32, i32, vp, vp, vp, i32, i32, vp, vp, vp], i32),
    "hf_sl_fock_workspace_size": ([i32, i32, i32, i32, i32, i32, i32, psz], i32),
    "hf_sl_fock": ([vp, i32, i32, i32, i32, i32, i32, i32, vp, vp, vp, vp, vp, vp, vp, sz], i32),
    "hf_fock_build_static_scratch": ([vp, i32, u32, i32, i32, i32, vp, vp, vp, vp, vp, vp, i32, vp, vp, vp,
                                      vp, vp, vp], i32),
    "hf_reduce_workspace_size": ([i32, i32, i32, psz], i32),
    "hf_energy": ([vp, i32, i32, i32, i32, vp, vp, vp, vp, i32, vp, vp, vp, sz], i32),
    "hf_occupation_entropy": ([vp, i32, i32, i32, i32, vp, vp, vp, vp, sz], i32),
    "hf_free_energy": ([vp, i32, i32, i32, i32, vp, vp, vp, f64, vp, vp, sz], i32),
    "hf_find_mu": ([vp, i32, i32, i32, i32, i32, vp, vp, f64, f64, i32, vp, vp], i32),
    "hf_density_from_Qp": ([vp, i32, i32, i32, vp, vp, vp], i32),
    "hf_fock_orbital": ([vp, i32, i32, i32, vp, vp, vp], i32),
    "hf_eigh": ([vp, i32, i32, i32, vp, vp, vp], i32),
    "hf_eigh_warm": ([vp, i32, i32, vp, vp, vp, vp], i32),
    "hf_cayley_retract": ([vp, i32, i32, i32, vp, f64, vp], i32),
    "hf_cayley_spectral": ([vp, i32, i32, i32, vp, vp, vp], i32),
    "hf_cayley_unitary": ([vp, i32, i32, i32, vp, vp, f64, vp], i32),
    "hf_diag_UFU": ([vp, i32, i32, i32, vp, vp, vp, f64, vp], i32),
    "hf_qr_retract": ([vp, i32, i32, i32, vp, f64, vp], i32),
    "hf_ops_workspace_size": ([psz], i32),
    "hf_fermi": ([vp, sz, vp, vp, f64, i32, f64, vp], i32),
    "hf_scf_residuals": ([vp, i32, i32, vp, vp, vp, vp, vp, vp, vp, vp], i32),
    "hf_gram": ([vp, i32, sz, i32, i32, vp, vp, vp, vp], i32),
    "hf_gram_row": ([vp, i32, i32, sz, i32, i32, vp, vp, vp, vp], i32),
    "hf_lincomb": ([vp, i32, sz, sz, vp, vp, vp], i32),
    "hf_axpby": ([vp, sz, i32, f64, vp, f64, vp, i32, vp], i32),
    "hf_axpby_real": ([vp, sz, f64, vp, f64, vp, vp], i32),
    "hf_jdot": ([vp, sz, i32, vp, vp, vp, vp, vp, vp, vp, vp], i32),
    "hf_orbital_grad": ([vp, sz, i32, vp, vp, vp, vp], i32),
    "hf_newton_prec": ([vp, sz, i32, vp, vp, vp, vp, f64, f64, f64, vp, vp, vp, vp, vp], i32),
    "hf_sub_scalar": ([vp, sz, vp, vp, f64], i32),
    "hf_newton_dP": ([vp, i32, i32, vp, vp, vp, vp, vp], i32),
    "hf_newton_hvp": ([vp, i32, i32, vp, vp, vp, vp, vp, vp, vp, f64, f64, f64, vp, vp, vp, vp, vp, vp], i32),
    "hf_matmul": ([vp, i32, i32, vp, vp, vp], i32),
    "hf_real_diag": ([vp, sz, i32, vp, vp], i32),
    "hf_cg_workspace_size": ([vp, vp, psz], i32),
    "hf_cg_solve": ([vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, sz], i32),
    "hf_cg_batch_workspace_size": ([vp, i32, vp, psz], i32),
    "hf_scf_workspace_size": ([vp, vp, psz], i32),
    "hf_scf_solve": ([vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, sz], i32),
    "hf_scf_batch_workspace_size": ([vp, i32, vp, psz], i32),
    "hf_scf_batch_graph_create": ([vp, i32, vp, vp, sz, vp], i32),
    "hf_scf_batch_graph_launch": ([vp, vp, vp], i32),
    "hf_scf_batch_graph_destroy": ([vp], i32),
    "hf_newton_workspace_size": ([vp, vp, psz], i32),
    "hf_newton_solve": ([vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, sz], i32),
    "hf_fock_vjp_workspace_size": ([i32, u32, i32, i32, i32, psz], i32),
    "hf_fock_build_vjp": ([vp, i32, u32, i32, i32, i32, vp, vp, vp, vp, vp, vp, sz], i32),
    "hf_energy_vjp": ([vp, i32, i32, i32, vp, vp, vp, vp, i32, vp, f64, vp, vp, vp], i32),
    "hf_free_energy_vjp": ([vp, i32, i32, i32, vp, vp, f64, f64, vp], i32),
    "hf_fourier_coeffs": ([vp, i32, i32, i32, vp, vp, i32, vp, vp], i32),
    "hf_cg_solve_batch": ([vp, vp, i32, vp, i32, vp, sz, vp], i32),
    "hf_cg_solve_batch_graph": ([vp, vp, i32, vp, vp, sz, vp], i32),
    "hf_cg_batch_graph_create": ([vp, i32, vp, vp, sz, vp], i32),
    "hf_cg_batch_graph_launch": ([vp, vp, vp], i32),
    "hf_cg_batch_graph_destroy": ([vp], i32),
}


class HFError(RuntimeError):
    """A CUDA-side failure reported by the hf_b200 library."""

    def __init__(self, status: int, msg: str):
        super().__init__(f"[{status}] {msg}")
        self.status = status


def lib():
    """Loads the library once; raises if it is not built."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not _LIB_PATH.exists():
                raise ImportError(
                    f"CUDA library not built: {_LIB_PATH} (run `python -m jax_hf_b200.build`)")
            L = C.CDLL(str(_LIB_PATH))
            for name, (args, res) in _SIGS.items():
                fn = getattr(L, name)
                fn.argtypes = args
                fn.restype = res
            _lib = L
    return _lib


def exported_symbols():
    return list(_SIGS)


def check(status: int) -> None:
    if status == HF_OK:
        return
    msg = lib().hf_last_error().decode(errors="replace")
    if status == HF_ERR_INVALID:
        raise ValueError(msg)
    raise HFError(status, msg)


def require_cuda(t: torch.Tensor) -> None:
    if not t.is_cuda:
        raise RuntimeError("jax_hf_b200 runs on CUDA tensors only (no CPU fallback)")


def stream_ptr(device=None) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def ptr(t) -> int | None:
    if t is None:
        return None
    return t.data_ptr()


def dtype_code(t: torch.Tensor) -> int:
    if t.dtype in (torch.complex128, torch.float64):
        return HF_C128
    if t.dtype in (torch.complex64, torch.float32):
        return HF_C64
    raise TypeError(f"unsupported dtype {t.dtype}")


_ws_cache: dict = {}


def workspace(nbytes: int, device, tag: str = "ws") -> torch.Tensor:
    """Caller-owned scratch from torch's caching allocator (256-byte aligned).

    One buffer per (tag, device, current stream): calls on different streams may
    run at the same time and never share scratch; calls on one stream are ordered.
    """
    key = (tag, str(device), torch.cuda.current_stream(device).cuda_stream)
    buf = _ws_cache.get(key)
    if buf is None or buf.numel() < nbytes:
        buf = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device)
        _ws_cache[key] = buf
    return buf
