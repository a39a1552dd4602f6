"""The C-ABI library loads and exports every declared symbol; host-side checks (CPU only)."""

import ctypes as C
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _declared():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        names |= set(re.findall(r"^(?:int|const char\*)\s+(hf_\w+)\s*\(", h.read_text(), re.M))
    return sorted(names)


def test_header_declares_entry_points():
    names = _declared()
    assert "hf_fock_build" in names and "hf_energy" in names and "hf_find_mu" in names


def test_library_exports_every_declared_symbol():
    from jax_hf_b200 import _lib
    L = _lib.lib()
    for name in _declared():
        assert hasattr(L, name), name
    assert set(_declared()) <= set(_lib.exported_symbols())


def test_workspace_size_query_runs_on_host():
    from jax_hf_b200 import _lib
    n = C.c_size_t(0)
    flags = _lib.FOCK_EXCHANGE | _lib.FOCK_VR_REAL
    _lib.check(_lib.lib().hf_fock_workspace_size(_lib.HF_C128, flags, 192, 192, 8, C.byref(n)))
    # spectrum scratch: 64 channels x 192^2 complex128, plus small terms
    assert n.value >= 64 * 192 * 192 * 16


def test_reference_validation_errors_map_to_valueerror():
    from jax_hf_b200 import _lib
    n = C.c_size_t(0)
    with pytest.raises(ValueError, match="at least one of Hartree or exchange"):
        _lib.check(_lib.lib().hf_fock_workspace_size(_lib.HF_C128, 0, 4, 4, 2, C.byref(n)))
    with pytest.raises(ValueError, match="hermitian_channel_packing requires a scalar"):
        _lib.check(_lib.lib().hf_fock_workspace_size(
            _lib.HF_C128, _lib.FOCK_EXCHANGE | _lib.FOCK_PACKING, 4, 4, 2, C.byref(n)))


def test_shape_limits_are_reported_on_the_host():
    from jax_hf_b200 import _lib
    n = C.c_size_t(0)
    ex = _lib.FOCK_EXCHANGE
    _lib.check(_lib.lib().hf_fock_workspace_size(_lib.HF_C128, ex, 3, 5, 32, C.byref(n)))
    assert n.value > 0
    with pytest.raises(_lib.HFError, match="nb > 32"):
        _lib.check(_lib.lib().hf_fock_workspace_size(_lib.HF_C128, ex, 4, 4, 33, C.byref(n)))
    for nk1, nk2, nb in ((0, 4, 2), (4, 0, 2), (4, 4, 0)):
        with pytest.raises(ValueError, match="must be positive"):
            _lib.check(_lib.lib().hf_fock_workspace_size(_lib.HF_C128, ex, nk1, nk2, nb, C.byref(n)))


def test_status_strings():
    from jax_hf_b200 import _lib
    assert _lib.lib().hf_status_string(0) == b"ok"
    assert _lib.lib().hf_version() >= 1
