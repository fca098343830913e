"""The C-ABI library builds for sm_100a, loads without a GPU and exports every
entry point that include/*.h declares (no compute calls here)."""
import ctypes
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    text = "\n".join(p.read_text() for p in sorted((ROOT / "include").glob("*.h")))
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(vqemps_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from vqemps import build, _lib
    build.build()
    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    names = declared_symbols()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) <= set(_lib.SYMBOLS)


def test_binding_loads_and_rejects_bad_arguments_without_a_gpu():
    from vqemps import _lib
    lib = _lib.load()
    # invalid arguments are rejected before any device call
    assert lib.vqemps_create(0, 99, 0.0, 0.0, ctypes.byref(ctypes.c_void_p())) == _lib.INVALID
    assert lib.vqemps_create(0, 16, -1.0, 0.0, ctypes.byref(ctypes.c_void_p())) == _lib.INVALID
    assert lib.vqemps_last_error(None) == b"null context"
    assert lib.vqemps_destroy(None) == _lib.OK
    assert lib.vqemps_mpnn_create(0, 4, 3, 100, 3, 5, ctypes.byref(ctypes.c_void_p())) == _lib.INVALID
    assert lib.vqemps_mpnn_last_error(None) == b"null network"


def test_built_for_sm_100a():
    from vqemps import build
    assert "arch=compute_100a,code=sm_100a" in " ".join(build.NVCC_FLAGS)
