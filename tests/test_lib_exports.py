"""libtbr.so loads and exports every entry point include/tbr.h declares (no device calls)."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "tbr.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(tbr_[a-z0-9_]+)\s*\(", src)))


def test_every_declared_symbol_is_exported():
    from turboransac_b200 import build, _lib
    build.build()
    L = ctypes.CDLL(_lib.LIB_PATH)
    syms = declared_symbols()
    assert len(syms) >= 20
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing
    assert set(syms) == set(_lib.EXPORTS)


def test_abi_version_and_defaults():
    from turboransac_b200 import _lib
    L = _lib.lib()
    assert L.tbr_abi_version() == 1
    o = _lib.RansacOptionsC()
    L.tbr_default_ransac_options(ctypes.byref(o))
    assert o.max_iterations == 100000 and o.success_prob == 0.9999 and o.max_reproj_error == 12.0
    b = _lib.BundleOptionsC()
    L.tbr_default_bundle_options(ctypes.byref(b))
    assert b.max_iterations == 100 and b.loss_type == 3 and b.step_tol == 1e-8


def test_no_device_is_a_clean_error():
    """Without a GPU, creating a context fails with a status code, not exit()."""
    from turboransac_b200 import _lib
    try:
        import torch
        if torch.cuda.is_available():
            return
    except Exception:
        pass
    L = _lib.lib()
    h = ctypes.c_void_p()
    st = L.tbr_context_create(0, 0, ctypes.byref(h))
    assert st == 3  # TBR_ERR_CUDA
    assert b"no CUDA device" in L.tbr_last_error()
