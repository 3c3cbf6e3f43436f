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


def test_submit_and_collect_refuse_bad_arguments_before_any_device_call():
    """The submitted batch calls check their arguments on the host: a NULL
    context, frame list or ticket pointer, and a ticket that was never handed
    out, are refused with TBR_ERR_INVALID_ARG and a message."""
    from turboransac_b200 import _lib
    L = _lib.lib()
    ro = _lib.RansacOptionsC()
    L.tbr_default_ransac_options(ctypes.byref(ro))
    fr = (_lib.FrameDescC * 1)()
    t = ctypes.c_void_p()
    assert L.tbr_estimate_batch_submit(None, fr, 1, ctypes.byref(ro), None, ctypes.byref(t)) == 1
    assert L.tbr_estimate_batch_device_submit(None, fr, 1, ctypes.byref(ro), None, None, ctypes.byref(t)) == 1
    assert L.tbr_estimate_batch_submit(ctypes.c_void_p(8), None, 1, ctypes.byref(ro), None, ctypes.byref(t)) == 1
    assert L.tbr_estimate_batch_submit(ctypes.c_void_p(8), fr, 0, ctypes.byref(ro), None, ctypes.byref(t)) == 1
    assert L.tbr_estimate_batch_submit(ctypes.c_void_p(8), fr, 1, ctypes.byref(ro), None, None) == 1
    assert L.tbr_estimate_batch_submit(ctypes.c_void_p(8), fr, 1025, ctypes.byref(ro), None, ctypes.byref(t)) == 1
    assert b"1024" in L.tbr_last_error()
    assert L.tbr_estimate_batch_collect(None, None, None) == 1
    assert L.tbr_estimate_batch_collect(ctypes.c_void_p(16), None, None) == 1  # never handed out
    assert b"unknown ticket" in L.tbr_last_error()
