"""Host-side batch plumbing without a GPU: the frame descriptors handed to the C
ABI (addresses, counts, cameras, seeds, thresholds, validation) and the packed
results returned to Python."""
import ctypes as C

import numpy as np
import pytest

from turboransac_b200 import RESULT_DTYPE, _lib, api, scenes


def descs(frames, **kw):
    ptr, keep = api._frame_descs(frames, **kw)
    return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_uint8)), (len(frames) * api._DESC_DTYPE.itemsize,)) \
        .view(api._DESC_DTYPE), keep


def test_descriptors_point_at_the_arrays_and_carry_frame_fields():
    fr = scenes.batched_frames(6, scale=0.2)
    d, keep = descs(fr)
    for i, f in enumerate(fr):
        assert d["points2D"][i] == f.uv.ctypes.data and d["points3D"][i] == f.xyz.ctypes.data
        assert d["n"][i] == f.n
        np.testing.assert_array_equal(d["K"][i], np.asarray(f.K, np.float64))
        assert int(d["seed"][i]) == f.seed & 0xFFFFFFFFFFFFFFFF
    d2, _ = descs(fr, max_reproj_error=3.5)
    assert (d2["max_reproj_error"] == 3.5).all()


def test_descriptors_convert_and_keep_noncontiguous_or_other_dtypes():
    f = scenes.batched_frames(1, scale=0.2)[0]
    g = scenes.Frame(**{**f.__dict__, "uv": np.asfortranarray(f.uv.astype(np.float32)),
                        "xyz": f.xyz[::1].copy()})
    d, keep = descs([g])
    conv = next(a for a in keep if isinstance(a, np.ndarray) and a.ndim == 2 and a.shape[1] == 2)
    assert conv.dtype == np.float64 and conv.flags.c_contiguous
    assert d["points2D"][0] == conv.ctypes.data  # the converted copy, kept alive
    np.testing.assert_allclose(conv, f.uv.astype(np.float32))


def test_descriptors_take_read_only_arrays_and_wrap_negative_seeds():
    f = scenes.batched_frames(1, scale=0.2)[0]
    uv = f.uv.copy()
    uv.flags.writeable = False
    g = scenes.Frame(**{**f.__dict__, "uv": uv, "seed": -1})
    d, _ = descs([g])
    assert d["points2D"][0] == uv.ctypes.data
    assert int(d["seed"][0]) == 0xFFFFFFFFFFFFFFFF


@pytest.mark.parametrize("bad", ["uv_cols", "xyz_cols", "count"])
def test_descriptors_reject_malformed_frames(bad):
    f = scenes.batched_frames(1, scale=0.2)[0]
    uv, xyz = f.uv, f.xyz
    if bad == "uv_cols":
        uv = np.zeros((f.n, 3))
    elif bad == "xyz_cols":
        xyz = np.zeros((f.n, 2))
    else:
        xyz = xyz[:-1]
    g = scenes.Frame(**{**f.__dict__, "uv": uv, "xyz": xyz})
    with pytest.raises(ValueError):
        api._frame_descs([g])


def test_results_unpack_as_dicts_or_one_record_array():
    n = 3
    res = (_lib.FrameResultC * n)()
    for i in range(n):
        res[i].q[0] = 1.0
        res[i].t[2] = float(i)
        res[i].status = i
        res[i].stats.samples = 1000 * (i + 1)
        res[i].stats.num_inliers = 10 + i
    arr = api._results(res, n, as_array=True)
    assert arr.dtype == RESULT_DTYPE and arr.shape == (n,)
    assert list(arr["stats"]["samples"]) == [1000, 2000, 3000]
    dicts = api._results(res, n)
    for i, r in enumerate(dicts):
        assert r["status"] == i and r["samples"] == 1000 * (i + 1) and r["num_inliers"] == 10 + i
        np.testing.assert_array_equal(r["t"], [0.0, 0.0, float(i)])
        assert r["q"][0] == 1.0


def test_camera_parameters_are_the_four_pinhole_values():
    cam = api.Camera_cuda(1, 640, 480, [525.0, 526.0, 319.5, 239.5])
    K = api._camera_K(cam)
    assert K.dtype == np.float64 and K.flags.c_contiguous and list(K) == [525.0, 526.0, 319.5, 239.5]
    for bad in ([525.0, 319.5, 239.5], [525.0, 525.0, 319.5, 239.5, 0.0]):
        with pytest.raises(ValueError):
            api._camera_K(api.Camera_cuda(1, 640, 480, bad))


def test_submitted_forms_check_frames_before_the_context():
    """estimate_batch_submit refuses malformed host frames, and the device form
    refuses frames that are not float64 CUDA tensors, on the host before any
    call reaches the library (no context or GPU is needed to see it)."""
    import dataclasses
    f = scenes.plain_frame(0)
    bad = dataclasses.replace(f, xyz=f.xyz[:-1])
    with pytest.raises(ValueError):
        api.estimate_batch_submit(None, [f, bad])
    with pytest.raises(ValueError):
        api.estimate_batch_device_submit(None, [f])  # numpy arrays, not CUDA tensors
    t = api.BatchTicket(None, None, [3], None)
    with pytest.raises(RuntimeError):  # nothing to collect
        t.collect()
