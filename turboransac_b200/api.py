"""Python mirror of the reference's absolute-pose interface, over libtbr.so.

Names, argument meaning and defaults follow the reference's C++ API
(Module/TbrCudaPnP/include/TbrCudaPnP/): ``RansacOptions_cuda``,
``BundleOptions_cuda``, ``RansacStats_cuda`` (utils.h:14-72), ``Camera_cuda``
(camera.cuh:10-85), ``CameraPose_cuda`` (pose.cuh:12-80),
``estimate_absolute_pose_cuda`` / ``get_inliers_mx`` (entry.h:13-25) and
``bundle_adjust_cuda`` (ba.cuh:17-24). Instead of exiting the process on a CUDA
error (cudaCheck.h:4-14) every call raises ``TbrError``.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import threading
import weakref

import numpy as np

from . import _lib
from ._lib import TbrError, check

__all__ = ["Batch", "Server", "estimate_batch", "RansacOptions_cuda", "BundleOptions_cuda", "RansacStats_cuda", "Camera_cuda",
           "CameraPose_cuda", "Context", "estimate_absolute_pose_cuda", "get_inliers_mx",
           "bundle_adjust_cuda", "TbrError"]


@dataclasses.dataclass
class RansacOptions_cuda:
    max_iterations: int = 100000      # reference meaning: samples per round (grid size)
    min_iterations: int = 1000
    dyn_num_trials_mult: float = 3.0
    success_prob: float = 0.9999
    max_reproj_error: float = 12.0
    max_epipolar_error: float = 1.0
    seed: int = 0
    progressive_sampling: bool = False
    max_prosac_iterations: int = 100000
    real_focal_check: bool = False
    score_initial_model: bool = False

    def to_c(self) -> _lib.RansacOptionsC:
        return _lib.RansacOptionsC(self.max_iterations, self.min_iterations, self.dyn_num_trials_mult,
                                   self.success_prob, self.max_reproj_error, self.max_epipolar_error,
                                   self.seed & 0xFFFFFFFFFFFFFFFF, int(self.progressive_sampling),
                                   self.max_prosac_iterations, int(self.real_focal_check),
                                   int(self.score_initial_model))


@dataclasses.dataclass
class BundleOptions_cuda:
    TRIVIAL, TRUNCATED, HUBER, CAUCHY, TRUNCATED_LE_ZACH = range(5)
    max_iterations: int = 100
    loss_type: int = 3
    loss_scale: float = 1.0
    gradient_tol: float = 1e-10
    step_tol: float = 1e-8
    initial_lambda: float = 1e-3
    min_lambda: float = 1e-10
    max_lambda: float = 1e10
    verbose: bool = False

    def to_c(self) -> _lib.BundleOptionsC:
        return _lib.BundleOptionsC(self.max_iterations, self.loss_type, self.loss_scale, self.gradient_tol,
                                   self.step_tol, self.initial_lambda, self.min_lambda, self.max_lambda,
                                   int(self.verbose))


@dataclasses.dataclass
class RansacStats_cuda:
    refinements: int = 0
    iterations: int = 0
    num_inliers: int = 0
    inlier_ratio: float = 0.0
    model_score: float = float("inf")
    # Beyond the reference (which returns these unfilled): engine details.
    details: dict = dataclasses.field(default_factory=dict)


@dataclasses.dataclass
class Camera_cuda:
    model_id: int = 1  # PINHOLE
    width: int = -1
    height: int = -1
    params: list = dataclasses.field(default_factory=lambda: [0.0, 0.0, 0.0, 0.0])  # fx, fy, cx, cy

    def focal(self) -> float:
        return 0.5 * (self.params[0] + self.params[1])

    def unproject(self, xp):
        fx, fy, cx, cy = self.params
        xp = np.asarray(xp, np.float64)
        return np.stack([(xp[..., 0] - cx) / fx, (xp[..., 1] - cy) / fy], axis=-1)

    def project(self, x):
        fx, fy, cx, cy = self.params
        x = np.asarray(x, np.float64)
        return np.stack([fx * x[..., 0] + cx, fy * x[..., 1] + cy], axis=-1)

    def rescale(self, scale: float) -> None:
        self.params = [p * scale for p in self.params]


def _quat_to_rotmat(q):
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


@dataclasses.dataclass
class CameraPose_cuda:
    """Unit quaternion q = (w, x, y, z) and t, with X_cam = R X + t."""

    q: np.ndarray = dataclasses.field(default_factory=lambda: np.array([1.0, 0.0, 0.0, 0.0]))
    t: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros(3))

    def R(self) -> np.ndarray:
        return _quat_to_rotmat(self.q)

    def Rt(self) -> np.ndarray:
        return np.hstack([self.R(), np.asarray(self.t).reshape(3, 1)])

    def Rt_homo(self) -> np.ndarray:
        m = np.eye(4)
        m[:3, :4] = self.Rt()
        return m

    def apply(self, X):
        return np.asarray(X) @ self.R().T + self.t

    def center(self) -> np.ndarray:
        return -self.R().T @ self.t


def _camera_K(camera):
    """(fx, fy, cx, cy): the four PINHOLE parameters the reference's camera
    reads (camera.cuh:24-67); any other count is refused here, before the C
    call reads four values."""
    K = np.ascontiguousarray(camera.params, np.float64).reshape(-1)
    if K.shape[0] != 4:
        raise ValueError(f"camera.params must hold (fx, fy, cx, cy), got {K.shape[0]} values")
    return K


def _f64(a, cols):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
    if a.ndim != 2 or a.shape[1] != cols:
        raise ValueError(f"expected an (N, {cols}) array, got {a.shape}")
    return a


class Context:
    """One device context: a CUDA stream plus a reusable device workspace."""

    def __init__(self, device: int = 0, workspace_bytes: int = 0):
        L = _lib.lib()
        h = C.c_void_p()
        check(L.tbr_context_create(device, workspace_bytes, C.byref(h)))
        self._h = h
        self._lock = threading.Lock()
        self._batches = weakref.WeakSet()  # destroyed before the context (they use its workspace)

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            for b in list(self._batches):
                b.close()
            _lib.lib().tbr_context_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- the reference's calls -------------------------------------------------
    def estimate_absolute_pose(self, points2D, points3D, camera: Camera_cuda,
                               ransac_opt: RansacOptions_cuda | None = None,
                               bundle_opt: BundleOptions_cuda | None = None, *, seed: int | None = None,
                               replay=None, force_samples: int = 0, skip_refine: bool = False,
                               honor_options: bool = False, hyp_per_thread: int = 0,
                               chunk_points: int = 0, max_total_samples: int = 0,
                               stop_rule_x86_quirk: bool = False, points_per_iter: int = 0):
        """Returns (RansacStats_cuda, CameraPose_cuda, inliers uint8[N])."""
        x = _f64(points2D, 2)
        X = _f64(points3D, 3)
        if x.shape[0] != X.shape[0]:
            raise ValueError("2D and 3D point counts must match")
        ro = (ransac_opt or RansacOptions_cuda()).to_c()
        bo = (bundle_opt or BundleOptions_cuda()).to_c()
        ext = _lib.ExtOptionsC()
        ext.honor_options = int(honor_options)
        ext.skip_refine = int(skip_refine)
        ext.force_samples = force_samples
        ext.max_total_samples = max_total_samples
        ext.seed = (seed or 0) & 0xFFFFFFFFFFFFFFFF
        ext.hyp_per_thread = hyp_per_thread
        ext.points_per_iter = points_per_iter
        ext.chunk_points = chunk_points
        ext.stop_rule_x86_quirk = int(stop_rule_x86_quirk)
        rep = None
        if replay is not None:
            rep = np.ascontiguousarray(np.asarray(replay, np.int32).reshape(-1, 3))
            ext.replay_idx = rep.ctypes.data
            ext.replay_count = rep.shape[0]
        K = _camera_K(camera)
        q = np.zeros(4)
        t = np.zeros(3)
        inl = np.zeros(x.shape[0], np.uint8)
        st = _lib.StatsC()
        with self._lock:
            check(_lib.lib().tbr_estimate_absolute_pose(
                self._h, x.ctypes.data, X.ctypes.data, x.shape[0], K.ctypes.data, camera.width,
                camera.height, C.byref(ro), C.byref(bo), C.byref(ext), q.ctypes.data, t.ctypes.data,
                inl.ctypes.data, C.byref(st)))
        stats = RansacStats_cuda(refinements=1 if not skip_refine else 0, iterations=st.samples,
                                 num_inliers=st.num_inliers, inlier_ratio=st.inlier_ratio,
                                 model_score=st.model_score, details=st.as_dict())
        return stats, CameraPose_cuda(q, t), inl

    def get_inliers(self, pose: CameraPose_cuda, x, X, sq_threshold: float):
        x = _f64(x, 2)
        X = _f64(X, 3)
        q = np.ascontiguousarray(pose.q, np.float64)
        t = np.ascontiguousarray(pose.t, np.float64)
        out = np.zeros(x.shape[0], np.uint8)
        cnt = C.c_int64()
        with self._lock:
            check(_lib.lib().tbr_get_inliers(self._h, q.ctypes.data, t.ctypes.data, x.ctypes.data,
                                             X.ctypes.data, x.shape[0], sq_threshold, out.ctypes.data,
                                             C.byref(cnt)))
        return out

    def bundle_adjust(self, x, X, camera: Camera_cuda, pose: CameraPose_cuda,
                      opt: BundleOptions_cuda | None = None, weights=None, honor_options=False):
        x = _f64(x, 2)
        X = _f64(X, 3)
        K = _camera_K(camera)
        q = np.array(pose.q, np.float64)
        t = np.array(pose.t, np.float64)
        bo = (opt or BundleOptions_cuda()).to_c()
        ext = _lib.ExtOptionsC()
        ext.honor_options = int(honor_options)
        w = None
        if weights is not None:
            w = np.ascontiguousarray(weights, np.float64)
        st = _lib.StatsC()
        with self._lock:
            check(_lib.lib().tbr_bundle_adjust(self._h, x.ctypes.data, X.ctypes.data, x.shape[0], K.ctypes.data,
                                               q.ctypes.data, t.ctypes.data, C.byref(bo),
                                               w.ctypes.data if w is not None else None, C.byref(ext),
                                               C.byref(st)))
        return CameraPose_cuda(q, t), st.as_dict()

    def debug_bounded_wait(self, polls: int = 1 << 16):
        """Failure-path check (tbr_debug_bounded_wait): a device wait that nothing
        completes gives up after `polls` tries; raises TbrError (TIMEOUT)."""
        with self._lock:
            check(_lib.lib().tbr_debug_bounded_wait(self._h, polls))

    def debug_score_samples(self, points2D, points3D, K, max_reproj_error, triples, counts=False, shape=None):
        """Per-hypothesis (ids, FP64 poses (H,3,4), FP32 scores in tau^2 units, counts or None).
        shape: a scoring shape (dict with hyp_per_thread, points_per_iter,
        chunk_points) for the FP32 pass; default: the built-in one."""
        ext = None
        if shape:
            ext = _lib.ExtOptionsC()
            ext.hyp_per_thread = int(shape.get("hyp_per_thread", 0))
            ext.points_per_iter = int(shape.get("points_per_iter", 0))
            ext.chunk_points = int(shape.get("chunk_points", 0))
        x = _f64(points2D, 2)
        X = _f64(points3D, 3)
        tr = np.ascontiguousarray(np.asarray(triples, np.int32).reshape(-1, 3))
        cap = 4 * tr.shape[0]
        ids = np.zeros(cap, np.int64)
        poses = np.zeros((cap, 12))
        s32 = np.zeros(cap, np.float32)
        cnt = np.zeros(cap, np.int64) if counts else None
        nh = C.c_int64()
        Kc = np.asarray(K, np.float64)
        with self._lock:
            check(_lib.lib().tbr_debug_score_samples(
                self._h, x.ctypes.data, X.ctypes.data, x.shape[0], Kc.ctypes.data, max_reproj_error,
                tr.ctypes.data, tr.shape[0], ids.ctypes.data, poses.ctypes.data, s32.ctypes.data,
                cnt.ctypes.data if counts else None, cap, C.byref(nh), C.byref(ext) if ext else None))
        m = nh.value
        return ids[:m], poses[:m].reshape(m, 3, 4), s32[:m], (cnt[:m] if counts else None)


_default_ctx = None
_default_lock = threading.Lock()


def default_context() -> Context:
    global _default_ctx
    with _default_lock:
        if _default_ctx is None:
            _default_ctx = Context()
        return _default_ctx


def estimate_absolute_pose_cuda(points2D, points3D, camera: Camera_cuda, ransac_opt: RansacOptions_cuda,
                                bundle_opt: BundleOptions_cuda, **kw):
    """entry.h:13-19: returns (RansacStats_cuda, CameraPose_cuda, inliers)."""
    return default_context().estimate_absolute_pose(points2D, points3D, camera, ransac_opt, bundle_opt, **kw)


def get_inliers_mx(pose: CameraPose_cuda, x, X, sq_threshold: float):
    """entry.h:22-25: inlier mask (uint8) with the reprojection and cheirality test."""
    return default_context().get_inliers(pose, x, X, sq_threshold)


def bundle_adjust_cuda(x, X, camera: Camera_cuda, pose: CameraPose_cuda, opt: BundleOptions_cuda,
                       weights=None):
    """ba.cuh:17-24: LM refinement; returns the refined CameraPose_cuda."""
    return default_context().bundle_adjust(x, X, camera, pose, opt, weights)[0]


_DESC_DTYPE = np.dtype(_lib.FrameDescC)
_RESULT_DTYPE = np.dtype(_lib.FrameResultC)


def _f64c(a):
    a = np.asarray(a)
    return a if (a.dtype == np.float64 and a.flags.c_contiguous) else np.ascontiguousarray(a, np.float64)


_U64 = 0xFFFFFFFFFFFFFFFF


_F64 = np.dtype(np.float64)


def _frame_descs(frames, seeds=None, max_reproj_error=0.0):
    """tbr_frame_desc entries for the frames' float64 arrays: (pointer for the C
    call, objects to keep alive until it returns). One pass over the frames
    (this runs once per batch call, so its per-frame cost counts)."""
    m = len(frames)
    keep = []
    p2, p3, ns, Ks = [0] * m, [0] * m, [0] * m, [None] * m
    from_buffer, addressof = C.c_char.from_buffer, C.addressof
    for i, fr in enumerate(frames):
        u, x = fr.uv, fr.xyz
        if type(u) is not np.ndarray or u.dtype != _F64 or not u.flags.c_contiguous:
            u = np.ascontiguousarray(u, np.float64)
        if type(x) is not np.ndarray or x.dtype != _F64 or not x.flags.c_contiguous:
            x = np.ascontiguousarray(x, np.float64)
        su, sx = u.shape, x.shape
        if len(su) != 2 or su[1] != 2 or len(sx) != 2 or sx[1] != 3 or su[0] != sx[0]:
            raise ValueError(f"frame {i}: uv must be (n, 2) and xyz (n, 3) with the same n")
        try:  # ctypes' buffer route is the cheapest address per array
            p2[i], p3[i] = addressof(from_buffer(u)), addressof(from_buffer(x))
        except (TypeError, ValueError, BufferError):  # read-only or empty arrays
            p2[i], p3[i] = u.ctypes.data, x.ctypes.data
        keep.append(u)
        keep.append(x)
        ns[i] = su[0]
        Ks[i] = fr.K
    a = np.zeros(m, _DESC_DTYPE)
    a["points2D"] = p2
    a["points3D"] = p3
    a["n"] = ns
    a["K"] = np.array(Ks, np.float64).reshape(m, 4)
    sd = [fr.seed for fr in frames] if seeds is None else list(seeds)
    try:
        a["seed"] = np.array(sd, np.uint64)
    except (OverflowError, ValueError, TypeError):
        a["seed"] = np.array([int(s) & _U64 for s in sd], np.uint64)
    a["max_reproj_error"] = (max_reproj_error if max_reproj_error
                             else [getattr(fr, "threshold_px", 0.0) for fr in frames])
    keep.append(a)
    return a.ctypes.data_as(C.POINTER(_lib.FrameDescC)), keep


_STAT_NAMES = _RESULT_DTYPE["stats"].names


RESULT_DTYPE = _RESULT_DTYPE
"""numpy dtype of one packed frame result (tbr_frame_result): fields q, t,
status and the stats record."""


def _results(res, n, as_array=False):
    a = np.frombuffer(res, dtype=_RESULT_DTYPE, count=n)
    if as_array:
        return a
    q, t, status = a["q"].copy(), a["t"].copy(), a["status"].tolist()
    keys = ("q", "t", "status") + _STAT_NAMES
    rows = a["stats"].tolist()
    return [dict(zip(keys, (q[i], t[i], status[i]) + rows[i])) for i in range(n)]


class Batch:
    """Frames uploaded once; run() replays one captured CUDA graph (device loop
    over engine steps) with the inputs resident in device memory."""

    def __init__(self, ctx: Context, frames, ransac_opt: RansacOptions_cuda | None = None,
                 hyp_per_thread: int = 0, chunk_points: int = 0, force_samples: int = 0,
                 points_per_iter: int = 0):
        self.ctx = ctx
        self.n = len(frames)
        arr, self._keep = _frame_descs(frames)
        ro = (ransac_opt or RansacOptions_cuda(max_iterations=1000, max_reproj_error=4.0)).to_c()
        ext = _lib.ExtOptionsC()
        ext.hyp_per_thread = hyp_per_thread
        ext.chunk_points = chunk_points
        ext.force_samples = force_samples
        ext.points_per_iter = points_per_iter
        h = C.c_void_p()
        with ctx._lock:
            check(_lib.lib().tbr_batch_create(ctx.handle, arr, self.n, C.byref(ro), C.byref(ext), C.byref(h)))
        self._h = h
        ctx._batches.add(self)

    def run(self):
        check(_lib.lib().tbr_batch_run(self._h))

    def sync(self):
        check(_lib.lib().tbr_batch_sync(self._h))

    def results(self):
        res = (_lib.FrameResultC * self.n)()
        check(_lib.lib().tbr_batch_results(self._h, res))
        return _results(res, self.n)

    def profile(self):
        """Per-kernel device ms of one host-stepped run (CUDA events) and pairs scored."""
        out = (_lib.KernelProfileC * 16)()
        n = C.c_int32()
        pairs = C.c_uint64()
        check(_lib.lib().tbr_batch_profile(self._h, out, 16, C.byref(n), C.byref(pairs)))
        return {out[i].name.decode(): (out[i].total_ms, out[i].launches) for i in range(n.value)}, pairs.value

    def autotune(self, repeats: int = 3):
        """Time every scoring shape (hypotheses per block x points per iteration x
        point tile) on this batch and keep the fastest; returns (best, all)."""
        ent = (_lib.TuneEntryC * 64)()
        n = C.c_int32()
        best = _lib.TuneEntryC()
        with self.ctx._lock:
            check(_lib.lib().tbr_batch_autotune(self._h, repeats, ent, 64, C.byref(n), C.byref(best)))
        return best.as_dict(), [ent[i].as_dict() for i in range(n.value)]

    def close(self):
        if self._h:
            _lib.lib().tbr_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def estimate_batch(ctx: Context, frames, ransac_opt: RansacOptions_cuda | None = None, masks: bool = False,
                   as_array: bool = False):
    """Host buffers in, results out, all frames in one call (tbr_estimate_batch).
    Returns one dict per frame, or with as_array=True the packed results as a
    numpy record array of RESULT_DTYPE (no per-frame Python objects; with masks
    the inlier masks are then returned beside it: (array, [masks]))."""
    arr, keep = _frame_descs(frames)
    ro = (ransac_opt or RansacOptions_cuda(max_iterations=1000, max_reproj_error=4.0)).to_c()
    ext = _lib.ExtOptionsC()
    res = (_lib.FrameResultC * len(frames))()
    mbufs = None
    mptrs = None
    if masks:
        mbufs = [np.zeros(f.n, np.uint8) for f in frames]
        mptrs = (C.c_void_p * len(frames))(*[m.ctypes.data for m in mbufs])
    with ctx._lock:
        check(_lib.lib().tbr_estimate_batch(ctx.handle, arr, len(frames), C.byref(ro), C.byref(ext), res,
                                            C.cast(mptrs, C.c_void_p) if masks else None))
    out = _results(res, len(frames), as_array)
    if as_array:
        return (out, mbufs) if masks else out
    if masks:
        for o, m in zip(out, mbufs):
            o["inliers"] = m
    return out


def estimate_batch_submit(ctx: Context, frames, ransac_opt: RansacOptions_cuda | None = None) -> "BatchTicket":
    """Queues the frames' whole run (tbr_estimate_batch_submit) and returns at
    once; BatchTicket.collect() waits for it and returns what estimate_batch
    returns. Submitting the next batch before collecting this one overlaps the
    host work of a call (descriptors, staging, launches, the result round trip)
    with the device work of the previous one; a context runs two submitted
    batches at a time. The frames' arrays are read while the batch runs, so
    the ticket keeps them referenced until collect."""
    arr, keep = _frame_descs(frames)
    ro = (ransac_opt or RansacOptions_cuda(max_iterations=1000, max_reproj_error=4.0)).to_c()
    ext = _lib.ExtOptionsC()
    h = C.c_void_p()
    with ctx._lock:
        check(_lib.lib().tbr_estimate_batch_submit(ctx.handle, arr, len(frames), C.byref(ro), C.byref(ext),
                                                   C.byref(h)))
    return BatchTicket(ctx, h, [keep[2 * i].shape[0] for i in range(len(frames))], keep)


class BatchTicket:
    """A submitted batch (estimate_batch_submit); collect() once."""

    def __init__(self, ctx: Context, handle, ns, keep):
        self.ctx, self._h, self._ns, self._keep = ctx, handle, ns, keep

    def collect(self, masks: bool = False, as_array: bool = False):
        """Waits for the batch and returns its results as estimate_batch does."""
        if not self._h:
            raise RuntimeError("ticket already collected")
        n = len(self._ns)
        res = (_lib.FrameResultC * n)()
        mbufs = mptrs = None
        if masks:
            mbufs = [np.zeros(k, np.uint8) for k in self._ns]
            mptrs = (C.c_void_p * n)(*[m.ctypes.data for m in mbufs])
        h, self._h = self._h, None
        try:
            with self.ctx._lock:
                check(_lib.lib().tbr_estimate_batch_collect(h, res, C.cast(mptrs, C.c_void_p) if masks else None))
        finally:
            self._keep = None
        out = _results(res, n, as_array)
        if as_array:
            return (out, mbufs) if masks else out
        if masks:
            for o, m in zip(out, mbufs):
                o["inliers"] = m
        return out

    def __del__(self):
        try:  # an uncollected ticket: release its frames' workspace
            if self._h:
                h, self._h = self._h, None
                _lib.lib().tbr_estimate_batch_collect(h, None, None)
        except Exception:
            pass


def _device_descs(frames):
    """tbr_frame_desc entries of frames with contiguous float64 CUDA tensors
    `uv` (n, 2) and `xyz` (n, 3): (record array, frame count)."""
    import torch
    f64 = torch.float64
    m = len(frames)
    uvs = [fr.uv for fr in frames]
    xyzs = [fr.xyz for fr in frames]
    for i, (u, x) in enumerate(zip(uvs, xyzs)):
        if not (getattr(u, "is_cuda", False) and getattr(x, "is_cuda", False) and u.dtype == f64 and x.dtype == f64
                and u.dim() == 2 and x.dim() == 2
                and u.is_contiguous() and x.is_contiguous()):
            raise ValueError(f"frame {i}: uv and xyz must be contiguous float64 CUDA tensors (n, 2), (n, 3)")
        su, sx = u.shape, x.shape
        if su[1] != 2 or sx[1] != 3:
            raise ValueError(f"frame {i}: uv must be (n, 2) and xyz (n, 3)")
        if su[0] != sx[0]:
            raise ValueError(f"frame {i}: 2D and 3D point counts differ")
    a = np.zeros(m, _DESC_DTYPE)
    a["points2D"] = [u.data_ptr() for u in uvs]
    a["points3D"] = [x.data_ptr() for x in xyzs]
    a["n"] = [u.shape[0] for u in uvs]
    a["K"] = np.array([fr.K for fr in frames], np.float64).reshape(m, 4)
    sd = [fr.seed for fr in frames]
    try:
        a["seed"] = np.array(sd, np.uint64)
    except (OverflowError, ValueError, TypeError):
        a["seed"] = np.array([int(s) & _U64 for s in sd], np.uint64)
    return a, m


def estimate_batch_device_submit(ctx: Context, frames, ransac_opt: RansacOptions_cuda | None = None,
                                 stream=None) -> "BatchTicket":
    """The submitted form of estimate_batch_device (tbr_estimate_batch_device_submit):
    queues the run and returns a BatchTicket at once. The frames' tensors must
    stay unchanged until collect; the ticket keeps them referenced."""
    import torch
    a, m = _device_descs(frames)
    ro = (ransac_opt or RansacOptions_cuda(max_iterations=1000, max_reproj_error=4.0)).to_c()
    ext = _lib.ExtOptionsC()
    st = stream if stream is not None else torch.cuda.current_stream()
    h = C.c_void_p()
    with ctx._lock:
        check(_lib.lib().tbr_estimate_batch_device_submit(ctx.handle, a.ctypes.data_as(C.POINTER(_lib.FrameDescC)),
                                                          m, C.byref(ro), C.byref(ext), C.c_void_p(st.cuda_stream),
                                                          C.byref(h)))
    return BatchTicket(ctx, h, [int(fr.uv.shape[0]) for fr in frames], [(fr.uv, fr.xyz) for fr in frames])


def estimate_batch_device(ctx: Context, frames, ransac_opt: RansacOptions_cuda | None = None, stream=None,
                          as_array: bool = False):
    """Frames whose correspondences are already on the context's GPU
    (tbr_estimate_batch_device). Each frame has `uv` (n, 2) and `xyz` (n, 3)
    float64 contiguous CUDA tensors (or objects with data_ptr()), `K` and
    `seed`. `stream`: a torch.cuda.Stream (default: torch's current stream) whose
    queued work the copy waits for. Results come back to the host, as dicts or
    (as_array=True) as one record array of RESULT_DTYPE."""
    import torch
    a, m = _device_descs(frames)
    ro = (ransac_opt or RansacOptions_cuda(max_iterations=1000, max_reproj_error=4.0)).to_c()
    ext = _lib.ExtOptionsC()
    res = (_lib.FrameResultC * m)()
    st = stream if stream is not None else torch.cuda.current_stream()
    with ctx._lock:
        check(_lib.lib().tbr_estimate_batch_device(ctx.handle, a.ctypes.data_as(C.POINTER(_lib.FrameDescC)), m,
                                                   C.byref(ro), C.byref(ext), C.c_void_p(st.cuda_stream), res,
                                                   None))
    return _results(res, m, as_array)


class DeviceFrame:
    """A frame's correspondences as CUDA tensors (for estimate_batch_device)."""

    def __init__(self, frame, device="cuda"):
        import torch
        self.uv = torch.as_tensor(np.ascontiguousarray(frame.uv, np.float64), device=device)
        self.xyz = torch.as_tensor(np.ascontiguousarray(frame.xyz, np.float64), device=device)
        self.K = tuple(float(k) for k in frame.K)
        self.seed = frame.seed
        self.n = int(self.uv.shape[0])


class Server:
    """Continuous-batching request loop (tbr_server_*): submit frames any time;
    a worker advances every resident frame one engine step at a time and admits
    new requests into free slots within the workspace budget.

    With copy=False (default) a submitted frame's arrays are read when the
    request is admitted (tbr_server_submit_nocopy): this object keeps them alive
    until poll() returns the request, and they must not be modified meanwhile.
    copy=True copies them at submit (tbr_server_submit)."""

    def __init__(self, ctx: Context, budget_bytes: int = 8 << 30, max_slots: int = 512, max_queue: int = 1 << 16,
                 ransac_opt: RansacOptions_cuda | None = None, copy: bool = False, scoring_shape: dict | None = None,
                 honor_options: bool = False):
        """scoring_shape: a Batch.autotune() result (hyp_per_thread, points_per_iter,
        chunk_points) for the server's scoring pass; default: the built-in shape.
        honor_options: apply the RANSAC options the reference ignores (see
        tbr_ext_options.honor_options)."""
        cfg = _lib.ServerConfigC()
        cfg.workspace_budget_bytes = budget_bytes
        cfg.max_slots = max_slots
        cfg.max_queue = max_queue
        cfg.ransac = (ransac_opt or RansacOptions_cuda(max_iterations=1000, max_reproj_error=4.0)).to_c()
        cfg.ext.honor_options = int(honor_options)
        if scoring_shape:
            cfg.ext.hyp_per_thread = int(scoring_shape.get("hyp_per_thread", 0))
            cfg.ext.points_per_iter = int(scoring_shape.get("points_per_iter", 0))
            cfg.ext.chunk_points = int(scoring_shape.get("chunk_points", 0))
        h = C.c_void_p()
        check(_lib.lib().tbr_server_create(ctx.handle, C.byref(cfg), C.byref(h)))
        self._h = h
        self._buf = (_lib.ServerResultC * 1024)()
        self._copy = copy
        self._keep = {}

    def submit(self, frame, seed: int | None = None, max_reproj_error: float = 0.0) -> int:
        arr, keep = _frame_descs([frame], None if seed is None else [seed], max_reproj_error)
        rid = C.c_uint64()
        if self._copy:
            check(_lib.lib().tbr_server_submit(self._h, arr, C.byref(rid)))
        else:
            check(_lib.lib().tbr_server_submit_nocopy(self._h, arr, C.byref(rid)))
            self._keep[rid.value] = keep
        return rid.value

    def stats(self) -> dict:
        st = _lib.ServerStatsC()
        check(_lib.lib().tbr_server_get_stats(self._h, C.byref(st)))
        return st.as_dict()

    def poll(self, max_results: int = 1024):
        n = C.c_int32()
        st = _lib.lib().tbr_server_poll(self._h, self._buf, min(max_results, 1024), C.byref(n))
        if st not in (0, 6):
            check(st)
        out = []
        for i in range(n.value):
            r = self._buf[i]
            self._keep.pop(r.request_id, None)
            out.append({"id": r.request_id, "status": r.status, "q": np.array(r.q[:]), "t": np.array(r.t[:]),
                        "latency_ms": r.submit_to_done_ms, **r.stats.as_dict()})
        return out

    def cancel(self, request_id: int):
        check(_lib.lib().tbr_server_cancel(self._h, request_id))

    def drain(self):
        check(_lib.lib().tbr_server_drain(self._h))

    def close(self):
        if self._h:
            _lib.lib().tbr_server_destroy(self._h)
            self._h = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
