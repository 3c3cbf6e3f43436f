"""ctypes bindings for the FP64 CPU oracle and the reference-source harness.

TEST INFRASTRUCTURE: imported only by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, always as the checker. The product package
(turboransac_b200) never imports this module.

* ``Oracle``     -- oracle/_build/liboracle.so, the FP64 restatement
                    (oracle/tbr_oracle.cpp).
* ``RefHarness`` -- oracle/_ref/libtbr_refhost.so, the reference's own header
                    code and entry.cu compiled on the host (present only where
                    the reference tree was available at build time).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libtbr_refhost.so")
# The reference tree (the TurboRANSAC checkout): TBR_REF_TREE, by default where
# this build environment mounts it.
REF_TREE = os.environ.get("TBR_REF_TREE", "/root/reference")
REF_SRC = os.path.join(REF_TREE, "Module", "TbrCudaPnP")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip32 = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_ip64 = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")


def build(ref: bool | None = None) -> None:
    """Compile the oracle (and, when the reference tree exists, oracle/_ref)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    if ref is None:
        ref = os.path.isdir(REF_SRC)
    if ref:
        subprocess.run(["make", "-s", "-C", HERE, "ref", "refcuda"], check=True)


class RansacCfg(C.Structure):
    _fields_ = [("samples_per_round", C.c_int64), ("max_total_samples", C.c_int64),
                ("success_prob", C.c_double), ("trials_mult", C.c_double),
                ("force_samples", C.c_int64), ("seed", C.c_uint64),
                ("replay", C.c_void_p), ("replay_count", C.c_int64), ("threads", C.c_int),
                ("quirk", C.c_int), ("min_samples", C.c_int64), ("prosac", C.c_int32),
                ("prosac_TN", C.c_double)]


class RansacOut(C.Structure):
    _fields_ = [("P", C.c_double * 12), ("score", C.c_double), ("count", C.c_int64),
                ("best_sample", C.c_int64), ("best_sol", C.c_int32), ("found", C.c_int32),
                ("samples", C.c_int64), ("rounds", C.c_int64), ("hypotheses", C.c_int64)]


class LMOpts(C.Structure):
    _fields_ = [("max_iterations", C.c_int64), ("loss_scale", C.c_double),
                ("gradient_tol", C.c_double), ("step_tol", C.c_double),
                ("initial_lambda", C.c_double), ("min_lambda", C.c_double),
                ("max_lambda", C.c_double), ("loss", C.c_int32), ("weights", C.c_void_p)]


class LMStats(C.Structure):
    _fields_ = [("iterations", C.c_int64), ("invalid_steps", C.c_int64),
                ("initial_cost", C.c_double), ("cost", C.c_double), ("lambda_", C.c_double),
                ("step_norm", C.c_double), ("grad_norm", C.c_double)]


class EstimateInfo(C.Structure):
    _fields_ = [("ransac", RansacOut), ("lm", LMStats), ("num_inliers", C.c_int64)]


def _cfg(samples_per_round=1000, seed=0, force_samples=0, replay=None, threads=1,
         max_total_samples=100000, success_prob=0.9999, trials_mult=3.0, quirk=False, min_samples=0,
         prosac=False, prosac_TN=100000.0):
    cfg = RansacCfg()
    cfg.quirk = int(quirk)
    cfg.min_samples = min_samples
    cfg.prosac = int(prosac)
    cfg.prosac_TN = float(prosac_TN)
    cfg.samples_per_round = samples_per_round
    cfg.max_total_samples = max_total_samples
    cfg.success_prob = success_prob
    cfg.trials_mult = trials_mult
    cfg.force_samples = force_samples
    cfg.seed = seed & 0xFFFFFFFFFFFFFFFF
    cfg.threads = threads
    if replay is not None:
        cfg.replay = replay.ctypes.data
        cfg.replay_count = replay.shape[0]
    return cfg


class Oracle:
    def __init__(self, path: str = LIB):
        if not os.path.exists(path):
            build(ref=False)
        L = self.lib = C.CDLL(path)
        L.orc_sample_triples.argtypes = [C.c_uint64, C.c_int64, C.c_int64, C.c_int64, _ip32]
        L.orc_philox4x32_10.argtypes = [C.POINTER(C.c_uint32)] * 3
        L.orc_p3p.argtypes = [_dp, _dp, _dp]
        L.orc_p3p.restype = C.c_int
        L.orc_bearing.argtypes = [C.c_double, C.c_double, _dp]
        L.orc_msac.argtypes = [_dp, _dp, C.c_int64, _dp, C.c_double, C.POINTER(C.c_double),
                               C.POINTER(C.c_int64)]
        L.orc_rotmat_to_quat.argtypes = [_dp, _dp]
        L.orc_quat_to_rotmat.argtypes = [_dp, _dp]
        L.orc_get_inliers.argtypes = [_dp, _dp, _dp, _dp, C.c_int64, C.c_double, C.c_void_p]
        L.orc_get_inliers.restype = C.c_int64
        L.orc_ransac.argtypes = [_dp, _dp, C.c_int64, C.c_double, C.POINTER(RansacCfg),
                                 C.POINTER(RansacOut), C.c_void_p, C.c_void_p, C.c_void_p,
                                 C.c_void_p, C.c_int64]
        L.orc_ransac.restype = C.c_int
        L.orc_lm.argtypes = [_dp, _dp, C.c_int64, _dp, _dp, _dp, C.POINTER(LMOpts),
                             C.POINTER(LMStats)]
        L.orc_estimate.argtypes = [_dp, _dp, C.c_int64, _dp, C.c_double, C.POINTER(RansacCfg),
                                   C.c_int, _dp, _dp, C.c_void_p, C.POINTER(EstimateInfo)]
        L.orc_estimate.restype = C.c_int
        L.orc_estimate_batch.argtypes = [_dp, _dp, _ip64, _dp, _u64p, C.c_int, C.c_double,
                                         C.c_int64, C.c_int, _dp, _dp, _ip64]
        L.orc_estimate_batch.restype = C.c_int
        L.orc_prosac_table.argtypes = [C.c_int64, C.c_double, _ip64]
        L.orc_prosac_triple.argtypes = [C.c_uint64, C.c_int64, C.c_int64, _ip64, _ip32]

    # -- pieces -------------------------------------------------------------
    def philox(self, ctr, key):
        c = (C.c_uint32 * 4)(*ctr)
        k = (C.c_uint32 * 2)(*key)
        o = (C.c_uint32 * 4)()
        self.lib.orc_philox4x32_10(c, k, o)
        return list(o)

    def sample_triples(self, seed: int, first: int, count: int, n: int) -> np.ndarray:
        out = np.empty((count, 3), dtype=np.int32)
        self.lib.orc_sample_triples(seed & 0xFFFFFFFFFFFFFFFF, first, count, n, out)
        return out

    def prosac_table(self, n: int, TN: float = 100000.0) -> np.ndarray:
        out = np.zeros(n - 2, np.int64)
        self.lib.orc_prosac_table(n, TN, out)
        return out

    def prosac_triples(self, seed: int, first: int, count: int, n: int, TN: float = 100000.0) -> np.ndarray:
        tp = self.prosac_table(n, TN)
        out = np.zeros((count, 3), np.int32)
        for s in range(count):
            self.lib.orc_prosac_triple(seed & 0xFFFFFFFFFFFFFFFF, first + s, n, tp, out[s])
        return out

    def p3p(self, x: np.ndarray, X: np.ndarray) -> np.ndarray:
        out = np.zeros((4, 12))
        n = self.lib.orc_p3p(np.ascontiguousarray(x, np.float64), np.ascontiguousarray(X, np.float64), out)
        return out[:n]

    def bearing(self, x: float, y: float) -> np.ndarray:
        out = np.zeros(3)
        self.lib.orc_bearing(x, y, out)
        return out

    def msac(self, xn, X, P, sq_thr):
        s = C.c_double()
        c = C.c_int64()
        xn = np.ascontiguousarray(xn, np.float64)
        X = np.ascontiguousarray(X, np.float64)
        self.lib.orc_msac(xn, X, xn.shape[0], np.ascontiguousarray(P, np.float64).reshape(12), sq_thr,
                          C.byref(s), C.byref(c))
        return s.value, c.value

    def rotmat_to_quat(self, R):
        q = np.zeros(4)
        self.lib.orc_rotmat_to_quat(np.ascontiguousarray(R, np.float64).reshape(9), q)
        return q

    def quat_to_rotmat(self, q):
        R = np.zeros(9)
        self.lib.orc_quat_to_rotmat(np.ascontiguousarray(q, np.float64), R)
        return R.reshape(3, 3)

    def get_inliers(self, q, t, xn, X, sq_thr):
        m = np.zeros(xn.shape[0], np.uint8)
        self.lib.orc_get_inliers(np.ascontiguousarray(q, np.float64), np.ascontiguousarray(t, np.float64),
                                 np.ascontiguousarray(xn, np.float64), np.ascontiguousarray(X, np.float64),
                                 xn.shape[0], sq_thr, m.ctypes.data)
        return m

    def ransac(self, xn, X, sq_thr, dump: int = 0, **kw):
        cfg = _cfg(**kw)
        out = RansacOut()
        hs = hc = hi = hp = None
        if dump:
            hs = np.zeros(dump)
            hc = np.zeros(dump, np.int64)
            hi = np.zeros(dump, np.int64)
            hp = np.zeros((dump, 12))
        xn = np.ascontiguousarray(xn, np.float64)
        X = np.ascontiguousarray(X, np.float64)
        rc = self.lib.orc_ransac(xn, X, xn.shape[0], sq_thr, C.byref(cfg), C.byref(out),
                                 hs.ctypes.data if dump else None, hc.ctypes.data if dump else None,
                                 hi.ctypes.data if dump else None, hp.ctypes.data if dump else None, dump)
        if rc:
            raise RuntimeError(f"orc_ransac failed: {rc}")
        res = {"P": np.array(out.P).reshape(3, 4), "score": out.score, "count": out.count,
               "best_sample": out.best_sample, "best_sol": out.best_sol, "found": out.found,
               "samples": out.samples, "rounds": out.rounds, "hypotheses": out.hypotheses}
        if dump:
            m = min(dump, out.hypotheses)
            res.update(hyp_scores=hs[:m], hyp_counts=hc[:m], hyp_ids=hi[:m], hyp_poses=hp[:m])
        return res

    def lm(self, x, X, cam, q, t, max_iterations=100, loss_scale=1.0, gradient_tol=1e-10,
           step_tol=1e-8, initial_lambda=1e-3, min_lambda=1e-10, max_lambda=1e10, loss=0, weights=None):
        """loss: 0 Cauchy (the reference), 1 truncated, 2 Huber, 3 trivial."""
        q = np.array(q, np.float64)
        t = np.array(t, np.float64)
        w = None if weights is None else np.ascontiguousarray(weights, np.float64)
        o = LMOpts(max_iterations, loss_scale, gradient_tol, step_tol, initial_lambda, min_lambda,
                   max_lambda, loss, w.ctypes.data if w is not None else None)
        st = LMStats()
        self.lib.orc_lm(np.ascontiguousarray(x), np.ascontiguousarray(X), x.shape[0],
                        np.asarray(cam, np.float64), q, t, C.byref(o), C.byref(st))
        return q, t, st

    def estimate(self, uv, xyz, K, max_reproj_error=4.0, skip_refine=False, **kw):
        """estimate_absolute_pose_cuda restated: returns dict(q, t, inliers, info)."""
        cfg = _cfg(**kw)
        q = np.zeros(4)
        t = np.zeros(3)
        inl = np.zeros(uv.shape[0], np.uint8)
        info = EstimateInfo()
        rc = self.lib.orc_estimate(np.ascontiguousarray(uv), np.ascontiguousarray(xyz), uv.shape[0],
                                   np.asarray(K, np.float64), max_reproj_error, C.byref(cfg),
                                   int(skip_refine), q, t, inl.ctypes.data, C.byref(info))
        if rc:
            raise RuntimeError(f"orc_estimate failed: {rc}")
        return {"q": q, "t": t, "inliers": inl, "info": info}

    def estimate_batch(self, frames, samples_per_round=1000, threads=None, max_reproj_error=4.0):
        threads = threads or os.cpu_count() or 1
        offs = np.zeros(len(frames) + 1, np.int64)
        offs[1:] = np.cumsum([f.n for f in frames])
        uv = np.ascontiguousarray(np.concatenate([f.uv for f in frames]))
        X = np.ascontiguousarray(np.concatenate([f.xyz for f in frames]))
        K = np.ascontiguousarray(np.concatenate([f.K for f in frames]))
        seeds = np.array([f.seed for f in frames], np.uint64)
        q = np.zeros(4 * len(frames))
        t = np.zeros(3 * len(frames))
        smp = np.zeros(len(frames), np.int64)
        rc = self.lib.orc_estimate_batch(uv, X, offs, K, seeds, len(frames), max_reproj_error,
                                         samples_per_round, threads, q, t, smp)
        if rc:
            raise RuntimeError(f"orc_estimate_batch failed: {rc}")
        return q.reshape(-1, 4), t.reshape(-1, 3), smp


class RefHarness:
    """The reference's own header code / entry.cu, host-compiled (oracle/_ref)."""

    def __init__(self, path: str = REF_LIB):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        L = self.lib = C.CDLL(path)
        L.ref_p3p.argtypes = [_dp, _dp, _dp]
        L.ref_p3p.restype = C.c_int
        L.ref_bearing.argtypes = [C.c_double, C.c_double, _dp]
        L.ref_msac.argtypes = [_dp, _dp, C.c_int64, _dp, C.c_double, C.POINTER(C.c_double),
                               C.POINTER(C.c_int64)]
        L.ref_rotmat_to_quat.argtypes = [_dp, _dp]
        L.ref_quat_to_rotmat.argtypes = [_dp, _dp]
        L.ref_quat_step_post.argtypes = [_dp, _dp, _dp]
        L.ref_solve_cholesky6.argtypes = [_dp, _dp, _dp]
        L.ref_cauchy_loss.argtypes = [C.c_double, C.c_double]
        L.ref_cauchy_loss.restype = C.c_double
        L.ref_cauchy_weight.argtypes = [C.c_double, C.c_double]
        L.ref_cauchy_weight.restype = C.c_double
        L.ref_lm.argtypes = [_dp, _dp, C.c_int64, _dp, _dp, _dp, C.c_int64, C.c_double]
        L.ref_estimate_from_pose.argtypes = [_dp, _dp, C.c_int64, _dp, C.c_double, _dp, _dp, _dp, _u8p]

    def p3p(self, x, X):
        out = np.zeros((4, 12))
        n = self.lib.ref_p3p(np.ascontiguousarray(x, np.float64), np.ascontiguousarray(X, np.float64), out)
        return out[:n]

    def bearing(self, x, y):
        out = np.zeros(3)
        self.lib.ref_bearing(x, y, out)
        return out

    def msac(self, xn, X, P, sq_thr):
        s = C.c_double()
        c = C.c_int64()
        self.lib.ref_msac(xn, X, xn.shape[0], np.ascontiguousarray(P, np.float64).reshape(12), sq_thr,
                          C.byref(s), C.byref(c))
        return s.value, c.value

    def rotmat_to_quat(self, R):
        q = np.zeros(4)
        self.lib.ref_rotmat_to_quat(np.ascontiguousarray(R, np.float64).reshape(9), q)
        return q

    def quat_to_rotmat(self, q):
        R = np.zeros(9)
        self.lib.ref_quat_to_rotmat(np.ascontiguousarray(q, np.float64), R)
        return R.reshape(3, 3)

    def quat_step_post(self, q, w):
        o = np.zeros(4)
        self.lib.ref_quat_step_post(np.asarray(q, np.float64), np.asarray(w, np.float64), o)
        return o

    def solve_cholesky6(self, A, b):
        x = np.zeros(6)
        self.lib.ref_solve_cholesky6(np.ascontiguousarray(A, np.float64).reshape(36),
                                     np.asarray(b, np.float64), x)
        return x

    def lm(self, x, X, cam, q, t, max_iterations=100, loss_scale=1.0):
        q = np.array(q, np.float64)
        t = np.array(t, np.float64)
        self.lib.ref_lm(np.ascontiguousarray(x), np.ascontiguousarray(X), x.shape[0],
                        np.asarray(cam, np.float64), q, t, max_iterations, loss_scale)
        return q, t

    def estimate_from_pose(self, uv, xyz, K, P, max_reproj_error=4.0):
        q = np.zeros(4)
        t = np.zeros(3)
        inl = np.zeros(uv.shape[0], np.uint8)
        self.lib.ref_estimate_from_pose(np.ascontiguousarray(uv), np.ascontiguousarray(xyz), uv.shape[0],
                                        np.asarray(K, np.float64), max_reproj_error,
                                        np.ascontiguousarray(P, np.float64).reshape(12), q, t, inl)
        return q, t, inl
