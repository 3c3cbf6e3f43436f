"""Runs the reference's own CUDA build (oracle/_ref/tbr_refcuda, made by
`make -C oracle refcuda`) on a list of frames -- measurement infrastructure for
the comparison arm, not part of the product.

Each frame is one call of the reference's estimate_absolute_pose_cuda
(entry.cu:28-144), timed around the whole call on the host clock as
TbrMain/src/main.cu:185-190 does. The reference prints inside every call; its
stdout goes to /dev/null here.
"""
from __future__ import annotations

import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BIN = os.path.join(HERE, "_ref", "tbr_refcuda")
CURAND_LIB = os.path.join(HERE, "_ref", "libtbr_refcurand.so")


def available() -> bool:
    return os.access(BIN, os.X_OK) and os.path.exists(CURAND_LIB) and os.path.exists(KERNEL_LIB)


def curand_triples(n: int, samples_per_round: int, rounds: int) -> np.ndarray:
    """The reference's minimal samples (cuRAND XORWOW, its seeds and redraw rule)
    for `rounds` rounds of `samples_per_round`, in sample order: (rounds*B, 3) int32."""
    import ctypes as C
    lib = C.CDLL(CURAND_LIB)
    lib.ref_curand_triples.argtypes = [C.c_int64, C.c_int64, C.c_int32, C.c_void_p]
    lib.ref_curand_triples.restype = C.c_int
    out = np.zeros((rounds * samples_per_round, 3), np.int32)
    rc = lib.ref_curand_triples(n, samples_per_round, rounds, out.ctypes.data)
    if rc:
        raise RuntimeError(f"ref_curand_triples failed ({rc})")
    return out


KERNEL_LIB = os.path.join(HERE, "_ref", "libtbr_refkernel.so")


def scoring_kernel(frame, samples: int = 4096, reps: int = 5, threshold_px: float = 4.0) -> dict:
    """The reference's RANSAC kernel on one round of `samples` blocks over the
    frame (its first-round cuRAND samples), timed on the device; pairs =
    P3P solutions x points, counted with the reference's own P3P restated by
    the oracle on the exported samples."""
    import ctypes as C

    from .oracle import Oracle
    K = np.asarray(frame.K, np.float64)
    f = 0.5 * (K[0] + K[1])
    xn = np.ascontiguousarray(np.stack([(frame.uv[:, 0] - K[2]) / K[0], (frame.uv[:, 1] - K[3]) / K[1]], 1))
    X = np.ascontiguousarray(frame.xyz, np.float64)
    lib = C.CDLL(KERNEL_LIB)
    lib.ref_scoring_kernel.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_int,
                                       C.POINTER(C.c_float), C.POINTER(C.c_double)]
    lib.ref_scoring_kernel.restype = C.c_int
    ms, best = C.c_float(), C.c_double()
    sq = (threshold_px / f) ** 2
    rc = lib.ref_scoring_kernel(xn.ctypes.data, X.ctypes.data, frame.n, samples, sq, reps, C.byref(ms),
                                C.byref(best))
    if rc:
        raise RuntimeError(f"ref_scoring_kernel failed ({rc})")
    o = Oracle()
    tri = curand_triples(frame.n, samples, 1)
    hyps = 0
    for a, b, c in tri:
        x = np.stack([o.bearing(*xn[i]) for i in (a, b, c)])
        hyps += o.p3p(x, X[[a, b, c]]).shape[0]
    pairs = hyps * frame.n
    return {"samples": samples, "hypotheses": hyps, "pairs": pairs, "kernel_ms": ms.value,
            "pairs_per_s": pairs / (ms.value / 1000.0), "best_score": best.value}


def _write_frames(path: str, frames) -> None:
    with open(path, "wb") as fh:
        fh.write(np.int64(len(frames)).tobytes())
        for f in frames:
            if f.n < 3:
                raise ValueError("the reference's sampler needs n >= 3")
            fh.write(np.int64(f.n).tobytes())
            fh.write(np.asarray(f.K, np.float64).tobytes())
            fh.write(np.array([640, 480], np.int32).tobytes())
            fh.write(np.ascontiguousarray(f.uv, np.float64).tobytes())
            fh.write(np.ascontiguousarray(f.xyz, np.float64).tobytes())


def run(frames, warmup: int = 3, max_iterations: int = 1000, reproj_px: float = 4.0,
        timeout: float = 600.0) -> dict:
    """Returns q (F,4), t (F,3), ms (F,) per call, inliers (F,)."""
    if not available():
        raise FileNotFoundError(BIN)
    with tempfile.TemporaryDirectory() as d:
        fin = os.path.join(d, "frames.bin")
        fout = os.path.join(d, "out.bin")
        _write_frames(fin, frames)
        subprocess.run([BIN, fin, fout, str(warmup), str(max_iterations), str(reproj_px)],
                       stdout=subprocess.DEVNULL, stderr=subprocess.PIPE, check=True, timeout=timeout)
        raw = np.fromfile(fout, dtype=np.uint8)
    rec = np.dtype([("q", "<f8", 4), ("t", "<f8", 3), ("ms", "<f8"), ("inl", "<i8")])
    out = raw.view(rec)
    if out.shape[0] != len(frames):
        raise RuntimeError("tbr_refcuda wrote %d results for %d frames" % (out.shape[0], len(frames)))
    return {"q": out["q"].copy(), "t": out["t"].copy(), "ms": out["ms"].copy(), "inliers": out["inl"].copy()}
