"""Runs the reference's own CUDA build (oracle/_ref/tbr_refcuda, made by
`make -C oracle refcuda`) on a list of frames -- BASELINE INFRASTRUCTURE.

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
    return os.access(BIN, os.X_OK) and os.path.exists(CURAND_LIB)


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
