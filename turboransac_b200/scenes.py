"""Seeded synthetic 2D-3D correspondence scenes for the absolute-pose workloads.

The reference is evaluated on 7-Scenes/STDLoc correspondences (TbrMain/src/
main.cu:21-97) that are not shipped with it; these generators stand in for
them with the shapes, sizes and value distributions of the five workloads:

* ``plain``     -- N=2000, 40 % inliers, sigma=1 px, 4 px threshold, B=1000
* ``scoring``   -- N=20000, 15 % inliers, sigma=1 px, exactly 4096 samples
* ``batched``   -- 256 frames, N log-uniform [500, 30000], w ~ U[0.10, 0.80],
                   sigma ~ U[0.5, 2]
* ``precision`` -- 4096 frames, N=5000, 30 % inliers, sigma in {0.25, 1, 3},
                   half with fx=fy=2000, 20 % near-degenerate (thin depth band
                   [3.9, 4.0] m or points within 1 cm of a plane)
* ``serving``   -- Poisson arrivals, N log-uniform [300, 50000],
                   w ~ U[0.05, 0.70], sigma=1 px

Camera: pinhole 640x480, fx=fy=525, cx=319.5, cy=239.5. Pose: rotation uniform
on SO(3), camera centre uniform in [-2, 2]^3 m, X_cam = R X + t with t = -R C.
Points: pixels uniform over the image, depth uniform in [0.5, 4] m,
back-projected to the world. Inliers get N(0, sigma^2) pixel noise; outliers
keep their pixel but get a 3-D point redrawn uniformly in the AABB of the
frame's clean points. Everything is generated in float64 and rounded to
float32 (the estimator consumes float64 casts of the float32 values).
"""
from __future__ import annotations

import dataclasses
import hashlib
import math

import numpy as np

WIDTH, HEIGHT = 640, 480
FX = FY = 525.0
CX, CY = 319.5, 239.5

CONFIG_IDS = {"plain": 0, "scoring": 1, "batched": 2, "precision": 3, "serving": 4}


@dataclasses.dataclass
class Frame:
    """One synthetic frame. Arrays are float64 holding float32-representable values."""

    uv: np.ndarray          # (N, 2) pixels
    xyz: np.ndarray         # (N, 3) world points, metres
    K: np.ndarray           # (4,) fx, fy, cx, cy
    R_gt: np.ndarray        # (3, 3) world-to-camera rotation
    t_gt: np.ndarray        # (3,)
    inlier_gt: np.ndarray   # (N,) bool
    seed: int               # per-frame sampler seed
    sigma: float
    threshold_px: float = 4.0
    degenerate: str = ""

    @property
    def n(self) -> int:
        return int(self.uv.shape[0])


def frame_seed(config: str | int, frame_id: int) -> int:
    """seed_frame = hash(config_id, frame_id): 64-bit, stable across platforms."""
    cid = CONFIG_IDS.get(config, config) if isinstance(config, str) else int(config)
    h = hashlib.blake2b(f"tbr:{cid}:{frame_id}".encode(), digest_size=8).digest()
    return int.from_bytes(h, "little")


def random_rotation(rng: np.random.Generator) -> np.ndarray:
    """Uniform rotation: a uniformly random unit quaternion (w, x, y, z)."""
    q = rng.standard_normal(4)
    q /= np.linalg.norm(q)
    return quat_to_rotmat(q)


def quat_to_rotmat(q: np.ndarray) -> np.ndarray:
    w, x, y, z = q
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)],
    ])


def make_frame(n: int, inlier_ratio: float, sigma: float, seed: int, *,
               K: tuple[float, float, float, float] = (FX, FY, CX, CY),
               depth_range: tuple[float, float] = (0.5, 4.0),
               plane: bool = False, threshold_px: float = 4.0) -> Frame:
    """Generate one frame from an integer seed (the same seed keys the sampler)."""
    rng = np.random.default_rng(seed)
    fx, fy, cx, cy = K
    R = random_rotation(rng)
    C = rng.uniform(-2.0, 2.0, 3)
    t = -R @ C
    u = rng.uniform(0.0, WIDTH, n)
    v = rng.uniform(0.0, HEIGHT, n)
    rays = np.stack([(u - cx) / fx, (v - cy) / fy, np.ones(n)], axis=1)
    degenerate = ""
    if plane:
        # Points within 1 cm of a random plane n.X = d0 in front of the camera
        # (tilt <= 45 deg). Each point stays on its pixel ray; pixels whose ray
        # meets the plane outside the depth range are redrawn.
        tilt = rng.uniform(0.0, math.pi / 4)
        az = rng.uniform(0.0, 2 * math.pi)
        normal = np.array([math.sin(tilt) * math.cos(az), math.sin(tilt) * math.sin(az), math.cos(tilt)])
        d0 = rng.uniform(1.5, 3.0)
        depth = np.empty(n)
        todo = np.arange(n)
        for _ in range(64):
            e = rng.uniform(-0.01, 0.01, todo.size)
            dd = (d0 + e) / (rays[todo] @ normal)
            ok = (dd >= depth_range[0]) & (dd <= depth_range[1])
            depth[todo[ok]] = dd[ok]
            todo = todo[~ok]
            if todo.size == 0:
                break
            u[todo] = rng.uniform(0.0, WIDTH, todo.size)
            v[todo] = rng.uniform(0.0, HEIGHT, todo.size)
            rays[todo] = np.stack([(u[todo] - cx) / fx, (v[todo] - cy) / fy, np.ones(todo.size)], axis=1)
        if todo.size:
            depth[todo] = d0 / (rays[todo] @ normal)
        degenerate = "plane"
    else:
        depth = rng.uniform(depth_range[0], depth_range[1], n)
        if depth_range != (0.5, 4.0):
            degenerate = "thin_depth"
    Xc = rays * depth[:, None]
    Xw = (Xc - t) @ R  # R^T (Xc - t)
    n_in = int(math.floor(inlier_ratio * n + 0.5))
    perm = rng.permutation(n)
    inl = np.zeros(n, dtype=bool)
    inl[perm[:n_in]] = True
    uv = np.stack([u, v], axis=1)
    uv[inl] += rng.normal(0.0, sigma, (n_in, 2))
    lo, hi = Xw.min(axis=0), Xw.max(axis=0)
    n_out = n - n_in
    Xw = Xw.copy()
    Xw[~inl] = rng.uniform(lo, hi, (n_out, 3))
    uv32 = uv.astype(np.float32).astype(np.float64)
    xyz32 = Xw.astype(np.float32).astype(np.float64)
    return Frame(uv=np.ascontiguousarray(uv32), xyz=np.ascontiguousarray(xyz32),
                 K=np.array(K, dtype=np.float64), R_gt=R, t_gt=t, inlier_gt=inl,
                 seed=seed, sigma=sigma, threshold_px=threshold_px, degenerate=degenerate)


def plain_frame(frame_id: int = 0) -> Frame:
    """N=2000, 40 % inliers, sigma 1 px."""
    return make_frame(2000, 0.40, 1.0, frame_seed("plain", frame_id))


def scoring_frame(frame_id: int = 0) -> Frame:
    """N=20000, 15 % inliers, sigma 1 px (scored with exactly 4096 samples)."""
    return make_frame(20000, 0.15, 1.0, frame_seed("scoring", frame_id))


def _log_uniform_int(rng: np.random.Generator, lo: int, hi: int) -> int:
    return int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))


def batched_frames(count: int = 256, first: int = 0, scale: float = 1.0) -> list[Frame]:
    """Uneven batch: N log-uniform [500, 30000] (times `scale`), w ~ U[0.1, 0.8]."""
    out = []
    for f in range(first, first + count):
        s = frame_seed("batched", f)
        rng = np.random.default_rng(s ^ 0x5EED)
        n = max(3, int(_log_uniform_int(rng, 500, 30000) * scale))
        w = rng.uniform(0.10, 0.80)
        sigma = rng.uniform(0.5, 2.0)
        out.append(make_frame(n, w, sigma, s))
    return out


def precision_frames(count: int = 4096, first: int = 0, n: int = 5000) -> list[Frame]:
    """Precision stress: sigma in {0.25, 1, 3}; half narrow FOV; 20 % near-degenerate."""
    out = []
    for f in range(first, first + count):
        s = frame_seed("precision", f)
        rng = np.random.default_rng(s ^ 0x5EED)
        sigma = float(rng.choice([0.25, 1.0, 3.0]))
        K = (2000.0, 2000.0, CX, CY) if rng.uniform() < 0.5 else (FX, FY, CX, CY)
        kind = rng.uniform()
        if kind < 0.10:
            fr = make_frame(n, 0.30, sigma, s, K=K, depth_range=(3.9, 4.0))
        elif kind < 0.20:
            fr = make_frame(n, 0.30, sigma, s, K=K, plane=True)
        else:
            fr = make_frame(n, 0.30, sigma, s, K=K)
        out.append(fr)
    return out


def serving_request(request_id: int) -> Frame:
    """One serving request: N log-uniform [300, 50000], w ~ U[0.05, 0.70], sigma 1 px."""
    s = frame_seed("serving", request_id)
    rng = np.random.default_rng(s ^ 0x5EED)
    n = _log_uniform_int(rng, 300, 50000)
    w = rng.uniform(0.05, 0.70)
    return make_frame(n, w, 1.0, s)


def poisson_arrivals(rate_hz: float, duration_s: float, seed: int = 7) -> np.ndarray:
    """Arrival times (s) of a Poisson stream."""
    rng = np.random.default_rng(seed)
    n = int(rate_hz * duration_s * 1.2) + 16
    t = np.cumsum(rng.exponential(1.0 / rate_hz, n))
    return t[t < duration_s]


def rotation_angle(M: np.ndarray) -> float:
    """Angle (rad) of a rotation matrix, accurate near zero: atan2(|vee(M - M^T)|/2, (tr M - 1)/2)."""
    s = 0.5 * math.sqrt((M[2, 1] - M[1, 2]) ** 2 + (M[0, 2] - M[2, 0]) ** 2 + (M[1, 0] - M[0, 1]) ** 2)
    c = 0.5 * (M[0, 0] + M[1, 1] + M[2, 2] - 1.0)
    return math.atan2(s, c)


def pose_error(R_est: np.ndarray, t_est: np.ndarray, R_gt: np.ndarray, t_gt: np.ndarray):
    """(rotation error in degrees, camera-centre error in cm), the metric of
    TbrMain/src/main.cu:141-158: angle of R_gt R_est^T and |C_est - C_gt|."""
    ae = math.degrees(rotation_angle(R_gt @ R_est.T))
    C_est = -R_est.T @ t_est
    C_gt = -R_gt.T @ t_gt
    te = float(np.linalg.norm(C_est - C_gt) * 100.0)
    return ae, te
