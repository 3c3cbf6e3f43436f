"""Generate the golden fixtures in tests/golden/ from the reference's own code.

Runs the reference's header code and entry.cu compiled on the host
(oracle/_ref/libtbr_refhost.so, built from the reference tree by
``make -C oracle ref``) on seeded inputs and stores inputs + outputs:

  p3p.npz        512 random P3P problems -> p3p<double> solutions (p3p.cuh:9-222)
  bearing.npz    bearing normalisation (ransac.cuh:196-200)
  msac.npz       compute_msac_scores summed over a frame for 16 poses (msac.cuh:18-56)
  quat.npz       rotmat_to_quat / quat_to_rotmat / quat_step_post (pose_utils.cuh)
  cholesky.npz   solve_cholesky<double,6> (lm_utils.cuh:14-100)
  lm.npz         lm_impl<CameraJacobianAccumulator_cuda> on 3 frames (lm.cuh, jaco.cuh)
  entry.npz      estimate_absolute_pose_cuda post-RANSAC path with an injected RANSAC
                 pose (entry.cu:28-144): inlier mask and refined (q, t)

Usage: python tests/golden/make_golden.py   (needs the reference tree, TBR_REF_TREE; run once)
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as orc  # noqa: E402
from turboransac_b200 import scenes  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def rand_bearings(rng, n):
    x = rng.standard_normal((n, 3, 3))
    x[..., 2] = np.abs(x[..., 2]) + 0.5
    return x / np.linalg.norm(x, axis=-1, keepdims=True)


def project_problem(rng, n):
    """P3P problems from a real pose (solvable) mixed with random ones."""
    xs, Xs = [], []
    for i in range(n):
        if i % 2 == 0:
            R = scenes.random_rotation(rng)
            t = rng.uniform(-1, 1, 3)
            Xc = rng.uniform(-1, 1, (3, 3))
            Xc[:, 2] = rng.uniform(1.0, 4.0, 3)
            X = (Xc - t) @ R
            x = Xc / np.linalg.norm(Xc, axis=1, keepdims=True)
        else:
            X = rng.uniform(-2, 2, (3, 3))
            x = rand_bearings(rng, 1)[0]
        xs.append(x)
        Xs.append(X)
    return np.array(xs), np.array(Xs)


def main():
    orc.build(ref=True)
    ref = orc.RefHarness()
    rng = np.random.default_rng(20260301)

    x, X = project_problem(rng, 512)
    nsol = np.zeros(512, np.int32)
    sols = np.zeros((512, 4, 12))
    for i in range(512):
        s = ref.p3p(x[i], X[i])
        nsol[i] = s.shape[0]
        sols[i, : s.shape[0]] = s
    np.savez_compressed(os.path.join(OUT, "p3p.npz"), x=x, X=X, nsol=nsol, sols=sols)

    pts = rng.uniform(-0.8, 0.8, (256, 2))
    bear = np.array([ref.bearing(a, b) for a, b in pts])
    np.savez_compressed(os.path.join(OUT, "bearing.npz"), pts=pts, bearing=bear)

    fr = scenes.make_frame(500, 0.4, 1.0, 11)
    xn = np.ascontiguousarray(np.stack([(fr.uv[:, 0] - fr.K[2]) / fr.K[0], (fr.uv[:, 1] - fr.K[3]) / fr.K[1]], 1))
    thr = 4.0 / (0.5 * (fr.K[0] + fr.K[1]))
    Ps = []
    for k in range(16):
        R = fr.R_gt if k == 0 else scenes.random_rotation(rng) if k > 8 else (
            scenes.quat_to_rotmat(np.array([1.0, *(rng.normal(0, 0.01, 3))]) / np.linalg.norm([1.0, *(rng.normal(0, 0.01, 3))])) @ fr.R_gt)
        t = fr.t_gt + (rng.normal(0, 0.02, 3) if k else 0)
        Ps.append(np.hstack([R, t[:, None]]))
    Ps = np.array(Ps)
    sc = np.zeros(16)
    cn = np.zeros(16, np.int64)
    for k in range(16):
        sc[k], cn[k] = ref.msac(xn, fr.xyz, Ps[k], thr * thr)
    np.savez_compressed(os.path.join(OUT, "msac.npz"), xn=xn, X=fr.xyz, P=Ps, sq_thr=thr * thr, score=sc,
                        count=cn)

    Rs = np.array([scenes.random_rotation(rng) for _ in range(128)])
    # include the trace <= 0 branches
    Rs[:32] = np.array([scenes.quat_to_rotmat(np.array([0.05 * rng.standard_normal(), *rng.standard_normal(3)]) /
                                              np.linalg.norm([0.05, 1, 1, 1])) for _ in range(32)])
    Rs[:32] = np.array([np.linalg.qr(r)[0] * np.sign(np.linalg.det(np.linalg.qr(r)[0])) for r in Rs[:32]])
    qs = np.array([ref.rotmat_to_quat(r) for r in Rs])
    qn = rng.standard_normal((128, 4))
    qn /= np.linalg.norm(qn, axis=1, keepdims=True)
    Rq = np.array([ref.quat_to_rotmat(q) for q in qn])
    ws = rng.normal(0, 0.3, (128, 3))
    ws[:32] *= 1e-7  # Taylor branch of quat_exp
    qstep = np.array([ref.quat_step_post(qn[i], ws[i]) for i in range(128)])
    np.savez_compressed(os.path.join(OUT, "quat.npz"), R=Rs, q_of_R=qs, q=qn, R_of_q=Rq, w=ws, q_step=qstep)

    As, bs, xs_ = [], [], []
    for i in range(64):
        J = rng.standard_normal((20, 6))
        A = J.T @ J + (1e-3 if i % 2 else 0) * np.eye(6)
        A = np.tril(A)  # the reference only fills the lower triangle
        b = rng.standard_normal(6)
        As.append(A)
        bs.append(b)
        xs_.append(ref.solve_cholesky6(A, b))
    np.savez_compressed(os.path.join(OUT, "cholesky.npz"), A=np.array(As), b=np.array(bs), x=np.array(xs_))

    lm = {}
    for k, (n, w, sig) in enumerate([(300, 1.0, 1.0), (800, 0.9, 0.5), (200, 1.0, 2.0)]):
        f = scenes.make_frame(n, w, sig, 1000 + k)
        scale = 1.0 / (0.5 * (f.K[0] + f.K[1]))
        x_in = f.uv * scale
        cam = f.K * scale
        q0 = orc.Oracle().rotmat_to_quat(scenes.quat_to_rotmat(np.array([1.0, 0.01, -0.02, 0.015]) /
                                                                np.linalg.norm([1.0, 0.01, -0.02, 0.015])) @ f.R_gt)
        t0 = f.t_gt + np.array([0.02, -0.01, 0.03])
        q1, t1 = ref.lm(x_in, f.xyz, cam, q0, t0, 100, scale)
        lm[f"x{k}"] = x_in
        lm[f"X{k}"] = f.xyz
        lm[f"cam{k}"] = cam
        lm[f"q0_{k}"] = q0
        lm[f"t0_{k}"] = t0
        lm[f"q1_{k}"] = q1
        lm[f"t1_{k}"] = t1
        lm[f"scale{k}"] = scale
    np.savez_compressed(os.path.join(OUT, "lm.npz"), **lm)

    ent = {}
    o = orc.Oracle()
    for k in range(3):
        f = scenes.make_frame(600, 0.4, 1.0, 2000 + k)
        xn = np.ascontiguousarray(np.stack([(f.uv[:, 0] - f.K[2]) / f.K[0], (f.uv[:, 1] - f.K[3]) / f.K[1]], 1))
        thr = 4.0 / (0.5 * (f.K[0] + f.K[1]))
        rs = o.ransac(xn, f.xyz, thr * thr, seed=f.seed, samples_per_round=1000)
        q, t, inl = ref.estimate_from_pose(f.uv, f.xyz, f.K, rs["P"], 4.0)
        ent[f"uv{k}"] = f.uv
        ent[f"X{k}"] = f.xyz
        ent[f"K{k}"] = f.K
        ent[f"P{k}"] = rs["P"]
        ent[f"q{k}"] = q
        ent[f"t{k}"] = t
        ent[f"inl{k}"] = inl
    np.savez_compressed(os.path.join(OUT, "entry.npz"), **ent)
    print("fixtures written to", OUT)


if __name__ == "__main__":
    main()
