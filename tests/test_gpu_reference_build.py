"""Parity against the reference's own CUDA build on the same B200, on the
reference's own minimal samples.

The reference's three src/*.cu are built unchanged for sm_100a (oracle/Makefile
target `refcuda`) and called once per frame through estimate_absolute_pose_cuda.
Its cuRAND draws are exported by a harness kernel that calls cuRAND with the
reference's seeds (turbo_ransac.cu:159-160, ransac.cuh:176-196) and replayed
through this library and through the FP64 oracle. Selection, stop rule
(x86 conversion of the overflowing bound), inliers and LM then have to land on
the reference's pose: within 1e-6 rad and 1e-6 m. Skipped where the reference
tree was not available to build oracle/_ref."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from helpers import quat_angle  # noqa: E402
from oracle import refcuda  # noqa: E402
from turboransac_b200 import BundleOptions_cuda, Camera_cuda, RansacOptions_cuda, scenes  # noqa: E402

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refcuda.available(), reason="reference CUDA build not present (oracle/_ref)")]

B = 1000
ROUNDS = 100  # the reference's 100000-sample cap


def frames():
    fr = [scenes.plain_frame(i) for i in range(4)]
    fr += [f for f in scenes.batched_frames(24) if f.n <= 12000][:6]
    return fr


def test_pose_matches_reference_cuda_build_on_its_samples(ctx, oracle):
    fr = frames()
    ref = refcuda.run(fr, warmup=1)
    ro = RansacOptions_cuda(max_iterations=B, success_prob=0.9999, max_reproj_error=4.0)
    worst = (0.0, 0.0)
    for k, f in enumerate(fr):
        tri = refcuda.curand_triples(f.n, B, ROUNDS)
        st, pose, inl = ctx.estimate_absolute_pose(f.uv, f.xyz, Camera_cuda(1, 640, 480, list(f.K)), ro,
                                                   BundleOptions_cuda(), replay=tri, stop_rule_x86_quirk=True)
        o = oracle.estimate(f.uv, f.xyz, f.K, 4.0, samples_per_round=B, replay=tri, quirk=True)
        assert st.details["best_sample"] == o["info"].ransac.best_sample
        np.testing.assert_array_equal(inl, o["inliers"])
        # the reference's own result on the same samples
        dr = quat_angle(pose.q, ref["q"][k])
        dt = float(np.abs(pose.t - ref["t"][k]).max())
        assert int(ref["inliers"][k]) == int(inl.sum()), f"frame {k}: inlier set differs from the reference build"
        assert dr < 1e-6 and dt < 1e-6, f"frame {k}: {dr:.2e} rad, {dt:.2e} m from the reference build"
        worst = (max(worst[0], dr), max(worst[1], dt))
    print(f"max deviation from the reference CUDA build: {worst[0]:.2e} rad, {worst[1]:.2e} m")
