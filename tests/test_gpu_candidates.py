"""FP64 re-rank candidates beyond the per-frame cap (4096 per step).

Every hypothesis whose FP32 score lies within the candidate band of its round's
running minimum is re-scored in FP64, so the selection is the FP64 pipeline's
(ransac.cuh:41-137: global minimum, first-found tie-break). These tests force
more candidates than fit:

  * a step of many forced samples whose hypotheses all tie (n = 3: every sample
    is a permutation of the one triple, every P3P solution fits all points) is
    redone in smaller steps and gives the FP64 oracle's selection, unflagged;
  * a single round of 4096 such samples cannot be split: the kept subset is
    the same on every run and alone or in a batch, and the flag is raised.
"""
import dataclasses

import numpy as np
import pytest

from helpers import quat_angle
from turboransac_b200 import BundleOptions_cuda, Camera_cuda, RansacOptions_cuda, estimate_batch, scenes

pytestmark = pytest.mark.gpu

CAM = Camera_cuda(1, 640, 480, [525.0, 525.0, 319.5, 239.5])


def tied_frame():
    return scenes.make_frame(3, 1.0, 0.0, 77)


def test_forced_step_beyond_cap_is_split_and_matches_oracle(ctx, oracle):
    f = tied_frame()
    ro = RansacOptions_cuda(max_iterations=4096, max_reproj_error=4.0)
    st, pose, inl = ctx.estimate_absolute_pose(f.uv, f.xyz, CAM, ro, BundleOptions_cuda(), seed=5,
                                               force_samples=4096)
    d = st.details
    o = oracle.estimate(f.uv, f.xyz, f.K, 4.0, seed=5, samples_per_round=4096, force_samples=4096)
    info = o["info"]
    assert d["hypotheses"] == info.ransac.hypotheses > 4096  # more ties than one step may re-rank
    assert d["samples"] == 4096 == info.ransac.samples
    assert d["best_sample"] == info.ransac.best_sample and d["best_solution"] == info.ransac.best_sol
    # every solution fits the three points exactly: the scores are FP64 rounding
    # noise (~1e-32), where only an absolute bound means anything
    assert abs(d["model_score"] - info.ransac.score) <= 1e-12 * info.ransac.score + 1e-28
    assert d["candidate_overflow"] == 0
    assert d["steps"] > 1  # the over-full step was redone in smaller ones
    np.testing.assert_array_equal(inl, o["inliers"])
    assert quat_angle(pose.q, o["q"]) < 1e-6 and np.abs(pose.t - o["t"]).max() < 1e-6


def test_single_round_beyond_cap_is_flagged_and_deterministic(ctx):
    f = tied_frame()
    ro = RansacOptions_cuda(max_iterations=4096, max_reproj_error=4.0)
    runs = [ctx.estimate_absolute_pose(f.uv, f.xyz, CAM, ro, BundleOptions_cuda(), seed=9) for _ in range(2)]
    (st0, p0, m0), (st1, p1, m1) = runs
    d0, d1 = st0.details, st1.details
    assert d0["hypotheses"] > 4096
    assert d0["candidate_overflow"] == 1 and d1["candidate_overflow"] == 1
    assert d0["best_sample"] == d1["best_sample"] and d0["best_solution"] == d1["best_solution"]
    assert d0["model_score"] == d1["model_score"]
    np.testing.assert_array_equal(p0.q, p1.q)
    np.testing.assert_array_equal(p0.t, p1.t)
    np.testing.assert_array_equal(m0, m1)
    # The same frame inside a batch keeps the same subset.
    mix = [dataclasses.replace(f, seed=9)] + [scenes.plain_frame(i) for i in range(3)]
    out = estimate_batch(ctx, mix, ro)
    r = out[0]
    assert r["candidate_overflow"] == 1
    assert r["best_sample"] == d0["best_sample"] and r["best_solution"] == d0["best_solution"]
    np.testing.assert_array_equal(r["q"], p0.q)
    np.testing.assert_array_equal(r["t"], p0.t)
    assert all(o["candidate_overflow"] == 0 for o in out[1:])


def test_redo_in_normal_mode_keeps_multi_round_steps_and_matches_oracle(ctx, oracle):
    """A small low-inlier frame of the serving pool (432 points, 100000 samples):
    its multi-round steps hold more than 4096 candidates, so such a step is
    redone, and later steps are sized by the candidate rate (several rounds each,
    not one). The sample count, the selection and the pose are the FP64
    oracle's; a batch with other frames gives the same."""
    f = scenes.serving_request(216)
    assert f.n == 432
    ro = RansacOptions_cuda(max_iterations=1000, max_reproj_error=4.0)
    st, pose, inl = ctx.estimate_absolute_pose(f.uv, f.xyz, CAM, ro, BundleOptions_cuda(), seed=f.seed)
    d = st.details
    o = oracle.estimate(f.uv, f.xyz, f.K, 4.0, seed=f.seed, samples_per_round=1000, threads=8)
    info = o["info"]
    assert d["samples"] == info.ransac.samples == 100000
    assert d["best_sample"] == info.ransac.best_sample and d["best_solution"] == info.ransac.best_sol
    assert abs(d["model_score"] - info.ransac.score) <= 1e-12 * info.ransac.score
    assert d["candidate_overflow"] == 0
    assert d["steps"] < d["rounds"] // 2  # steps of several rounds after the redo
    np.testing.assert_array_equal(inl, o["inliers"])
    assert quat_angle(pose.q, o["q"]) < 1e-6 and np.abs(pose.t - o["t"]).max() < 1e-6
    mixed = estimate_batch(ctx, scenes.batched_frames(6, scale=0.3) + [f], ro)
    r = mixed[-1]
    assert r["samples"] == d["samples"] and r["best_sample"] == d["best_sample"]
    assert quat_angle(r["q"], pose.q) < 1e-9
