"""CUDA path (through the C ABI) against the FP64 oracle on identical samples.

Tolerances (the parity bar):
  * P3P hypotheses: same solution count per sample, poses within 1e-9
  * FP32 MSAC scores: within 1e-5 relative of the FP64 scores
  * inlier counts: exact except for points within 1e-4 px of the threshold
  * selected best hypothesis: same sample and solution, FP64 score within 1e-12 relative
  * final pose: within 1e-6 rad and 1e-6 m of the FP64 pipeline
"""
import numpy as np
import pytest

from helpers import near_threshold, normalized, quat_angle, sq_thr
from turboransac_b200 import (BundleOptions_cuda, Camera_cuda, CameraPose_cuda, RansacOptions_cuda, TbrError,
                              scenes)

pytestmark = pytest.mark.gpu


def cam_of(f):
    return Camera_cuda(1, 640, 480, list(f.K))


# Scoring shapes: on the tensor cores (tcgen05, TF32 split operands; the
# default) and on the FP32 pipe.
TENSOR = {"points_per_iter": 128}
FP32 = {"hyp_per_thread": 4, "points_per_iter": 2}


@pytest.mark.parametrize("shape", [None, FP32, dict(FP32, hyp_per_thread=8), dict(TENSOR, chunk_points=256)],
                         ids=["default", "fp32", "fp32-hr8", "tensor-chunk256"])
def test_debug_scores_counts_vs_oracle(ctx, oracle, shape):
    f = scenes.plain_frame(1)
    S = 512
    tr = oracle.sample_triples(f.seed, 0, S, f.n)
    ids, poses, s32, cnt = ctx.debug_score_samples(f.uv, f.xyz, f.K, 4.0, tr, counts=True, shape=shape)
    xn = normalized(f)
    sq = sq_thr(f)
    o = oracle.ransac(xn, f.xyz, sq, dump=4 * S, replay=tr, force_samples=S, samples_per_round=S)
    np.testing.assert_array_equal(ids, o["hyp_ids"])
    np.testing.assert_allclose(poses.reshape(-1, 12), o["hyp_poses"], rtol=1e-9, atol=1e-9)
    s64 = o["hyp_scores"] / sq
    rel = np.abs(s32.astype(np.float64) - s64) / s64
    assert rel.max() < 1e-5, rel.max()
    focal = 0.5 * (f.K[0] + f.K[1])
    for k in range(ids.size):
        d = abs(int(cnt[k]) - int(o["hyp_counts"][k]))
        if d:
            allowed = near_threshold(o["hyp_poses"][k].reshape(3, 4), xn, f.xyz, focal).sum()
            assert d <= allowed, (k, d, allowed)


@pytest.mark.parametrize("frame_id", [0, 3])
def test_plain_call_matches_oracle(ctx, oracle, frame_id):
    f = scenes.plain_frame(frame_id)
    ro = RansacOptions_cuda(max_iterations=1000, success_prob=0.9999, max_reproj_error=4.0)
    st, pose, inl = ctx.estimate_absolute_pose(f.uv, f.xyz, cam_of(f), ro, BundleOptions_cuda(), seed=f.seed)
    o = oracle.estimate(f.uv, f.xyz, f.K, 4.0, seed=f.seed, samples_per_round=1000)
    d = st.details
    info = o["info"]
    assert d["samples"] == info.ransac.samples
    assert d["best_sample"] == info.ransac.best_sample and d["best_solution"] == info.ransac.best_sol
    assert d["ransac_inliers"] == info.ransac.count
    assert abs(d["model_score"] - info.ransac.score) <= 1e-12 * info.ransac.score
    assert d["num_inliers"] == info.num_inliers
    np.testing.assert_array_equal(inl, o["inliers"])
    assert quat_angle(pose.q, o["q"]) < 1e-6
    assert np.abs(pose.t - o["t"]).max() < 1e-6
    ae, te = scenes.pose_error(pose.R(), pose.t, f.R_gt, f.t_gt)
    assert ae < 5 and te < 5


def test_scoring_bound_config_matches_oracle(ctx, oracle):
    """N=20000, 15 % inliers, exactly 4096 samples (no early stop)."""
    f = scenes.scoring_frame(0)
    ro = RansacOptions_cuda(max_iterations=4096, max_reproj_error=4.0)
    st, pose, inl = ctx.estimate_absolute_pose(f.uv, f.xyz, cam_of(f), ro, BundleOptions_cuda(), seed=f.seed,
                                               force_samples=4096)
    o = oracle.estimate(f.uv, f.xyz, f.K, 4.0, seed=f.seed, samples_per_round=4096, force_samples=4096, threads=8)
    info = o["info"]
    d = st.details
    assert d["samples"] == 4096 == info.ransac.samples
    assert d["hypotheses"] == info.ransac.hypotheses
    assert d["best_sample"] == info.ransac.best_sample and d["best_solution"] == info.ransac.best_sol
    assert d["ransac_inliers"] == info.ransac.count
    assert quat_angle(pose.q, o["q"]) < 1e-6 and np.abs(pose.t - o["t"]).max() < 1e-6
    np.testing.assert_array_equal(inl, o["inliers"])


@pytest.mark.parametrize("shape", [TENSOR, FP32], ids=["tensor", "fp32"])
def test_scoring_shapes_match_oracle(ctx, oracle, shape):
    """Both scoring kernels decide like the FP64 pipeline: the scoring-bound
    frame (4096 samples, 15 % inliers, N = 20000) and a frame that needs many
    rounds give the oracle's samples, selection and pose."""
    f = scenes.scoring_frame(0)
    ro = RansacOptions_cuda(max_iterations=4096, max_reproj_error=4.0)
    st, pose, inl = ctx.estimate_absolute_pose(f.uv, f.xyz, cam_of(f), ro, BundleOptions_cuda(), seed=f.seed,
                                               force_samples=4096, **shape)
    o = oracle.estimate(f.uv, f.xyz, f.K, 4.0, seed=f.seed, samples_per_round=4096, force_samples=4096, threads=8)
    d, info = st.details, o["info"]
    assert d["hypotheses"] == info.ransac.hypotheses
    assert d["best_sample"] == info.ransac.best_sample and d["best_solution"] == info.ransac.best_sol
    assert d["ransac_inliers"] == info.ransac.count
    assert quat_angle(pose.q, o["q"]) < 1e-6 and np.abs(pose.t - o["t"]).max() < 1e-6
    np.testing.assert_array_equal(inl, o["inliers"])
    f = scenes.make_frame(3000, 0.10, 1.0, 4242)
    ro = RansacOptions_cuda(max_iterations=1000, max_reproj_error=4.0)
    st, pose, inl = ctx.estimate_absolute_pose(f.uv, f.xyz, cam_of(f), ro, BundleOptions_cuda(), seed=f.seed,
                                               **shape)
    o = oracle.estimate(f.uv, f.xyz, f.K, 4.0, seed=f.seed, samples_per_round=1000, threads=8)
    d, info = st.details, o["info"]
    assert d["samples"] == info.ransac.samples and d["best_sample"] == info.ransac.best_sample
    assert quat_angle(pose.q, o["q"]) < 1e-6 and np.abs(pose.t - o["t"]).max() < 1e-6


def test_multi_round_termination_matches_oracle(ctx, oracle):
    """10 % inliers: ~28 rounds of 1000 under the reference's stop rule, run by the
    engine in a couple of speculative steps; samples, selection and pose must be
    those of the sequential round loop."""
    f = scenes.make_frame(3000, 0.10, 1.0, 4242)
    ro = RansacOptions_cuda(max_iterations=1000, max_reproj_error=4.0)
    st, pose, inl = ctx.estimate_absolute_pose(f.uv, f.xyz, cam_of(f), ro, BundleOptions_cuda(), seed=f.seed)
    o = oracle.estimate(f.uv, f.xyz, f.K, 4.0, seed=f.seed, samples_per_round=1000, threads=8)
    info = o["info"]
    d = st.details
    assert info.ransac.rounds > 5
    assert d["samples"] == info.ransac.samples and d["rounds"] == info.ransac.rounds
    assert d["hypotheses"] == info.ransac.hypotheses
    assert d["best_sample"] == info.ransac.best_sample
    assert quat_angle(pose.q, o["q"]) < 1e-6 and np.abs(pose.t - o["t"]).max() < 1e-6


def test_replayed_samples(ctx, oracle):
    f = scenes.plain_frame(5)
    rng = np.random.default_rng(1)
    tr = np.stack([rng.choice(f.n, 3, replace=False) for _ in range(3000)]).astype(np.int32)
    ro = RansacOptions_cuda(max_iterations=300, max_reproj_error=4.0)
    st, pose, inl = ctx.estimate_absolute_pose(f.uv, f.xyz, cam_of(f), ro, BundleOptions_cuda(), replay=tr)
    o = oracle.estimate(f.uv, f.xyz, f.K, 4.0, replay=tr, samples_per_round=300)
    assert st.details["samples"] == o["info"].ransac.samples
    assert st.details["best_sample"] == o["info"].ransac.best_sample
    assert quat_angle(pose.q, o["q"]) < 1e-6 and np.abs(pose.t - o["t"]).max() < 1e-6


def test_edge_cases(ctx, oracle):
    ro = RansacOptions_cuda(max_iterations=64, max_reproj_error=4.0)
    cam = Camera_cuda(1, 640, 480, [525.0, 525.0, 319.5, 239.5])
    with pytest.raises(TbrError):
        ctx.estimate_absolute_pose(np.zeros((2, 2)), np.zeros((2, 3)), cam, ro)
    with pytest.raises(ValueError):
        ctx.estimate_absolute_pose(np.zeros((5, 2)), np.zeros((4, 3)), cam, ro)
    # exactly three points: every sample is a permutation of the one triple
    f = scenes.make_frame(3, 1.0, 0.0, 77)
    st, pose, inl = ctx.estimate_absolute_pose(f.uv, f.xyz, cam, ro, seed=3)
    o = oracle.estimate(f.uv, f.xyz, f.K, 4.0, seed=3, samples_per_round=64)
    assert st.details["best_sample"] == o["info"].ransac.best_sample
    np.testing.assert_array_equal(inl, o["inliers"])
    # all points identical: P3P degenerates, no hypothesis is valid or all are NaN-poses
    uv = np.tile([[300.0, 200.0]], (10, 1))
    X = np.tile([[0.1, 0.2, 2.0]], (10, 1))
    st, pose, inl = ctx.estimate_absolute_pose(uv, X, cam, ro, seed=1)
    o = oracle.estimate(uv, X, np.array(cam.params), 4.0, seed=1, samples_per_round=64)
    assert st.details["samples"] == o["info"].ransac.samples
    # ragged small n
    for n in (4, 5, 7, 65, 129):
        f = scenes.make_frame(n, 0.8, 0.5, 100 + n)
        st, pose, inl = ctx.estimate_absolute_pose(f.uv, f.xyz, cam, ro, seed=f.seed)
        o = oracle.estimate(f.uv, f.xyz, f.K, 4.0, seed=f.seed, samples_per_round=64)
        assert st.details["best_sample"] == o["info"].ransac.best_sample
        assert quat_angle(pose.q, o["q"]) < 1e-6 and np.abs(pose.t - o["t"]).max() < 1e-6


def test_get_inliers_matches_oracle(ctx, oracle):
    f = scenes.plain_frame(2)
    xn = normalized(f)
    q = oracle.rotmat_to_quat(f.R_gt)
    m = ctx.get_inliers(CameraPose_cuda(q, f.t_gt), xn, f.xyz, sq_thr(f))
    np.testing.assert_array_equal(m, oracle.get_inliers(q, f.t_gt, xn, f.xyz, sq_thr(f)))


def test_bundle_adjust_matches_reference_fixture(ctx):
    import os
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "lm.npz"))
    for k in range(3):
        cam = Camera_cuda(1, 640, 480, list(d[f"cam{k}"]))
        pose, st = ctx.bundle_adjust(d[f"x{k}"], d[f"X{k}"], cam, CameraPose_cuda(d[f"q0_{k}"], d[f"t0_{k}"]),
                                     BundleOptions_cuda(loss_scale=float(d[f"scale{k}"])))
        assert quat_angle(pose.q, d[f"q1_{k}"]) < 1e-6
        assert np.abs(pose.t - d[f"t1_{k}"]).max() < 1e-6


@pytest.mark.parametrize("quirk", [False, True])
def test_stop_rule_overflow_modes(ctx, oracle, quirk):
    """A first round whose best has almost no inliers makes the stop bound
    overflow int: the x86 quirk stops after one round, the default saturates."""
    from turboransac_b200 import scenes as sc
    f = sc.batched_frames(256)[169]
    ro = RansacOptions_cuda(max_iterations=1000, max_reproj_error=4.0)
    st, pose, inl = ctx.estimate_absolute_pose(f.uv, f.xyz, cam_of(f), ro, BundleOptions_cuda(), seed=f.seed,
                                               stop_rule_x86_quirk=quirk)
    o = oracle.estimate(f.uv, f.xyz, f.K, 4.0, seed=f.seed, samples_per_round=1000, threads=8, quirk=quirk)
    assert st.details["samples"] == o["info"].ransac.samples
    assert st.details["best_sample"] == o["info"].ransac.best_sample
    assert (o["info"].ransac.samples == 1000) == quirk
    assert quat_angle(pose.q, o["q"]) < 1e-6 and np.abs(pose.t - o["t"]).max() < 1e-6


def test_nonfinite_points_are_outliers(ctx, oracle):
    """NaN / inf correspondences are never inliers (comparisons with NaN fail in
    msac.cuh:46 and entry.cu:22); the FP32 filter stages them as outliers, and
    samples that contain them give non-finite P3P poses that score n * tau^2."""
    f = scenes.plain_frame(3)
    uv, xyz = f.uv.copy(), f.xyz.copy()
    rng = np.random.default_rng(5)
    bad = rng.choice(f.n, 120, replace=False)
    xyz[bad[:40], 0] = np.nan
    xyz[bad[40:60], 2] = np.inf
    uv[bad[60:100], 1] = np.nan
    uv[bad[100:], 0] = -np.inf
    ro = RansacOptions_cuda(max_iterations=1000, success_prob=0.9999, max_reproj_error=4.0)
    st, pose, inl = ctx.estimate_absolute_pose(uv, xyz, cam_of(f), ro, BundleOptions_cuda(), seed=f.seed)
    o = oracle.estimate(uv, xyz, f.K, 4.0, seed=f.seed, samples_per_round=1000)
    d, info = st.details, o["info"]
    assert d["samples"] == info.ransac.samples
    assert d["best_sample"] == info.ransac.best_sample and d["best_solution"] == info.ransac.best_sol
    assert abs(d["model_score"] - info.ransac.score) <= 1e-12 * info.ransac.score
    np.testing.assert_array_equal(inl, o["inliers"])
    assert not inl[bad].any()
    assert quat_angle(pose.q, o["q"]) < 1e-6 and np.abs(pose.t - o["t"]).max() < 1e-6


def test_large_frame_cluster_lm_matches_oracle(ctx, oracle):
    """N = 25000 at 60 % inliers: the LM of this frame runs on a cluster of CTAs
    (distributed-shared-memory sums); pose within 1e-6 of the FP64 pipeline."""
    f = scenes.make_frame(25000, 0.60, 1.0, 9191)
    ro = RansacOptions_cuda(max_iterations=1000, max_reproj_error=4.0)
    st, pose, inl = ctx.estimate_absolute_pose(f.uv, f.xyz, cam_of(f), ro, BundleOptions_cuda(), seed=f.seed)
    o = oracle.estimate(f.uv, f.xyz, f.K, 4.0, seed=f.seed, samples_per_round=1000, threads=8)
    d = st.details
    assert d["num_inliers"] == o["info"].num_inliers and d["num_inliers"] >= 10000
    assert d["best_sample"] == o["info"].ransac.best_sample
    np.testing.assert_array_equal(inl, o["inliers"])
    assert quat_angle(pose.q, o["q"]) < 1e-6 and np.abs(pose.t - o["t"]).max() < 1e-6


def test_honoured_ransac_options_match_oracle(ctx, oracle):
    """honor_options: min_iterations, success_prob and dyn_num_trials_mult of
    RansacOptions_cuda (utils.h:16-19, ignored by the reference) take effect and
    give the oracle's samples, selection and pose."""
    f = scenes.plain_frame(2)
    for kw in ({"min_iterations": 5000}, {"success_prob": 0.99, "dyn_num_trials_mult": 1.0},
               {"min_iterations": 2500, "success_prob": 0.999999}):
        ro = RansacOptions_cuda(max_iterations=1000, max_reproj_error=4.0, **kw)
        st, pose, inl = ctx.estimate_absolute_pose(f.uv, f.xyz, cam_of(f), ro, BundleOptions_cuda(), seed=f.seed,
                                                   honor_options=True)
        o = oracle.estimate(f.uv, f.xyz, f.K, 4.0, seed=f.seed, samples_per_round=1000,
                            min_samples=kw.get("min_iterations", 0), success_prob=kw.get("success_prob", 0.9999),
                            trials_mult=kw.get("dyn_num_trials_mult", 3.0))
        d, info = st.details, o["info"]
        assert d["samples"] == info.ransac.samples, kw
        if "min_iterations" in kw:
            assert d["samples"] >= kw["min_iterations"]
        assert d["best_sample"] == info.ransac.best_sample
        np.testing.assert_array_equal(inl, o["inliers"])
        assert quat_angle(pose.q, o["q"]) < 1e-6 and np.abs(pose.t - o["t"]).max() < 1e-6


@pytest.mark.parametrize("loss_type", [0, 1, 2, 3])
def test_bundle_adjust_honoured_loss_and_weights(ctx, oracle, loss_type):
    """honor_options on bundle_adjust_cuda: BundleOptions_cuda::loss_type
    (TRIVIAL, TRUNCATED, HUBER, CAUCHY; the reference always runs Cauchy) and
    per-point weights (ignored by the reference) against the FP64 oracle LM."""
    import os
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "lm.npz"))
    rng = np.random.default_rng(17 + loss_type)
    for k in range(3):
        x, X, K = d[f"x{k}"], d[f"X{k}"], d[f"cam{k}"]
        scale = float(d[f"scale{k}"])
        w = rng.uniform(0.5, 2.0, x.shape[0])
        cam = Camera_cuda(1, 640, 480, list(K))
        pose, st = ctx.bundle_adjust(x, X, cam, CameraPose_cuda(d[f"q0_{k}"], d[f"t0_{k}"]),
                                     BundleOptions_cuda(loss_scale=scale, loss_type=loss_type), weights=w,
                                     honor_options=True)
        oq, ot, ost = oracle.lm(x, X, K, d[f"q0_{k}"], d[f"t0_{k}"], loss_scale=scale,
                                loss={0: 3, 1: 1, 2: 2, 3: 0}[loss_type], weights=w)
        assert quat_angle(pose.q, oq) < 1e-6, (loss_type, k)
        assert np.abs(pose.t - ot).max() < 1e-6, (loss_type, k)


def test_prosac_sampling_matches_oracle(ctx, oracle):
    """honor_options + progressive_sampling (utils.h:23-25, declared but not
    implemented by the reference): PROSAC draws over correspondences sorted by
    quality (here inliers first); samples, selection and pose equal the oracle's."""
    f = scenes.make_frame(3000, 0.15, 1.0, 5151)
    order = np.concatenate([np.flatnonzero(f.inlier_gt), np.flatnonzero(~f.inlier_gt)])
    uv, xyz = f.uv[order].copy(), f.xyz[order].copy()
    for TN in (100000, 20000):
        ro = RansacOptions_cuda(max_iterations=1000, max_reproj_error=4.0, progressive_sampling=True,
                                max_prosac_iterations=TN)
        st, pose, inl = ctx.estimate_absolute_pose(uv, xyz, cam_of(f), ro, BundleOptions_cuda(), seed=f.seed,
                                                   honor_options=True)
        o = oracle.estimate(uv, xyz, f.K, 4.0, seed=f.seed, samples_per_round=1000, threads=8, prosac=True,
                            prosac_TN=float(TN))
        d, info = st.details, o["info"]
        assert d["samples"] == info.ransac.samples
        assert d["best_sample"] == info.ransac.best_sample and d["best_solution"] == info.ransac.best_sol
        np.testing.assert_array_equal(inl, o["inliers"])
        assert quat_angle(pose.q, o["q"]) < 1e-6 and np.abs(pose.t - o["t"]).max() < 1e-6
        ae, te = scenes.pose_error(pose.R(), pose.t, f.R_gt, f.t_gt)
        assert ae < 5 and te < 5


def test_large_frame_and_workspace_limit(oracle):
    """N = 100000 (the paper's large-N regime) matches the oracle; a frame that
    does not fit the context's workspace is refused with OOM, and the context
    stays usable."""
    from turboransac_b200 import Context, TbrError
    big = Context(0, 2 << 30)
    f = scenes.make_frame(100000, 0.5, 1.0, 777)
    ro = RansacOptions_cuda(max_iterations=1000, max_reproj_error=4.0)
    st, pose, inl = big.estimate_absolute_pose(f.uv, f.xyz, cam_of(f), ro, BundleOptions_cuda(), seed=f.seed)
    o = oracle.estimate(f.uv, f.xyz, f.K, 4.0, seed=f.seed, samples_per_round=1000, threads=16)
    assert st.details["best_sample"] == o["info"].ransac.best_sample
    np.testing.assert_array_equal(inl, o["inliers"])
    assert quat_angle(pose.q, o["q"]) < 1e-6 and np.abs(pose.t - o["t"]).max() < 1e-6
    big.close()
    small = Context(0, 256 << 20)
    g = scenes.make_frame(2000000, 0.5, 1.0, 778)
    with pytest.raises(TbrError) as e:
        small.estimate_absolute_pose(g.uv, g.xyz, cam_of(g), ro, BundleOptions_cuda(), seed=g.seed)
    assert "OOM" in str(e.value) or "workspace" in str(e.value)
    h = scenes.plain_frame(0)
    st, pose, inl = small.estimate_absolute_pose(h.uv, h.xyz, cam_of(h), ro, BundleOptions_cuda(), seed=h.seed)
    assert st.num_inliers > 0
    small.close()
