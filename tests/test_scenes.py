import numpy as np

from turboransac_b200 import scenes


def test_plain_frame_shapes_and_inliers():
    f = scenes.plain_frame(0)
    assert f.n == 2000 and f.inlier_gt.sum() == 800
    assert np.all(f.uv.astype(np.float32).astype(np.float64) == f.uv)
    # inliers reproject within a few sigma
    Xc = f.xyz @ f.R_gt.T + f.t_gt
    p = Xc[:, :2] / Xc[:, 2:3] * 525.0 + np.array([319.5, 239.5])
    e = np.linalg.norm(p - f.uv, axis=1)
    assert np.median(e[f.inlier_gt]) < 2.0
    assert np.median(e[~f.inlier_gt]) > 20.0


def test_seeds_are_stable():
    assert scenes.frame_seed("plain", 0) == scenes.frame_seed(0, 0)
    assert scenes.frame_seed("plain", 0) != scenes.frame_seed("plain", 1)
    a = scenes.batched_frames(3)
    b = scenes.batched_frames(3)
    assert all(np.array_equal(x.uv, y.uv) for x, y in zip(a, b))


def test_precision_and_serving_generators():
    fr = scenes.precision_frames(40)
    assert all(f.n == 5000 for f in fr)
    assert any(f.degenerate == "plane" for f in fr) and any(f.K[0] == 2000.0 for f in fr)
    r = scenes.serving_request(3)
    assert 300 <= r.n <= 50000
    t = scenes.poisson_arrivals(2000.0, 1.0)
    assert 1800 < t.size < 2200


def test_pose_error_metric():
    R = scenes.random_rotation(np.random.default_rng(0))
    t = np.array([0.1, 0.2, 0.3])
    assert scenes.pose_error(R, t, R, t) == (0.0, 0.0)
