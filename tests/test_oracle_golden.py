"""The FP64 oracle against fixtures generated by the reference's own code
(tests/golden/make_golden.py over oracle/_ref), and against published
Philox4x32-10 known answers."""
import os

import numpy as np
import pytest

G = os.path.join(os.path.dirname(__file__), "golden")


def load(name):
    return np.load(os.path.join(G, name))


def test_philox_known_answers(oracle):
    # Random123 philox4x32_10 known-answer vectors (Salmon et al., SC'11).
    assert oracle.philox([0, 0, 0, 0], [0, 0]) == [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]
    assert oracle.philox([0xffffffff] * 4, [0xffffffff] * 2) == [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]
    assert oracle.philox([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0]) == \
        [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]


def test_triples_distinct_and_in_range(oracle):
    for n in (3, 4, 5, 17, 2000, 1 << 20):
        tr = oracle.sample_triples(12345, 0, 4096, n)
        assert tr.min() >= 0 and tr.max() < n
        assert np.all(tr[:, 0] != tr[:, 1]) and np.all(tr[:, 0] != tr[:, 2]) and np.all(tr[:, 1] != tr[:, 2])
    # n = 3: every ordered triple is a permutation, all 6 appear
    tr = oracle.sample_triples(7, 0, 600, 3)
    assert len({tuple(r) for r in tr}) == 6
    # roughly uniform marginals
    tr = oracle.sample_triples(99, 0, 60000, 10)
    h = np.bincount(tr.ravel(), minlength=10) / tr.size
    assert np.all(np.abs(h - 0.1) < 0.01)


def test_p3p_matches_reference(oracle):
    d = load("p3p.npz")
    for i in range(d["x"].shape[0]):
        s = oracle.p3p(d["x"][i], d["X"][i])
        assert s.shape[0] == d["nsol"][i]
        np.testing.assert_array_equal(s, d["sols"][i, : s.shape[0]])


def test_bearing_matches_reference(oracle):
    d = load("bearing.npz")
    b = np.array([oracle.bearing(a, c) for a, c in d["pts"]])
    np.testing.assert_array_equal(b, d["bearing"])


def test_msac_matches_reference(oracle):
    d = load("msac.npz")
    for k in range(d["P"].shape[0]):
        s, c = oracle.msac(d["xn"], d["X"], d["P"][k], float(d["sq_thr"]))
        assert c == d["count"][k]
        assert s == d["score"][k]


def test_quaternions_match_reference(oracle):
    d = load("quat.npz")
    for i in range(d["R"].shape[0]):
        np.testing.assert_array_equal(oracle.rotmat_to_quat(d["R"][i]), d["q_of_R"][i])
        np.testing.assert_array_equal(oracle.quat_to_rotmat(d["q"][i]), d["R_of_q"][i])


def test_lm_matches_reference(oracle):
    d = load("lm.npz")
    for k in range(3):
        q, t, st = oracle.lm(d[f"x{k}"], d[f"X{k}"], d[f"cam{k}"], d[f"q0_{k}"], d[f"t0_{k}"],
                             loss_scale=float(d[f"scale{k}"]))
        np.testing.assert_allclose(q, d[f"q1_{k}"], rtol=0, atol=1e-12)
        np.testing.assert_allclose(t, d[f"t1_{k}"], rtol=0, atol=1e-12)


def test_estimate_post_ransac_matches_reference_entry(oracle):
    """entry.cu's orchestration (inliers with the pre-LM pose, pixel/f LM inputs,
    1/f Cauchy scale) reproduced by the oracle given the same RANSAC pose."""
    d = load("entry.npz")
    for k in range(3):
        uv, X, K = d[f"uv{k}"], d[f"X{k}"], d[f"K{k}"]
        r = oracle.estimate(uv, X, K, seed=int(0), skip_refine=False, replay=None, force_samples=0)
        # same pipeline from the injected pose
        xn = np.ascontiguousarray(np.stack([(uv[:, 0] - K[2]) / K[0], (uv[:, 1] - K[3]) / K[1]], 1))
        R = d[f"P{k}"][:, :3]
        q0 = oracle.rotmat_to_quat(R)
        thr = 4.0 / (0.5 * (K[0] + K[1]))
        inl = oracle.get_inliers(q0, d[f"P{k}"][:, 3], xn, X, thr * thr)
        np.testing.assert_array_equal(inl, d[f"inl{k}"])
        s = 1.0 / (0.5 * (K[0] + K[1]))
        m = inl.astype(bool)
        q, t, _ = oracle.lm(np.ascontiguousarray(uv[m] * s), np.ascontiguousarray(X[m]), K * s, q0,
                            d[f"P{k}"][:, 3], loss_scale=s)
        np.testing.assert_allclose(q, d[f"q{k}"], rtol=0, atol=1e-12)
        np.testing.assert_allclose(t, d[f"t{k}"], rtol=0, atol=1e-12)
        assert r["q"].shape == (4,)


def test_ransac_termination_rule(oracle):
    from turboransac_b200 import scenes
    f = scenes.plain_frame(0)
    xn = np.ascontiguousarray(np.stack([(f.uv[:, 0] - f.K[2]) / f.K[0], (f.uv[:, 1] - f.K[3]) / f.K[1]], 1))
    thr = 4.0 / 525.0
    r = oracle.ransac(xn, f.xyz, thr * thr, seed=f.seed, samples_per_round=1000)
    # 40 % inliers -> K = 418 < 1000: one round (turbo_ransac.cu:223-257)
    assert r["rounds"] == 1 and r["samples"] == 1000 and r["found"]
    r2 = oracle.ransac(xn, f.xyz, thr * thr, seed=f.seed, samples_per_round=100)
    assert r2["rounds"] >= 5  # K = 418 -> stop after the first round with > 418 samples


def test_live_oracle_vs_reference_harness(oracle, ref_harness):
    rng = np.random.default_rng(5)
    for _ in range(2000):
        X = rng.uniform(-3, 3, (3, 3))
        x = rng.standard_normal((3, 3))
        x[:, 2] = np.abs(x[:, 2]) + 0.2
        x /= np.linalg.norm(x, axis=1, keepdims=True)
        a, b = oracle.p3p(x, X), ref_harness.p3p(x, X)
        assert a.shape == b.shape
        np.testing.assert_array_equal(a, b)


def test_stop_rule_quirk_vs_saturation(oracle):
    from turboransac_b200 import scenes
    f = scenes.batched_frames(256)[223]
    xn = np.ascontiguousarray(np.stack([(f.uv[:, 0] - f.K[2]) / f.K[0], (f.uv[:, 1] - f.K[3]) / f.K[1]], 1))
    thr = 4.0 / 525.0
    q = oracle.ransac(xn, f.xyz, thr * thr, seed=f.seed, samples_per_round=1000, quirk=True, threads=8)
    s = oracle.ransac(xn, f.xyz, thr * thr, seed=f.seed, samples_per_round=1000, quirk=False, threads=8)
    assert q["samples"] == 1000 and q["count"] < 10   # INT_MIN ends the loop after one round
    assert s["samples"] > 1000 and s["count"] > 300   # saturating rule keeps sampling


def test_oracle_min_samples_delays_the_stop(oracle):
    from helpers import normalized, sq_thr
    from turboransac_b200 import scenes
    f = scenes.plain_frame(2)
    xn = normalized(f)
    thr = sq_thr(f)
    a = oracle.ransac(xn, f.xyz, thr, seed=f.seed)
    b = oracle.ransac(xn, f.xyz, thr, seed=f.seed, min_samples=4000)
    assert a["samples"] < 4000 <= b["samples"]
    assert b["score"] <= a["score"]


def test_oracle_prosac_schedule(oracle):
    """PROSAC growth table and draws (Chum & Matas, CVPR 2005): T' strictly
    increasing from 1, ending near T_N; every draw before the subset reaches n
    holds the newest point m-1 and two distinct points below it; afterwards the
    draws are the uniform ones."""
    n, TN = 500, 20000.0
    tp = oracle.prosac_table(n, TN)
    assert tp[0] == 1 and np.all(np.diff(tp) >= 1)
    assert TN <= tp[-1] <= TN + n
    tr = oracle.prosac_triples(11, 0, 3000, n, TN)
    for s, (a, b, c) in enumerate(tr):
        t = s + 1
        m = 3 + int(np.searchsorted(tp[:n - 3], t, side="right"))
        assert c == m - 1 and a != b and max(a, b) < m - 1
    late = oracle.prosac_triples(11, int(tp[-1]) + 5, 50, n, TN)
    np.testing.assert_array_equal(late, oracle.sample_triples(11, int(tp[-1]) + 5, 50, n))
