"""Batched (graph-captured) and served (continuous batching) forms: each frame's
result is the one the plain per-frame call gives -- alone and in the mix."""
import time

import numpy as np
import pytest

from helpers import quat_angle
from turboransac_b200 import (Batch, BundleOptions_cuda, Camera_cuda, RansacOptions_cuda, Server, estimate_batch,
                              scenes)

pytestmark = pytest.mark.gpu

RO = RansacOptions_cuda(max_iterations=1000, max_reproj_error=4.0)


def plain(ctx, f):
    st, pose, inl = ctx.estimate_absolute_pose(f.uv, f.xyz, Camera_cuda(1, 640, 480, list(f.K)), RO,
                                               BundleOptions_cuda(), seed=f.seed)
    return st.details, pose


def mixed_frames():
    fr = scenes.batched_frames(24, scale=0.5)
    fr += [scenes.make_frame(6000, 0.08, 1.0, 9001), scenes.make_frame(400, 0.6, 0.5, 9002)]
    return fr


def same(d, pose_q, pose_t, ref_d, ref_pose):
    assert d["samples"] == ref_d["samples"]
    assert d["best_sample"] == ref_d["best_sample"]
    assert d["num_inliers"] == ref_d["num_inliers"]
    assert quat_angle(pose_q, ref_pose.q) < 1e-9
    assert np.abs(np.asarray(pose_t) - ref_pose.t).max() < 1e-9


def test_batch_graph_matches_plain_calls(ctx):
    fr = mixed_frames()
    ref = [plain(ctx, f) for f in fr]
    b = Batch(ctx, fr, RO)
    for _ in range(2):  # the graph is replayed: second run must give the same
        b.run()
        b.sync()
        res = b.results()
        for r, f, (d, pose) in zip(res, fr, ref):
            assert r["status"] == 0
            same(r, r["q"], r["t"], d, pose)
    prof, pairs = b.profile()
    assert prof["k_score"][1] >= 1 and pairs > 0
    b.close()


def test_estimate_batch_host_buffers(ctx):
    fr = mixed_frames()[:8]
    out = estimate_batch(ctx, fr, RO, masks=True)
    for o, f in zip(out, fr):
        d, pose = plain(ctx, f)
        same(o, o["q"], o["t"], d, pose)
        assert int(o["inliers"].sum()) == d["num_inliers"]


def test_server_results_match_plain_and_alone(ctx):
    fr = mixed_frames()
    ref = [plain(ctx, f) for f in fr]
    srv = Server(ctx, budget_bytes=2 << 30, max_slots=64)
    # alone: one request at a time
    alone = {}
    for i in (0, len(fr) - 2):
        rid = srv.submit(fr[i])
        srv.drain()
        (r,) = srv.poll()
        assert r["id"] == rid and r["status"] == 0
        alone[i] = r
    # in the mix: everything submitted in a burst while others run
    ids = {}
    for i, f in enumerate(fr):
        ids[srv.submit(f)] = i
        if i % 5 == 0:
            time.sleep(0.002)
    srv.drain()
    got = srv.poll()
    assert len(got) == len(fr)
    for r in got:
        i = ids[r["id"]]
        assert r["status"] == 0
        d, pose = ref[i]
        same(r, r["q"], r["t"], d, pose)
        if i in alone:
            np.testing.assert_array_equal(r["q"], alone[i]["q"])
            np.testing.assert_array_equal(r["t"], alone[i]["t"])
    srv.close()


def test_server_cancel_and_errors(ctx):
    srv = Server(ctx, budget_bytes=1 << 30, max_slots=8)
    f = scenes.make_frame(3000, 0.06, 1.0, 77)
    rid = srv.submit(f)
    srv.cancel(rid)
    srv.drain()
    (r,) = srv.poll()
    assert r["id"] == rid and r["status"] in (0, 5)  # finished before the cancel landed, or cancelled
    class Tiny:  # two points: refused with INVALID_ARG, the server keeps running
        uv = np.zeros((2, 2))
        xyz = np.zeros((2, 3))
        K = f.K
        seed = 1
    from turboransac_b200 import TbrError
    with pytest.raises(TbrError):
        srv.submit(Tiny())
    rid2 = srv.submit(scenes.make_frame(500, 0.5, 1.0, 78))
    srv.drain()
    (r2,) = srv.poll()
    assert r2["id"] == rid2 and r2["status"] == 0
    srv.close()


def test_autotune_keeps_results(ctx):
    """Every scoring shape gives the same results (the FP64 re-rank decides), and
    the tuned batch keeps returning them."""
    fr = mixed_frames()
    b = Batch(ctx, fr, RO)
    b.run()
    b.sync()
    before = b.results()
    best, tried = b.autotune(repeats=1)
    # 32 hypotheses per block (tensor cores) and 64-256 (FP32 kernel) x point tiles
    assert len(tried) == 41 and all(t["ms"] > 0 for t in tried)
    assert {t["hyp_per_block"] for t in tried} == {32, 64, 128, 192, 256}
    assert {128, 256, 512} <= {t["chunk_points"] for t in tried}
    assert sum(t["points_per_iter"] == 128 for t in tried) == 5  # the tensor-core shape with 5 tilings
    assert best["ms"] == min(t["ms"] for t in tried)
    b.run()
    b.sync()
    after = b.results()
    b.close()
    for r0, r1 in zip(before, after):
        assert r1["status"] == 0
        assert r1["samples"] == r0["samples"] and r1["best_sample"] == r0["best_sample"]
        assert r1["num_inliers"] == r0["num_inliers"]
        assert quat_angle(r1["q"], r0["q"]) < 1e-12 and np.abs(r1["t"] - r0["t"]).max() < 1e-12


def test_device_resident_inputs_match_host_inputs(ctx):
    """tbr_estimate_batch_device: correspondences handed over as CUDA tensors
    give the host call's results."""
    import torch

    from turboransac_b200 import DeviceFrame, estimate_batch_device
    fr = mixed_frames()
    host = estimate_batch(ctx, fr, RO)
    dev_frames = [DeviceFrame(f) for f in fr]
    torch.cuda.synchronize()
    for _ in range(2):
        got = estimate_batch_device(ctx, dev_frames, RO)
        for a, b in zip(got, host):
            assert a["status"] == 0
            assert a["samples"] == b["samples"] and a["best_sample"] == b["best_sample"]
            assert a["num_inliers"] == b["num_inliers"]
            assert quat_angle(a["q"], b["q"]) < 1e-12 and np.abs(a["t"] - b["t"]).max() < 1e-12
    # host pointers are refused, not read as device memory
    import ctypes as C

    from turboransac_b200 import _lib
    arr = (_lib.FrameDescC * 1)()
    f = fr[0]
    arr[0].points2D = f.uv.ctypes.data
    arr[0].points3D = f.xyz.ctypes.data
    arr[0].n = f.n
    for k in range(4):
        arr[0].K[k] = float(f.K[k])
    res = (_lib.FrameResultC * 1)()
    ro = RO.to_c()
    st = _lib.lib().tbr_estimate_batch_device(ctx.handle, arr, 1, C.byref(ro), None, None, res, None)
    assert st != 0


def test_estimate_batch_beyond_context_capacity(ctx):
    """More frames than the context holds at once (1024) run in consecutive
    groups; every result equals the plain call's."""
    fr = [scenes.make_frame(300, 0.6, 1.0, 20000 + i) for i in range(1100)]
    got = estimate_batch(ctx, fr, RO)
    assert len(got) == 1100 and all(r["status"] == 0 for r in got)
    for i in (0, 511, 1023, 1024, 1099):
        d, pose = plain(ctx, fr[i])
        same(got[i], got[i]["q"], got[i]["t"], d, pose)


def test_server_honoured_options_match_plain(ctx):
    """The server with honor_options (PROSAC over sorted correspondences, a raised
    minimum sample count) gives the plain call's results under the same options."""
    ro = RansacOptions_cuda(max_iterations=1000, max_reproj_error=4.0, progressive_sampling=True,
                            max_prosac_iterations=30000, min_iterations=3000)
    fr = []
    for i in range(6):
        f = scenes.make_frame(2500, 0.3, 1.0, 31000 + i)
        order = np.concatenate([np.flatnonzero(f.inlier_gt), np.flatnonzero(~f.inlier_gt)])
        f.uv, f.xyz, f.inlier_gt = f.uv[order].copy(), f.xyz[order].copy(), f.inlier_gt[order]
        fr.append(f)
    srv = Server(ctx, budget_bytes=1 << 30, max_slots=64, ransac_opt=ro, honor_options=True)
    ids = [srv.submit(f) for f in fr]
    srv.drain()
    got = {r["id"]: r for r in srv.poll()}
    srv.close()
    for rid, f in zip(ids, fr):
        r = got[rid]
        st, pose, _ = ctx.estimate_absolute_pose(f.uv, f.xyz, Camera_cuda(1, 640, 480, list(f.K)), ro,
                                                 BundleOptions_cuda(), seed=f.seed, honor_options=True)
        assert r["status"] == 0 and r["samples"] == st.details["samples"] >= 3000
        assert r["best_sample"] == st.details["best_sample"]
        assert quat_angle(r["q"], pose.q) < 1e-9 and np.abs(r["t"] - pose.t).max() < 1e-9


def test_pinned_host_inputs_match_pageable(ctx):
    """Frames in page-locked host memory go up without the staging copy (a
    mix of pinned and pageable frames in one call); results are unchanged."""
    import dataclasses

    import torch
    fr = mixed_frames() + [scenes.make_frame(30000, 0.5, 1.0, 9100 + i) for i in range(4)]  # > 512 KiB each
    ref = estimate_batch(ctx, fr, RO)
    keep, mixed = [], []
    for i, f in enumerate(fr):
        if i % 3 == 2:
            mixed.append(f)
            continue
        tu = torch.empty(f.uv.shape, dtype=torch.float64, pin_memory=True)
        tx = torch.empty(f.xyz.shape, dtype=torch.float64, pin_memory=True)
        tu.numpy()[...] = f.uv
        tx.numpy()[...] = f.xyz
        keep += [tu, tx]
        mixed.append(dataclasses.replace(f, uv=tu.numpy(), xyz=tx.numpy()))
    got = estimate_batch(ctx, mixed, RO)
    for a, b in zip(got, ref):
        assert a["status"] == 0 and a["samples"] == b["samples"] and a["best_sample"] == b["best_sample"]
        np.testing.assert_array_equal(a["q"], b["q"])
        np.testing.assert_array_equal(a["t"], b["t"])


def test_staggered_admission_matches_resident_run(ctx):
    """A host-buffer batch above 16 MiB is admitted in groups that join the
    running step loop as their uploads land (later groups wait as kPending).
    Samples, best sample, inliers, masks and poses equal the device-input call,
    which admits every frame before the loop starts."""
    import dataclasses

    import torch

    from turboransac_b200 import DeviceFrame, estimate_batch_device
    rng = np.random.default_rng(77)
    fr = [scenes.make_frame(12000, float(rng.uniform(0.12, 0.8)), 1.0, 41000 + i) for i in range(40)]
    assert sum(40 * f.n for f in fr) >= 16 << 20
    keep, mixed = [], []
    for i, f in enumerate(fr):  # every third frame page-locked (direct upload inside a later group)
        if i % 3:
            mixed.append(f)
            continue
        tu = torch.empty(f.uv.shape, dtype=torch.float64, pin_memory=True)
        tx = torch.empty(f.xyz.shape, dtype=torch.float64, pin_memory=True)
        tu.numpy()[...] = f.uv
        tx.numpy()[...] = f.xyz
        keep += [tu, tx]
        mixed.append(dataclasses.replace(f, uv=tu.numpy(), xyz=tx.numpy()))
    dev = estimate_batch_device(ctx, [DeviceFrame(f) for f in fr], RO)
    tail = list(range(len(fr) - 3, len(fr)))  # frames of the last admission group
    ref_masks = [ctx.estimate_absolute_pose(fr[i].uv, fr[i].xyz, Camera_cuda(1, 640, 480, list(fr[i].K)), RO,
                                            BundleOptions_cuda(), seed=fr[i].seed)[2] for i in tail]
    for _ in range(2):
        got = estimate_batch(ctx, mixed, RO, masks=True)
        assert max(r["steps"] for r in got) >= 2
        for a, b in zip(got, dev):
            assert a["status"] == 0
            assert a["samples"] == b["samples"] and a["best_sample"] == b["best_sample"]
            assert a["num_inliers"] == b["num_inliers"] and a["lm_iterations"] == b["lm_iterations"]
            np.testing.assert_array_equal(a["q"], b["q"])
            np.testing.assert_array_equal(a["t"], b["t"])
        for i, m in zip(tail, ref_masks):
            np.testing.assert_array_equal(got[i]["inliers"].astype(bool), np.asarray(m).astype(bool))


def test_tensor_scoring_batch_matches_fp32_shape(ctx):
    """A batch scored on the tensor cores (points_per_iter=128, several point-chunk
    sizes) gives the FP32 shape's results: the FP64 re-rank decides, the filter
    only has to keep the best within its band."""
    fr = mixed_frames() + [scenes.make_frame(30000, 0.15, 1.0, 9300), scenes.make_frame(700, 0.5, 2.0, 9301)]
    b = Batch(ctx, fr, RO, hyp_per_thread=4, points_per_iter=2)
    b.run()
    b.sync()
    ref = b.results()
    b.close()
    for chunk in (0, 256, 2048, 8192):
        b = Batch(ctx, fr, RO, hyp_per_thread=2, points_per_iter=128, chunk_points=chunk)
        for _ in range(2):
            b.run()
            b.sync()
            got = b.results()
            for r0, r1 in zip(ref, got):
                assert r1["status"] == 0
                assert r1["samples"] == r0["samples"] and r1["best_sample"] == r0["best_sample"]
                assert r1["num_inliers"] == r0["num_inliers"]
                np.testing.assert_array_equal(r1["q"], r0["q"])
                np.testing.assert_array_equal(r1["t"], r0["t"])
        b.close()


def test_server_tensor_scoring_shape_matches_plain(ctx):
    """The server running the tensor-core scoring shape (an autotuner result it
    can be handed) returns the plain call's results."""
    fr = mixed_frames()
    ref = [plain(ctx, f) for f in fr]
    srv = Server(ctx, budget_bytes=2 << 30, max_slots=64,
                 scoring_shape={"hyp_per_thread": 1, "points_per_iter": 128, "chunk_points": 8192})
    ids = {srv.submit(f): i for i, f in enumerate(fr)}
    srv.drain()
    got = srv.poll()
    srv.close()
    assert len(got) == len(fr)
    for r in got:
        d, pose = ref[ids[r["id"]]]
        assert r["status"] == 0
        same(r, r["q"], r["t"], d, pose)


def test_context_close_releases_its_batches_first(ctx):
    """Closing a context closes the batches made on it (they use its workspace);
    a server takes only the device and keeps working after its context closes."""
    from turboransac_b200 import Context
    f = scenes.make_frame(800, 0.5, 1.0, 31001)
    d, pose = plain(ctx, f)
    c2 = Context(0, 1 << 30)
    b = Batch(c2, [f], RO)
    srv = Server(c2, budget_bytes=1 << 30, max_slots=4)
    b.run()
    b.sync()
    (r,) = b.results()
    same(r, r["q"], r["t"], d, pose)
    c2.close()
    assert b._h is None
    b.close()  # a second close is a no-op
    rid = srv.submit(f)
    srv.drain()
    (s,) = srv.poll()
    assert s["id"] == rid and s["status"] == 0
    same(s, s["q"], s["t"], d, pose)
    srv.close()


def test_context_destroy_frees_live_batches_through_the_c_abi(ctx):
    """A C caller that destroys the context before its batch: the context frees
    the batch, later calls on the dead handle are refused and its destroy is a
    no-op (no use after free)."""
    from turboransac_b200 import Context, _lib
    L = _lib.lib()
    f = scenes.make_frame(800, 0.5, 1.0, 31002)
    c2 = Context(0, 1 << 30)
    b = Batch(c2, [f], RO)
    h = b._h
    c2._batches.discard(b)  # as a C caller: only the C library knows about the batch
    L.tbr_context_destroy(c2.handle)
    c2._h = None
    assert L.tbr_batch_run(h) == 1 and b"destroyed" in L.tbr_last_error()
    res = (_lib.FrameResultC * 1)()
    assert L.tbr_batch_results(h, res) == 1
    L.tbr_batch_destroy(h)  # no-op
    b._h = None
    d, pose = plain(ctx, f)  # other contexts are unaffected
    (r,) = estimate_batch(ctx, [f], RO)
    same(r, r["q"], r["t"], d, pose)


def test_batched_calls_reject_what_the_plain_call_rejects(ctx):
    """max_iterations < 1, a threshold <= 0 and non-positive focal lengths are
    INVALID_ARG in every batched entry point, as in the plain call; the context
    keeps working."""
    import dataclasses

    import torch

    from turboransac_b200 import TbrError, estimate_batch_device
    f = scenes.make_frame(500, 0.5, 1.0, 31002)
    bad_cam = dataclasses.replace(f, K=np.array([0.0, 525.0, 319.5, 239.5]))
    bad_opts = [RansacOptions_cuda(max_iterations=0, max_reproj_error=4.0),
                RansacOptions_cuda(max_iterations=1000, max_reproj_error=0.0)]
    from turboransac_b200 import DeviceFrame
    df, dbad = DeviceFrame(f), DeviceFrame(bad_cam)
    for ro in bad_opts:
        with pytest.raises(TbrError):
            estimate_batch(ctx, [f, f], ro)
        with pytest.raises(TbrError):
            estimate_batch_device(ctx, [df], ro)
        with pytest.raises(TbrError):
            Batch(ctx, [f], ro)
        with pytest.raises(TbrError):
            Server(ctx, budget_bytes=1 << 30, max_slots=4, ransac_opt=ro)
    with pytest.raises(TbrError):
        estimate_batch(ctx, [f, bad_cam], RO)
    with pytest.raises(TbrError):
        estimate_batch_device(ctx, [dbad], RO)
    with pytest.raises(TbrError):
        Batch(ctx, [bad_cam], RO)
    torch.cuda.synchronize()
    (r,) = estimate_batch(ctx, [f], RO)
    d, pose = plain(ctx, f)
    same(r, r["q"], r["t"], d, pose)


def test_batched_workload_full_size(ctx, oracle):
    """The bench's batched workload at full size (256 frames, N log-uniform
    [500, 30000]): the resident graph run and the host-buffer call (staggered
    zero-copy admission) agree bit for bit, at least 99 % of the frames meet
    5 deg / 5 cm, and every frame's sample count and pose equal the FP64
    oracle's on the same samples (pose within 1e-6 rad / 1e-6 m)."""
    import os

    from helpers import pose_errors
    from helpers import quat_angle as qa
    fr = scenes.batched_frames(256)
    b = Batch(ctx, fr, RO)
    b.run()
    b.sync()
    res = b.results()
    b.close()
    host = estimate_batch(ctx, fr, RO)
    ok = 0
    for f, a, c in zip(fr, res, host):
        assert a["status"] == 0 and c["status"] == 0
        assert a["candidate_overflow"] == 0 and c["candidate_overflow"] == 0
        assert a["samples"] == c["samples"] and a["best_sample"] == c["best_sample"]
        assert a["num_inliers"] == c["num_inliers"]
        np.testing.assert_array_equal(a["q"], c["q"])
        np.testing.assert_array_equal(a["t"], c["t"])
        ae, te = pose_errors(a["q"], a["t"], f)
        ok += ae < 5 and te < 5
    assert ok >= 0.99 * len(fr)
    q, t, smp = oracle.estimate_batch(fr, samples_per_round=1000, threads=os.cpu_count())
    bad = [(i, res[i]["samples"], int(smp[i]), qa(res[i]["q"], q[i]), float(np.abs(np.asarray(res[i]["t"]) - t[i]).max()))
           for i in range(len(fr))
           if res[i]["samples"] != smp[i] or qa(res[i]["q"], q[i]) >= 1e-6
           or np.abs(np.asarray(res[i]["t"]) - t[i]).max() >= 1e-6]
    assert not bad, bad


def test_serving_workload_matches_plain_and_sample_cap_matches_oracle(ctx, oracle):
    """Requests of the serving workload (N log-uniform [300, 50000], w down to
    0.05) plus a 5 %-inlier frame that runs into the 100000-sample cap: the
    server (rounds per step bounded for serving) returns the plain call's
    results, and the capped frame equals the FP64 oracle's sample count and pose."""
    fr = [scenes.serving_request(i) for i in range(40)] + [scenes.make_frame(20000, 0.05, 1.0, 9400)]
    ref = [plain(ctx, f) for f in fr]
    srv = Server(ctx, budget_bytes=4 << 30, max_slots=64)
    ids = {srv.submit(f): i for i, f in enumerate(fr)}
    srv.drain()
    got = srv.poll(1024)
    srv.close()
    assert len(got) == len(fr)
    for r in got:
        d, pose = ref[ids[r["id"]]]
        assert r["status"] == 0
        assert r["candidate_overflow"] == 0 and d["candidate_overflow"] == 0
        same(r, r["q"], r["t"], d, pose)
    d, pose = ref[-1]
    assert d["samples"] == 100000
    f = fr[-1]
    o = oracle.estimate(f.uv, f.xyz, f.K, 4.0, seed=f.seed, samples_per_round=1000, threads=8)
    assert o["info"].ransac.samples == 100000 and o["info"].ransac.best_sample == d["best_sample"]
    assert quat_angle(pose.q, o["q"]) < 1e-6 and np.abs(pose.t - o["t"]).max() < 1e-6
