"""Submitted batches (tbr_estimate_batch_submit / tbr_estimate_batch_collect):
every frame's result and inlier mask is the one tbr_estimate_batch gives --
with two batches in flight, collected out of order, across the wait of a third
submission, across synchronous calls on the same context, after a refused
submission, and never after the context is gone."""
import numpy as np
import pytest

from turboransac_b200 import (Camera_cuda, Context, DeviceFrame, RansacOptions_cuda, TbrError, estimate_batch,
                              estimate_batch_device, estimate_batch_device_submit, estimate_batch_submit, scenes)

pytestmark = pytest.mark.gpu

RO = RansacOptions_cuda(max_iterations=1000, max_reproj_error=4.0)


def same(got, ref, masks=True):
    assert len(got) == len(ref)
    for a, b in zip(got, ref):
        assert a["status"] == 0
        assert a["samples"] == b["samples"] and a["best_sample"] == b["best_sample"]
        assert a["num_inliers"] == b["num_inliers"]
        np.testing.assert_array_equal(a["q"], b["q"])
        np.testing.assert_array_equal(a["t"], b["t"])
        if masks:
            np.testing.assert_array_equal(a["inliers"], b["inliers"])


def groups():
    a = scenes.batched_frames(10, scale=0.5)
    b = scenes.batched_frames(12, first=40, scale=0.5) + [scenes.make_frame(6000, 0.08, 1.0, 9301)]
    # Above 16 MiB of pageable host data: admitted in groups, the late ones
    # copied into the call's staging buffer and read from there during the run.
    c = [scenes.make_frame(30000, 0.5, 1.0, 9310 + i) for i in range(15)]
    return a, b, c


def test_submitted_batches_match_the_batch_call(ctx):
    a, b, c = groups()
    ref = [estimate_batch(ctx, g, RO, masks=True) for g in (a, b, c)]
    ta = estimate_batch_submit(ctx, a, RO)
    tb = estimate_batch_submit(ctx, b, RO)
    tc = estimate_batch_submit(ctx, c, RO)  # waits for a's device work first
    same(tb.collect(masks=True), ref[1])  # out of order
    same(ta.collect(masks=True), ref[0])
    td = estimate_batch_submit(ctx, a, RO)
    same(tc.collect(masks=True), ref[2])
    same(td.collect(), ref[0], masks=False)
    with pytest.raises(RuntimeError):
        td.collect()


def test_synchronous_calls_between_submit_and_collect(ctx):
    a, b, c = groups()
    ref_a, ref_b = estimate_batch(ctx, a, RO, masks=True), estimate_batch(ctx, b, RO, masks=True)
    f = b[-1]
    st0, pose0, _ = ctx.estimate_absolute_pose(f.uv, f.xyz, Camera_cuda(1, 640, 480, list(f.K)), RO, seed=f.seed)
    ta = estimate_batch_submit(ctx, a, RO)
    tb = estimate_batch_submit(ctx, b, RO)
    st, pose, _ = ctx.estimate_absolute_pose(f.uv, f.xyz, Camera_cuda(1, 640, 480, list(f.K)), RO, seed=f.seed)
    assert st.details["samples"] == st0.details["samples"]
    np.testing.assert_array_equal(pose.q, pose0.q)
    same(estimate_batch(ctx, a[:4], RO, masks=True), ref_a[:4])
    same(ta.collect(masks=True), ref_a)
    same(tb.collect(masks=True), ref_b)


def test_submission_beyond_the_free_slots_is_refused(ctx):
    small = [scenes.make_frame(40, 0.7, 0.5, 9400 + i) for i in range(600)]
    ref = estimate_batch(ctx, small[:8], RO)
    t1 = estimate_batch_submit(ctx, small, RO)
    with pytest.raises(TbrError) as e:  # 1200 frames held at once: more than the context's 1024 slots
        estimate_batch_submit(ctx, small, RO)
    assert e.value.status == 7
    got = t1.collect()
    same(got[:8], ref, masks=False)
    t2 = estimate_batch_submit(ctx, small[:8], RO)  # the slots are free again
    same(t2.collect(), ref, masks=False)


def test_collect_after_context_destroy_is_refused(ctx):
    c2 = Context(0, 1 << 30)
    f = scenes.make_frame(800, 0.5, 1.0, 9500)
    t = estimate_batch_submit(c2, [f], RO)
    c2.close()  # frees the uncollected ticket
    with pytest.raises(TbrError) as e:
        t.collect()
    assert e.value.status == 1
    (r,) = estimate_batch_submit(ctx, [f], RO).collect()  # other contexts are unaffected
    (ref,) = estimate_batch(ctx, [f], RO)
    same([r], [ref], masks=False)


def test_device_input_submissions_match_the_device_call(ctx):
    """Device-resident correspondences through the submitted form, in flight
    beside host submissions: the results of the device call and of the host
    call, bit for bit, masks included."""
    import torch
    a, b, c = groups()
    da, dc = [DeviceFrame(f) for f in a], [DeviceFrame(f) for f in c]
    torch.cuda.synchronize()
    ref_a = estimate_batch_device(ctx, da, RO)
    ref_b = estimate_batch(ctx, b, RO)
    ref_c = estimate_batch(ctx, c, RO, masks=True)
    t1 = estimate_batch_device_submit(ctx, da, RO)
    t2 = estimate_batch_submit(ctx, b, RO)
    t3 = estimate_batch_device_submit(ctx, dc, RO)  # waits for t1's device work first
    same(t1.collect(), ref_a, masks=False)
    same(t3.collect(masks=True), ref_c)
    same(t2.collect(), ref_b, masks=False)
    with pytest.raises(ValueError):  # host arrays are refused by the device form
        estimate_batch_device_submit(ctx, a, RO)


def test_submission_beyond_the_free_workspace_is_refused():
    """A small workspace: the second batch's points do not fit beside the
    uncollected first one (TBR_ERR_OOM); the first is unaffected and the
    second fits once the first is collected."""
    c2 = Context(0, 512 << 20)
    try:
        big = [scenes.make_frame(30000, 0.5, 1.0, 9600 + i) for i in range(40)]
        ref = estimate_batch(c2, big, RO)
        t1 = estimate_batch_submit(c2, big, RO)
        with pytest.raises(TbrError) as e:
            estimate_batch_submit(c2, big, RO)
        assert e.value.status == 2
        same(t1.collect(), ref, masks=False)
        same(estimate_batch_submit(c2, big, RO).collect(), ref, masks=False)
    finally:
        c2.close()
