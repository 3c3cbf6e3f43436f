"""Device-side waits are bounded: a wait that nothing completes gives up, the
host reads TIMEOUT from the device's error word, and the context keeps working.
No GPU fault, trap or hang is involved: the kernel polls an mbarrier a fixed
number of times and returns."""
import numpy as np
import pytest

from turboransac_b200 import BundleOptions_cuda, Camera_cuda, RansacOptions_cuda, TbrError, scenes

pytestmark = pytest.mark.gpu


def test_expired_wait_reports_timeout_and_context_survives(ctx, oracle):
    for polls in (1, 1 << 12):
        with pytest.raises(TbrError) as e:
            ctx.debug_bounded_wait(polls)
        assert e.value.status == 4  # TBR_ERR_TIMEOUT
    with pytest.raises(TbrError) as e:
        ctx.debug_bounded_wait(0)
    assert e.value.status == 1  # INVALID_ARG: the limit must be 1 .. 2^22
    # The next estimate on the same context is unaffected.
    f = scenes.plain_frame(2)
    ro = RansacOptions_cuda(max_iterations=1000, success_prob=0.9999, max_reproj_error=4.0)
    st, pose, inl = ctx.estimate_absolute_pose(f.uv, f.xyz, Camera_cuda(1, 640, 480, list(f.K)), ro,
                                               BundleOptions_cuda(), seed=f.seed)
    o = oracle.estimate(f.uv, f.xyz, f.K, 4.0, seed=f.seed, samples_per_round=1000)
    assert st.details["samples"] == o["info"].ransac.samples
    assert st.details["best_sample"] == o["info"].ransac.best_sample
    np.testing.assert_array_equal(inl, o["inliers"])
