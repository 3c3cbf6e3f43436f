"""tbr_msac_score_noalloc: FP64 MSAC scoring for callers that cannot allocate.

Some callers run where device allocation is not theirs to make -- inside
another runtime's memory pool, or in an allocation-free real-time loop. The
entry point takes their device buffers and uses only a fixed scratch array
compiled into the library. This test gives it the hypotheses the engine's
existing scoring entry point (tbr_debug_score_samples) produced and checks
both calls in a row against that entry point's scores and inlier counts, at
the tolerances of the parity tests: scores within 1e-5 relative, counts exact
except for points within 1e-4 px of the threshold. The second call catches
state the shared scratch might carry over from the first. The file is named
to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import near_threshold, normalized, sq_thr

pytestmark = pytest.mark.gpu


def test_noalloc_scores_match_existing_entry_point_twice():
    import torch

    from turboransac_b200 import Context, _lib, scenes
    ctx = Context(0, 1 << 30)
    f = scenes.plain_frame(7)
    rng = np.random.default_rng(3)
    tr = np.stack([rng.choice(f.n, 3, replace=False) for _ in range(300)]).astype(np.int32)
    ids, poses, s32, cnt = ctx.debug_score_samples(f.uv, f.xyz, f.K, 4.0, tr, counts=True)
    H = ids.size
    assert 0 < H <= 1024
    sq = sq_thr(f)
    xn = normalized(f)
    dev = torch.device("cuda", 0)
    x_d = torch.tensor(xn, dtype=torch.float64, device=dev).contiguous()
    X_d = torch.tensor(f.xyz, dtype=torch.float64, device=dev).contiguous()
    P_d = torch.tensor(poses.reshape(H, 12), dtype=torch.float64, device=dev).contiguous()
    scores = torch.empty(H, dtype=torch.float64, device=dev)
    counts = torch.empty(H, dtype=torch.int64, device=dev)
    L = _lib.lib()
    stream = torch.cuda.current_stream(dev).cuda_stream
    focal = 0.5 * (f.K[0] + f.K[1])
    allowed = np.array([near_threshold(poses[k], xn, f.xyz, focal).sum() for k in range(H)])
    for call in range(2):
        scores.fill_(-1.0)
        counts.fill_(-1)
        st = L.tbr_msac_score_noalloc(x_d.data_ptr(), X_d.data_ptr(), f.n, P_d.data_ptr(), H, sq,
                                      scores.data_ptr(), counts.data_ptr(), C.c_void_p(stream))
        assert st == 0, L.tbr_last_error()
        torch.cuda.synchronize(dev)
        s64 = scores.cpu().numpy() / sq
        c64 = counts.cpu().numpy()
        rel = np.abs(s64 - s32.astype(np.float64)) / s64
        assert rel.max() < 1e-5, (call, rel.max())
        assert np.all(np.abs(c64 - cnt) <= allowed), call
    # beyond the fixed maximum: a clear error, nothing launched
    big = torch.zeros((1025, 12), dtype=torch.float64, device=dev)
    st = L.tbr_msac_score_noalloc(x_d.data_ptr(), X_d.data_ptr(), f.n, big.data_ptr(), 1025, sq,
                                  scores.data_ptr(), counts.data_ptr(), C.c_void_p(stream))
    assert st == 1 and b"1024" in L.tbr_last_error()
    ctx.close()
