"""tbr_msac_score_noalloc: FP64 MSAC scoring for callers that cannot allocate.

Some callers run where device allocation is not theirs to make -- inside
another runtime's memory pool, or in an allocation-free real-time loop. The
entry point takes their device buffers and uses only a fixed scratch array
compiled into the library. These tests give it the hypotheses the engine's
existing scoring entry point (tbr_debug_score_samples) produced and check two
calls in a row against that entry point (FP32 scores within 1e-5 relative,
counts exact except for points within 1e-4 px of the threshold) and against
the FP64 oracle, which restates msac.cuh:18-56 and ransac.cuh:322 (scores
within 1e-12 relative, counts exact). The second call catches state the
shared scratch might carry over from the first; free device memory is the
same before and after the calls. The file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import near_threshold, normalized, sq_thr

pytestmark = pytest.mark.gpu


def _device_arrays(dev, xn, xyz, poses):
    import torch
    x_d = torch.tensor(xn, dtype=torch.float64, device=dev).contiguous()
    X_d = torch.tensor(xyz, dtype=torch.float64, device=dev).contiguous()
    P_d = torch.tensor(np.asarray(poses).reshape(-1, 12), dtype=torch.float64, device=dev).contiguous()
    H = P_d.shape[0]
    return x_d, X_d, P_d, torch.empty(H, dtype=torch.float64, device=dev), torch.empty(H, dtype=torch.int64,
                                                                                        device=dev)


def _call(L, x_d, X_d, n, P_d, H, sq, scores, counts, stream):
    return L.tbr_msac_score_noalloc(x_d.data_ptr(), X_d.data_ptr(), n, P_d.data_ptr(), H, sq, scores.data_ptr(),
                                    counts.data_ptr(), C.c_void_p(stream))


def _oracle_scores(oracle, xn, xyz, poses, sq):
    out = [oracle.msac(xn, xyz, P, sq) for P in np.asarray(poses).reshape(-1, 12)]
    return np.array([o[0] for o in out]), np.array([o[1] for o in out], np.int64)


def test_noalloc_scores_match_existing_entry_point_and_oracle_twice(oracle):
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
    x_d, X_d, P_d, scores, counts = _device_arrays(dev, xn, f.xyz, poses)
    L = _lib.lib()
    stream = torch.cuda.current_stream(dev).cuda_stream
    focal = 0.5 * (f.K[0] + f.K[1])
    allowed = np.array([near_threshold(poses[k], xn, f.xyz, focal).sum() for k in range(H)])
    o_s, o_c = _oracle_scores(oracle, xn, f.xyz, poses, sq)
    # A first round loads the device code it uses (this library's and torch's
    # fill and copy kernels); after it no call may change free device memory.
    scores.fill_(-1.0)
    counts.fill_(-1)
    assert _call(L, x_d, X_d, f.n, P_d, H, sq, scores, counts, stream) == 0, L.tbr_last_error()
    torch.cuda.synchronize(dev)
    scores.cpu(), counts.cpu()
    torch.cuda.synchronize(dev)
    free0 = torch.cuda.mem_get_info(dev)[0]
    for call in range(2):
        scores.fill_(-1.0)
        counts.fill_(-1)
        st = _call(L, x_d, X_d, f.n, P_d, H, sq, scores, counts, stream)
        assert st == 0, L.tbr_last_error()
        torch.cuda.synchronize(dev)
        s64 = scores.cpu().numpy()
        c64 = counts.cpu().numpy()
        rel = np.abs(s64 / sq - s32.astype(np.float64)) / (s64 / sq)
        assert rel.max() < 1e-5, (call, rel.max())
        assert np.all(np.abs(c64 - cnt) <= allowed), call
        assert np.abs(s64 - o_s).max() <= 1e-12 * np.abs(o_s).max(), (call, np.abs(s64 - o_s).max())
        np.testing.assert_array_equal(c64, o_c)
    assert torch.cuda.mem_get_info(dev)[0] == free0
    # beyond the fixed maximum, or a threshold that is not positive and finite:
    # a clear error, nothing launched
    big = torch.zeros((1025, 12), dtype=torch.float64, device=dev)
    st = _call(L, x_d, X_d, f.n, big, 1025, sq, scores, counts, stream)
    assert st == 1 and b"1024" in L.tbr_last_error()
    for bad in (0.0, -1.0, float("nan"), float("inf")):
        st = _call(L, x_d, X_d, f.n, P_d, H, bad, scores, counts, stream)
        assert st == 1 and b"sq_threshold" in L.tbr_last_error()
    ctx.close()


@pytest.mark.parametrize("n,H", [(5, 7), (31, 64), (2000, 1024)], ids=["n5", "n31", "poses1024"])
def test_noalloc_edge_sizes_match_oracle(oracle, n, H):
    """Fewer points than the 32 point chunks (empty chunks) and exactly the
    1024-pose maximum, two calls in a row, against the FP64 oracle."""
    import torch

    from turboransac_b200 import _lib, scenes
    f = scenes.make_frame(n, 0.6, 1.0, 500 + n)
    xn = normalized(f)
    sq = sq_thr(f)
    rng = np.random.default_rng(n)
    poses = []
    for _ in range(H):  # ground truth perturbed, so that counts vary between poses
        dq = np.r_[1.0, 0.02 * rng.standard_normal(3)]
        R = f.R_gt @ scenes.quat_to_rotmat(dq / np.linalg.norm(dq))
        t = f.t_gt + 0.05 * rng.standard_normal(3)
        poses.append(np.hstack([R, t[:, None]]))
    poses = np.array(poses)
    dev = torch.device("cuda", 0)
    x_d, X_d, P_d, scores, counts = _device_arrays(dev, xn, f.xyz, poses)
    L = _lib.lib()
    stream = torch.cuda.current_stream(dev).cuda_stream
    o_s, o_c = _oracle_scores(oracle, xn, f.xyz, poses, sq)
    for call in range(2):
        scores.fill_(-1.0)
        counts.fill_(-1)
        assert _call(L, x_d, X_d, n, P_d, H, sq, scores, counts, stream) == 0, L.tbr_last_error()
        torch.cuda.synchronize(dev)
        s64 = scores.cpu().numpy()
        assert np.abs(s64 - o_s).max() <= 1e-12 * np.abs(o_s).max(), (call, np.abs(s64 - o_s).max())
        np.testing.assert_array_equal(counts.cpu().numpy(), o_c)
