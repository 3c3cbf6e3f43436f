"""Arithmetic of the tensor-core scoring shape, on the CPU: each FP32 operand of
the projection z = c . [X 1] is split into a TF32 part (rounded to nearest, 10
explicit mantissa bits) and the TF32-rounded remainder; the four cross terms are
exact FP32 products, and their FP32 sum stays within 2^-20 of the magnitude sum
of the exact product -- near FP32 accuracy, where one TF32 product per term is
only good to about 2^-11. The device kernel's own scores are checked against
the FP64 oracle by the GPU parity tests; this pins the split that lets TF32 MMA
stand in for the FP32 projection."""
import numpy as np


def tf32_rn(x):
    """Round float32 values to TF32 (10 explicit mantissa bits), half away from
    zero on the magnitude, as the kernel's bit operation does."""
    u = np.asarray(x, np.float32).view(np.uint32)
    return ((u + np.uint32(0x1000)) & np.uint32(0xFFFFE000)).view(np.float32)


def split(x):
    hi = tf32_rn(x)
    lo = tf32_rn((x - hi).astype(np.float32))
    return hi, lo


def scoring_rows(rng, m):
    """FP32 scoring rows of m hypotheses: rows 0 and 1 divided by the normalised
    threshold (4 px at f = 525), translation in the points' centred frame."""
    q = rng.normal(size=(m, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    R = np.stack([np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)], -1),
                  np.stack([2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)], -1),
                  np.stack([2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)], -1)], 1)
    t = np.concatenate([rng.uniform(-0.5, 0.5, (m, 2)), rng.uniform(1.0, 3.0, (m, 1))], 1)
    tau = 4.0 / 525.0
    rows = np.concatenate([R, t[:, :, None]], 2)  # (m, 3, 4)
    rows[:, :2] /= tau
    return rows.astype(np.float32)


def test_split_operands_keep_fp32_accuracy():
    rng = np.random.default_rng(7)
    rows = scoring_rows(rng, 64).reshape(-1, 4)                 # (192, 4)
    pts = rng.uniform(-2.0, 2.0, (4096, 3)).astype(np.float32)  # centred world points
    A = np.concatenate([pts, np.ones((len(pts), 1), np.float32)], 1)
    exact = A.astype(np.float64) @ rows.astype(np.float64).T    # (points, row)
    mag = np.abs(A.astype(np.float64)) @ np.abs(rows.astype(np.float64)).T
    ah, al = split(A)
    ch, cl = split(rows)
    al[:, 3] = 0.0  # the constant 1 column is exact: its remainder is not a K term
    # The four cross terms per K index, summed in FP32 in a shuffled order (the
    # MMA's order is not specified).
    terms = [ah[:, None, :] * ch[None, :, :], al[:, None, :] * ch[None, :, :],
             ah[:, None, :] * cl[None, :, :], al[:, None, :] * cl[None, :, :]]
    terms = np.concatenate(terms, 2).astype(np.float32)  # (points, rows, 16)
    order = rng.permutation(terms.shape[2])
    z = np.zeros(exact.shape, np.float32)
    for k in order:
        z = (z + terms[:, :, k]).astype(np.float32)
    err = np.abs(z.astype(np.float64) - exact)
    assert (err <= 2.0 ** -20 * mag).all(), (err / mag).max()
    # A plain FP32 product reaches about 2^-22 here; one TF32 product per term
    # only about 2^-10: the split is what makes the tensor-core projection an
    # FP32 one.
    z1 = (tf32_rn(A).astype(np.float64) @ tf32_rn(rows).astype(np.float64).T)
    assert (np.abs(z1 - exact) / mag).max() > 2.0 ** -14


def test_cross_term_products_are_exact_in_fp32():
    rng = np.random.default_rng(8)
    a = rng.normal(size=100000).astype(np.float32) * np.float32(100.0)
    b = rng.normal(size=100000).astype(np.float32)
    for x in split(a):
        for y in split(b):
            p32 = (x * y).astype(np.float64)
            p64 = x.astype(np.float64) * y.astype(np.float64)
            np.testing.assert_array_equal(p32, p64)
