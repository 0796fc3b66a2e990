"""CPU: the accuracy bound behind the far tiles of the spatial mode.

For positions rounded to float (the high parts of the double-single split),
the single-float difference xj_hi - xi_hi differs from the exact difference
by at most 2^-24 (|xi| + |xj|) per component plus its own rounding.  A far
tile is one whose box (of high parts) is at least |x|max * 2^-23 / delta
from the warp's box, so every component error is within (delta + 2^-24) of
the pair distance.  Checked here in numpy on pairs drawn at every scale,
including the close binaries that make the double-single path necessary.
"""
import numpy as np

DELTA = 1e-6


def _far_errors(x_i, x_j, delta):
    hi_i = x_i.astype(np.float32)
    hi_j = x_j.astype(np.float32)
    d_hi = (hi_j.astype(np.float64) - hi_i.astype(np.float64))
    gap = np.sqrt((d_hi ** 2).sum(1))  # a pair is its own box: gap = |dr_hi|
    xmax = np.maximum(np.abs(hi_i).max(1), np.abs(hi_j).max(1)).astype(np.float64)
    far = gap >= xmax * 2.0 ** -23 / delta
    d_f32 = (hi_j - hi_i).astype(np.float64)  # the kernel's 3-operation difference
    exact = x_j - x_i
    dist = np.sqrt((exact ** 2).sum(1))
    err = np.abs(d_f32 - exact).max(1) / dist
    return far, err


def test_far_pairs_meet_the_bound():
    rng = np.random.default_rng(0)
    n = 400_000
    scale = 10.0 ** rng.uniform(-3, 1, n)
    x_i = rng.normal(size=(n, 3)) * scale[:, None]
    sep = 10.0 ** rng.uniform(-7, 1, n)  # binaries 1e-7 apart up to distant pairs
    u = rng.normal(size=(n, 3))
    x_j = x_i + sep[:, None] * u / np.linalg.norm(u, axis=1)[:, None]
    for delta in (1e-6, 1e-5, 1e-4):
        far, err = _far_errors(x_i, x_j, delta)
        assert far.sum() > n // 10
        assert np.all(err[far] <= delta + 2.0 ** -24), (delta, err[far].max())


def test_close_pairs_are_never_far():
    """The pairs that need the double-single difference (error of the
    single-float one above delta) all fail the far test."""
    rng = np.random.default_rng(1)
    n = 200_000
    x_i = rng.uniform(-2, 2, size=(n, 3))
    sep = 10.0 ** rng.uniform(-8, -4, n)
    u = rng.normal(size=(n, 3))
    x_j = x_i + sep[:, None] * u / np.linalg.norm(u, axis=1)[:, None]
    far, err = _far_errors(x_i, x_j, DELTA)
    assert np.all(~far[err > DELTA + 2.0 ** -24])
    assert np.mean(err > DELTA) > 0.5  # most of these pairs do need it
