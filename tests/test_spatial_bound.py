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


def _morton30(p, lo, scale):
    q = np.clip((p - lo) * scale, 0, 1023).astype(np.int64)
    k = np.zeros(len(p), np.int64)
    for b in range(10):
        for c in range(3):
            k |= ((q[:, c] >> b) & 1) << (3 * b + c)
    return k


def test_far_tiles_never_hold_a_nearest_neighbour():
    """The far test of the force kernel, restated in numpy on a clustered
    system: j in Morton order in tiles of 256 with boxes of the float high
    parts, i (a subset) in Morton order in warps of 128, each i's bound the
    exact minimum ds2 over the tile whose key range holds its key.  A tile
    is far for a warp when every i is >= far_c max(|x|) from its box and
    the squared distance, less the margin, exceeds the bound; then no pair
    of the tile may be the i's nearest neighbour (checked by brute force),
    and a large share of the tiles is far."""
    from sapporo2_b200 import ic
    rng = np.random.default_rng(3)
    x, _, _ = ic.plummer(20000, seed=11)
    x, _, _, _ = ic.add_binaries(x, np.zeros_like(x), np.full(len(x), 1.0 / len(x)), 0.1, 12)
    n = len(x)
    far_c = 2.0 ** -23 / DELTA
    shrink = min(0.9999, 1 - 8 * DELTA)
    hi = x.astype(np.float32).astype(np.float64)
    lo, scale = hi.min(0), 1023.99 / (hi.max(0) - hi.min(0)).max()
    kj = _morton30(hi, lo, scale)
    oj = np.argsort(kj, kind="stable")
    xs, ks, hs = x[oj], kj[oj], hi[oj]
    nt = (n + 255) // 256
    tiles = [slice(t * 256, min(n, (t + 1) * 256)) for t in range(nt)]
    blo = np.array([hs[t].min(0) for t in tiles])
    bhi = np.array([hs[t].max(0) for t in tiles])
    babs = np.array([np.abs(hs[t]).max() for t in tiles])
    tkey = ks[::256]
    sel = rng.choice(n, 4096, replace=False)
    ki = _morton30(hi[sel], lo, scale)
    sel = sel[np.argsort(ki, kind="stable")]
    far_pairs = 0
    for w in range(0, len(sel), 128):
        idx = sel[w:w + 128]
        xi, hi_i = x[idx], hi[idx]
        seed = np.maximum(np.searchsorted(tkey, _morton30(hi_i, lo, scale), side="right") - 1, 0)
        d2_all = ((xs[None, :, :] - xi[:, None, :]) ** 2).sum(2)
        d2_all[d2_all == 0] = np.inf  # the self pair (same particle)
        bound = np.array([d2_all[q, tiles[seed[q]]].min() for q in range(len(idx))])
        nn = d2_all.min(1)
        for t, tsl in enumerate(tiles):
            g = np.maximum(0, np.maximum(blo[t][None] - hi_i, hi_i - bhi[t][None]))
            g2 = (g ** 2).sum(1)
            xm = np.maximum(babs[t], np.abs(hi_i).max(1)) * far_c
            if not np.all((g2 >= xm ** 2) & (g2 * shrink > bound)):
                continue
            far_pairs += 1
            assert np.all(d2_all[:, tsl].min(1) > nn), (w, t)
    assert far_pairs > 0.3 * nt * (len(sel) // 128), far_pairs
