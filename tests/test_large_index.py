"""GPU: index ranges beyond 2^31 bytes -- 2^23 j-particles (512 MB of force
records, 1.5 GB of state) against a sample of i, and 2^22 i-particles with
neighbour lists (4 GB of list slots) against a small j set; sampled i are
checked against the FP64 oracle."""
import numpy as np
import pytest

import sapporo2_b200 as sp
from oracle import oracle as O
from tests import cases as T

pytestmark = pytest.mark.gpu


def _system(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1.0, 1.0, (n, 3))
    v = rng.normal(0.0, 0.3, (n, 3))
    m = np.full(n, 1.0 / n)
    return x, v, m


def test_eight_million_j(gpu):
    nj, ni = 1 << 23, 512
    x, v, m = _system(nj, 41)
    ids = np.arange(nj, dtype=np.int32)
    sel = np.sort(np.random.default_rng(42).choice(nj, ni, replace=False))
    z = np.zeros((nj, 3))
    with sp.Sapporo(order=sp.FOURTH, precision=sp.DOUBLESINGLE) as s:
        s.set_j_particles(ids, ids, np.zeros(nj), m, x, v, z, z)
        s.set_time(0.0)
        s.start(nj, ids[sel], x[sel], v[sel], None, 1e-6, np.zeros(ni))
        got = s.results(nj)
    want = O.force_subset(1, np.arange(ni, dtype=np.int32), x[sel], v[sel], None,
                          np.zeros(ni), ids[sel], x, v, None, m, ids, 1e-6)
    T.check_forces(got, want, 1)


def test_four_million_i_with_lists(gpu):
    nj, ni = 512, 1 << 22
    xj, vj, mj = _system(nj, 43)
    xi, vi, _ = _system(ni, 44)
    idj = np.arange(nj, dtype=np.int32)
    idi = np.arange(nj, nj + ni, dtype=np.int32)  # no i is a j
    h2 = np.full(ni, 0.05)
    z = np.zeros((nj, 3))
    with sp.Sapporo(order=sp.FOURTH, precision=sp.DOUBLESINGLE, n_pipes=ni) as s:
        s.set_j_particles(idj, idj, np.zeros(nj), mj, xj, vj, z, z)
        s.set_time(0.0)
        s.start(nj, idi, xi, vi, None, 1e-6, h2)
        got = s.results(nj)
        cnt, lst = s.neighbour_lists()
    sel = np.sort(np.random.default_rng(45).choice(ni, 1024, replace=False))
    want = O.force(1, xi[sel], vi[sel], None, h2[sel], idi[sel], xj, vj, None, mj, idj, 1e-6)
    T.check_forces({f: got[f][sel] for f in ("acc", "pot", "jrk")}, want, 1)
    assert np.mean(want["ngb_count"]) > 1  # lists are exercised
    for q, i in enumerate(sel):
        g = set(int(t) for t in lst[i, :int(cnt[i])])
        w = set(int(t) for t in want["ngb_list"][q, :int(want["ngb_count"][q])])
        for jd in g ^ w:  # only pairs within 1e-6 of the h2 boundary may differ
            d2 = float(((xj[jd] - xi[i]) ** 2).sum())
            assert abs(d2 - h2[i]) <= 1e-6 * h2[i], (i, jd, d2)
    # the last i (the largest list offset) was written where it belongs
    w_last = O.force(1, xi[-1:], vi[-1:], None, h2[-1:], idi[-1:], xj, vj, None, mj, idj, 1e-6)
    assert int(cnt[-1]) == int(w_last["ngb_count"][0])
