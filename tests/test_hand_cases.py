"""GPU: hand-made cases with known answers, through the sapporo class --
two bodies against the closed form, a binary 1e-6 apart at unit radius (the
reason the position difference is double-single), a j exactly on the h2
boundary (the list test is strict: h2 > ds2), neighbour counts of 255,
256 and 257 (overflow from 256 on), and a softened pair next to the zero of
its snap (the reason close pairs are summed in FP64)."""
import numpy as np
import pytest

import sapporo2_b200 as sp

pytestmark = pytest.mark.gpu

PRECS = [(sp.DOUBLESINGLE, 1e-6), (sp.DOUBLE, 1e-13)]


def _run(order, prec, x, v, m, xi, vi, h2, eps2, ids=None, ids_i=None, a=None):
    n, ni = len(m), len(xi)
    ids = np.arange(n) if ids is None else ids
    ids_i = np.arange(ni) if ids_i is None else ids_i
    z = np.zeros((n, 3))
    with sp.Sapporo(order=order, precision=prec) as s:
        s.set_j_particles(np.arange(n), ids, np.zeros(n), m, x, v, z, z, z, z)
        s.set_time(0.0)
        s.start(n, ids_i, xi, vi, a if a is not None else np.zeros((ni, 3)), eps2, h2)
        r = s.results(n)
        r["ovf"] = s.read_ngb_list()
        r["lists"] = [s.get_ngb_list(i, sp.NGB_PB) for i in range(ni)]
    return r


def _pair(xj, vj, mj, xi, vi, eps2):
    dr, dv = np.subtract(xj, xi), np.subtract(vj, vi)
    r2 = dr @ dr + eps2
    inv = 1 / np.sqrt(r2)
    acc = mj * inv ** 3 * dr
    jrk = mj * inv ** 3 * (dv - 3 * (dr @ dv) / r2 * dr)
    return acc, jrk, -mj * inv


@pytest.mark.parametrize("order", [sp.FOURTH, sp.SIXTH])
@pytest.mark.parametrize("prec,tol", PRECS)
def test_two_bodies_closed_form(gpu, order, prec, tol):
    x = np.array([[-0.5, 0.1, 0.0], [0.5, -0.1, 0.2]])
    v = np.array([[0.0, 0.5, 0.1], [0.0, -0.5, -0.1]])
    m = np.array([0.4, 0.6])
    eps2 = 1e-4
    r = _run(order, prec, x, v, m, x, v, np.zeros(2), eps2)
    for i, j in ((0, 1), (1, 0)):
        acc, jrk, pot = _pair(x[j], v[j], m[j], x[i], v[i], eps2)
        assert np.linalg.norm(r["acc"][i] - acc) <= tol * np.linalg.norm(acc)
        assert np.linalg.norm(r["jrk"][i] - jrk) <= tol * np.linalg.norm(jrk)
        assert abs(r["pot"][i] - pot) <= tol * abs(pot)
        assert r["nnb"][i] == j


@pytest.mark.parametrize("prec,tol", PRECS)
def test_binary_one_micron_apart_at_unit_radius(gpu, prec, tol):
    """A float position difference would be wrong by up to 6 % here; the
    double-single one is exact to ~1e-9 relative."""
    sep = 1.0e-6
    x = np.array([[1.0, 0.25, -0.5], [1.0 + sep, 0.25, -0.5]])
    v = np.array([[0.0, 1.0, 0.0], [0.0, -1.0, 0.0]])
    m = np.array([1e-6, 1e-6])
    r = _run(sp.FOURTH, prec, x, v, m, x, v, np.full(2, 1e-10), 0.0)
    for i, j in ((0, 1), (1, 0)):
        acc, jrk, pot = _pair(x[j], v[j], m[j], x[i], v[i], 0.0)
        assert np.linalg.norm(r["acc"][i] - acc) <= tol * np.linalg.norm(acc)
        assert np.linalg.norm(r["jrk"][i] - jrk) <= tol * np.linalg.norm(jrk)
        assert r["nnb"][i] == j and r["lists"][i][1] == 1


@pytest.mark.parametrize("prec", [sp.DOUBLESINGLE, sp.DOUBLE])
def test_exact_h2_boundary_is_not_a_neighbour(gpu, prec):
    """ds2 = 0.25 exactly (representable in float and double): h2 = 0.25 does
    not list it (strict h2 > ds2, kernels.cu:584), the next float up does."""
    x = np.array([[0.0, 0.0, 0.0], [0.5, 0.0, 0.0], [0.0, 3.0, 0.0]])
    m = np.full(3, 1e-3)
    v = np.zeros((3, 3))
    up = float(np.nextafter(np.float32(0.25), np.float32(1.0)))
    for h2, want in ((0.25, []), (up, [1])):
        r = _run(sp.FOURTH, prec, x, v, m, x[:1], v[:1], np.array([h2]), 1e-6)
        ovf, n, ids = r["lists"][0]
        assert ovf == 0 and n == len(want) and list(ids) == want


@pytest.mark.parametrize("prec", [sp.DOUBLESINGLE, sp.DOUBLE])
@pytest.mark.parametrize("k", [255, 256, 257])
def test_neighbour_overflow_at_256(gpu, prec, k):
    rng = np.random.default_rng(k)
    n_in, n_out = k, 400
    # k j inside radius 0.4 of the origin, the rest beyond 0.6; i at the origin
    # is not one of the j (its id is absent), so the count is exactly k
    u = rng.normal(size=(n_in + n_out, 3))
    u /= np.linalg.norm(u, axis=1)[:, None]
    rad = np.concatenate([rng.uniform(0.05, 0.4, n_in), rng.uniform(0.6, 2.0, n_out)])
    x = u * rad[:, None]
    m = np.full(len(x), 1e-4)
    v = np.zeros_like(x)
    r = _run(sp.FOURTH, prec, x, v, m, np.zeros((1, 3)), np.zeros((1, 3)), np.array([0.25]),
             1e-6, ids_i=np.array([10 ** 6]))
    ovf, n, ids = r["lists"][0]
    assert n == k
    assert r["ovf"] == (1 if k >= 256 else 0) and ovf == (1 if k >= 256 else 0)
    if k < 256:
        np.testing.assert_array_equal(ids, np.arange(n_in))
    else:  # the list holds 256 of the k, all genuine neighbours
        assert len(ids) == 256 and len(set(ids)) == 256 and ids.max() < n_in
    assert r["nnb"][0] == int(np.argmin(rad))


def _snap_pair(xj, vj, aj, mj, xi, vi, ai, eps2):
    """Snap of one softened pair, in FP64 (kernels.cu:642-667)."""
    dr, dv, da = (np.subtract(q, p) for q, p in ((xj, xi), (vj, vi), (aj, ai)))
    r2 = dr @ dr + eps2
    inv3 = r2 ** -1.5
    al = (dr @ dv) / r2
    be = (dv @ dv + dr @ da) / r2 + al * al
    jij = mj * inv3 * dv - 3 * al * mj * inv3 * dr
    return mj * inv3 * da - 6 * al * jij - 3 * be * mj * inv3 * dr


@pytest.mark.parametrize("near", [16.0, 0.0])
def test_softened_pair_near_its_snap_zero(gpu, near):
    """Two bodies receding radially from each other at r^2 = 1.5 eps^2 (1 +
    1e-4), just off the separation where the radial snap of a softened pair
    vanishes (6 r^2 = 9 eps^2): the snap is 3e-4 of its scale there, so FP32
    rounding of the pair's terms alone is a ~2e-3 relative error.  The FP64
    near-pair sum (default factor 16: pairs within 4 softening lengths) keeps
    it near 1e-8 (the FP32 rounding of the stored mass); with the factor 0
    (every pair in FP32, as the reference's double-single kernels) it is
    above 1e-4.  One of the two is at unit radius, like a cluster particle."""
    eps2 = 1e-6
    r = np.sqrt(1.5 * eps2 * (1 + 1e-4))
    x = np.array([[1.0, 0.0, 0.0], [1.0 + r, 0.0, 0.0]])
    # velocities exact in FP32, so the records' rounding does not enter
    v = np.array([[0.25, 0.0, 0.0], [1.25, 0.0, 0.0]])
    m = np.array([1e-6, 1e-6])
    z = np.zeros((2, 3))
    with sp.Sapporo(order=sp.SIXTH, precision=sp.DOUBLESINGLE) as s:
        s.set_near(near)
        s.set_j_particles(np.arange(2), np.arange(2), np.zeros(2), m, x, v, z, z, z, z)
        s.set_time(0.0)
        s.start(2, np.arange(2), x, v, z, eps2, np.zeros(2))
        got = s.results(2)
    for i, j in ((0, 1), (1, 0)):
        want = _snap_pair(x[j], v[j], z[j], m[j], x[i], v[i], z[i], eps2)
        scale = m[j] * (r * r + eps2) ** -1.5 / np.sqrt(r * r + eps2)  # |dv| = 1
        err = np.linalg.norm(got["snp"][i] - want) / np.linalg.norm(want)
        print(f"near {near}: |snap| / scale = {np.linalg.norm(want) / scale:.1e}, rel err {err:.2e}")
        if near > 0:
            assert err < 1e-5
        else:
            assert err > 1e-4
