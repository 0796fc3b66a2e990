"""GPU parity: the library (through the sapporo class) against the FP64
oracle on seeded Plummer inputs, both precisions, both orders."""
import numpy as np
import pytest

import sapporo2_b200 as sp
from tests import cases as T

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("eps2", [1e-6, 0.0])
@pytest.mark.parametrize("order", [1, 2])
def test_fp64_kernel_matches_oracle(gpu, order, eps2):
    case = T.build_case(order, 2048, seed=11, binaries=0.1, eps2=eps2, t_spread=eps2 > 0)
    want = T.oracle_force(case)
    got = T.run_library(case, sp.DOUBLE)
    # all-FP64 kernel: only summation order and rsqrt rounding differ.  The
    # unsoftened snap is ill-conditioned (each binary's two a_j ~5e8 cancel):
    # the oracle summed in two j orders differs by 4e-11 median, 5e-9 max
    med, mx = (1e-13, 1e-9) if eps2 > 0 else (1e-9, 1e-7)
    st = T.check_forces(got, want, order, median_tol=med, max_tol=mx)
    assert T.check_nn(case, got["nnb"], want) == 0
    T.check_neighbours(case, got["ngb_sets"], got["ngb_count"], want)
    print(st)


@pytest.mark.parametrize("eps2", [1e-6, 0.0])
@pytest.mark.parametrize("order", [1, 2])
def test_mixed_kernel_matches_oracle(gpu, order, eps2):
    """Softened and unsoftened (eps2 = 0: no near-pair FP64 sums, binaries
    1e-6..1e-4 apart in plain double-single arithmetic).  Unsoftened, the j
    are given at t_i: a Taylor step of up to 7/1024 along the orbits of such
    binaries (accelerations ~5e8) would throw them far out of the system.

    Unsoftened 6th order is checked without snap: the snap of every i sums
    m r^-3 (a_j - a_i) over each binary's two members, whose accelerations
    (~5e8, opposite) cancel; taken in FP32, as the reference's sixth_DS
    kernel takes them too (kernels.cu:642-644, Tvel = float), their rounding
    (~15 per component) leaves a snap error of ~1e-2 relative.  That case
    needs the FP64 kernels (the reference's 6th-order interface defaults to
    them, sapporo6thlib.cpp:29), which test_fp64_kernel_matches_oracle
    checks at eps2 = 0."""
    case = T.build_case(order, 2048, seed=12, binaries=0.1, eps2=eps2, t_spread=eps2 > 0)
    want = T.oracle_force(case)
    got = T.run_library(case, sp.DOUBLESINGLE)
    fields = ["acc", "pot", "jrk"] if (order == 2 and eps2 == 0) else None
    st = T.check_forces(got, want, order, fields=fields)
    T.check_nn(case, got["nnb"], want)
    T.check_neighbours(case, got["ngb_sets"], got["ngb_count"], want)
    print(st)


@pytest.mark.parametrize("order,precision", [(1, 1), (2, 1), (2, 2)])
@pytest.mark.parametrize("launch", [(1, 2, 0), (2, 2, 3), (4, 2, 0), (8, 2, 5), (16, 1, 2),
                                    (32, 1, 0), (1, 1, 7), (1, 4, 0), (2, 4, 3)])
def test_launch_shapes_agree(gpu, order, precision, launch):
    """Every (threads-per-i, i-per-thread, j-slices) shape gives the same
    physics; ragged i and j counts exercise the partial tiles."""
    if launch[1] == 4 and precision == sp.DOUBLE:
        pytest.skip("4 i per thread is a mixed-precision shape")
    case = T.build_case(order, 1000, seed=13, binaries=0.1)
    sel = np.arange(3, 900, 2)
    want = T.oracle_force(case, sel=sel)
    got = T.run_library(case, precision, sel=sel, launch=launch)
    tol = (1e-13, 1e-9) if precision == sp.DOUBLE else (T.MEDIAN_TOL, T.MAX_TOL)
    T.check_forces(got, want, order, *tol)
    T.check_nn(case, got["nnb"], want, sel=sel)
    T.check_neighbours(case, got["ngb_sets"], got["ngb_count"], want, sel=sel)


@pytest.mark.parametrize("order", [1, 2])
@pytest.mark.parametrize("permute", [False, True])
@pytest.mark.parametrize("launch", [(1, 4, 0), (1, 2, 0), (2, 2, 3)])
def test_self_pair_both_tile_paths(gpu, order, permute, launch):
    """Tiles whose ids cannot contain a warp's i skip the self-pair compare;
    ids in address order (mostly skipped) and permuted ids (never skipped)
    give the oracle's answer, with the self pair excluded either way."""
    case = T.build_case(order, 1500, seed=15, binaries=0.1, permute_ids=permute)
    want = T.oracle_force(case)
    got = T.run_library(case, sp.DOUBLESINGLE, launch=launch)
    T.check_forces(got, want, order)
    T.check_nn(case, got["nnb"], want)
    assert not np.any(got["nnb"] == case["id"])
    T.check_neighbours(case, got["ngb_sets"], got["ngb_count"], want)


@pytest.mark.parametrize("ni", [1, 2, 31, 127, 129, 255, 257])
def test_small_active_sets(gpu, ni):
    case = T.build_case(2, 3000, seed=14)
    sel = np.random.default_rng(ni).choice(3000, ni, replace=False)
    want = T.oracle_force(case, sel=sel)
    got = T.run_library(case, sp.DOUBLESINGLE, sel=sel)
    T.check_forces(got, want, 2)
    T.check_nn(case, got["nnb"], want, sel=sel)
    T.check_neighbours(case, got["ngb_sets"], got["ngb_count"], want, sel=sel)


@pytest.mark.parametrize("eps2", [0.0, 1e-6])
def test_fp64_kernel_rsqrt_over_scales(gpu, eps2):
    """1/sqrt in the FP64 kernels over eight decades of distance: one j at
    the origin, i at distances 1e-6 .. 1e2, against long-double sums."""
    rng = np.random.default_rng(17)
    n_i = 2000
    d = 10.0 ** rng.uniform(-6, 2, n_i)
    u = rng.normal(size=(n_i, 3))
    xi = d[:, None] * u / np.linalg.norm(u, axis=1)[:, None]
    with sp.Sapporo(order=sp.FOURTH, precision=sp.DOUBLE) as s:
        z = np.zeros((1, 3))
        s.set_j_particles([0], [0], [0.0], [1.0], z, z, z, z)
        s.set_time(0.0)
        s.start(1, np.arange(1, n_i + 1), xi, np.zeros((n_i, 3)), None, eps2, np.zeros(n_i))
        got = s.results(1)
    xl = xi.astype(np.longdouble)
    r2 = (xl * xl).sum(1) + np.longdouble(eps2)
    inv = 1 / np.sqrt(r2)
    acc = (-xl * (inv ** 3)[:, None]).astype(np.float64)
    pot = (-inv).astype(np.float64)
    ea = np.linalg.norm(got["acc"] - acc, axis=1) / np.linalg.norm(acc, axis=1)
    ep = np.abs(got["pot"] - pot) / np.abs(pot)
    assert ea.max() < 2e-15 and ep.max() < 1e-15, (ea.max(), ep.max())


def test_near_pair_factor_is_checked(gpu):
    with sp.Sapporo(order=2, precision=sp.DOUBLESINGLE) as s:
        for bad in (-1.0, float("nan"), 2e6):
            with pytest.raises(sp.SapporoError):
                s.set_near(bad)
        s.set_near(0.0)
        s.set_near(64.0)


@pytest.mark.parametrize("order,precision,ni,nj,shapes", [
    (1, sp.DOUBLESINGLE, 16384, 16384, {(4, 2)}),
    (2, sp.DOUBLESINGLE, 4096, 16384, {(8, 2)}),
    (2, sp.DOUBLESINGLE, 256, 131072, {(8, 2), (16, 1), (32, 1)}),
    (2, sp.DOUBLESINGLE, 1 << 20, 1 << 20, {(1, 4), (2, 4)}),
    (1, sp.DOUBLE, 2048, 16384, {(16, 1)}),
    (2, sp.DOUBLE, 16384, 131072, {(8, 2)}),
])
def test_planner_shape_families(gpu, order, precision, ni, nj, shapes):
    """The launch planner's shape families by call size (mid-size calls take
    the measured best family; calls of 2^32 pairs and more the cost model's
    free choice); any plan computes the same forces (other tests)."""
    with sp.Sapporo(order=order, precision=precision) as s:
        tpi, ip, ns = s.plan(ni, nj)
    assert (tpi, ip) in shapes and ns >= 1, (tpi, ip, ns)
