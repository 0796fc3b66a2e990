"""Seeded test cases and comparison helpers shared by the test files.

Inputs come from sapporo2_b200.ic (Plummer spheres, binaries); the j-particle
derivatives and the i-particle predictions come from the FP64 oracle.
"""
from __future__ import annotations

import numpy as np

from oracle import oracle as O
from sapporo2_b200 import ic

# Tolerances of the parity contract: forces within 1e-6 relative median and
# 1e-4 relative max of the same-order reference / FP64 answer; neighbour sets
# exact except pairs within 1e-6 relative of the h2 boundary.
MEDIAN_TOL = 1e-6
MAX_TOL = 1e-4
H2_BAND = 1e-6


def build_case(order: int, n: int, seed: int, eps2: float = 1e-6, binaries: float = 0.0,
               salpeter: bool = False, nngb: float = 32.0, id_offset: int = 100,
               t_spread: bool = True, permute_ids: bool = False) -> dict:
    m = ic.salpeter(n, seed) if salpeter else None
    x, v, m = ic.plummer(n, seed, masses=m)
    if binaries > 0:
        x, v, m, _ = ic.add_binaries(x, v, m, binaries, seed + 11)
    ids = (np.arange(n) + id_offset).astype(np.int32)
    if permute_ids:  # ids unrelated to the addresses: every j tile spans all ids
        ids = ids[np.random.default_rng(seed + 7).permutation(n)]
    fn = O.derivative_fn()
    a, j, _ = fn(1, x, v, None, m, ids, eps2)
    s = c = None
    if order >= 2:
        _, _, s = fn(2, x, v, a, m, ids, eps2)
        c = ic.crackle_from(x, a, j)
    rng = np.random.default_rng(seed + 99)
    ti = 1.0
    t0 = ti - (rng.integers(0, 8, n) * 2.0 ** -10 if t_spread else np.zeros(n))
    px, pv, pa = O.predict(order, ti, t0, x, v, a, j, s, c)
    h2 = ic.plummer_h2(px, m, nngb)
    return dict(order=order, n=n, x=x, v=v, m=m, a=a, j=j, s=s, c=c, id=ids, t0=t0, ti=ti,
                px=px, pv=pv, pa=pa, h2=h2, eps2=eps2)


def oracle_force(case: dict, sel=None, lists=True) -> dict:
    o = case["order"]
    xi, vi, ai, h2, idi = case["px"], case["pv"], case["pa"], case["h2"], case["id"]
    if sel is not None:
        xi, vi, h2, idi = xi[sel], vi[sel], h2[sel], idi[sel]
        ai = ai[sel] if ai is not None else None
    return O.force(o, xi, vi, ai, h2, idi, case["px"], case["pv"], case["pa"], case["m"],
                   case["id"], case["eps2"], lists=lists)


def run_library(case: dict, precision: int, sel=None, lists=True, launch=None,
                spatial=None, devices=None) -> dict:
    """Drives the sapporo class exactly as an integrator would: stage all j,
    set_time, startGravCalc on the selected i, getGravResults, neighbour
    readout.  `spatial` = (mode, delta) sets the spatial mode first;
    `devices` = a device list for open (the j spread over its entries)."""
    import sapporo2_b200 as sp
    o, n = case["order"], case["n"]
    with sp.Sapporo(order=o, precision=precision, devices=devices) as s:
        if launch:
            s.set_launch(*launch)
        if spatial is not None:
            s.set_spatial(*spatial)
        s.set_j_particles(np.arange(n), case["id"], case["t0"], case["m"], case["x"], case["v"],
                          case["a"], case["j"], case["s"], case["c"])
        s.set_time(case["ti"])
        idx = np.arange(n) if sel is None else np.asarray(sel)
        s.start(n, case["id"][idx], case["px"][idx], case["pv"][idx],
                case["pa"][idx] if case["pa"] is not None else None, case["eps2"],
                case["h2"][idx])
        r = s.results(n, ngb=True)
        if devices is None:
            r["raw"] = s.raw_results(len(idx)).copy()
        if spatial is not None:
            r["far_tiles"] = s.spatial_stats()  # (far, all) (warp, tile) pairs
        if lists:
            r["overflow"] = s.read_ngb_list()
            cnts, lsts = [], []
            for i in range(len(idx)):
                _, nb, ids = s.get_ngb_list(i, sp.NGB_PB)
                cnts.append(nb)
                lsts.append(ids)
            r["ngb_count"] = np.array(cnts)
            r["ngb_sets"] = lsts
    return r


def rel_err(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Per-particle |a - b| / |b| for vectors ([n, 3]) or scalars ([n])."""
    if a.ndim == 1:
        return np.abs(a - b) / np.maximum(np.abs(b), 1e-300)
    return np.linalg.norm(a - b, axis=1) / np.maximum(np.linalg.norm(b, axis=1), 1e-300)


def check_forces(got: dict, want: dict, order: int, median_tol=MEDIAN_TOL, max_tol=MAX_TOL,
                 fields=None) -> dict:
    fields = fields or (["acc", "pot", "jrk"] + (["snp"] if order >= 2 else []))
    stats = {}
    for f in fields:
        e = rel_err(got[f], want[f])
        stats[f] = (float(np.median(e)), float(e.max()))
        assert np.all(np.isfinite(got[f])), f"{f}: non-finite values"
        assert stats[f][0] <= median_tol, f"{f}: median rel err {stats[f][0]:.3e} > {median_tol}"
        assert stats[f][1] <= max_tol, f"{f}: max rel err {stats[f][1]:.3e} > {max_tol}"
    return stats


def _ds2(case, i_idx, j_ids):
    jpos = {int(k): p for k, p in zip(case["id"], case["px"])}
    xi = case["px"][i_idx]
    return np.array([float(((jpos[int(q)] - xi) ** 2).sum()) for q in j_ids])


def check_neighbours(case: dict, got_sets, got_counts, want: dict, sel=None) -> int:
    """Neighbour sets equal except pairs within H2_BAND of the h2 boundary.
    Returns the number of exempted boundary pairs."""
    idx = np.arange(case["n"]) if sel is None else np.asarray(sel)
    exempt = 0
    for q, i in enumerate(idx):
        wc = int(want["ngb_count"][q])
        h2 = case["h2"][i]
        gc = int(got_counts[q])
        if wc >= 256 or gc >= 256:
            # overflow flags (count >= 256, sapporohostclass.cpp:827-829) must
            # agree; they may differ only where pairs within the h2 band can
            # carry one count across 256
            if (wc >= 256) != (gc >= 256):
                d2 = ((case["px"] - case["px"][i]) ** 2).sum(1)
                band = int(np.sum(np.abs(d2 - h2) <= H2_BAND * h2))
                assert min(wc, gc) + band >= 256, \
                    f"i={i}: overflow flag differs (want count {wc}, got {gc}, band pairs {band})"
                exempt += band
            continue
        ws = set(int(t) for t in want["ngb_list"][q, :wc])
        gs = set(int(t) for t in got_sets[q])
        diff = ws ^ gs
        if diff:
            d2 = _ds2(case, i, sorted(diff))
            band = np.abs(d2 - h2) / h2
            assert np.all(band <= H2_BAND), f"i={i}: neighbour sets differ off the boundary {sorted(diff)} band={band}"
            exempt += len(diff)
    return exempt


def check_nn(case: dict, got_nnb, want: dict, sel=None) -> int:
    """Nearest-neighbour ids equal except near-ties (second candidate within
    1e-6 relative in ds2).  Returns the number of exempted near-ties."""
    idx = np.arange(case["n"]) if sel is None else np.asarray(sel)
    bad = np.nonzero(np.asarray(got_nnb) != want["nnb"])[0]
    for q in bad:
        i = idx[q]
        d = _ds2(case, i, [got_nnb[q], want["nnb"][q]])
        assert abs(d[0] - d[1]) <= 1e-6 * max(d[1], 1e-300), \
            f"i={i}: nn {got_nnb[q]} (ds2 {d[0]:.6e}) vs {want['nnb'][q]} (ds2 {d[1]:.6e})"
    return len(bad)
