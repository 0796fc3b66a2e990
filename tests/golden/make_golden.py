"""Generates the golden fixtures of tests/golden/ from the reference's own
CUDA kernels (oracle/_ref: lib/CUDAKernels/kernels.cu compiled unchanged for
sm_100a and launched with the reference geometry).  Run on a GPU box:

    python tests/golden/make_golden.py

For each order (4th, 6th) it stores a seeded input set (raw j state at t0,
t_i, h2, ids), the reference predictor's output, and the outputs of the
reference gravity kernels in DOUBLE and DOUBLESINGLE precision (acc, jerk,
snap, pot, nearest neighbour, neighbour counts and sorted lists), computed on
the reference-predicted j with i = every particle predicted to t_i.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import oracle as O  # noqa: E402
from sapporo2_b200 import ic  # noqa: E402

HERE = Path(__file__).resolve().parent


def make(order: int, n: int, seed: int, nngb: float) -> dict:
    x, v, m = ic.plummer(n, seed)
    x, v, m, _ = ic.add_binaries(x, v, m, 0.1, seed + 11)
    ids = (np.arange(n) + 100).astype(np.int32)
    eps2 = 1e-6
    fn = O.derivative_fn()
    a, j, _ = fn(1, x, v, None, m, ids, eps2)
    s = c = None
    if order == 2:
        _, _, s = fn(2, x, v, a, m, ids, eps2)
        c = ic.crackle_from(x, a, j)
    rng = np.random.default_rng(seed + 99)
    ti = 1.0
    t0 = ti - rng.integers(0, 8, n) * 2.0 ** -10
    # reference predictor -> j inputs of the reference gravity kernels
    rpx, rpv, rpa = O.ref_predict(order, ti, t0, x, m, v, a, j, s, c)
    h2 = ic.plummer_h2(rpx, m, nngb)
    out = dict(order=order, n=n, seed=seed, eps2=eps2, ti=ti, t0=t0, x=x, v=v, m=m, a=a, j=j,
               id=ids, h2=h2, ref_px=rpx, ref_pv=rpv)
    if order == 2:
        out.update(s=s, c=c, ref_pa=rpa)
    for prec, tag in ((2, "dp"), (1, "ds")):
        r = O.ref_gravity(order, prec, rpx, rpv, rpa if order == 2 else None, h2, ids, rpx, rpv,
                          rpa if order == 2 else None, m, ids, eps2)
        out[f"{tag}_acc"], out[f"{tag}_jrk"], out[f"{tag}_pot"] = r["acc"], r["jrk"], r["pot"]
        if order == 2:
            out[f"{tag}_snp"] = r["snp"]
        out[f"{tag}_nnb"], out[f"{tag}_ds2"] = r["nnb"], r["ds2min"]
        cnt = r["ngb_count"]
        out[f"{tag}_cnt"] = cnt
        flat, offs = [], [0]
        for i in range(n):
            lst = np.sort(r["ngb_list"][i, :cnt[i]]) if cnt[i] < 256 else np.zeros(0, np.int32)
            flat.append(lst)
            offs.append(offs[-1] + len(lst))
        out[f"{tag}_ngb"] = np.concatenate(flat).astype(np.int32)
        out[f"{tag}_ngb_off"] = np.array(offs, dtype=np.int64)
    return out


def main():
    if not O.ref_available():
        raise SystemExit("oracle/_ref is not built (make -C oracle on a machine with the reference tree)")
    for order, n, seed, nngb in ((1, 768, 21, 24.0), (2, 768, 22, 24.0)):
        d = make(order, n, seed, nngb)
        path = HERE / f"ref_kernels_order{2 * order + 2}.npz"
        np.savez_compressed(path, **{k: v for k, v in d.items() if v is not None})
        print(f"wrote {path} ({path.stat().st_size} bytes)")


if __name__ == "__main__":
    main()
