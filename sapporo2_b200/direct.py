"""FP64 direct summation on the GPU through the library's all-FP64 kernels.

Used to set up workloads (the j-particle acceleration, jerk and snap that a
Hermite integrator would hand to the library) at sizes where a CPU direct
sum is impractical.  It drives the public `sapporo` class with precision
DOUBLE, so it is the same code path as any caller's.
"""
from __future__ import annotations

import numpy as np

from . import DOUBLE, FOURTH, SIXTH, Sapporo


def fp64_direct(order: int, x, v, a, m, ids, eps2: float, device: int = 0):
    """acc, jerk (and snap for order 6th) of every particle from all others,
    all particles at one time (no prediction)."""
    n = len(m)
    o = SIXTH if order >= 2 else FOURTH
    acc, jrk, snp = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros((n, 3))
    zero = np.zeros((n, 3))
    with Sapporo(device=device, order=o, precision=DOUBLE) as s:
        s.set_j_particles(np.arange(n), ids, np.zeros(n), m, x, v,
                          a if a is not None else zero, zero,
                          zero if o == SIXTH else None, zero if o == SIXTH else None)
        s.set_no_time()
        step = s.get_n_pipes()
        for i0 in range(0, n, step):
            sl = slice(i0, min(n, i0 + step))
            s.start(n, ids[sl], x[sl], v[sl], a[sl] if (a is not None and o == SIXTH) else None,
                    eps2, np.zeros(sl.stop - sl.start))
            r = s.results(n, ngb=False)
            acc[sl], jrk[sl], snp[sl] = r["acc"], r["jrk"], r["snp"]
    return acc, jrk, snp
