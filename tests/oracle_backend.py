"""A CPU stand-in for the library's `Sapporo` class, built on the FP64
oracle, so the integrator's host logic (corrector, block steps, neighbour
overflow re-evaluation, radius policies) is tested without a GPU."""
import numpy as np

from oracle import oracle as O


class OracleBackend:
    def __init__(self, n, lists=False):
        z = np.zeros((n, 3))
        self.n = n
        self.t = np.zeros(n)
        self.m = np.zeros(n)
        self.id = np.zeros(n, dtype=np.int32)
        self.x, self.v, self.a, self.j, self.s, self.c = (z.copy() for _ in range(6))
        self.ti = 0.0
        self.calls = 0
        self.lists = lists

    def set_j_particles(self, address, id, t, mass, x, v, a, jrk, snp=None, crk=None, eps=None):
        address = np.asarray(address)
        self.id[address], self.t[address], self.m[address] = id, t, mass
        self.x[address], self.v[address], self.a[address], self.j[address] = x, v, a, jrk
        self.s[address] = snp if snp is not None else 0.0
        self.c[address] = crk if crk is not None else 0.0

    def set_time(self, t):
        self.ti = float(t)

    def start(self, nj, id, xi, vi, ai=None, eps2=0.0, h2=None):
        px, pv, pa = O.predict(2, self.ti, self.t[:nj], self.x[:nj], self.v[:nj], self.a[:nj],
                               self.j[:nj], self.s[:nj], self.c[:nj])
        ni = len(id)
        self._r = O.force(2, xi, vi, ai if ai is not None else np.zeros((ni, 3)),
                          np.zeros(ni) if h2 is None else h2, id, px, pv, pa, self.m[:nj],
                          self.id[:nj], eps2, lists=self.lists)
        self.calls += 1

    def results(self, nj, ni=None, ngb=True):
        return self._r

    def neighbour_counts(self, ni=None):
        return self._r["ngb_count"].copy()

    def raw_results(self, ni=None):
        """Records in the device layout: acc, pot, jerk, snap, ds2 of the
        nearest neighbour rounded to float (1e11 when none), its id."""
        r = self._r
        n = len(r["pot"])
        out = np.zeros((n, 12))
        out[:, 0:3], out[:, 3], out[:, 4:7], out[:, 7:10] = r["acc"], r["pot"], r["jrk"], r["snp"]
        none = r["nnb"] < 0
        out[:, 10] = np.where(none, 1.0e11, r["ds2min"].astype(np.float32).astype(np.float64))
        out[:, 11] = np.where(none, -1, r["nnb"])
        return out

    def neighbour_lists(self, ni=None):
        return self._r["ngb_count"].copy(), self._r["ngb_list"].copy()

    def close(self):
        pass
