"""Block-timestep 6th-order Hermite integrator driving the library.

Predictor: Taylor series to crackle on the host for the active i, on the GPU
for all j (the library).  Corrector: the 6th-order Hermite scheme of
Nitadori & Makino (2008), with crackle at the end of the step from the
quintic interpolation of a, jerk, snap.  Steps dt = 2^-k on a block grid.

Each force evaluation requests neighbour lists with a radius chosen by a
policy (`FixedH2` or `LearnedH2`); particles whose list overflows (count >=
256) are re-evaluated with the count-scaled radius until none overflows.
Forces do not depend on the radius, so the trajectory is the same whatever
the policy; only the neighbour work differs.
"""
from __future__ import annotations

import time

import numpy as np

from . import DOUBLESINGLE, NGB_PB, SIXTH, Sapporo
from .learned_h2 import TARGET, H2Net, features, log_density, retry_h2, target_log_ratio

# [C, P, Q] = M^-1 [A, J, S] for the quintic interpolation of a(t)
_MINV = np.linalg.inv(np.array([[1 / 6, 1 / 24, 1 / 120], [1 / 2, 1 / 6, 1 / 24],
                                [1.0, 1 / 2, 1 / 6]]))


class FixedH2:
    """The plain fixed rule: one radius for every particle, the one holding
    TARGET neighbours at the local density of the half-mass radius.  A global
    radius necessarily overflows the core (a Plummer core is ~12x denser than
    the half-mass shell) and starves the halo."""

    name = "fixed"

    def start(self, sim, samples):
        pass

    def propose(self, sim, idx):
        return np.full(len(idx), sim.h2_fix)

    def observe(self, sim, idx, h2_used, counts):
        pass


class CountScaledH2:
    """Non-learned per-particle rule, for comparison: the previous radius
    scaled by (TARGET / previous count)^(2/3)."""

    name = "count-scaled"

    def start(self, sim, samples):
        pass

    def propose(self, sim, idx):
        return retry_h2(sim.h2_prev[idx], np.maximum(sim.n_prev[idx], 0.5))

    def observe(self, sim, idx, h2_used, counts):
        pass


class LearnedH2:
    """The GPU-trained network proposes h2 from the particle's previous
    evaluation and its history (as a correction to the count-scaled radius).
    It is pretrained on the counts of the two start-up force passes (two
    radii) and then learns online from first-attempt counts.  The history is
    a running mean of each particle's log density over its evaluations
    (weight `w` on the newest), kept here and updated after every step."""

    name = "learned"

    def __init__(self, sap, seed=5, epochs=1, lr=1e-4, pre_epochs=300, max_batch=8192,
                 max_pre=65536, train_every=4, w=0.5):
        self.net = H2Net(sap, seed=seed)
        # start from a zero correction: the count-scaled radius is already a
        # good proposal, the network only adds what it learns consistently
        self.net.zero_output_layer()
        self.epochs, self.lr, self.pre_epochs = epochs, lr, pre_epochs
        self.max_batch, self.max_pre, self.train_every = max_batch, max_pre, train_every
        self.rng = np.random.default_rng(seed)
        self.losses = []
        self.train_s = 0.0
        self.pretrain_s = 0.0
        self.propose_s = 0.0
        self.n_obs = 0
        self.w = w
        self.lrho = None  # running mean of log density per particle

    def start(self, sim, samples):
        t0 = time.perf_counter()
        self.lrho = log_density(sim.n_prev, sim.h2_prev)
        f = np.concatenate([s[0] for s in samples])
        y = np.concatenate([s[1] - self.net.base_log_ratio(s[2]) for s in samples])
        if len(f) > self.max_pre:
            take = self.rng.choice(len(f), self.max_pre, replace=False)
            f, y = f[take], y[take]
        self.net.fit_standardisation(f)
        for _ in range(self.pre_epochs // 50):
            self.losses.append(self.net.train(self.net.standardise(f), y, 50, 3e-3))
        self.pretrain_s += time.perf_counter() - t0

    def propose(self, sim, idx):
        t0 = time.perf_counter()
        h2 = self.net.propose(sim.n_prev[idx], sim.h2_prev[idx], sim.a[idx], sim.j[idx],
                              self.lrho[idx])
        self.propose_s += time.perf_counter() - t0
        return h2

    def observe(self, sim, idx, h2_used, counts):
        """One online update on (at most max_batch of) this step's first
        attempts, every train_every-th block step; then the history of the
        evaluated particles takes in this step's counts."""
        self.n_obs += 1
        if (self.n_obs - 1) % self.train_every == 0:
            t0 = time.perf_counter()
            take = np.arange(len(idx))
            if len(take) > self.max_batch:
                take = self.rng.choice(len(idx), self.max_batch, replace=False)
            q = idx[take]
            loss = self.net.learn(sim.n_prev[q], sim.h2_prev[q], sim.a[q], sim.j[q],
                                  h2_used[take], counts[take], lrho_mean=self.lrho[q],
                                  epochs=self.epochs, lr=self.lr)
            self.losses.append(loss)
            self.train_s += time.perf_counter() - t0
        self.lrho[idx] += self.w * (log_density(counts, h2_used) - self.lrho[idx])


def half_mass_h2(x, m, target=TARGET):
    """Radius holding `target` neighbours at the density of the half-mass
    shell (particles within 10 % of the median radius)."""
    r = np.linalg.norm(x, axis=1)
    rh = np.median(r)
    r1, r2 = rh / 1.1, rh * 1.1
    shell = (r >= r1) & (r < r2)
    rho = shell.sum() / (4.0 / 3.0 * np.pi * (r2 ** 3 - r1 ** 3))
    return (target / (4.0 / 3.0 * np.pi * rho)) ** (2.0 / 3.0)


class BlockHermite6:
    def __init__(self, x, v, m, eps2, policy_factory, eta=0.02, eta_init=0.01,
                 dt_max=2.0 ** -3, dt_min=2.0 ** -24, precision=DOUBLESINGLE, device=0,
                 backend=None):
        self.n = len(m)
        self.x, self.v, self.m = x.copy(), v.copy(), m.copy()
        self.ids = np.arange(self.n, dtype=np.int32)
        self.eps2, self.eta, self.dt_max, self.dt_min = eps2, eta, dt_max, dt_min
        # backend: an object with the Sapporo methods used below (set_j_particles,
        # set_time, start, results, neighbour_counts, close); default the GPU
        self.sap = backend if backend is not None else Sapporo(
            device=device, order=SIXTH, precision=precision, n_pipes=max(self.n, 16384))
        self.policy = policy_factory(self.sap) if callable(policy_factory) else policy_factory
        z = np.zeros((self.n, 3))
        self.a, self.j, self.s, self.c = z.copy(), z.copy(), z.copy(), z.copy()
        self.t = np.zeros(self.n)
        self.h2_fix = half_mass_h2(self.x, self.m)
        self.stats = {"evaluated": 0, "overflow": 0, "retries": 0, "rounds": 0,
                      "in_range": 0, "in_tight": 0, "abs_log_err": 0.0, "force_s": 0.0,
                      "step_s": 0.0, "steps": 0, "interactions": 0.0}
        # two passes at t = 0: acc and jerk, then snap with the i acceleration;
        # their neighbour counts (radii h2_fix / 4 and h2_fix) are the
        # policies' start-up samples
        all_i = np.arange(self.n)
        self._push(all_i)
        h2a = np.full(self.n, self.h2_fix / 4.0)
        r, cnt_a = self._force(all_i, self.x, self.v, z, h2a, 0.0, retry=False)
        self.a, self.j = r["acc"], r["jrk"]
        self._push(all_i)
        h2b = np.full(self.n, self.h2_fix)
        r, cnt_b = self._force(all_i, self.x, self.v, self.a, h2b, 0.0, retry=False)
        self.s = r["snp"]
        self.h2_prev = h2b.copy()
        self.n_prev = cnt_b.astype(np.float64)
        samples = []
        for h2u, cnt in ((h2a, cnt_a), (h2b, cnt_b)):
            f = features(cnt, h2u, self.a, self.j)
            samples.append((f, target_log_ratio(h2u, h2u, cnt), cnt))
        self.policy.start(self, samples)
        an, jn = np.linalg.norm(self.a, axis=1), np.linalg.norm(self.j, axis=1)
        self.dt = self._quantize(eta_init * an / np.maximum(jn, 1e-300), np.zeros(self.n),
                                 np.full(self.n, dt_max))
        self._push(all_i)
        self.e0 = self.energy()
        for k in self.stats:
            self.stats[k] = 0 if not isinstance(self.stats[k], float) else 0.0

    # -------------------------------------------------------------------
    def _push(self, idx):
        self.sap.set_j_particles(idx, self.ids[idx], self.t[idx], self.m[idx], self.x[idx],
                                 self.v[idx], self.a[idx], self.j[idx], self.s[idx], self.c[idx])

    def _force(self, idx, xi, vi, ai, h2, ti, retry=True):
        """Force with lists on particles idx; overflowing ones are re-evaluated
        with the count-scaled radius.  Returns results and final counts."""
        t0 = time.perf_counter()
        self.sap.set_time(ti)
        self.sap.start(self.n, self.ids[idx], xi, vi, ai, self.eps2, h2)
        r = self.sap.results(self.n, ngb=True)
        cnt = self.sap.neighbour_counts().astype(np.int64)
        first = cnt.copy()
        self.stats["interactions"] += float(len(idx)) * self.n
        h2 = np.array(h2, dtype=np.float64)
        over = np.nonzero(cnt >= NGB_PB)[0] if retry else np.zeros(0, dtype=np.int64)
        self.stats["overflow"] += len(over)
        while len(over):
            self.stats["rounds"] += 1
            self.stats["retries"] += len(over)
            h2[over] = retry_h2(h2[over], cnt[over])
            self.sap.start(self.n, self.ids[idx[over]], xi[over], vi[over], ai[over], self.eps2,
                           h2[over])
            self.sap.results(self.n, ngb=False)
            c2 = self.sap.neighbour_counts()
            self.stats["interactions"] += float(len(over)) * self.n
            cnt[over] = c2
            over = over[c2 >= NGB_PB]
        self.stats["evaluated"] += len(idx)
        self.stats["in_range"] += int(np.sum((first >= TARGET / 2) & (first <= 2 * TARGET)))
        # a tighter band (+-25 % in the count) and the mean |log(count/target)|
        self.stats["in_tight"] += int(np.sum((first >= 0.75 * TARGET) & (first <= 1.25 * TARGET)))
        self.stats["abs_log_err"] += float(np.sum(np.abs(np.log(np.maximum(first, 0.5) / TARGET))))
        self.stats["force_s"] += time.perf_counter() - t0
        self.h2_used, self.first_counts = h2, first
        return r, cnt

    def _quantize(self, dt, t, dt_old):
        k = np.floor(np.log2(np.maximum(dt, self.dt_min)))
        dtq = np.ldexp(1.0, k.astype(int))
        dtq = np.minimum(dtq, np.minimum(self.dt_max, 2.0 * dt_old))
        dtq = np.maximum(dtq, self.dt_min)
        # commensurate with the current time
        while True:
            bad = np.fmod(t, dtq) != 0
            if not bad.any():
                return dtq
            dtq[bad] *= 0.5

    # -------------------------------------------------------------------
    def step(self):
        ts = time.perf_counter()
        tn = np.min(self.t + self.dt)
        act = np.nonzero(self.t + self.dt == tn)[0]
        h = tn - self.t[act]
        hh = h[:, None]
        x0, v0, a0, j0, s0, c0 = (q[act] for q in (self.x, self.v, self.a, self.j, self.s, self.c))
        h2, h3, h4, h5 = hh * hh / 2, hh ** 3 / 6, hh ** 4 / 24, hh ** 5 / 120
        xp = x0 + hh * v0 + h2 * a0 + h3 * j0 + h4 * s0 + h5 * c0
        vp = v0 + hh * a0 + h2 * j0 + h3 * s0 + h4 * c0
        ap = a0 + hh * j0 + h2 * s0 + h3 * c0
        h2_try = self.policy.propose(self, act)
        r, cnt = self._force(act, xp, vp, ap, h2_try, tn)
        self.policy.observe(self, act, h2_try, self.first_counts)
        a1, j1, s1 = r["acc"], r["jrk"], r["snp"]
        # 6th-order Hermite corrector (Nitadori & Makino 2008)
        v1 = v0 + hh / 2 * (a0 + a1) - hh * hh / 10 * (j1 - j0) + hh ** 3 / 120 * (s0 + s1)
        x1 = x0 + hh / 2 * (v0 + v1) - hh * hh / 10 * (a1 - a0) + hh ** 3 / 120 * (j0 + j1)
        A = a1 - a0 - j0 * hh - s0 * hh * hh / 2
        J = (j1 - j0 - s0 * hh) * hh
        S = (s1 - s0) * hh * hh
        CPQ = np.einsum("ab,bnk->ank", _MINV, np.stack([A, J, S]))
        c1 = (CPQ[0] + CPQ[1] + CPQ[2] / 2) / hh ** 3
        self.x[act], self.v[act], self.a[act], self.j[act], self.s[act], self.c[act] = \
            x1, v1, a1, j1, s1, c1
        self.t[act] = tn
        an, jn = np.linalg.norm(a1, axis=1), np.linalg.norm(j1, axis=1)
        sn, cn = np.linalg.norm(s1, axis=1), np.linalg.norm(c1, axis=1)
        dt = np.sqrt(self.eta * (an * sn + jn * jn) / np.maximum(jn * cn + sn * sn, 1e-300))
        self.dt[act] = self._quantize(dt, self.t[act], self.dt[act])
        self.h2_prev[act] = self.h2_used
        self.n_prev[act] = cnt
        self._push(act)
        self.stats["steps"] += 1
        self.stats["step_s"] += time.perf_counter() - ts
        return len(act)

    def energy(self):
        """Total energy at the latest particle time: every particle predicted
        there (host Taylor series for i, the library's predictor for j),
        potential from the GPU."""
        tmax = float(np.max(self.t))
        hh = (tmax - self.t)[:, None]
        xp = self.x + hh * (self.v + hh / 2 * (self.a + hh / 3 * (self.j + hh / 4 * (
            self.s + hh / 5 * self.c))))
        vp = self.v + hh * (self.a + hh / 2 * (self.j + hh / 3 * (self.s + hh / 4 * self.c)))
        ap = self.a + hh * (self.j + hh / 2 * (self.s + hh / 3 * self.c))
        self.sap.set_time(tmax)
        self.sap.start(self.n, self.ids, xp, vp, ap, self.eps2, np.zeros(self.n))
        r = self.sap.results(self.n, ngb=False)
        ek = 0.5 * float(np.sum(self.m * np.sum(vp * vp, axis=1)))
        ep = 0.5 * float(np.sum(self.m * r["pot"]))
        return ek + ep

    def close(self):
        if hasattr(self.policy, "net"):
            self.policy.net.close()
        self.sap.close()
