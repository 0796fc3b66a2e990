"""Learned neighbour radius: the network of sapb_mlp.cu proposes each
particle's h2 from five features of its previous force evaluation, and is
trained online on the neighbour counts the force kernel reports.

Features (standardised with statistics frozen at the first training call):
log of the local density estimate rho = n_prev / (4/3 pi h_prev^3), log |a|,
log |jerk|, the particle's running mean L of log rho over its past
evaluations less log rho (how far the last count strays from the
particle's history: Poisson noise of a count of ~32 is ~18 %), log h2_prev.
The proposal is
log(h2 / h2_prev) = 2/3 log(target / n_prev) + network output: the network
learns the correction to the count-scaled radius (density drift along the
orbit, shrinkage of a noisy last count toward the particle's history).  Target for a particle evaluated
with h2_used that found n neighbours: the radius that would have given the
target count in a locally uniform medium,
log(h2_used / h2_prev) + 2/3 log(target / max(n, 1/2)), minus the
count-scaled part.

The fixed rule with overflow re-evaluation (`retry_h2`) stays as the fallback
and judge: any overflowing particle is re-evaluated with the count-scaled
radius, so results never depend on the network.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import Sapporo, SapporoError, _check, load_library

TARGET = 32.0
CAP = 256


def log_density(n, h2) -> np.ndarray:
    """log of n / (4/3 pi h^3), n = max(count, 1/2)."""
    n = np.maximum(np.asarray(n, dtype=np.float64), 0.5)
    return np.log(n / (4.0 / 3.0 * np.pi * np.asarray(h2, dtype=np.float64) ** 1.5))


def features(n_prev, h2_prev, acc, jrk, lrho_mean=None) -> np.ndarray:
    """The network's five inputs (before standardisation); lrho_mean is the
    particle's running mean of log density (None: no history yet, the last
    evaluation's own value)."""
    h2 = np.asarray(h2_prev, dtype=np.float64)
    lr = log_density(n_prev, h2)
    lm = lr if lrho_mean is None else np.asarray(lrho_mean, dtype=np.float64)
    a = np.linalg.norm(acc, axis=1) + 1e-30
    j = np.linalg.norm(jrk, axis=1) + 1e-30
    return np.stack([lr, np.log(a), np.log(j), lm - lr, np.log(h2)], axis=1)


def target_log_ratio(h2_used, h2_prev, n_obs, target=TARGET) -> np.ndarray:
    n = np.maximum(np.asarray(n_obs, dtype=np.float64), 0.5)
    return np.log(np.asarray(h2_used) / np.asarray(h2_prev)) + (2.0 / 3.0) * np.log(target / n)


def retry_h2(h2, count, target=TARGET) -> np.ndarray:
    """Radius for re-evaluating an overflowing particle (exact counts)."""
    return np.asarray(h2) * (target / np.maximum(np.asarray(count, dtype=np.float64), 1.0)) ** (2.0 / 3.0)


class H2Net:
    """The network on the GPU of an open :class:`Sapporo` instance."""

    def __init__(self, owner: Sapporo, seed: int = 5):
        self.lib = load_library()
        self.owner = owner
        self.np = self.lib.sapb_mlp_num_params()
        h = C.c_void_p()
        _check(self.lib.sapb_mlp_create(owner.dev, C.c_ulonglong(seed), C.byref(h)), "mlp_create",
               owner.dev)
        self.h = h
        self.mu = None
        self.sd = None

    def close(self):
        if self.h:
            self.lib.sapb_mlp_destroy(self.h)
            self.h = None

    def params(self) -> np.ndarray:
        p = np.zeros(self.np, dtype=np.float32)
        _check(self.lib.sapb_mlp_get_params(self.h, p.ctypes.data_as(C.POINTER(C.c_float))),
               "mlp_get", self.owner.dev)
        return p

    def zero_output_layer(self):
        """Output weights and bias set to zero (the last 65 parameters, W4
        and b4): the network then proposes no correction until training
        finds a consistent one."""
        p = self.params()
        p[-(64 + 1):] = 0.0
        self.set_params(p)

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        _check(self.lib.sapb_mlp_set_params(self.h, p.ctypes.data_as(C.POINTER(C.c_float))),
               "mlp_set", self.owner.dev)

    @staticmethod
    def _f(a):
        return np.ascontiguousarray(a, dtype=np.float32)

    def forward(self, x) -> np.ndarray:
        x = self._f(x)
        y = np.zeros(len(x), dtype=np.float32)
        _check(self.lib.sapb_mlp_forward(self.h, len(x), x.ctypes.data_as(C.POINTER(C.c_float)),
                                         y.ctypes.data_as(C.POINTER(C.c_float))), "mlp_forward",
               self.owner.dev)
        return y

    def gradient(self, x, t):
        x, t = self._f(x), self._f(t)
        g = np.zeros(self.np, dtype=np.float32)
        loss = C.c_float()
        _check(self.lib.sapb_mlp_gradient(self.h, len(x), x.ctypes.data_as(C.POINTER(C.c_float)),
                                          t.ctypes.data_as(C.POINTER(C.c_float)),
                                          g.ctypes.data_as(C.POINTER(C.c_float)), C.byref(loss)),
               "mlp_gradient", self.owner.dev)
        return g, loss.value

    def train(self, x, t, epochs=20, lr=1e-3) -> float:
        x, t = self._f(x), self._f(t)
        loss = C.c_float()
        _check(self.lib.sapb_mlp_train(self.h, len(x), x.ctypes.data_as(C.POINTER(C.c_float)),
                                       t.ctypes.data_as(C.POINTER(C.c_float)), int(epochs),
                                       float(lr), C.byref(loss)), "mlp_train", self.owner.dev)
        return loss.value

    # ---- standardised use -------------------------------------------------
    def fit_standardisation(self, f, floor=0.5):
        """Freezes the feature scaling (mean, std floored at `floor`: the
        features are logarithms, so a constant start-up feature such as one
        global h2 must not blow up later variations)."""
        self.mu = f.mean(0)
        self.sd = np.maximum(f.std(0), floor)

    def standardise(self, f):
        if self.mu is None:
            self.fit_standardisation(f)
        return (f - self.mu) / self.sd

    @staticmethod
    def base_log_ratio(n_prev, target=TARGET) -> np.ndarray:
        """The count-scaled step the network corrects: log of
        (target / previous count)^(2/3)."""
        return (2.0 / 3.0) * np.log(target / np.maximum(np.asarray(n_prev, dtype=np.float64), 0.5))

    # The correction may shrink h2 by up to e^MAX_DOWN but grow it by at most
    # e^MAX_UP (x1.45 in the expected count): an overflow costs a whole
    # re-evaluation of the particle, a list below the target range costs
    # nothing, so the network is not allowed to gamble on growing a radius.
    MAX_DOWN = 1.0
    MAX_UP = 0.25

    def propose(self, n_prev, h2_prev, acc, jrk, lrho_mean=None, clip=4.0) -> np.ndarray:
        """h2 for the next evaluation: the count-scaled radius times the
        network's bounded correction; the whole log-ratio is clipped to
        +-clip.  Features, standardisation, network and correction run in
        one kernel (sapb_mlp_propose) from the raw per-particle state."""
        if self.mu is None:
            self.fit_standardisation(features(n_prev, h2_prev, acc, jrk, lrho_mean))
        n = len(h2_prev)
        rec = np.empty((n, 9), dtype=np.float32)
        rec[:, 0] = n_prev
        rec[:, 1] = h2_prev
        rec[:, 2:5] = acc
        rec[:, 5:8] = jrk
        rec[:, 8] = log_density(n_prev, h2_prev) if lrho_mean is None else lrho_mean
        mu = self._f(self.mu)
        sd = self._f(self.sd)
        out = np.empty(n, dtype=np.float32)
        fp = C.POINTER(C.c_float)
        _check(self.lib.sapb_mlp_propose(self.h, n, rec.ctypes.data_as(fp), mu.ctypes.data_as(fp),
                                         sd.ctypes.data_as(fp), float(TARGET),
                                         float(self.MAX_DOWN), float(self.MAX_UP), float(clip),
                                         out.ctypes.data_as(fp)), "mlp_propose", self.owner.dev)
        return out.astype(np.float64)

    def propose_host(self, n_prev, h2_prev, acc, jrk, lrho_mean=None, clip=4.0) -> np.ndarray:
        """The same proposal with the features built on the host (FP64) and
        only the network on the GPU -- the reference for propose()."""
        f = self.standardise(features(n_prev, h2_prev, acc, jrk, lrho_mean))
        corr = np.clip(self.forward(f).astype(np.float64), -self.MAX_DOWN, self.MAX_UP)
        r = self.base_log_ratio(n_prev) + corr
        return np.asarray(h2_prev) * np.exp(np.clip(r, -clip, clip))

    def learn(self, n_prev, h2_prev, acc, jrk, h2_used, n_obs, lrho_mean=None, epochs=20,
              lr=2e-3) -> float:
        """One online update: the correction that would have given the target
        count, from the count the force kernel found with h2_used (clipped to
        the correction's bounds, so a particle that found no neighbour does
        not drag the fit)."""
        f = self.standardise(features(n_prev, h2_prev, acc, jrk, lrho_mean))
        y = target_log_ratio(h2_used, h2_prev, n_obs) - self.base_log_ratio(n_prev)
        return self.train(f, np.clip(y, -self.MAX_DOWN, self.MAX_UP), epochs, lr)
