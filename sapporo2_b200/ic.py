"""Seeded synthetic N-body inputs for the benchmark and the tests.

No public dataset is involved: the workloads are Plummer spheres in Henon
units (G = M = 1, E = -1/4) sampled with the published Aarseth, Henon &
Wielen (1974) recipe, optionally with a Salpeter mass function and a fraction
of particles placed in circular binaries, plus the time structure the
Hermite schemes need (particle times, block time steps, active sets).
"""
from __future__ import annotations

import numpy as np

PLUMMER_A = 3.0 * np.pi / 16.0  # Plummer scale radius in Henon units


def plummer(n: int, seed: int, rcut: float = 10.0, masses: np.ndarray | None = None):
    """Positions, velocities and masses of an n-body Plummer sphere.

    Radii from the inverse cumulative mass, velocities by von Neumann
    rejection on q^2 (1 - q^2)^{7/2} (Aarseth, Henon & Wielen 1974), scaled
    to Henon units; radii beyond `rcut` (Henon units) are resampled.  The
    centre of mass is moved to rest at the origin.
    """
    rng = np.random.default_rng(seed)
    x = np.empty((n, 3))
    v = np.empty((n, 3))
    filled = 0
    while filled < n:
        m = int((n - filled) * 1.05) + 16
        X1 = rng.random(m)
        X1 = np.clip(X1, 1e-12, 1.0 - 1e-12)
        r = 1.0 / np.sqrt(X1 ** (-2.0 / 3.0) - 1.0)
        keep = r * PLUMMER_A <= rcut
        r = r[keep]
        k = min(len(r), n - filled)
        r = r[:k]
        # isotropic directions
        ct = rng.uniform(-1.0, 1.0, k)
        ph = rng.uniform(0.0, 2.0 * np.pi, k)
        st = np.sqrt(1.0 - ct * ct)
        dirs = np.stack([st * np.cos(ph), st * np.sin(ph), ct], axis=1)
        # speed: q with g(q) = q^2 (1-q^2)^3.5 by rejection (max of g < 0.1)
        q = np.empty(k)
        todo = np.arange(k)
        while len(todo):
            X4 = rng.random(len(todo))
            X5 = rng.random(len(todo))
            ok = 0.1 * X5 < X4 * X4 * (1.0 - X4 * X4) ** 3.5
            q[todo[ok]] = X4[ok]
            todo = todo[~ok]
        speed = q * np.sqrt(2.0) * (1.0 + r * r) ** (-0.25)
        ct = rng.uniform(-1.0, 1.0, k)
        ph = rng.uniform(0.0, 2.0 * np.pi, k)
        st = np.sqrt(1.0 - ct * ct)
        vdir = np.stack([st * np.cos(ph), st * np.sin(ph), ct], axis=1)
        x[filled:filled + k] = dirs * (r * PLUMMER_A)[:, None]
        v[filled:filled + k] = vdir * (speed / np.sqrt(PLUMMER_A))[:, None]
        filled += k
    if masses is None:
        masses = np.full(n, 1.0 / n)
    x -= (masses[:, None] * x).sum(0) / masses.sum()
    v -= (masses[:, None] * v).sum(0) / masses.sum()
    return x, v, masses


def salpeter(n: int, seed: int, mlo: float = 0.1, mhi: float = 100.0, slope: float = 2.35):
    """Masses dN/dm ~ m^-slope on [mlo, mhi], rescaled to total mass 1."""
    rng = np.random.default_rng(seed)
    e = 1.0 - slope
    u = rng.random(n)
    m = (mlo ** e + u * (mhi ** e - mlo ** e)) ** (1.0 / e)
    return m / m.sum()


def add_binaries(x, v, m, frac: float, seed: int, amin=1e-6, amax=1e-4):
    """Turns a fraction `frac` of the particles into circular binaries: pairs
    (2k, 2k+1) of a random subset keep their centre of mass at the first
    member's position/velocity and are placed at separation a ~ logU(amin,
    amax) with the circular relative speed sqrt(G (m1 + m2) / a)."""
    rng = np.random.default_rng(seed)
    n = len(m)
    npairs = int(frac * n) // 2
    if npairs == 0:
        return x, v, m, np.zeros((0, 2), dtype=np.int64)
    idx = rng.permutation(n)[: 2 * npairs].reshape(npairs, 2)
    p, s = idx[:, 0], idx[:, 1]
    a = np.exp(rng.uniform(np.log(amin), np.log(amax), npairs))
    ct = rng.uniform(-1, 1, npairs)
    ph = rng.uniform(0, 2 * np.pi, npairs)
    st = np.sqrt(1 - ct * ct)
    nhat = np.stack([st * np.cos(ph), st * np.sin(ph), ct], axis=1)
    # a unit vector perpendicular to nhat
    helper = np.where(np.abs(nhat[:, 2:3]) < 0.9, [[0.0, 0.0, 1.0]], [[1.0, 0.0, 0.0]])
    that = np.cross(nhat, helper)
    that /= np.linalg.norm(that, axis=1)[:, None]
    m1, m2 = m[p], m[s]
    mt = m1 + m2
    vrel = np.sqrt(mt / a)
    xc, vc = x[p].copy(), v[p].copy()
    x[p] = xc + (m2 / mt * a)[:, None] * nhat
    x[s] = xc - (m1 / mt * a)[:, None] * nhat
    v[p] = vc + (m2 / mt * vrel)[:, None] * that
    v[s] = vc - (m1 / mt * vrel)[:, None] * that
    return x, v, m, idx


def plummer_h2(x: np.ndarray, m: np.ndarray, nngb: float = 32.0):
    """Per-particle h2 so that the expected neighbour count within sqrt(h2)
    is `nngb`, from the analytic Plummer density at each particle's radius
    (local mean particle mass)."""
    r2 = (x * x).sum(1)
    rho = 3.0 / (4.0 * np.pi * PLUMMER_A ** 3) * (1.0 + r2 / PLUMMER_A ** 2) ** (-2.5)
    mbar = m.mean()
    h3 = nngb * mbar / (4.0 / 3.0 * np.pi * rho)
    return h3 ** (2.0 / 3.0)


def crackle_from(x, a, jrk):
    """Crackle (2nd derivative of jerk) for the 6th-order predictor input,
    from the harmonic estimate c = -w^2 j with w^2 = |a| / max(|x|, 1e-3).
    It only feeds the predictor and is parity-neutral input data."""
    w2 = np.linalg.norm(a, axis=1) / np.maximum(np.linalg.norm(x, axis=1), 1e-3)
    return -w2[:, None] * jrk


def block_timesteps(n: int, seed: int, kmin: int = 3, kmax: int = 12):
    """dt = 2^-k with k uniform in [kmin, kmax]."""
    rng = np.random.default_rng(seed)
    k = rng.integers(kmin, kmax + 1, n)
    return k, np.ldexp(1.0, -k)


def block_state(k: np.ndarray, step: int, kmax: int = 12):
    """At global time T = step * 2^-kmax: each particle's last update time
    t0 = floor(T / dt) * dt and the active set (dt divides T)."""
    T = np.ldexp(float(step), -kmax)
    dt = np.ldexp(1.0, -k)
    t0 = np.floor(T / dt) * dt
    active = np.nonzero(t0 == T)[0]
    return T, t0, active


def make_config(name: str, n: int | None = None, seed: int | None = None) -> dict:
    """Input state of one of the documented workloads (positions/velocities
    at each particle's own time t0; derivatives are filled in separately by a
    direct summation, see `fill_derivatives`).

    C1  Plummer equal mass, 4th order, eps2 = 1e-6, t0 = t_i - U{0..7} 2^-10,
        all active, lists off.
    C2  Plummer equal mass, 6th order, block steps dt = 2^-k (k in 3..12),
        h2 for ~32 neighbours, lists on.
    C3  Plummer + Salpeter masses + 10 % circular binaries, 6th order,
        t0 = t_i - U{0..7} 2^-10, all active.
    C5  Plummer equal mass + 10 % circular binaries, 6th order, lists on.
    """
    defaults = {"C1": (16384, 1), "C2": (131072, 2), "C3": (1 << 20, 3), "C5": (262144, 5)}
    n0, s0 = defaults[name]
    n = n or n0
    seed = s0 if seed is None else seed
    rng = np.random.default_rng(seed + 1000)
    cfg = {"name": name, "n": n, "seed": seed, "eps2": 1e-6}
    if name == "C1":
        x, v, m = plummer(n, seed)
        cfg.update(order=1, x=x, v=v, m=m, ti=1.0)
        cfg["t0"] = cfg["ti"] - rng.integers(0, 8, n) * 2.0 ** -10
        cfg["h2"] = np.zeros(n)
        cfg["lists"] = False
    elif name in ("C2",):
        x, v, m = plummer(n, seed)
        k, dt = block_timesteps(n, seed + 7)
        cfg.update(order=2, x=x, v=v, m=m, k=k, dt=dt)
        cfg["h2"] = plummer_h2(x, m, 32.0)
        cfg["lists"] = True
    elif name in ("C3", "C5"):
        m = salpeter(n, seed) if name == "C3" else np.full(n, 1.0 / n)
        x, v, m = plummer(n, seed, masses=m)
        x, v, m, pairs = add_binaries(x, v, m, 0.10, seed + 11)
        cfg.update(order=2, x=x, v=v, m=m, pairs=pairs, ti=1.0)
        cfg["t0"] = cfg["ti"] - rng.integers(0, 8, n) * 2.0 ** -10
        cfg["h2"] = plummer_h2(x, m, 32.0)
        cfg["lists"] = name == "C5"
    cfg["id"] = np.arange(n, dtype=np.int32)
    return cfg


def fill_derivatives(cfg: dict, force_fn) -> dict:
    """Sets the j acceleration, jerk (and snap, crackle for 6th order) from a
    direct summation at each particle's own state.  `force_fn(order, x, v, a,
    m, ids, eps2)` returns (acc, jrk, snp) for all particles (an FP64
    direct-summation routine)."""
    order = cfg["order"]
    x, v, m, ids, eps2 = cfg["x"], cfg["v"], cfg["m"], cfg["id"], cfg["eps2"]
    acc, jrk, _ = force_fn(1, x, v, None, m, ids, eps2)
    cfg["a"], cfg["j"] = acc, jrk
    if order >= 2:
        _, _, snp = force_fn(2, x, v, acc, m, ids, eps2)
        cfg["s"] = snp
        cfg["c"] = crackle_from(x, acc, jrk)
    return cfg


def predict_fp64(order: int, ti: float, t0, x, v, a, j, s=None, c=None):
    """FP64 Taylor prediction to ti in the Horner form of the device
    predictor (used to build the i-particle inputs of the workloads)."""
    dt = (ti - np.asarray(t0))[:, None]
    dt2, dt3 = dt * (1.0 / 2.0), dt * (1.0 / 3.0)
    if order >= 2:
        dt4, dt5 = dt * (1.0 / 4.0), dt * (1.0 / 5.0)
        px = x + dt * (v + dt2 * (a + dt3 * (j + dt4 * (s + dt5 * c))))
        pv = v + dt * (a + dt2 * (j + dt3 * (s + dt4 * c)))
        pa = a + dt * (j + dt2 * (s + dt3 * c))
        return px, pv, pa
    px = x + dt * (v + dt2 * (a + dt3 * j))
    pv = v + dt * (a + dt2 * j)
    return px, pv, None
