"""The neighbour-radius network: the FP64 CPU oracle is pinned by finite
differences (CPU); the GPU forward, backward and training kernels are
checked against it (GPU)."""
import numpy as np
import pytest

from oracle import mlp_oracle as M


def _params(seed):
    rng = np.random.default_rng(seed)
    p = []
    for name, shp in M.SHAPES:
        fan = shp[1] if len(shp) == 2 else M.H
        lim = np.sqrt(6.0 / fan) if name.startswith("W") else 0.1
        p.append(rng.uniform(-lim, lim, shp).ravel())
    return np.concatenate(p)


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    p = _params(2)
    x = rng.normal(size=(40, M.IN))
    t = rng.normal(size=40)
    g = M.gradient(p, x, t)
    idx = rng.choice(M.NP, 60, replace=False)
    for k in idx:
        e = np.zeros(M.NP)
        e[k] = 1e-6
        fd = (M.loss(p + e, x, t) - M.loss(p - e, x, t)) / 2e-6
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(g[k])), (k, fd, g[k])


gpu = pytest.mark.gpu


@gpu
def test_gpu_forward_and_gradient_match_oracle(gpu):
    import sapporo2_b200 as sp
    from sapporo2_b200.learned_h2 import H2Net
    rng = np.random.default_rng(3)
    with sp.Sapporo(order=sp.SIXTH) as s:
        net = H2Net(s, seed=11)
        p = net.params().astype(np.float64)
        for n in (1, 127, 128, 1000):
            x = rng.normal(size=(n, M.IN)).astype(np.float32)
            t = rng.normal(size=n).astype(np.float32)
            y = net.forward(x)
            yo, _ = M.forward(p, x)
            assert np.max(np.abs(y - yo)) <= 1e-5 * max(1.0, np.max(np.abs(yo)))
            g, loss = net.gradient(x, t)
            go = M.gradient(p, x, t)
            assert abs(loss - M.loss(p, x, t)) <= 1e-5 * max(1.0, M.loss(p, x, t))
            err = np.linalg.norm(g - go) / np.linalg.norm(go)
            assert err <= 1e-4, err
        net.close()


@gpu
def test_gpu_training_fits_a_smooth_target(gpu):
    import sapporo2_b200 as sp
    from sapporo2_b200.learned_h2 import H2Net
    rng = np.random.default_rng(4)
    x = rng.normal(size=(4096, M.IN)).astype(np.float32)
    t = (0.7 * x[:, 0] - 0.4 * x[:, 3] + 0.2 * np.tanh(x[:, 1] * x[:, 2])).astype(np.float32)
    with sp.Sapporo(order=sp.SIXTH) as s:
        net = H2Net(s, seed=12)
        l0 = M.loss(net.params().astype(np.float64), x, t)
        for _ in range(10):
            net.train(x, t, epochs=50, lr=3e-3)
        l1 = M.loss(net.params().astype(np.float64), x, t)
        net.close()
    assert l1 < 0.02 * l0, (l0, l1)


@gpu
def test_gpu_proposal_kernel_matches_the_host_features(gpu):
    """sapb_mlp_propose (features, standardisation, network, bounded
    correction in one kernel) against features built on the host."""
    import sapporo2_b200 as sp
    from sapporo2_b200.learned_h2 import H2Net
    rng = np.random.default_rng(8)
    n = 3000
    n_prev = rng.integers(0, 300, n).astype(np.float64)
    h2 = 10.0 ** rng.uniform(-6, -1, n)
    acc = rng.normal(size=(n, 3)) * 10.0 ** rng.uniform(-2, 2, (n, 1))
    jrk = rng.normal(size=(n, 3)) * 10.0 ** rng.uniform(-1, 3, (n, 1))
    from sapporo2_b200.learned_h2 import log_density
    hist = log_density(n_prev, h2) + rng.normal(scale=0.3, size=n)
    with sp.Sapporo(order=sp.SIXTH) as s:
        net = H2Net(s, seed=13)
        for lm in (None, hist):
            want = net.propose_host(n_prev, h2, acc, jrk, lm)
            got = net.propose(n_prev, h2, acc, jrk, lm)
            np.testing.assert_allclose(got, want, rtol=2e-5)
        net.close()
