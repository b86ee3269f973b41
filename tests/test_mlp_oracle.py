"""The CPU oracle of the surrogate network: BF16 rounding and the analytic gradient of the
FP64 network against central finite differences."""
import numpy as np

from oracle import mlp as mo


def test_bf16_rounding_nearest_even():
    one = 1.0
    ulp = 2.0 ** -7                         # BF16 spacing at 1
    assert mo.bf16([one])[0] == one
    assert mo.bf16([one + ulp / 2])[0] == one            # tie -> even (1.0)
    assert mo.bf16([one + 1.5 * ulp])[0] == one + 2 * ulp  # tie -> even (1 + 2 ulp)
    assert mo.bf16([one + 0.75 * ulp])[0] == one + ulp
    assert mo.bf16([-3.0])[0] == -3.0
    x = np.random.default_rng(0).normal(size=1000)
    r = mo.bf16(x)
    assert np.all(np.abs(r - x) <= np.abs(x) * 2.0 ** -8 * 1.0001)


def _net(hidden=16, n_emb=3, seed=0):
    L = mo.layout(hidden, n_emb)
    rng = np.random.default_rng(seed)
    th = rng.normal(0, 0.3, L["total"])
    return mo.MlpOracle(th, hidden, n_emb, bf16_mode=False)


def test_fp64_gradient_matches_finite_differences():
    net = _net()
    rng = np.random.default_rng(1)
    x = rng.normal(size=(10, 64))
    conf = rng.integers(-1, 3, 10)
    t = rng.normal(size=10)
    _, g = net.backward(x, t, conf)
    idx = rng.choice(net.L["b4"][0] + 1, 60, replace=False).tolist()
    idx += [net.L["emb"][0] + i for i in range(0, 96, 7)]
    h = 1e-6
    for i in idx:
        th0 = net.theta[i]
        net.theta[i] = th0 + h
        lp = net.loss(x, t, conf)
        net.theta[i] = th0 - h
        lm = net.loss(x, t, conf)
        net.theta[i] = th0
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_adam_reference_step():
    th = np.array([1.0, -2.0])
    g = np.array([0.5, -0.25])
    m = np.zeros(2)
    v = np.zeros(2)
    mo.MlpOracle.adam(th, g, m, v, 1, 0.1)
    # first step: m_hat = g, v_hat = g^2 -> step = lr * sign(g)
    assert np.allclose(th, [0.9, -1.9], atol=1e-6)
