"""CPU checks of the warm-start network's restatement (oracle/mlp.py): its
gradient against central finite differences in FP64, and the BF16 rounding
helper.  The GPU's forward and backward passes are checked against this
restatement in tests/test_gpu_learned.py."""
import numpy as np

from oracle import mlp


def _params(seed):
    rng = np.random.default_rng(seed)
    p = {"W1": np.zeros((mlp.H, mlp.K1)), "b1": rng.normal(0, 0.1, mlp.H),
         "W2": rng.normal(0, 0.2, (mlp.H, mlp.H)), "b2": rng.normal(0, 0.1, mlp.H),
         "W3": rng.normal(0, 0.2, (mlp.H, mlp.H)), "b3": rng.normal(0, 0.1, mlp.H),
         "W4": np.zeros((mlp.OUTPAD, mlp.H)), "b4": np.zeros(mlp.OUTPAD)}
    p["W1"][:, :mlp.N_IN] = rng.normal(0, 0.5, (mlp.H, mlp.N_IN))
    p["W4"][:mlp.OUT] = rng.normal(0, 0.2, (mlp.OUT, mlp.H))
    p["b4"][:mlp.OUT] = rng.normal(0, 0.1, mlp.OUT)
    return mlp.pack(p)


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    th = _params(1)
    scale = np.ones(mlp.N_IN, np.float32)
    n = 24
    x = rng.normal(0, 1, (n, mlp.N_IN))
    t = rng.uniform(0.2, 1.0, n)
    t[::5] = np.nan  # no root: only the contact term
    c = (rng.uniform(0, 1, n) > 0.5).astype(float)
    loss, g = mlp.loss_and_grad(th, scale, x, t, c)
    live = [i for i in range(mlp.COUNT)
            if not (i < mlp.OFF["b1"][0] and (i % mlp.K1) >= mlp.N_IN)
            and not (mlp.OFF["W4"][0] <= i < mlp.OFF["b4"][0]
                     and (i - mlp.OFF["W4"][0]) // mlp.H >= mlp.OUT)
            and not (i >= mlp.OFF["b4"][0] + mlp.OUT)]
    idx = rng.choice(live, 60, replace=False)
    h = 1e-6
    for i in idx:
        tp, tm = th.copy(), th.copy()
        tp[i] += h
        tm[i] -= h
        fd = (mlp.loss_and_grad(tp, scale, x, t, c)[0] - mlp.loss_and_grad(tm, scale, x, t, c)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, g[i])
    assert loss > 0


def test_bf16_rounding():
    v = np.array([1.0, 1.00390625, 1.005859375, -3.140625, 1e-3], np.float32)
    r = mlp.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0  # a tie rounds to even
    assert r[2] == 1.0078125
    assert r[3] == -3.140625
    assert abs(r[4] - 1e-3) <= 1e-3 * 2 ** -8
