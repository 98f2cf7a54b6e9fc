"""GPU tests of the learned warm start (xdem_mlp_*, xdem_set_warm_start).

  - forward and gradient of the network on the tensor cores against the CPU
    restatement with the GPU's BF16 rounding points (oracle/mlp.py): outputs
    within 5e-3 of their scale, gradient within 1e-2 relative L2 (BF16
    rounding of a value that lands on a different side of a rounding tie
    between the two FP32/FP64 accumulations changes it by one BF16 step);
  - training on pairs harvested from a sheared packing lowers the loss;
  - with the trained network attached, a closest-approach world gives the
    plain solver's results (state within 1e-10 relative, identical contact
    pairs) in fewer Newton iterations per solve, in FP64 and in the mixed
    path (whose FP64 pairs take the warm start).  The comparison runs on a
    packing where the plain iteration converges for every pair: where it
    cycles (the reference's loop never returns there, the solver stops at its
    cap) there is no answer to reproduce, and a warm start that converges
    gives a different value.
"""
import numpy as np
import pytest

from oracle import mlp as omlp
from xdem_b200 import abi
from xdem_b200.learned import Mlp, warm_stats
from xdem_b200.world import World, make_control

from helpers import compare_states, dense_ellipse_case, ellipse_case, same_pairs
from xdem_b200 import inputs

pytestmark = pytest.mark.gpu


def _samples(n, seed):
    rng = np.random.default_rng(seed)
    x = np.stack([rng.uniform(-4, 4, n), rng.uniform(-4, 4, n), rng.uniform(-1, 1, n),
                  rng.uniform(-1, 1, n), rng.uniform(1, 3, n), rng.uniform(0.5, 4, n),
                  rng.uniform(0.5, 1.5, n)], 1).astype(np.float32)
    t = rng.uniform(0.2, 1.0, n).astype(np.float32)
    t[rng.uniform(0, 1, n) < 0.2] = np.nan
    c = (rng.uniform(0, 1, n) < 0.4).astype(np.float32)
    return x, t, c


def test_mlp_forward_matches_oracle():
    net = Mlp(seed=5)
    th, sc = net.get_params()
    x, _, _ = _samples(1001, 1)  # ragged: not a multiple of the 16-row tiles
    y = net.forward(x)
    yo, _ = omlp.forward(th, sc, x, mode="bf16")
    scale = np.max(np.abs(yo))
    assert np.max(np.abs(y - yo)) <= 5e-3 * scale, np.max(np.abs(y - yo)) / scale


def test_mlp_gradient_matches_oracle():
    net = Mlp(seed=7)
    th, sc = net.get_params()
    x, t, c = _samples(1000, 2)
    g, loss = net.gradient(x, t, c)
    lo, go = omlp.loss_and_grad(th, sc, x, t, c, mode="bf16")
    assert abs(loss - lo) <= 1e-3 * abs(lo)
    rel = np.linalg.norm(g - go) / np.linalg.norm(go)
    cos = float(np.dot(g, go) / (np.linalg.norm(g) * np.linalg.norm(go)))
    assert rel <= 1e-2 and cos >= 0.9999, (rel, cos)
    # padding stays zero
    assert np.all(g[:omlp.OFF["b1"][0]].reshape(omlp.H, omlp.K1)[:, omlp.N_IN:] == 0)


@pytest.fixture(scope="module")
def trained():
    """A network trained on pairs harvested from a sheared ellipse packing."""
    p, contacts, prm = dense_ellipse_case(n=3000, seed=41, kind=abi.WORLD_LEES_EDWARDS)
    w = World(prm)
    w.raise_mask = ~abi.ERR_NEWTON
    w.set_particles(p)
    w.set_contacts(contacts)
    net = Mlp(seed=3)
    for _ in range(20):
        w.run(5, make_control())
        net.harvest(w, stride=1)
    n = net.dataset_size()
    x, t, c = net.dataset()
    losses = net.train(epochs=60, batch=1024, lr=2e-3, seed=1)
    w.close()
    return net, (p, contacts, prm), n, x, t, c, losses


def test_harvest_and_training(trained):
    net, _, n, x, t, c, losses = trained
    assert n > 20000
    assert np.isfinite(x).all()
    ok = np.isfinite(t)
    # the root lies between 1 and the analytic start sqrt(δ+1): a fraction
    # below 1 of the start, or above 1 where the reference exchanged the
    # eigenvalues (δ < 0)
    assert ok.mean() > 0.3 and np.all(t[ok] > 0)
    assert set(np.unique(c)) <= {0.0, 1.0}
    assert losses[-1] < 0.3 * losses[0], losses
    # the trained network predicts the root fraction well on its data
    y = net.forward(x[ok][:4000])
    assert np.median(np.abs(y[:, 0] - t[ok][:4000])) < 0.05


@pytest.mark.parametrize("precision", [abi.PRECISION_FP64, abi.PRECISION_MIXED])
def test_warm_start_same_results_fewer_iterations(trained, precision):
    net = trained[0]
    p, prm = ellipse_case(n=2500, seed=44, kind=abi.WORLD_LEES_EDWARDS, aspect=inputs.c2_aspect,
                          compress=1.3)
    prm.precision = precision
    worlds = []
    for use in (False, True):
        w = World(prm)
        w.set_particles(p)
        if use:
            net.attach(w)
        w.reset_newton_stats()
        w.run(40, make_control(update_stress=True))
        worlds.append(w)
    plain, warm = worlds
    compare_states(warm.get_state(), plain.get_state(), 1e-10)
    assert same_pairs(warm.get_contacts(), plain.get_contacts())
    s0, i0, c0 = plain.newton_stats()
    s1, i1, _ = warm.newton_stats()
    assert c0 == 0  # every plain solve converged
    assert s1 == s0 > 0
    ws = warm_stats(warm)
    if precision == abi.PRECISION_FP64:
        assert ws["offered"] > 0 and ws["used"] > 0.2 * ws["offered"], ws
        assert i1 / s1 < i0 / s0, (i0 / s0, i1 / s1)
        assert ws["logit_right"] > 0.6 * ws["offered"], ws
    else:
        # only the few pairs the mixed path hands to the FP64 construction
        # take the warm start
        assert i1 <= i0, (i0, i1)


def test_tensor_core_barrier_wait_is_bounded():
    """A completion barrier that nothing arrives on: the kernels' wait gives up
    after its limit and reports a timeout instead of hanging."""
    import ctypes as C
    from xdem_b200 import abi
    lib = abi.load_library()
    ms = C.c_double(0.0)
    assert lib.xdem_selftest_bounded_wait(C.byref(ms)) == abi.ERR_TIMEOUT
    assert 0.0 < ms.value < 5000.0
    # the context stays usable
    net = Mlp(seed=3)
    x = _samples(200, 4)[0]
    assert np.all(np.isfinite(net.forward(x)))
