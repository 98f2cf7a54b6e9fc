"""Host side of the learned warm start of the closest-approach Newton
iteration (include/xdem_gpu.h, xdem_mlp_*): a network that predicts the root
of the reference's quartic (EllipticParticle.cpp:92-100, 163) as a fraction
of Newton's analytic start, plus a contact logit, trained on the GPU on pairs
harvested from worlds.  The network only moves Newton's starting point; the
iteration still runs to the reference's tolerance (see ellipse_closest in
xdem_b200/csrc/geometry.cuh), so results are the plain solver's wherever the
plain iteration's root lies in [min(1, sqrt(δ+1)), max(1, sqrt(δ+1))]; a
plain iteration that wanders long can end outside that interval, and the
warm-started solve then returns the interval's root instead."""
import ctypes as C

import numpy as np

from . import abi

N_IN = 7


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class Mlp:
    """The warm-start network (7 -> 64 -> 64 -> 64 -> 2, SiLU, BF16 weights)."""

    def __init__(self, seed=0):
        self.lib = abi.load_library()
        h = C.c_void_p()
        st = self.lib.xdem_mlp_create(seed, C.byref(h))
        if st:
            raise abi.XdemError(st, "xdem_mlp_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.xdem_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st, where):
        if st:
            raise abi.XdemError(st, where)

    @property
    def param_count(self):
        return int(self.lib.xdem_mlp_param_count())

    def get_params(self):
        th = np.zeros(self.param_count, np.float32)
        sc = np.zeros(N_IN, np.float32)
        self._check(self.lib.xdem_mlp_get_params(self.h, _fp(th), _fp(sc)), "get_params")
        return th, sc

    def set_params(self, theta=None, scale=None):
        th = None if theta is None else np.ascontiguousarray(theta, np.float32)
        sc = None if scale is None else np.ascontiguousarray(scale, np.float32)
        self._check(self.lib.xdem_mlp_set_params(self.h, None if th is None else _fp(th),
                                                 None if sc is None else _fp(sc)), "set_params")

    def forward(self, x):
        x = np.ascontiguousarray(x, np.float32)
        y = np.zeros((len(x), 2), np.float32)
        self._check(self.lib.xdem_mlp_forward(self.h, len(x), _fp(x), _fp(y)), "forward")
        return y

    def gradient(self, x, target, contact):
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(target, np.float32)
        c = np.ascontiguousarray(contact, np.float32)
        g = np.zeros(self.param_count, np.float32)
        loss = C.c_float(0.0)
        self._check(self.lib.xdem_mlp_gradient(self.h, len(x), _fp(x), _fp(t), _fp(c), _fp(g),
                                               C.byref(loss)), "gradient")
        return g, float(loss.value)

    def add_samples(self, x, target, contact):
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(target, np.float32)
        c = np.ascontiguousarray(contact, np.float32)
        self._check(self.lib.xdem_mlp_add_samples(self.h, len(x), _fp(x), _fp(t), _fp(c)),
                    "add_samples")

    def dataset_size(self):
        n = C.c_int64(0)
        self._check(self.lib.xdem_mlp_dataset(self.h, C.byref(n), None, None, None), "dataset")
        return int(n.value)

    def dataset(self):
        n = self.dataset_size()
        x = np.zeros((n, N_IN), np.float32)
        t = np.zeros(n, np.float32)
        c = np.zeros(n, np.float32)
        nn = C.c_int64(0)
        self._check(self.lib.xdem_mlp_dataset(self.h, C.byref(nn), _fp(x), _fp(t), _fp(c)), "dataset")
        return x, t, c

    def clear_dataset(self):
        self._check(self.lib.xdem_mlp_clear_dataset(self.h), "clear_dataset")

    def train(self, epochs, batch=4096, lr=1e-3, seed=0, max_samples=0):
        losses = np.zeros(epochs, np.float32)
        self._check(self.lib.xdem_mlp_train(self.h, epochs, batch, lr, seed, max_samples,
                                            _fp(losses)), "train")
        return losses

    def harvest(self, world, stride=1, max_new=1 << 20):
        """Appends pairs of the world's last candidate list to the training set."""
        n = C.c_int64(0)
        self._check(self.lib.xdem_harvest_pairs(world.h, self.h, stride, max_new, C.byref(n)),
                    "harvest_pairs")
        return int(n.value)

    def attach(self, world):
        """Gives the world's closest-approach Newton iteration this warm start."""
        self._check(self.lib.xdem_set_warm_start(world.h, self.h), "set_warm_start")
        world._warm_net = self

    @staticmethod
    def detach(world):
        lib = abi.load_library()
        lib.xdem_set_warm_start(world.h, None)
        world._warm_net = None


def warm_stats(world):
    """{offered, used, rejected, restarted, logit_right} since the last
    reset_newton_stats of the world."""
    out = (C.c_int64 * 5)()
    st = world.lib.xdem_get_warm_stats(world.h, out)
    if st:
        raise abi.XdemError(st, "get_warm_stats")
    keys = ("offered", "used", "rejected", "restarted", "logit_right")
    return {k: int(v) for k, v in zip(keys, out)}
