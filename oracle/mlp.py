"""TEST INFRASTRUCTURE ONLY — CPU restatement of the warm-start network of
xdem_b200/csrc/mlp.cuh and learn.cu (no counterpart in the reference, which
has no learned component): forward pass, loss and gradient in numpy.

mode="fp64": plain FP64 arithmetic (checked against finite differences).
mode="bf16": FP64 arithmetic with the values rounded to BF16 where the GPU
rounds them (inputs, weights, hidden activations and the back-propagated
pre-activation gradients that feed the tensor cores), the checker of the
GPU's forward and backward passes.
Parameter layout (FP32 vector): W1[64][16], b1[64], W2[64][64], b2[64],
W3[64][64], b3[64], W4[8][64], b4[8].
"""
import numpy as np

N_IN, K1, H, OUT, OUTPAD = 7, 16, 64, 2, 8
LOGIT_WEIGHT = 0.1

OFF = {}
_o = 0
for _name, _size in (("W1", H * K1), ("b1", H), ("W2", H * H), ("b2", H), ("W3", H * H), ("b3", H),
                     ("W4", OUTPAD * H), ("b4", OUTPAD)):
    OFF[_name] = (_o, _size)
    _o += _size
COUNT = _o


def bf16(a):
    """round to the nearest BF16 (ties to even), returned as float64"""
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(theta):
    th = np.asarray(theta, np.float64)
    p = {}
    for name, (o, s) in OFF.items():
        p[name] = th[o:o + s].copy()
    p["W1"] = p["W1"].reshape(H, K1)
    p["W2"] = p["W2"].reshape(H, H)
    p["W3"] = p["W3"].reshape(H, H)
    p["W4"] = p["W4"].reshape(OUTPAD, H)
    return p


def pack(p):
    th = np.zeros(COUNT)
    for name, (o, s) in OFF.items():
        th[o:o + s] = np.asarray(p[name]).reshape(-1)
    return th


def _sig(z):
    return 1.0 / (1.0 + np.exp(-z))


def forward(theta, scale, x, mode="fp64"):
    """outputs (n, 2) and the intermediates for the backward pass"""
    r = bf16 if mode == "bf16" else (lambda a: np.asarray(a, np.float64))
    p = unpack(theta)
    xs = (np.asarray(x, np.float32) * np.asarray(scale, np.float32)).astype(np.float64)
    x16 = np.zeros((len(xs), K1))
    x16[:, :N_IN] = r(xs)
    W = [r(p["W1"]), r(p["W2"]), r(p["W3"]), r(p["W4"])]
    z1 = x16 @ W[0].T + p["b1"]
    h1 = r(z1 * _sig(z1))
    z2 = h1 @ W[1].T + p["b2"]
    h2 = r(z2 * _sig(z2))
    z3 = h2 @ W[2].T + p["b3"]
    h3 = r(z3 * _sig(z3))
    y = h3 @ W[3][:OUT].T + p["b4"][:OUT]
    return y, dict(x16=x16, z=(z1, z2, z3), h=(h1, h2, h3), W=W)


def loss_and_grad(theta, scale, x, target, contact, mode="fp64"):
    """mean loss and its gradient (COUNT,) with the GPU's loss:
    valid * (y0 - target)^2 + 0.1 * BCE-with-logits(y1, contact)"""
    r = bf16 if mode == "bf16" else (lambda a: np.asarray(a, np.float64))
    n = len(x)
    y, c = forward(theta, scale, x, mode)
    t = np.asarray(target, np.float64)
    ct = np.asarray(contact, np.float64)
    valid = np.isfinite(t)
    tz = np.where(valid, t, 0.0)
    y0, y1 = y[:, 0], y[:, 1]
    sp = np.where(y1 > 0, y1 + np.log1p(np.exp(-y1)), np.log1p(np.exp(y1)))
    loss = np.sum(np.where(valid, (y0 - tz) ** 2, 0.0) + LOGIT_WEIGHT * (sp - ct * y1)) / n
    dy = np.zeros((n, 2))
    dy[:, 0] = np.where(valid, 2.0 * (y0 - tz) / n, 0.0)
    dy[:, 1] = LOGIT_WEIGHT * (_sig(y1) - ct) / n
    (z1, z2, z3), (h1, h2, h3), W = c["z"], c["h"], c["W"]

    def dsilu(z):
        s = _sig(z)
        return s * (1.0 + z * (1.0 - s))
    dz3 = r((dy @ W[3][:OUT]) * dsilu(z3))
    dz2 = r((dz3 @ W[2]) * dsilu(z2))
    dz1 = r((dz2 @ W[1]) * dsilu(z1))
    g = {
        "W1": dz1.T @ c["x16"], "b1": dz1.sum(0),
        "W2": dz2.T @ h1, "b2": dz2.sum(0),
        "W3": dz3.T @ h2, "b3": dz3.sum(0),
        "W4": np.zeros((OUTPAD, H)), "b4": np.zeros(OUTPAD),
    }
    g["W4"][:OUT] = dy.T @ h3
    g["b4"][:OUT] = dy.sum(0)
    g["W1"][:, N_IN:] = 0.0
    return loss, pack(g)
