"""The centre-line screen of the mixed-precision candidate kernels
(separated_on_centre_line in xdem_b200/csrc/pairs.cuh) drops a candidate pair
of ellipses when the centre distance exceeds the sum of the two half-widths
along the line of centres.  The exact distance of closest approach along that
line is at most the sum, so neither contact law finds a contact there.  These
CPU tests hold the checker's closest-approach and intersection laws (and the
compiled reference's, where it is built) to that on pairs drawn at and just
beyond the screen's threshold, with the aspect ratios and sizes of the shear
workloads, and show what share of the listed non-touching pairs the screen
removes.

The screen runs in mixed precision only: the reference's construction reports
a contact for such a pair in its degenerate branch (a Newton result that is
not finite gives d' = 1 + a2', EllipticParticle.cpp:168-170), which random
pairs do not reach but the FP64 path must reproduce.
"""
import numpy as np
import pytest

import oracle
from xdem_b200 import abi

MARGIN = 1.001  # the device test: |d|² > (H_i + H_j) * MARGIN


def _half_width_sum(dx, dy, a1, b1, t1, a2, b2, t2):
    """H_i + H_j with H = sqrt(a²(d·k)² + b²(d×k)²), k the major axis."""
    def H(a, b, t):
        c, s = np.cos(t), np.sin(t)
        p, q = dx * c + dy * s, dx * s - dy * c
        return np.sqrt(a * a * p * p + b * b * q * q)
    return H(a1, b1, t1) + H(a2, b2, t2)


def _pairs(seed, N, beyond):
    """Pairs with a/b ~ U[1,3], b in {0.5, 0.7}; centre distance between the
    screen's threshold and the bounding-circle sum when beyond, else anywhere
    inside the bounding circles."""
    rng = np.random.default_rng(seed)
    b1 = rng.choice([0.5, 0.7], N)
    a1 = b1 * rng.uniform(1.0, 3.0, N)
    b2 = rng.choice([0.5, 0.7], N)
    a2 = b2 * rng.uniform(1.0, 3.0, N)
    t1 = rng.uniform(-30.0, 30.0, N)
    t2 = rng.uniform(-30.0, 30.0, N)
    ang = rng.uniform(0.0, 2.0 * np.pi, N)
    ux, uy = np.cos(ang), np.sin(ang)
    hs = _half_width_sum(ux, uy, a1, b1, t1, a2, b2, t2)  # half-width sum along û
    if beyond:
        # biased towards the threshold, where a wrong screen would show first
        f = rng.uniform(0.0, 1.0, N) ** 3
        dist = hs * MARGIN * (1.0 + 1e-9) + f * np.maximum(a1 + a2 - hs * MARGIN, 0.0)
    else:
        dist = (a1 + a2) * rng.uniform(0.5, 1.0, N)
    x0, y0 = rng.uniform(-800.0, 800.0, N), rng.uniform(-800.0, 800.0, N)
    zero = np.zeros(N)
    pi = np.stack([np.ones(N), a1, a1 / b1, x0, y0, zero, zero, t1, zero], 1)
    pj = np.stack([np.ones(N), a2, a2 / b2, x0 + dist * ux, y0 + dist * uy, zero, zero, t2, zero], 1)
    dx, dy = pj[:, 3] - pi[:, 3], pj[:, 4] - pi[:, 4]
    screened = dx * dx + dy * dy > _half_width_sum(dx, dy, a1, b1, t1, a2, b2, t2) * MARGIN
    return pi, pj, screened


@pytest.mark.parametrize("method", [abi.ELLIPSE_CLOSEST_APPROACH, abi.ELLIPSE_INTERSECTION])
@pytest.mark.parametrize("which", ["port", "reference"])
def test_no_contact_beyond_the_screen(method, which):
    if which == "reference" and not oracle.ref_available():
        pytest.skip("compiled reference absent")
    pi, pj, screened = _pairs(11 + method, 200000, beyond=True)
    assert screened.mean() > 0.99
    out, _ = oracle.pair_geometry(pi[screened], pj[screened], np.zeros((screened.sum(), 4)), method,
                                  which)
    assert not out[:, 0].any(), np.where(out[:, 0])[0][:5]


def test_screen_removes_most_non_touching_pairs():
    pi, pj, screened = _pairs(5, 200000, beyond=False)
    out, _ = oracle.pair_geometry(pi, pj, np.zeros((len(pi), 4)), abi.ELLIPSE_CLOSEST_APPROACH,
                                  "port")
    touching = out[:, 0] == 1
    assert not (screened & touching).any()
    assert 0.3 < touching.mean() < 0.7
    assert screened[~touching].mean() > 0.7
