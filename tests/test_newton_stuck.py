"""Closest-approach Newton iterations that never terminate in the reference.

NewtonRaphsonForQuartic (EllipticParticle.cpp:613-626) has no iteration cap;
on some deeply overlapping pairs (δ < 0) its iterate wanders among negative
values where the quartic has no root and the reference never returns.  Both
the checker and the CUDA path stop such an iteration when it repeats an
earlier iterate exactly (the reference's loop is a function of the iterate
alone, so it would cycle forever) or at 1,000 iterations, take the quartic's
root on [min(1, s), max(1, s)] (s = sqrt(δ+1), the analytic start) by
bisection, and raise XDEM_ERR_NEWTON.  Where the reference returns, nothing
changes: a converging iteration never repeats an iterate.

Fixture: tests/golden/newton_stuck.npz (make_newton_stuck.py), 40
pairs found by a seeded search, with the checker's outputs.
"""
import os

import numpy as np
import pytest

import oracle
from xdem_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = os.path.join(HERE, "golden", "newton_stuck.npz")


def _quartic(A, B, C, D, E, x):
    return A * x ** 4 + B * x ** 3 + C * x ** 2 + D * x + E


def test_known_cycle_stops_and_bisects():
    """The input that cycles forever in the reference stops on a repeated
    iterate or the cap, and the bisection returns the root between the
    analytic start and 1 to the last double."""
    A, B, C, D, E = (-0.26036636837902971, -0.32298145246944276, 0.12112405448664837,
                     0.28164745468898272, 0.087345098145840058)
    s = 0.51812102010664518
    r, it, stuck = oracle.newton_quartic(A, B, C, D, E, s)
    assert stuck and it <= 1000
    q = oracle.bisect_quartic(A, B, C, D, E, s, r)
    assert s <= q <= 1.0
    lo, hi = np.nextafter(q, 0.0), np.nextafter(q, 2.0)
    f = lambda x: _quartic(A, B, C, D, E, x)  # noqa: E731
    assert f(q) == 0.0 or np.sign(f(lo)) != np.sign(f(hi))


def test_converging_iterations_are_the_reference_loop():
    """Cycle detection never fires on an iteration that converges: the
    checker's result equals a plain restatement of the reference loop over
    many slow and fast cases (Python floats are IEEE doubles, and the loop is
    written with the reference's operations)."""
    rng = np.random.default_rng(3)

    def plain(A, B, C, D, E, init):
        A0, B0, C0 = 4.0 * A, 3.0 * B, 2.0 * C
        r0, r, it = init, 0.0, 0
        while abs(r0 - r) > 1e-10 and it < 1000:
            r = r0
            r0 -= ((A * (r0 * r0 * r0 * r0) + B * (r0 * r0 * r0) + C * (r0 * r0) + D * r0 + E)
                   / (A0 * (r0 * r0 * r0) + B0 * (r0 * r0) + C0 * r0 + D))
            it += 1
        return r0, it

    seen_slow = 0
    for _ in range(3000):
        coef = rng.normal(0.0, 1.0, 5)
        init = float(rng.uniform(0.2, 1.5))
        r, it, stuck = oracle.newton_quartic(*coef, init)
        if stuck:
            continue
        rp, itp = plain(*coef, init)
        assert (r == rp or (np.isnan(r) and np.isnan(rp))) and it == itp
        seen_slow += it > 30
    assert seen_slow > 10


def test_fixture_pairs_are_stuck_and_resolved():
    """Every fixture pair raises XDEM_ERR_NEWTON in the checker, most of them
    stop on a repeated iterate well before the cap, and the checker still
    produces the fixture's outputs (its geometry comes from the bisected
    root, so it is finite)."""
    d = np.load(FIX)
    out, st = oracle.pair_geometry(d["pi"], d["pj"], d["off"], abi.ELLIPSE_CLOSEST_APPROACH, "port")
    assert st & abi.ERR_NEWTON
    np.testing.assert_array_equal(out, d["out"])
    assert np.all(out[:, 16] <= 1000)
    assert np.sum(out[:, 16] < 1000) >= len(out) // 2
    hit = out[:, 0] == 1
    assert np.all(np.isfinite(out[hit, 1:16]))
    for k in range(len(out)):
        _, stk = oracle.pair_geometry(d["pi"][k:k + 1], d["pj"][k:k + 1], d["off"][k:k + 1],
                                      abi.ELLIPSE_CLOSEST_APPROACH, "port")
        assert stk & abi.ERR_NEWTON, k


def test_converged_roots_outside_the_interval():
    """Where the reference returns, its root is not always the one in
    [min(1, s), max(1, s)]: over 200,000 seeded deep overlaps with the
    fixture's shapes, some converged solves end outside that interval
    (mostly at a negative root), and their share grows with the iteration
    count (a long wander before converging).  The interval's root (what the
    bisection, or a learned start clamped to the interval, finds) is then a
    different answer, which is why a solve that converges is never cut short
    in its favour."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_newton_stuck",
                                                  os.path.join(HERE, "golden", "make_newton_stuck.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    pi, pj = mod.deep_pairs(np.random.default_rng(5), 200_000)
    out, _ = oracle.closest_quartic(pi, pj, np.zeros((len(pi), 4)))
    solved = (out[:, 7] > 0) & (out[:, 8] == 0)
    o = out[solved]
    lo, hi = np.minimum(1.0, o[:, 5]), np.maximum(1.0, o[:, 5])
    outside = ~((o[:, 6] >= lo * (1 - 1e-12)) & (o[:, 6] <= hi * (1 + 1e-12)))
    assert outside.sum() > 0
    short, long_ = o[:, 7] < 10, o[:, 7] >= 20
    assert outside[long_].mean() > 10 * outside[short].mean()
    assert np.mean(o[outside, 6] < 0) > 0.5
    for c in o[outside][:20]:
        rb = oracle.bisect_quartic(*c[:5], c[5], np.nan)
        assert not (abs(rb - c[6]) <= 1e-9 * max(1.0, abs(c[6])))


@pytest.mark.gpu
def test_gpu_stuck_pairs_match_checker():
    """The CUDA closest-approach law on the fixture pairs.  The quartic's
    coefficients come from cos/sin of the orientations, which may round
    differently from glibc's; the wandering Newton iterate amplifies that, so
    the iteration may stop at another step.  The root it is meant to find is
    well conditioned, so wherever both stop on the same iteration count the
    geometry agrees within the FP64 bar, and the pairs flagged raise
    XDEM_ERR_NEWTON on the device as well."""
    from xdem_b200.world import pair_geometry
    d = np.load(FIX)
    og, st = pair_geometry(d["pi"], d["pj"], d["off"], abi.ELLIPSE_CLOSEST_APPROACH)
    assert st & abi.ERR_NEWTON
    oc = d["out"]
    same = og[:, 16] == oc[:, 16]
    assert same.sum() >= len(oc) // 2, (same.sum(), len(oc))
    assert np.array_equal(og[same, 0], oc[same, 0])
    hit = same & (oc[:, 0] == 1)
    for col in range(1, 16):
        a, b = og[hit, col], oc[hit, col]
        scale = max(np.max(np.abs(b)), 1e-300)
        assert np.max(np.abs(a - b)) <= 1e-10 * scale, col
