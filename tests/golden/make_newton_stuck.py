"""Generates tests/golden/newton_stuck.npz: ellipse pairs on which the
closest-approach Newton iteration of the reference (NewtonRaphsonForQuartic,
EllipticParticle.cpp:613-626) never terminates.

The compiled reference does not return on these pairs (its loop has no cap),
so the fixture holds only the inputs and the C restatement's outputs
(oracle/liboracle.so), which stops the iteration at a repeated iterate or its
cap and takes the quartic's root on [min(1, s), max(1, s)] by bisection.
Pairs are found by a seeded random search over deep overlaps with the shapes
of the shear workloads (a/b ~ U[1,3], b in {0.5, 0.7}).  Run from the
repository root:

    python tests/golden/make_newton_stuck.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from xdem_b200 import abi  # noqa: E402


def deep_pairs(rng, N):
    b1 = rng.choice([0.5, 0.7], N)
    a1 = b1 * rng.uniform(1.0, 3.0, N)
    b2 = rng.choice([0.5, 0.7], N)
    a2 = b2 * rng.uniform(1.0, 3.0, N)
    t1 = rng.uniform(-30.0, 30.0, N)
    t2 = rng.uniform(-30.0, 30.0, N)
    ang = rng.uniform(0.0, 2.0 * np.pi, N)
    dist = (a1 + a2) * rng.uniform(0.02, 0.7, N)
    zero = np.zeros(N)
    pi = np.stack([np.ones(N), a1, a1 / b1, zero, zero, zero, zero, t1, zero], 1)
    pj = np.stack([np.ones(N), a2, a2 / b2, dist * np.cos(ang), dist * np.sin(ang), zero, zero, t2,
                   zero], 1)
    return pi, pj


def main(want=40, seed=7):
    rng = np.random.default_rng(seed)
    keep_i, keep_j = [], []
    while sum(len(k) for k in keep_i) < want:
        pi, pj = deep_pairs(rng, 500_000)
        out, _ = oracle.pair_geometry(pi, pj, np.zeros((len(pi), 4)), abi.ELLIPSE_CLOSEST_APPROACH,
                                      "port")
        # a converging solve needs at most a few hundred iterations; the ones
        # that stop on a repeat or the cap are recognised by re-running Newton
        cand = np.nonzero(out[:, 16] >= 50)[0]
        for k in cand:
            _, st = oracle.pair_geometry(pi[k:k + 1], pj[k:k + 1], np.zeros((1, 4)),
                                         abi.ELLIPSE_CLOSEST_APPROACH, "port")
            if st & abi.ERR_NEWTON:
                keep_i.append(pi[k:k + 1])
                keep_j.append(pj[k:k + 1])
    pi = np.concatenate(keep_i)[:want]
    pj = np.concatenate(keep_j)[:want]
    off = np.zeros((len(pi), 4))
    out, st = oracle.pair_geometry(pi, pj, off, abi.ELLIPSE_CLOSEST_APPROACH, "port")
    np.savez_compressed(os.path.join(HERE, "newton_stuck.npz"), pi=pi, pj=pj, off=off,
                        out=out, status=st, source="C restatement (oracle/liboracle.so)")
    print(f"{len(pi)} pairs, iterations {out[:, 16].min():.0f}..{out[:, 16].max():.0f}")


if __name__ == "__main__":
    main()
