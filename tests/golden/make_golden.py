"""Generates the golden fixtures in this folder from the COMPILED REFERENCE
(oracle/_ref/libxdem_ref.so: the unmodified reference sources driven by
oracle/ref_harness.cpp).  Run from the repository root where the reference
sources were available at build time:

    python tests/golden/make_golden.py [fixture names, e.g. world_discs_segments_periodic]

(with names, only those fixtures are written)

Every fixture holds seeded inputs and the reference's outputs:
  pairs_<law>.npz    single-pair contact geometry (BaseParticle::
                     calculateContactGeometry) for random near-contact pairs,
                     incl. aligned, crossed and exactly touching cases;
  world_<case>.npz   a small world advanced a few steps by the reference's own
                     step methods: initial particles, parameters, control, and
                     the final state, contacts, forces, stress, box and
                     Lees-Edwards scalars.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import oracle  # noqa: E402
from xdem_b200 import abi  # noqa: E402

from helpers import clump_case, controls, disc_case, ellipse_case, segment_case  # noqa: E402


def random_pairs(seed, N, shape, b_range, asp_range, near):
    rng = np.random.default_rng(seed)
    b1, b2 = rng.uniform(*b_range, N), rng.uniform(*b_range, N)
    k1, k2 = rng.uniform(*asp_range, N), rng.uniform(*asp_range, N)
    a1, a2 = b1 * k1, b2 * k2
    ang = rng.uniform(0, 2 * np.pi, N)
    dist = rng.uniform(*near, N) * (a1 + a2)
    sh = np.full(N, float(shape))
    pi = np.stack([sh, a1, k1, rng.normal(0, 3, N), rng.normal(0, 3, N), rng.normal(0, .1, N),
                   rng.normal(0, .1, N), rng.uniform(0, np.pi, N), rng.normal(0, .1, N)], 1)
    pj = np.stack([sh, a2, k2, pi[:, 3] + dist * np.cos(ang), pi[:, 4] + dist * np.sin(ang),
                   rng.normal(0, .1, N), rng.normal(0, .1, N), rng.uniform(0, np.pi, N),
                   rng.normal(0, .1, N)], 1)
    off = np.zeros((N, 4))
    off[:, :2] = rng.choice([-20.0, 0.0, 20.0], (N, 2))
    pj[:, 3:5] -= off[:, :2]          # the image of j sits where it was drawn
    off[:, 2:] = rng.normal(0, 0.05, (N, 2))
    return pi, pj, off


ONLY = set(sys.argv[1:])


def wanted(name):
    return not ONLY or name in ONLY


def make_pairs():
    cases = {
        "circle": (0, 0, (0.3, 0.7), (1.0, 1.0), (0.8, 1.02)),
        "closest": (1, abi.ELLIPSE_CLOSEST_APPROACH, (0.4, 0.7), (1.0, 3.0), (0.5, 1.05)),
        "intersection": (1, abi.ELLIPSE_INTERSECTION, (0.4, 0.7), (1.0, 3.0), (0.5, 1.05)),
    }
    for name, (shape, method, br, ar, near) in cases.items():
        if not wanted(f"pairs_{name}"):
            continue
        pi, pj, off = random_pairs(1000 + len(name), 600, shape, br, ar, near)
        if shape == 1:
            pi[:40, 7] = pj[:40, 7] = 0.0
            pj[40:80, 7] = np.pi / 2
        else:
            pi[:10, 1], pj[:10, 1] = 0.5, 0.25
            pi[:10, 3:5] = 0.0
            pj[:10, 3], pj[:10, 4] = 0.75, 0.0
            off[:10, :2] = 0.0
        out, st = oracle.pair_geometry(pi, pj, off, method, "ref")
        np.savez_compressed(os.path.join(HERE, f"pairs_{name}.npz"), pi=pi, pj=pj, off=off,
                            out=out, method=method)
        print(name, int(out[:, 0].sum()), "contacts of", len(pi))


def save_world(name, p, prm, ctl, nsteps, mass=None):
    if not wanted(f"world_{name}"):
        return
    w = oracle.RefWorld(prm)
    w.set_particles(p)
    if prm.world_kind == abi.WORLD_PERIODIC_CONTROL:
        w.setVirtualBoundaryMass()
    done = w.run(nsteps, ctl)
    st = w.get_state()
    c = w.get_contacts()
    f = w.get_force_and_torque()
    arrs = {f"p_{k}": v for k, v in p.items() if isinstance(v, np.ndarray)}
    arrs.update({f"s_{k}": v for k, v in st.items()})
    arrs.update({f"c_{k}": v for k, v in c.items()})
    arrs.update({f"f_{k}": v for k, v in f.items()})
    arrs["params"] = np.frombuffer(bytes(prm), np.uint8)
    arrs["control"] = np.frombuffer(bytes(ctl), np.uint8)
    arrs["nsteps"] = np.array(done)
    arrs["stress"] = w.getStress()
    arrs["boundary"] = w.getBoundary()
    arrs["lees_edwards"] = w.getLeesEdwards()
    arrs["z_phi"] = w.quadron_z_phi()
    np.savez_compressed(os.path.join(HERE, f"world_{name}.npz"), **arrs)
    print(name, done, "steps", len(c["id_i"]), "contacts")


def make_worlds():
    ctl = controls()
    p, prm = disc_case(n=160, phi=0.80, seed=31)
    save_world("discs_periodic", p, prm, ctl["stress"], 25)
    p, prm = disc_case(n=160, phi=0.78, seed=32, kind=abi.WORLD_PERIODIC_CONTROL)
    save_world("discs_control_stress_xy", p, prm, ctl["stress_xy"], 25)
    p, prm = ellipse_case(n=160, seed=33, kind=abi.WORLD_LEES_EDWARDS,
                          method=abi.ELLIPSE_CLOSEST_APPROACH, compress=1.9, shift_rate=0.2)
    save_world("ellipses_closest_lees_edwards", p, prm, ctl["stress"], 20)
    p, prm = ellipse_case(n=160, seed=34, kind=abi.WORLD_PERIODIC_CONTROL,
                          method=abi.ELLIPSE_INTERSECTION, compress=1.9)
    save_world("ellipses_intersection_control_strain", p, prm, ctl["strain"], 20)
    p, prm = clump_case(nfree=60, nclump=15, seed=35)
    save_world("clumps_periodic", p, prm, ctl["stress"], 20)
    p, prm = segment_case(n=220, seed=36)
    save_world("discs_segments_periodic", p, prm, ctl["stress"], 25)
    p, prm = segment_case(n=220, seed=37, kind=abi.WORLD_LEES_EDWARDS, shift_strain_rate=0.1)
    save_world("discs_segments_lees_edwards", p, prm, ctl["stress"], 25)


if __name__ == "__main__":
    if not oracle.ref_available():
        sys.exit("the compiled reference (oracle/_ref) is required")
    make_pairs()
    make_worlds()
