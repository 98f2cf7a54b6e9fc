"""GPU tests of the mixed-precision path (XDEM_PRECISION_MIXED): FP32 contact
geometry and forces, FP64 positions, velocities, tangential springs and
Lees-Edwards shift, FP64 evaluation of the closest-approach distance.

It is compared with the FP64 checker (oracle/, pinned to the compiled
reference) and with the FP64 GPU path on identical inputs.  Tolerances, each
the stated error of the mixed path:
  - contact pair sets: identical to FP64 (the overlap that decides contact is
    evaluated in FP64 from the FP32 solve; pairs within 1e-9 of tangency are
    the only ones allowed to differ, and the tests below contain none);
  - per-pair geometry: overlap within 1e-6 relative (plus 1e-12 absolute),
    normals, contact points and branch vectors within 2e-6, velocities
    within 2e-6 of their largest magnitude;
  - forces after one step from an identical state: within 1e-5 of the
    largest contact force, per contact (the force tolerance the mixed mode
    promises), torques likewise;
  - mean shear stress of a Lees-Edwards shear run: within 0.5 %.
"""
import numpy as np
import pytest

import oracle
from xdem_b200 import abi, inputs
from xdem_b200.world import World, make_control, pair_geometry

from helpers import disc_case, ellipse_case, same_pairs

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-5


def _ellipse_pairs(N, seed, aspect_hi=3.0):
    rng = np.random.default_rng(seed)
    b1 = rng.choice([0.5, 0.7], N)
    a1 = b1 * rng.uniform(1.0, aspect_hi, N)
    b2 = rng.choice([0.5, 0.7], N)
    a2 = b2 * rng.uniform(1.0, aspect_hi, N)
    ang = rng.uniform(0, 2 * np.pi, N)
    dist = rng.uniform(0.5, 1.05, N) * (a1 + a2)
    pi = np.stack([np.ones(N), a1, a1 / b1, rng.normal(0, 5, N), rng.normal(0, 5, N),
                   rng.normal(0, .1, N), rng.normal(0, .1, N), rng.uniform(-20, 20, N),
                   rng.normal(0, .1, N)], 1)
    pj = pi.copy()
    pj[:, 1], pj[:, 2] = a2, a2 / b2
    pj[:, 3] = pi[:, 3] + dist * np.cos(ang)
    pj[:, 4] = pi[:, 4] + dist * np.sin(ang)
    pj[:, 5:7] = rng.normal(0, .1, (N, 2))
    pj[:, 7] = rng.uniform(-20, 20, N)
    return pi, pj


def test_mixed_pair_geometry_closest_approach():
    pi, pj = _ellipse_pairs(20000, 3)
    off = np.zeros((len(pi), 4))
    om, sm = pair_geometry(pi, pj, off, abi.ELLIPSE_CLOSEST_APPROACH, precision=abi.PRECISION_MIXED)
    oc, sc = oracle.pair_geometry(pi, pj, off, abi.ELLIPSE_CLOSEST_APPROACH, "port")
    assert np.array_equal(om[:, 0], oc[:, 0]), np.where(om[:, 0] != oc[:, 0])
    c = oc[:, 0] == 1
    assert c.sum() > 5000
    ov_m, ov_c = om[c, 9], oc[c, 9]
    assert np.all(np.abs(ov_m - ov_c) <= 1e-6 * np.abs(ov_c) + 1e-12)
    for cols in ((1, 2), (3, 4), (5, 6), (7, 8)):
        assert np.max(np.abs(om[c][:, cols] - oc[c][:, cols])) <= 2e-6, cols
    for cols in ((10, 11), (12, 13), (14, 15)):
        scale = np.max(np.abs(oc[c][:, cols]))
        assert np.max(np.abs(om[c][:, cols] - oc[c][:, cols])) <= 2e-6 * scale, cols


def test_mixed_pair_geometry_circles_overlap_is_fp64():
    rng = np.random.default_rng(8)
    N = 4000
    r1 = rng.choice([0.5, 0.7], N)
    r2 = rng.choice([0.5, 0.7], N)
    ang = rng.uniform(0, 2 * np.pi, N)
    dist = rng.uniform(0.8, 1.02, N) * (r1 + r2)
    pi = np.stack([np.zeros(N), r1, np.ones(N), rng.normal(0, 30, N), rng.normal(0, 30, N),
                   rng.normal(0, .1, N), rng.normal(0, .1, N), np.zeros(N), rng.normal(0, .1, N)], 1)
    pj = pi.copy()
    pj[:, 1] = r2
    pj[:, 3] = pi[:, 3] + dist * np.cos(ang)
    pj[:, 4] = pi[:, 4] + dist * np.sin(ang)
    pj[:, 5:7] = rng.normal(0, .1, (N, 2))
    pj[:, 8] = rng.normal(0, .1, N)
    off = np.zeros((N, 4))
    om, _ = pair_geometry(pi, pj, off, precision=abi.PRECISION_MIXED)
    oc, _ = oracle.pair_geometry(pi, pj, off, 0, "port")
    np.testing.assert_array_equal(om[:, 0], oc[:, 0])
    c = oc[:, 0] == 1
    np.testing.assert_array_equal(om[c, 9], oc[c, 9])  # the FP64 overlap expression
    assert np.max(np.abs(om[c][:, 1:3] - oc[c][:, 1:3])) <= 2e-6


def _one_step_pair(p, prm_fp64, prm_mixed):
    c = oracle.PortWorld(prm_fp64)
    c.set_particles(p)
    g = World(prm_mixed)
    g.set_particles(p)
    c.takeTimeStep()
    g.takeTimeStep()
    return g.get_contacts(), c.get_contacts()


def _force_err(cm, cc):
    f_m = np.hypot(cm["fn_x"] + cm["ft_x"], cm["fn_y"] + cm["ft_y"])
    scale = np.max(np.hypot(cc["fn_x"] + cc["ft_x"], cc["fn_y"] + cc["ft_y"]))
    dfx = (cm["fn_x"] + cm["ft_x"]) - (cc["fn_x"] + cc["ft_x"])
    dfy = (cm["fn_y"] + cm["ft_y"]) - (cc["fn_y"] + cc["ft_y"])
    del f_m
    return np.max(np.hypot(dfx, dfy)) / scale


@pytest.mark.parametrize("kind", [abi.WORLD_PERIODIC, abi.WORLD_LEES_EDWARDS])
def test_mixed_ellipse_world_one_step_forces(kind):
    from ctypes import sizeof, memmove, byref
    p, prm = ellipse_case(n=3000, seed=21, kind=kind, aspect=inputs.c4_aspect, compress=1.3)
    pm = abi.Params()
    memmove(byref(pm), byref(prm), sizeof(abi.Params))
    pm.precision = abi.PRECISION_MIXED
    cm, cc = _one_step_pair(p, prm, pm)
    assert same_pairs(cm, cc)
    assert len(cc["id_i"]) > 1000
    assert _force_err(cm, cc) <= FORCE_TOL
    tscale = max(np.max(np.abs(cc["torque_i"])), 1e-300)
    assert np.max(np.abs(cm["torque_i"] - cc["torque_i"])) <= FORCE_TOL * tscale
    assert np.max(np.abs(cm["normal_x"] - cc["normal_x"])) <= 2e-6


def test_mixed_disc_world_one_step_forces():
    from ctypes import sizeof, memmove, byref
    p, prm = disc_case(n=2000, phi=0.82, seed=4, kind=abi.WORLD_LEES_EDWARDS, shift_strain_rate=0.05)
    pm = abi.Params()
    memmove(byref(pm), byref(prm), sizeof(abi.Params))
    pm.precision = abi.PRECISION_MIXED
    cm, cc = _one_step_pair(p, prm, pm)
    assert same_pairs(cm, cc)
    assert _force_err(cm, cc) <= FORCE_TOL


def test_mixed_lees_edwards_history_and_mean_shear_stress():
    """Several hundred steps of shear: the contact history carries over in
    both runs, and the time-averaged shear stress agrees within 0.5 %."""
    from ctypes import sizeof, memmove, byref
    p, prm = ellipse_case(n=4000, seed=33, kind=abi.WORLD_LEES_EDWARDS, aspect=inputs.c4_aspect,
                          compress=1.35, shift_rate=0.1)
    pm = abi.Params()
    memmove(byref(pm), byref(prm), sizeof(abi.Params))
    pm.precision = abi.PRECISION_MIXED
    g64, gmx = World(prm), World(pm)
    for w in (g64, gmx):
        w.raise_mask = ~abi.ERR_NEWTON
        w.set_particles(p)
    ctl = make_control(update_stress=True)
    s64, smx = [], []
    for _ in range(40):
        g64.run(20, ctl)
        gmx.run(20, ctl)
        s64.append(g64.getStress()[1])
        smx.append(gmx.getStress()[1])
    m64, mmx = np.mean(s64), np.mean(smx)
    assert abs(m64) > 0
    assert abs(mmx - m64) <= 5e-3 * abs(m64), (m64, mmx)
    assert g64.count_contacts() > 2000
    # the contact set after 800 steps is still nearly the same
    c64, cmx = g64.get_contacts(), gmx.get_contacts()
    k64 = set(zip(c64["id_i"].tolist(), c64["id_j"].tolist()))
    kmx = set(zip(cmx["id_i"].tolist(), cmx["id_j"].tolist()))
    assert len(k64 ^ kmx) <= 0.01 * len(k64)
