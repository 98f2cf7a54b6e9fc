"""GPU parity: the CUDA path (through the C-ABI) against the C restatement
(oracle/), which tests/test_oracle_vs_reference.py pins to the compiled
reference.

Tolerances.  The CUDA FP64 path performs the reference's operations in the
reference's order with -fmad=false; it differs only where CUDA's cos, sin,
atan2 and pow round differently from glibc's (within a few ulp).  Hence:
  - contact pair sets: identical (bit-exact integer sets);
  - circle geometry: bit-exact (only + - * / sqrt);
  - one step from an identical state: every contact field and every particle
    sum within 1e-10 relative to the largest magnitude of that field (the
    FP64 bar); ellipse pair geometry within 1e-10 where the problem is well
    conditioned and within a few times the checker's own 1-ulp sensitivity
    near tangency (the intersection quartic has a near-double root there);
  - short trajectories: within 1e-9 relative after 30-50 steps;
  - determinism: two GPU runs agree bit for bit.
"""
import numpy as np
import pytest

import oracle
from xdem_b200 import abi
from xdem_b200.world import World, make_control, pair_geometry

from helpers import (setup_control, clump_case, compare_contacts, compare_pair_geometry, compare_states, controls,
                     disc_case, ellipse_case, rel_err, same_pairs)

pytestmark = pytest.mark.gpu

ONE_STEP_TOL = 1e-10
TRAJ_TOL = 1e-9


def _pair(p, prm):
    g = World(prm)
    g.set_particles(p)
    c = oracle.PortWorld(prm)
    c.set_particles(p)
    if prm.world_kind == abi.WORLD_PERIODIC_CONTROL:
        g.setVirtualBoundaryMass()
        c.setVirtualBoundaryMass()
    return g, c


def _compare_worlds(g, c, tol):
    compare_contacts(g.get_contacts(), c.get_contacts(), tol)
    compare_states(g.get_state(), c.get_state(), tol)
    fg, fc = g.get_force_and_torque(), c.get_force_and_torque()
    for k in ("fx", "fy", "torque"):
        assert rel_err(fg[k], fc[k]) <= tol, k
    assert np.array_equal(fg["num_contacts"], fc["num_contacts"])
    assert np.array_equal(g.get_state()["is_rattler"], c.get_state()["is_rattler"])


def test_device_present():
    import ctypes as C
    lib = abi.load_library()
    n = C.c_int32(0)
    assert lib.xdem_device_count(C.byref(n)) == 0 and n.value >= 1


@pytest.mark.parametrize("method", [abi.ELLIPSE_CLOSEST_APPROACH, abi.ELLIPSE_INTERSECTION])
def test_pair_geometry_ellipses(method):
    rng = np.random.default_rng(42 + method)
    N = 4000
    b1 = rng.uniform(0.4, 0.7, N)
    a1 = b1 * rng.uniform(1.0, 3.0, N)
    b2 = rng.uniform(0.4, 0.7, N)
    a2 = b2 * rng.uniform(1.0, 3.0, N)
    ang = rng.uniform(0, 2 * np.pi, N)
    dist = rng.uniform(0.5, 1.05, N) * (a1 + a2)
    pi = np.stack([np.ones(N), a1, a1 / b1, rng.normal(0, 5, N), rng.normal(0, 5, N),
                   rng.normal(0, .1, N), rng.normal(0, .1, N), rng.uniform(0, np.pi, N),
                   rng.normal(0, .1, N)], 1)
    pj = pi.copy()
    pj[:, 1], pj[:, 2] = a2, a2 / b2
    pj[:, 3] = pi[:, 3] + dist * np.cos(ang)
    pj[:, 4] = pi[:, 4] + dist * np.sin(ang)
    pj[:, 5:7] = rng.normal(0, .1, (N, 2))
    pj[:, 7] = rng.uniform(0, np.pi, N)
    # aligned and crossed orientations
    pi[:200, 7] = 0.0
    pj[:200, 7] = 0.0
    pj[200:400, 7] = np.pi / 2
    off = np.zeros((N, 4))
    og, sg = pair_geometry(pi, pj, off, method)
    oc, sc = oracle.pair_geometry(pi, pj, off, method, "port")
    assert sg == sc
    assert np.array_equal(og[:, 0], oc[:, 0]), np.where(og[:, 0] != oc[:, 0])
    assert (og[:, 0] == 1).sum() > 500
    compare_pair_geometry(og, oc, pi, pj, off, method)


def test_pair_geometry_circles():
    rng = np.random.default_rng(7)
    N = 2000
    r1 = rng.choice([0.5, 0.7], N)
    r2 = rng.choice([0.5, 0.7], N)
    ang = rng.uniform(0, 2 * np.pi, N)
    dist = rng.uniform(0.8, 1.02, N) * (r1 + r2)
    pi = np.stack([np.zeros(N), r1, np.ones(N), np.zeros(N), np.zeros(N), rng.normal(0, .1, N),
                   rng.normal(0, .1, N), np.zeros(N), rng.normal(0, .1, N)], 1)
    pj = np.stack([np.zeros(N), r2, np.ones(N), dist * np.cos(ang), dist * np.sin(ang),
                   rng.normal(0, .1, N), rng.normal(0, .1, N), np.zeros(N), rng.normal(0, .1, N)], 1)
    # exactly touching (exactly representable): overlap 0 counts as contact
    pi[:10, 1], pj[:10, 1] = 0.5, 0.25
    pj[:10, 3], pj[:10, 4] = 0.75, 0.0
    off = np.zeros((N, 4))
    og, _ = pair_geometry(pi, pj, off)
    oc, _ = oracle.pair_geometry(pi, pj, off, 0, "port")
    np.testing.assert_array_equal(og[:, :16], oc[:, :16])  # + - * / sqrt only: bit-exact
    assert og[:10, 0].all()


@pytest.mark.parametrize("kind", [abi.WORLD_PERIODIC, abi.WORLD_PERIODIC_CONTROL,
                                  abi.WORLD_LEES_EDWARDS])
def test_discs_one_step(kind):
    p, prm = disc_case(n=400, phi=0.82, seed=1, kind=kind, shift_strain_rate=0.05)
    g, c = _pair(p, prm)
    g.takeTimeStep()
    c.takeTimeStep()
    _compare_worlds(g, c, ONE_STEP_TOL)


@pytest.mark.parametrize("method", [abi.ELLIPSE_CLOSEST_APPROACH, abi.ELLIPSE_INTERSECTION])
@pytest.mark.parametrize("kind", [abi.WORLD_PERIODIC, abi.WORLD_PERIODIC_CONTROL,
                                  abi.WORLD_LEES_EDWARDS])
def test_ellipses_one_step(kind, method):
    p, prm = ellipse_case(n=600, seed=2, kind=kind, method=method, compress=1.6)
    g, c = _pair(p, prm)
    g.takeTimeStep()
    c.takeTimeStep()
    assert c.count_contacts() > 100
    _compare_worlds(g, c, ONE_STEP_TOL)


@pytest.mark.parametrize("name", ["plain", "stress", "strain", "stress_xy", "uniform",
                                  "uniform_limit"])
def test_discs_trajectory_controls(name):
    kind = abi.WORLD_PERIODIC_CONTROL if name != "plain" else abi.WORLD_PERIODIC
    p, prm = disc_case(n=300, phi=0.80, seed=4, kind=kind)
    g, c = _pair(p, prm)
    setup_control(name, g, c)
    ctl = controls()[name]
    assert g.run(50, ctl) == 50
    assert c.run(50, ctl) == 50
    _compare_worlds(g, c, TRAJ_TOL)
    assert rel_err(g.getBoundary(), c.getBoundary()) <= TRAJ_TOL
    if ctl.update_stress:
        assert rel_err(g.getStress(), c.getStress()) <= TRAJ_TOL


@pytest.mark.parametrize("method", [abi.ELLIPSE_CLOSEST_APPROACH, abi.ELLIPSE_INTERSECTION])
def test_lees_edwards_ellipses_trajectory(method):
    p, prm = ellipse_case(n=500, seed=9, kind=abi.WORLD_LEES_EDWARDS, method=method, compress=1.5,
                          shift_rate=0.2)
    g, c = _pair(p, prm)
    ctl = make_control(update_stress=True)
    g.run(40, ctl)
    c.run(40, ctl)
    _compare_worlds(g, c, TRAJ_TOL)
    assert rel_err(g.getLeesEdwards(), c.getLeesEdwards()) <= 1e-15
    assert rel_err(g.getStress(), c.getStress()) <= TRAJ_TOL


def test_clumps_trajectory():
    p, prm = clump_case()
    g, c = _pair(p, prm)
    ctl = make_control(update_stress=True)
    g.run(30, ctl)
    c.run(30, ctl)
    _compare_worlds(g, c, TRAJ_TOL)
    sg, sc = g.get_state(), c.get_state()
    assert rel_err(sg["branch_x"], sc["branch_x"]) <= TRAJ_TOL
    assert rel_err(g.getStress(), c.getStress()) <= TRAJ_TOL


def test_substeps_equal_fused_step():
    """Calling the reference's sub-steps one by one gives the fused step's result."""
    p, prm = disc_case(n=300, phi=0.8, seed=6)
    a = World(prm)
    a.set_particles(p)
    b = World(prm)
    b.set_particles(p)
    for _ in range(3):
        a.takeTimeStep()
        b.modifyParticlePosition()
        b.findPossibleContacts()
        b.updateContacts()
        b.collectForceAndTorque()
        b.takeTimeIntegral()
    sa, sb = a.get_state(), b.get_state()
    for k in ("x", "y", "vx", "vy", "rot", "rot_vel"):
        np.testing.assert_array_equal(sa[k], sb[k])


def test_lees_edwards_substeps_equal_fused_step():
    """LE takeTimeStep folds apply/removeBackgroudVelocity into the kernels;
    the explicit sub-step sequence gives the same bits."""
    p, prm = ellipse_case(n=300, seed=3, kind=abi.WORLD_LEES_EDWARDS, compress=1.5)
    a = World(prm)
    a.set_particles(p)
    b = World(prm)
    b.set_particles(p)
    for _ in range(3):
        a.takeTimeStep()
        b.modifyParticlePosition()
        b.applyBackgroudVelocity()
        b.findPossibleContacts()
        b.updateContacts()
        b.removeBackgroudVelocity()
        b.collectForceAndTorque()
        b.takeTimeIntegral()
        b.updateLeesEdwardBoundary()
    sa, sb = a.get_state(), b.get_state()
    for k in ("x", "y", "vx", "vy", "rot", "rot_vel"):
        np.testing.assert_array_equal(sa[k], sb[k])


def test_many_resorts_match_checker():
    """Runs long enough for several memory-order refreshes (each captured chunk
    starts with one), with state read back and written again in between."""
    p, prm = disc_case(n=500, phi=0.80, seed=14)
    g, c = _pair(p, prm)
    ctl = make_control(update_stress=True)
    for chunk in (70, 64, 1, 33):
        g.run(chunk, ctl)
        c.run(chunk, ctl)
        _compare_worlds(g, c, TRAJ_TOL)
    # a state round trip through the id-ordered boundary leaves the run unchanged
    st = g.get_state()
    g.upload_state(st["x"], st["y"], st["vx"], st["vy"], st["rot"], st["rot_vel"])
    g.run(40, ctl)
    c.run(40, ctl)
    _compare_worlds(g, c, TRAJ_TOL)


def test_run_deterministic():
    p, prm = ellipse_case(n=500, seed=8, compress=1.5)
    out = []
    for _ in range(2):
        g = World(prm)
        g.set_particles(p)
        g.run(30, make_control(update_stress=True))
        out.append((g.get_state(), g.get_contacts(), g.getStress()))
    for k in ("x", "y", "vx", "vy", "rot", "rot_vel"):
        np.testing.assert_array_equal(out[0][0][k], out[1][0][k])
    assert same_pairs(out[0][1], out[1][1])
    np.testing.assert_array_equal(out[0][2], out[1][2])


def test_contact_upload_roundtrip():
    """Contacts downloaded from the checker and uploaded to the GPU world give
    the same next step (checkpoint/resume of the contact history)."""
    p, prm = disc_case(n=300, phi=0.82, seed=12)
    c = oracle.PortWorld(prm)
    c.set_particles(p)
    c.run(20)
    st = c.get_state()
    q = dict(p)
    for k in ("x", "y", "vx", "vy", "rot", "rot_vel"):
        q[k] = st[k].copy()
    g = World(prm)
    g.set_particles(q)
    g.set_contacts(c.get_contacts())
    compare_contacts(g.get_contacts(), c.get_contacts(), 0.0)
    g.takeTimeStep()
    c.takeTimeStep()
    _compare_worlds(g, c, ONE_STEP_TOL)


def test_history_of_non_candidates_carried_over():
    """An old contact whose pair is not a candidate any more keeps its history
    (the reference's map entry survives, BaseParticle.cpp:95 erases only
    candidates) and its force still enters the force sum.  Contacts of a
    settled packing plus three entries between particles far apart are
    uploaded to the GPU world and to the checker; after five steps both hold
    the same contacts (the three carried over unchanged) and the same state."""
    p, prm = disc_case(n=300, phi=0.82, seed=12)
    c = oracle.PortWorld(prm)
    c.set_particles(p)
    c.run(20)
    st = c.get_state()
    q = dict(p)
    for k in ("x", "y", "vx", "vy", "rot", "rot_vel"):
        q[k] = st[k].copy()
    cont = c.get_contacts()
    existing = set(zip(cont["id_i"].tolist(), cont["id_j"].tolist()))
    box = prm.xmax - prm.xmin
    far = []
    for i in range(len(q["x"])):
        for j in range(i + 1, len(q["x"])):
            dx = abs(q["x"][i] - q["x"][j])
            dy = abs(q["y"][i] - q["y"][j])
            dx, dy = min(dx, box - dx), min(dy, (prm.ymax - prm.ymin) - dy)
            if dx > 0.3 * box and dy > 0.3 * box and (i, j) not in existing:
                far.append((i, j))
                break
        if len(far) == 3:
            break
    assert len(far) == 3
    extra = {k: np.concatenate([v, v[:3]]) for k, v in cont.items()}
    extra["id_i"][-3:] = [f[0] for f in far]
    extra["id_j"][-3:] = [f[1] for f in far]
    g = World(prm)
    g.set_particles(q)
    g.set_contacts(extra)
    c2 = oracle.PortWorld(prm)
    c2.set_particles(q)
    c2.set_contacts(extra)
    g.run(5)
    c2.run(5)
    _compare_worlds(g, c2, TRAJ_TOL)
    gc = g.get_contacts()
    keys = list(zip(gc["id_i"].tolist(), gc["id_j"].tolist()))
    for (i, j), k in zip(far, range(len(extra["id_i"]) - 3, len(extra["id_i"]))):
        at = keys.index((i, j))
        for f in ("shear_x", "shear_y", "fn_x", "fn_y", "ft_x", "ft_y", "damping"):
            assert gc[f][at] == extra[f][k], (i, j, f)


def test_stop_on_pressure():
    p, prm = disc_case(n=300, phi=0.75, seed=13, kind=abi.WORLD_PERIODIC_CONTROL)
    g, c = _pair(p, prm)
    ctl = make_control(update_stress=True, box_law=abi.BOX_STRAIN, p0=-5e-3, p1=-5e-3,
                       reset_rattlers=False, stop_pressure=2.0)
    ng = g.run(2000, ctl)
    nc = c.run(2000, ctl)
    assert ng == nc and ng < 2000
    _compare_worlds(g, c, TRAJ_TOL)


@pytest.mark.parametrize("kind", [abi.WORLD_PERIODIC, abi.WORLD_LEES_EDWARDS])
def test_quadron_z_phi_on_device(kind):
    """QuadronAnalysis's rattler-free Z and solid fraction computed on the
    device equal the checker's (pinned to the compiled reference) after a run."""
    p, prm = disc_case(n=600, phi=0.80, seed=23, kind=kind, shift_strain_rate=0.05)
    g, c = _pair(p, prm)
    ctl = make_control()
    g.run(60, ctl)
    c.run(60, ctl)
    zg, zc = g.quadron_z_phi(), c.quadron_z_phi()
    assert zc[0] > 0
    assert zg[0] == zc[0]
    assert abs(zg[1] - zc[1]) <= 1e-12 * zc[1]
