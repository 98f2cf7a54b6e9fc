"""GPU tests of fixed wall segments (SegmentObject): disc-segment contacts of
both orders (CircularParticle.cpp:94-129 with the disc as P1,
SegmentObject.cpp:45-80 with the segment as P1), checked against the FP64
checker, which the compiled reference pins bit for bit
(tests/test_oracle_vs_reference.py) and the golden fixtures
world_discs_segments_*.npz pin on the GPU box.

Tolerances: one step from an identical state 1e-10 relative per field (the
disc-segment construction is sqrt/divide only, correctly rounded on both
sides, so it agrees to the last bit; particle sums differ in order), 50-step
trajectories 1e-9, the mixed path within its stated force tolerance (1e-5 of
the largest contact force), the candidate lists and snapshots bit for bit.
"""
import numpy as np
import pytest

import oracle
from xdem_b200 import abi, inputs
from xdem_b200.world import World, make_control

from helpers import (compare_contacts, compare_states, controls, disc_case, rel_err, same_pairs,
                     segment_case)

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


def _wall_contacts(p, c):
    seg = np.flatnonzero(p["shape"] == abi.SHAPE_SEGMENT)
    return int(np.isin(c["id_i"], seg).sum()), int(np.isin(c["id_j"], seg).sum())


@pytest.mark.parametrize("kind", [abi.WORLD_PERIODIC, abi.WORLD_PERIODIC_CONTROL,
                                  abi.WORLD_LEES_EDWARDS])
def test_segments_one_step(kind):
    p, prm = segment_case(kind=kind, seed=31, shift_strain_rate=0.05)
    g, c = _pair(p, prm)
    g.takeTimeStep()
    c.takeTimeStep()
    cg, cc = g.get_contacts(), c.get_contacts()
    first, second = _wall_contacts(p, cc)
    assert first >= 2 and second >= 10
    compare_contacts(cg, cc, ONE_STEP_TOL)
    compare_states(g.get_state(), c.get_state(), ONE_STEP_TOL)
    fg, fc = g.get_force_and_torque(), c.get_force_and_torque()
    for k in ("fx", "fy", "torque"):
        assert rel_err(fg[k], fc[k]) <= ONE_STEP_TOL, k


@pytest.mark.parametrize("name", ["stress", "strain", "stress_xy"])
def test_segments_trajectory(name):
    kind = abi.WORLD_PERIODIC if name == "stress" else abi.WORLD_PERIODIC_CONTROL
    p, prm = segment_case(kind=kind, seed=32, long_walls=(name == "stress"))
    g, c = _pair(p, prm)
    ctl = controls()[name]
    assert g.run(50, ctl) == c.run(50, ctl) == 50
    compare_contacts(g.get_contacts(), c.get_contacts(), TRAJ_TOL)
    sg = g.get_state()
    compare_states(sg, c.get_state(), TRAJ_TOL)
    assert rel_err(g.getStress(), c.getStress()) <= TRAJ_TOL
    assert rel_err(g.getBoundary(), c.getBoundary()) <= TRAJ_TOL
    seg = p["shape"] == abi.SHAPE_SEGMENT
    for key in ("vx", "vy", "rot_vel", "rot"):  # SKIP_TIME_INTEGRAL
        np.testing.assert_array_equal(sg[key][seg], p[key][seg])
    assert sum(_wall_contacts(p, g.get_contacts())) >= 10


def test_segment_vertices_round_trip():
    p, prm = segment_case(seed=33)
    g = World(prm)
    g.set_particles(p)
    out = {k: np.zeros(len(p["x"])) for k in abi.SEGMENT_FIELDS}
    s = abi.Particles()
    s.n = len(p["x"])
    for k, v in out.items():
        setattr(s, k, v.ctypes.data_as(abi.C.POINTER(abi.C.c_double)))
    assert g.lib.xdem_get_particles(g.h, abi.C.byref(s)) == 0
    for k in abi.SEGMENT_FIELDS:
        np.testing.assert_array_equal(out[k], p[k])


def test_segments_mixed_precision():
    p, prm = segment_case(kind=abi.WORLD_LEES_EDWARDS, seed=34, shift_strain_rate=0.05)
    c = oracle.PortWorld(prm)
    c.set_particles(p)
    prm.precision = abi.PRECISION_MIXED
    g = World(prm)
    g.set_particles(p)
    g.takeTimeStep()
    c.takeTimeStep()
    cg, cc = g.get_contacts(), c.get_contacts()
    assert same_pairs(cg, cc)
    assert sum(_wall_contacts(p, cc)) >= 10
    scale = np.max(np.hypot(cc["fn_x"] + cc["ft_x"], cc["fn_y"] + cc["ft_y"]))
    dfx = (cg["fn_x"] + cg["ft_x"]) - (cc["fn_x"] + cc["ft_x"])
    dfy = (cg["fn_y"] + cg["ft_y"]) - (cc["fn_y"] + cc["ft_y"])
    assert np.max(np.hypot(dfx, dfy)) <= 1e-5 * scale


def test_segments_candidate_lists_and_full_scan_agree():
    p, prm = segment_case(kind=abi.WORLD_LEES_EDWARDS, seed=35, shift_strain_rate=0.2)
    a, b = World(prm), World(prm)
    b.set_candidate_lists(0)
    for w in (a, b):
        w.set_particles(p)
        w.run(80, make_control(update_stress=True))
    sa, sb = a.get_state(), b.get_state()
    for key in ("x", "y", "vx", "vy", "rot", "rot_vel"):
        np.testing.assert_array_equal(sa[key], sb[key], err_msg=key)
    ca, cb = a.get_contacts(), b.get_contacts()
    for key in ca:
        np.testing.assert_array_equal(ca[key], cb[key], err_msg=key)
    assert a.candidate_list_stats()["builds"] >= 1


def test_segments_snapshot_resume(tmp_path):
    p, prm = segment_case(seed=36)
    a = World(prm)
    a.set_particles(p)
    ctl = make_control(update_stress=True)
    a.run(40, ctl)
    a.save_snapshot(tmp_path / "walls.xdem")
    b = World(prm)
    b.load_snapshot(tmp_path / "walls.xdem")
    for w in (a, b):
        w.run(45, ctl)
    sa, sb = a.get_state(), b.get_state()
    for key in ("x", "y", "vx", "vy", "rot", "rot_vel"):
        np.testing.assert_array_equal(sa[key], sb[key], err_msg=key)
    ca, cb = a.get_contacts(), b.get_contacts()
    assert sum(_wall_contacts(p, ca)) > 0
    for key in ca:
        np.testing.assert_array_equal(ca[key], cb[key], err_msg=key)
    np.testing.assert_array_equal(np.asarray(a.getStress()), np.asarray(b.getStress()))


def test_segment_meeting_an_ellipse_is_unsupported():
    """The reference exits (SegmentObject.cpp:24-26, EllipticParticle.cpp:30);
    the GPU path and the checker raise UNSUPPORTED_PAIR."""
    e = inputs.assemble(np.array([abi.SHAPE_ELLIPSE], np.int32), np.array([0.8]), np.array([2.0]),
                        np.array([0.0]), np.array([0.3]), np.zeros(1), np.zeros(1), np.zeros(1),
                        np.zeros(1))
    d, box = inputs.disc_system(40, phi=0.3, seed=2)
    far = np.hypot(d["x"], d["y"]) > 4.0  # no disc near the pair
    d = {k: np.ascontiguousarray(v[far]) for k, v in d.items()}
    d["up_level"] = np.arange(int(far.sum()), dtype=np.int32)
    s = inputs.segments([-0.5], [0.0], [0.5], [0.0])
    p = inputs.concatenate(s, e, d)
    from xdem_b200.world import make_params
    prm = make_params(abi.WORLD_PERIODIC, 1e-3, box, inputs.KN, inputs.KT, inputs.RESTITUTION,
                      inputs.FRICTION)
    for w in (World(prm), oracle.PortWorld(prm)):
        w.raise_mask = 0
        w.set_particles(p)
        w.takeTimeStep()
        assert w.last_status & abi.ERR_UNSUPPORTED_PAIR
