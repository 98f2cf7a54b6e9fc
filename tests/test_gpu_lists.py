"""GPU tests of the candidate lists kept across steps (xdem_set_candidate_lists):
a world with the lists and a world with the full 3x3 scan every step produce
the same contacts and state bit for bit — in a Lees-Edwards shear (the shift
travels, particles cross the sheared edge), under a strain-controlled box law
(affine scaling), for clumps, after host state uploads, in a batch, with
lists that overflow, and where nine cells may hold the 200-candidate cap's
count (the last two read the cell-ordered records on steps without a list
rebuild)."""
import numpy as np
import pytest

from xdem_b200 import abi
from xdem_b200.world import World, make_control, make_params

from helpers import clump_case, dense_ellipse_case, disc_case

pytestmark = pytest.mark.gpu


def _pair_of_worlds(p, prm, skin=0.1, contacts=None):
    a, b = World(prm), World(prm)
    a.set_candidate_lists(0)
    b.set_candidate_lists(48, skin)
    for w in (a, b):
        w.raise_mask = ~abi.ERR_NEWTON
        w.set_particles(p)
        if contacts is not None:
            w.set_contacts(contacts)
    return a, b


def _same(a, b):
    sa, sb = a.get_state(), b.get_state()
    for key in ("x", "y", "vx", "vy", "rot", "rot_vel"):
        np.testing.assert_array_equal(sa[key], sb[key], err_msg=key)
    ca, cb = a.get_contacts(), b.get_contacts()
    for key in ca:
        np.testing.assert_array_equal(ca[key], cb[key], err_msg=key)
    return len(ca["id_i"])


@pytest.mark.parametrize("precision", [abi.PRECISION_FP64, abi.PRECISION_MIXED])
def test_lists_match_full_scan_lees_edwards(precision):
    p, contacts, prm = dense_ellipse_case(n=2000, seed=61, kind=abi.WORLD_LEES_EDWARDS,
                                          shift_rate=2.0)
    prm.precision = precision
    a, b = _pair_of_worlds(p, prm, skin=0.05, contacts=contacts)
    for w in (a, b):
        w.run(150, make_control(update_stress=True))
    assert _same(a, b) > 1500
    assert abs(a.getLeesEdwards()[0]) > 0
    assert b.candidate_list_stats()["builds"] > 2


def test_lists_match_full_scan_strain_control_and_uploads():
    p, prm = disc_case(n=1200, phi=0.78, seed=9, kind=abi.WORLD_PERIODIC_CONTROL)
    a, b = _pair_of_worlds(p, prm)
    ctl = make_control(update_stress=True, box_law=abi.BOX_STRAIN, p0=-2e-3, p1=-2e-3)
    for w in (a, b):
        w.run(60, ctl)
    # a host upload of the state the world already has, then more steps
    s = a.get_state()
    for w in (a, b):
        w.upload_state(s["x"], s["y"], s["vx"], s["vy"], s["rot"], s["rot_vel"])
        w.run(40, ctl)
    assert _same(a, b) > 500


def test_lists_match_full_scan_clumps():
    """Also: a sub-disc outside the periodic box (its clump's centre inside)
    is wrapped on its own at each step's start and placed at the clump's
    centre plus its branch again by the time integral; that jump of one box
    length is no move, so the lists are not rebuilt every step."""
    p, prm = clump_case(nfree=150, nclump=40, seed=17, phi=0.62)
    a, b = _pair_of_worlds(p, prm)
    for w in (a, b):
        w.run(120, make_control())
    assert _same(a, b) > 50
    s = b.get_state()
    xmin, xmax, ymin, ymax = b.getBoundary()
    sub = np.nonzero(p["up_level"] != np.arange(len(p["up_level"])))[0]
    outside = (s["x"][sub] < xmin) | (s["x"][sub] > xmax) | (s["y"][sub] < ymin) | (s["y"][sub] > ymax)
    assert np.any(outside), "no sub-disc outside the box: the case needs one"
    builds = b.candidate_list_stats()["builds"]
    assert builds < 30, f"{builds} list builds in 120 steps"


@pytest.mark.parametrize("kind", ["compression", "shear"])
def test_lists_match_full_scan_clumps_moving_box(kind):
    """Clumps under a strain-controlled compression (the box law scales every
    position, and the time integral puts each sub-disc back at its clump's
    centre plus its branch) and in a Lees-Edwards shear (sub-discs cross the
    sheared edge on their own)."""
    p, prm = clump_case(nfree=150, nclump=40, seed=23, phi=0.6)
    if kind == "compression":
        prm.world_kind = abi.WORLD_PERIODIC_CONTROL
        ctl = make_control(update_stress=True, box_law=abi.BOX_STRAIN, p0=-2e-3, p1=-2e-3)
    else:
        prm.world_kind = abi.WORLD_LEES_EDWARDS
        prm.shift_strain_rate = 2.0
        ctl = make_control(update_stress=True)
    a, b = _pair_of_worlds(p, prm)
    for w in (a, b):
        w.run(100, ctl)
    assert _same(a, b) > 20


def test_lists_match_full_scan_list_overflow():
    """Lists of three entries overflow for most particles, which then take
    the full 3x3 scan every step from the cell records (written every step
    while a list of the last build overflowed); plain steps."""
    p, prm = disc_case(n=1500, phi=0.80, seed=21)
    a, b = World(prm), World(prm)
    a.set_candidate_lists(0)
    b.set_candidate_lists(3, 0.1)
    for w in (a, b):
        w.set_particles(p)
        w.run(80, make_control())
    assert _same(a, b) > 1000
    assert b.candidate_list_stats()["builds"] >= 1


def test_lists_match_full_scan_candidate_cap_reachable():
    """Small discs (r 0.25) with a few large ones (r 1.2, which set the cell
    size to 2.01 x 1.2) at solid fraction 0.65 put up to 23 records in a
    cell, so nine cells may hold the 200-candidate cap's count and the bound
    is counted from the cell records every step (below the cap itself: no
    capacity error)."""
    from xdem_b200 import inputs
    rng = np.random.default_rng(5)
    n = 3000
    r = np.where(rng.permutation(n) < 40, 1.2, 0.25)
    box = inputs.box_for(float(np.sum(np.pi * r * r)), 0.5)
    x, y = inputs.rsa_positions(r, box, 6)
    p = inputs.assemble(np.zeros(n, np.int32), r, np.ones(n), x, y, rng.normal(0, 0.05, n),
                        rng.normal(0, 0.05, n), np.zeros(n), np.zeros(n))
    box = inputs.scale_to_fraction(p, box, float(np.sum(p["volume"])), 0.65)
    side = 2.01 * 1.2
    nx, ny = int((box[1] - box[0]) // side), int((box[3] - box[2]) // side)
    counts, _, _ = np.histogram2d(p["x"], p["y"], bins=(nx, ny),
                                  range=((box[0], box[1]), (box[2], box[3])))
    assert 9 * counts.max() + 1 >= 200
    prm = make_params(abi.WORLD_PERIODIC, inputs.time_step(p), box, inputs.KN, inputs.KT,
                      inputs.RESTITUTION, inputs.FRICTION)
    a, b = _pair_of_worlds(p, prm)
    for w in (a, b):
        w.run(60, make_control())
    assert _same(a, b) > 100
