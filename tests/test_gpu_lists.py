"""GPU tests of the candidate lists kept across steps (xdem_set_candidate_lists):
a world with the lists and a world with the full 3x3 scan every step produce
the same contacts and state bit for bit — in a Lees-Edwards shear (the shift
travels, particles cross the sheared edge), under a strain-controlled box law
(affine scaling), for clumps, after host state uploads, and in a batch."""
import numpy as np
import pytest

from xdem_b200 import abi
from xdem_b200.world import World, make_control

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
    p, prm = clump_case(nfree=150, nclump=40, seed=17, phi=0.62)
    a, b = _pair_of_worlds(p, prm)
    for w in (a, b):
        w.run(120, make_control())
    assert _same(a, b) > 50
