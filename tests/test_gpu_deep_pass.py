"""The FP64 closest-approach path evaluates the pairs that the centre-line
class marks deep (centre distance below 0.7 of the two half-widths along the
line of centres) in a pass of their own, launched ahead of the regular pair
pass, which starts beside it as a programmatic dependent launch.  The long
Newton iterations of deep overlaps then start with the step's other pairs
instead of ending the pair phase.  Nothing is dropped in FP64 (the class only
orders the evaluation), and every pair is evaluated by the same operations
whichever pass takes it.

With per-kernel profiling on, the regular pass is an ordinary launch after
the deep pass; both orders must give the same state, contacts, stress and
Newton counters bit for bit, through direct steps and through the CUDA-graph
chunks of a run."""
import numpy as np
import pytest

from xdem_b200 import abi
from xdem_b200.world import World, make_control

from helpers import dense_ellipse_case

pytestmark = pytest.mark.gpu


def test_fp64_deep_pass_beside_the_regular_pass_is_bit_identical():
    p, contacts, prm = dense_ellipse_case(n=4000, seed=35, kind=abi.WORLD_LEES_EDWARDS,
                                          shift_rate=0.1)
    assert prm.precision == abi.PRECISION_FP64
    worlds = [World(prm), World(prm)]
    worlds[1].set_profiling(True)
    for w in worlds:
        w.raise_mask = ~abi.ERR_NEWTON
        w.set_particles(p)
        w.set_contacts(contacts)
        w.reset_newton_stats()
    ctl = make_control(update_stress=True)
    for w in worlds:
        for _ in range(3):
            w.takeTimeStep()
        w.run(70, ctl)
    prof = worlds[1].profile()
    assert prof["k_pair_deep"][0] == 73
    s0, s1 = worlds[0].get_state(), worlds[1].get_state()
    for k in s0:
        np.testing.assert_array_equal(s0[k], s1[k], err_msg=k)
    c0, c1 = worlds[0].get_contacts(), worlds[1].get_contacts()
    for k in c0:
        np.testing.assert_array_equal(c0[k], c1[k], err_msg=k)
    assert len(c0["id_i"]) > 4000
    np.testing.assert_array_equal(worlds[0].getStress(), worlds[1].getStress())
    assert worlds[0].newton_stats() == worlds[1].newton_stats()


def test_fp64_deep_pass_equals_full_scan_order():
    """The same world with candidate lists off (the full 3x3 scan lists the
    pairs, deep ones included, in another order) gives the same state bit
    for bit: the deep/regular split depends on nothing but the pair."""
    p, contacts, prm = dense_ellipse_case(n=3000, seed=36, kind=abi.WORLD_PERIODIC)
    worlds = [World(prm), World(prm)]
    worlds[1].set_candidate_lists(0)
    for w in worlds:
        w.raise_mask = ~abi.ERR_NEWTON
        w.set_particles(p)
        w.set_contacts(contacts)
        w.run(40, make_control(update_stress=True))
    s0, s1 = worlds[0].get_state(), worlds[1].get_state()
    for k in s0:
        np.testing.assert_array_equal(s0[k], s1[k], err_msg=k)
    np.testing.assert_array_equal(worlds[0].getStress(), worlds[1].getStress())
