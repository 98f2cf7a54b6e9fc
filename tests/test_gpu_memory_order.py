"""Results do not depend on the device memory order of the particles.

The arrays are re-sorted by cell every few steps (xdem_set_memory_order_refresh)
so that neighbours sit at nearby addresses; contact ownership, force-sum order
and history matching go by id and every cell test by position, so the
interval must not change any result.  The regime where a dependence would
show is a hard compression of an RSA packing: deep overlaps, closest-approach
Newton iterations that never terminate in the reference (stopped and
bisected here), candidate lists rebuilt often.  Three worlds that differ only
in the refresh interval (31, 63, never) run the same strain-controlled
compression of 65,536 ellipses (a/b ~ U[1,3], b in {0.5, 0.7}, from an RSA of
bounding discs at 0.40 towards 0.85) and must end bit for bit equal, with the
same Newton counters.  The run must stay finite: a NaN position (the
reference's closest-approach arithmetic can produce one) bins into a clamped
cell, which is where an order dependence could enter, and raises
XDEM_ERR_NONFINITE.
"""
import math

import numpy as np
import pytest

from xdem_b200 import abi, inputs
from xdem_b200.world import World, make_control, make_params

pytestmark = pytest.mark.gpu


def test_refresh_interval_does_not_change_a_hard_compression():
    n = 65536
    p, box = inputs.ellipse_system(n, b=inputs.c2_b, aspect=inputs.c4_aspect, phi_rsa_circle=0.40,
                                   phi=None, seed=3)
    dt = inputs.time_step(p)
    prm = make_params(abi.WORLD_PERIODIC_CONTROL, dt, box, inputs.KN, inputs.KT,
                      inputs.RESTITUTION, inputs.FRICTION, global_damping=0.1)
    worlds = []
    for interval in (31, 63, 0):
        w = World(prm)
        w.raise_mask = ~abi.ERR_NEWTON
        w.set_memory_order_refresh(interval)
        w.set_particles(p)
        worlds.append(w)
    vol = float(p["volume"].sum())
    steps = 1500
    s_step = math.sqrt(vol / ((box[1] - box[0]) * (box[3] - box[2])) / 0.85) ** (1.0 / steps)
    ctl = make_control(box_law=abi.BOX_STRAIN, reset_rattlers=False)
    done = 0
    while done < steps:
        b = worlds[0].getBoundary()
        ctl.p0 = ctl.p1 = (s_step - 1.0) / ((b[1] - b[0]) * dt)
        for w in worlds:
            assert w.run(100, ctl) == 100
        done += 100
    for w in worlds:
        w.run(300, make_control())
    solves, iters, stuck = worlds[0].newton_stats()
    assert stuck > 0, "the run should reach non-terminating Newton iterations"
    ref = worlds[0].get_state()
    c0 = worlds[0].get_contacts()
    assert len(c0["id_i"]) > n
    for w in worlds[1:]:
        st = w.get_state()
        for k in ("x", "y", "vx", "vy", "rot", "rot_vel"):
            np.testing.assert_array_equal(st[k], ref[k], err_msg=k)
        c = w.get_contacts()
        for k in c0:
            np.testing.assert_array_equal(c[k], c0[k], err_msg=k)
        assert w.newton_stats() == (solves, iters, stuck)
    np.testing.assert_array_equal(worlds[1].getBoundary(), worlds[0].getBoundary())
