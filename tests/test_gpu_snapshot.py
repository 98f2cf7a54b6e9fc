"""GPU tests of binary snapshots (xdem_save_snapshot / xdem_load_snapshot),
the checkpoint/resume replacing the reference's text dumps
(BaseParticle.cpp:158-186, ContactInformation.h:51-60, read4File_particle).

A world loaded from a snapshot holds the saved particles, contact history
and world scalars; since a step's results do not depend on the memory order
of the particles or on when the candidate lists were last built, the loaded
world and the saved one must then take the same steps bit for bit.
"""
import ctypes as C

import numpy as np
import pytest

from xdem_b200 import abi
from xdem_b200.world import World, make_control, make_params

from helpers import clump_case, dense_ellipse_case, disc_case, ellipse_case

pytestmark = pytest.mark.gpu

STATE = ("x", "y", "vx", "vy", "rot", "rot_vel")


def _same_world(a, b):
    sa, sb = a.get_state(), b.get_state()
    for key in STATE:
        np.testing.assert_array_equal(sa[key], sb[key], err_msg=key)
    ca, cb = a.get_contacts(), b.get_contacts()
    assert len(ca["id_i"]) > 0
    for key in ca:
        np.testing.assert_array_equal(ca[key], cb[key], err_msg=key)
    np.testing.assert_array_equal(np.asarray(a.getStress()), np.asarray(b.getStress()))
    np.testing.assert_array_equal(np.asarray(a.getBoundary()), np.asarray(b.getBoundary()))


def _resume(prm, setup, ctl, tmp_path, before=45, after=70):
    a = World(prm)
    a.raise_mask = ~abi.ERR_NEWTON
    setup(a)
    a.run(before, ctl)
    path = tmp_path / "world.xdem"
    a.save_snapshot(path)
    b = World(prm)
    b.raise_mask = ~abi.ERR_NEWTON
    b.load_snapshot(path)
    assert b.n == a.n
    _same_world(a, b)
    for w in (a, b):
        w.run(after, ctl)
    _same_world(a, b)
    return a, b


@pytest.mark.parametrize("precision", [abi.PRECISION_FP64, abi.PRECISION_MIXED])
def test_sheared_ellipses_resume_exactly(precision, tmp_path):
    q, contacts, prm = dense_ellipse_case(n=1200, seed=4, steps=800, relax=200)
    prm.precision = precision

    def setup(w):
        w.set_particles(q)
        w.set_contacts(contacts)

    _resume(prm, setup, make_control(update_stress=True), tmp_path)


def test_discs_under_stress_control_resume_exactly(tmp_path):
    p, prm = disc_case(n=900, phi=0.80, seed=8, kind=abi.WORLD_PERIODIC_CONTROL)
    ctl = make_control(update_stress=True, box_law=abi.BOX_STRESS_XY, p0=5.0,
                       scale_rattlers=0.99, sequence=abi.SEQ_SUBSTEPS)

    def setup(w):
        w.set_particles(p)
        w.setVirtualBoundaryMass()

    _resume(prm, setup, ctl, tmp_path)


def test_clumps_under_strain_control_resume_exactly(tmp_path):
    p, prm = clump_case(nfree=100, nclump=30, seed=3, phi=0.6)
    ctl = make_control(update_stress=True, box_law=abi.BOX_STRAIN, p0=-2e-3, p1=-2e-3)
    _resume(prm, lambda w: w.set_particles(p), ctl, tmp_path)


def test_batch_resumes_exactly(tmp_path):
    systems = [disc_case(n=300, phi=0.80, seed=2),
               ellipse_case(n=250, seed=9, kind=abi.WORLD_PERIODIC, compress=1.3),
               disc_case(n=400, phi=0.78, seed=6)]
    prm0 = systems[0][1]
    boxes = [[prm.xmin, prm.xmax, prm.ymin, prm.ymax] for _, prm in systems]
    dts = [prm.dt for _, prm in systems]
    a, b = _resume(prm0, lambda w: w.set_batch([p for p, _ in systems], boxes, dts),
                   make_control(update_stress=True), tmp_path)
    na, fa = a.batch_info()
    nb, fb = b.batch_info()
    assert na == nb == 3
    np.testing.assert_array_equal(fa, fb)
    np.testing.assert_array_equal(a.batch_stress(), b.batch_stress())
    np.testing.assert_array_equal(a.batch_count_contacts(), b.batch_count_contacts())


def test_load_refuses_other_kinds_and_damaged_files(tmp_path):
    p, prm = disc_case(n=200, phi=0.8, seed=1)
    a = World(prm)
    a.set_particles(p)
    a.run(5)
    path = tmp_path / "w.xdem"
    a.save_snapshot(path)
    lib = a.lib
    other = make_params(abi.WORLD_LEES_EDWARDS, prm.dt, [prm.xmin, prm.xmax, prm.ymin, prm.ymax],
                        prm.normal_stiffness, prm.shear_stiffness, prm.restitution_coeff,
                        prm.frictional_coeff)
    b = World(other)
    assert lib.xdem_load_snapshot(b.h, str(path).encode()) == abi.ERR_ARGUMENT
    data = path.read_bytes()
    cut = tmp_path / "cut.xdem"
    cut.write_bytes(data[: len(data) // 2])
    c = World(prm)
    assert lib.xdem_load_snapshot(c.h, str(cut).encode()) == abi.ERR_ARGUMENT
    bad = tmp_path / "bad.xdem"
    bad.write_bytes(b"NOTASNAP" + data[8:])
    assert lib.xdem_load_snapshot(c.h, str(bad).encode()) == abi.ERR_ARGUMENT
    assert lib.xdem_load_snapshot(c.h, str(tmp_path / "missing").encode()) == abi.ERR_ARGUMENT
    empty = World(prm)
    assert lib.xdem_save_snapshot(empty.h, str(tmp_path / "e.xdem").encode()) == abi.ERR_ARGUMENT
    # a refused load leaves the world usable
    c.load_snapshot(path)
    c.run(3)
    assert C.c_int32(c.n).value == len(p["x"])
