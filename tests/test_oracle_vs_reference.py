"""Pins the C restatement (oracle/xdem_oracle.c) to the compiled reference
(oracle/_ref, the unmodified reference sources driven by
oracle/ref_harness.cpp).

Expected agreement: bit for bit on every contact law and per-contact field
from identical state, on box laws, Lees-Edwards updates and stress.  The one
systematic difference is the order in which a particle's own contacts are
summed (ascending partner here, unordered_map order in the reference,
BaseWorld.cpp:26-56), which changes particle sums in the last bit; after one
step states agree to 1e-15 relative and stay within 1e-10 over short runs.
The reference's Newton loop has no iteration cap, so every reference run on
ellipses happens on mild overlaps (deep overlaps can make it loop forever).
"""
import numpy as np
import pytest

import oracle
from xdem_b200 import abi, inputs

from helpers import (setup_control, clump_case, compare_contacts, compare_states, controls, disc_case,
                     ellipse_case, rel_err, same_pairs, segment_case)

pytestmark = [pytest.mark.reference,
              pytest.mark.skipif(not oracle.ref_available(), reason="compiled reference absent")]


def _worlds(p, prm):
    r = oracle.RefWorld(prm)
    r.set_particles(p)
    c = oracle.PortWorld(prm)
    c.set_particles(p)
    if prm.world_kind == abi.WORLD_PERIODIC_CONTROL:
        r.setVirtualBoundaryMass()
        c.setVirtualBoundaryMass()
    return r, c


def _random_pairs(seed, N, shape, a_range, asp_range, near=(0.5, 1.05)):
    rng = np.random.default_rng(seed)
    b1 = rng.uniform(*a_range, N)
    b2 = rng.uniform(*a_range, N)
    k1 = rng.uniform(*asp_range, N)
    k2 = rng.uniform(*asp_range, N)
    a1, a2 = b1 * k1, b2 * k2
    ang = rng.uniform(0, 2 * np.pi, N)
    dist = rng.uniform(*near, N) * (a1 + a2)
    sh = np.full(N, shape, float)
    pi = np.stack([sh, a1, k1, rng.normal(0, 3, N), rng.normal(0, 3, N), rng.normal(0, .1, N),
                   rng.normal(0, .1, N), rng.uniform(0, np.pi, N), rng.normal(0, .1, N)], 1)
    pj = np.stack([sh, a2, k2, pi[:, 3] + dist * np.cos(ang), pi[:, 4] + dist * np.sin(ang),
                   rng.normal(0, .1, N), rng.normal(0, .1, N), rng.uniform(0, np.pi, N),
                   rng.normal(0, .1, N)], 1)
    off = np.zeros((N, 4))
    off[:, 2:] = rng.normal(0, 0.05, (N, 2))
    return pi, pj, off


@pytest.mark.parametrize("method", [abi.ELLIPSE_CLOSEST_APPROACH, abi.ELLIPSE_INTERSECTION])
def test_pair_geometry_ellipses_bit_exact(method):
    pi, pj, off = _random_pairs(100 + method, 3000, 1, (0.4, 0.7), (1.0, 3.0))
    pi[:100, 7] = pj[:100, 7] = 0.0          # aligned
    pj[100:200, 7] = np.pi / 2                # crossed
    og, _ = oracle.pair_geometry(pi, pj, off, method, "port")
    orf, _ = oracle.pair_geometry(pi, pj, off, method, "ref")
    assert og[:, 0].sum() > 800
    np.testing.assert_array_equal(og[:, :16], orf[:, :16])


def test_pair_geometry_circles_bit_exact():
    pi, pj, off = _random_pairs(7, 3000, 0, (0.3, 0.7), (1.0, 1.0), near=(0.8, 1.02))
    # exactly touching (every quantity exactly representable): overlap is 0
    pi[:20, 1], pj[:20, 1] = 0.5, 0.25
    pi[:20, 3:5] = 0.0
    pj[:20, 3], pj[:20, 4] = 0.75, 0.0
    og, _ = oracle.pair_geometry(pi, pj, off, 0, "port")
    orf, _ = oracle.pair_geometry(pi, pj, off, 0, "ref")
    np.testing.assert_array_equal(og[:, :16], orf[:, :16])
    assert og[:20, 0].all()  # overlap 0 is a contact (CircularParticle.cpp:73-77)


def test_eigen_ordering_follows_integer_abs():
    """matrix2d::eigen compares int-truncated magnitudes (MathMatrix2d.h:122);
    pairs whose eigenvalues share an integer part swap roles.  Both must agree
    on such pairs, including contact flags."""
    pi, pj, off = _random_pairs(55, 2000, 1, (0.5, 0.6), (1.0, 1.3))
    og, _ = oracle.pair_geometry(pi, pj, off, 0, "port")
    orf, _ = oracle.pair_geometry(pi, pj, off, 0, "ref")
    np.testing.assert_array_equal(og[:, :16], orf[:, :16])


@pytest.mark.parametrize("kind", [abi.WORLD_PERIODIC, abi.WORLD_PERIODIC_CONTROL,
                                  abi.WORLD_LEES_EDWARDS])
def test_discs_one_step(kind):
    p, prm = disc_case(n=300, phi=0.82, seed=21, kind=kind, shift_strain_rate=0.05)
    r, c = _worlds(p, prm)
    r.takeTimeStep()
    c.takeTimeStep()
    compare_contacts(r.get_contacts(), c.get_contacts(), 0.0)
    compare_states(r.get_state(), c.get_state(), 1e-15)


@pytest.mark.parametrize("method", [abi.ELLIPSE_CLOSEST_APPROACH, abi.ELLIPSE_INTERSECTION])
@pytest.mark.parametrize("kind", [abi.WORLD_PERIODIC, abi.WORLD_PERIODIC_CONTROL,
                                  abi.WORLD_LEES_EDWARDS])
def test_ellipses_one_step(kind, method):
    p, prm = ellipse_case(n=400, seed=22, kind=kind, method=method, compress=1.6)
    r, c = _worlds(p, prm)
    r.takeTimeStep()
    c.takeTimeStep()
    assert r.count_contacts() > 50
    compare_contacts(r.get_contacts(), c.get_contacts(), 0.0)
    compare_states(r.get_state(), c.get_state(), 1e-15)


@pytest.mark.parametrize("name", ["plain", "stress", "strain", "stress_xy", "uniform",
                                  "uniform_limit"])
def test_discs_trajectory_controls(name):
    kind = abi.WORLD_PERIODIC_CONTROL if name != "plain" else abi.WORLD_PERIODIC
    p, prm = disc_case(n=250, phi=0.80, seed=23, kind=kind)
    r, c = _worlds(p, prm)
    setup_control(name, r, c)
    ctl = controls()[name]
    assert r.run(40, ctl) == c.run(40, ctl) == 40
    compare_contacts(r.get_contacts(), c.get_contacts(), 1e-10)
    compare_states(r.get_state(), c.get_state(), 1e-10)
    assert rel_err(r.getBoundary(), c.getBoundary()) <= 1e-12
    assert rel_err(r.getStress(), c.getStress()) <= 1e-10


def test_lees_edwards_trajectory():
    p, prm = ellipse_case(n=300, seed=24, kind=abi.WORLD_LEES_EDWARDS, compress=1.4,
                          shift_rate=0.3)
    r, c = _worlds(p, prm)
    ctl = controls()["stress"]
    r.run(30, ctl)
    c.run(30, ctl)
    compare_contacts(r.get_contacts(), c.get_contacts(), 1e-10)
    compare_states(r.get_state(), c.get_state(), 1e-10)
    np.testing.assert_array_equal(r.getLeesEdwards(), c.getLeesEdwards())


def test_clumps_trajectory():
    p, prm = clump_case(nfree=80, nclump=20, seed=25)
    r, c = _worlds(p, prm)
    ctl = controls()["stress"]
    r.run(25, ctl)
    c.run(25, ctl)
    compare_contacts(r.get_contacts(), c.get_contacts(), 1e-10)
    sr, sc = r.get_state(), c.get_state()
    compare_states(sr, sc, 1e-10)
    assert rel_err(sr["branch_x"], sc["branch_x"]) <= 1e-12
    assert rel_err(r.getStress(), c.getStress()) <= 1e-10


@pytest.mark.parametrize("kind", [abi.WORLD_PERIODIC, abi.WORLD_PERIODIC_CONTROL,
                                  abi.WORLD_LEES_EDWARDS])
def test_segments_one_step(kind):
    """Disc-segment contacts of both orders (CircularParticle.cpp:94-129,
    SegmentObject.cpp:45-80), image pairs included."""
    p, prm = segment_case(kind=kind, seed=31, shift_strain_rate=0.05)
    r, c = _worlds(p, prm)
    r.takeTimeStep()
    c.takeTimeStep()
    cr = r.get_contacts()
    seg = np.flatnonzero(p["shape"] == abi.SHAPE_SEGMENT)
    first = np.isin(cr["id_i"], seg)
    second = np.isin(cr["id_j"], seg)
    assert first.sum() >= 2 and second.sum() >= 10
    compare_contacts(cr, c.get_contacts(), 0.0)
    compare_states(r.get_state(), c.get_state(), 1e-15)


@pytest.mark.parametrize("name", ["stress", "strain"])
def test_segments_trajectory(name):
    kind = abi.WORLD_PERIODIC_CONTROL if name == "strain" else abi.WORLD_PERIODIC
    p, prm = segment_case(kind=kind, seed=32, long_walls=(name == "stress"))
    r, c = _worlds(p, prm)
    ctl = controls()[name]
    assert r.run(40, ctl) == c.run(40, ctl) == 40
    compare_contacts(r.get_contacts(), c.get_contacts(), 1e-10)
    sr, sc = r.get_state(), c.get_state()
    compare_states(sr, sc, 1e-10)
    seg = p["shape"] == abi.SHAPE_SEGMENT
    for key in ("vx", "vy", "rot_vel"):  # walls never move (SKIP_TIME_INTEGRAL)
        np.testing.assert_array_equal(sr[key][seg], p[key][seg])
    assert rel_err(r.getStress(), c.getStress()) <= 1e-10


def test_clump_properties_match_reference():
    """xdem_clump_properties restates GluedParticle::calculateParticleProperties."""
    import ctypes as C
    rng = np.random.default_rng(3)
    lib = abi.load_library()
    d = C.POINTER(C.c_double)
    fns = oracle.ref_lib()
    for k in (2, 3, 5):
        shape = np.zeros(k, np.int32)
        r = rng.uniform(0.3, 0.6, k)
        x = rng.uniform(-0.8, 0.8, k)
        y = rng.uniform(-0.8, 0.8, k)
        asp = np.ones(k)
        rot = np.zeros(k)
        a_out, a_bx, a_by = np.zeros(7), np.zeros(k), np.zeros(k)
        b_out, b_bx, b_by = np.zeros(7), np.zeros(k), np.zeros(k)
        args = (shape.ctypes.data_as(C.POINTER(C.c_int32)), r.ctypes.data_as(d),
                asp.ctypes.data_as(d), x.ctypes.data_as(d), y.ctypes.data_as(d),
                rot.ctypes.data_as(d), 1.0)
        assert lib.xdem_clump_properties(k, *args, a_out.ctypes.data_as(d), a_bx.ctypes.data_as(d),
                                         a_by.ctypes.data_as(d)) == 0
        fns["clump_properties"](k, *args, b_out.ctypes.data_as(d), b_bx.ctypes.data_as(d),
                                b_by.ctypes.data_as(d))
        np.testing.assert_array_equal(a_out, b_out)
        np.testing.assert_array_equal(a_bx, b_bx)
        np.testing.assert_array_equal(a_by, b_by)


def test_particle_properties_match_reference():
    rng = np.random.default_rng(4)
    shape = rng.integers(0, 2, 100).astype(np.int32)
    shape[::7] = abi.SHAPE_SEGMENT
    r = rng.uniform(0.3, 1.5, 100)
    asp = np.where(shape == 1, rng.uniform(1, 3, 100), 1.0)
    a = inputs.particle_properties(shape, r, asp, 1.7)
    b = oracle.ref_particle_properties(shape, r, asp, 1.7)
    for k in a:
        np.testing.assert_array_equal(a[k], b[k])


def test_quadron_coordination_and_solid_fraction():
    """Rattler removal + Z + phi: the restatement's peeling against the
    reference's QuadronAnalysis (QuadronAnalysis.cpp:663-732, 980-986)."""
    p, prm = disc_case(n=400, phi=0.78, seed=26)
    r, c = _worlds(p, prm)
    r.run(30)
    c.run(30)
    assert same_pairs(r.get_contacts(), c.get_contacts())
    zr = r.quadron_z_phi()
    zc = c.quadron_z_phi()
    assert zr[0] > 0
    np.testing.assert_allclose(zc, zr, rtol=1e-15)


def test_virtual_boundary_mass():
    """setVirtualBoundaryMass (PeriodicControlWorld.cpp:58-66)."""
    p, prm = disc_case(n=100, kind=abi.WORLD_PERIODIC_CONTROL)
    r, c = _worlds(p, prm)
    assert r.control_mass() == pytest.approx(p["mass"].sum() / (100 * 10.0), rel=1e-15)
