"""GPU tests of batched worlds (xdem_batch_set_particles): several
independent systems in one handle, every kernel of a step covering all of
them.

A system in a batch performs exactly the operations it performs alone (its
own box, time step, cells and contact-model constants; ids shifted by the
system's first id; force sums in the same id order), so its state and
contacts must equal, bit for bit, those of the same system run as a world of
its own, which the parity tests pin to the checker.  Per-system stresses are
summed in a different tree than a single world's and agree within 1e-12.
"""
import numpy as np
import pytest

from xdem_b200 import abi, inputs
from xdem_b200.world import World, make_control, make_params

from helpers import clump_case, disc_case, ellipse_case

pytestmark = pytest.mark.gpu


def _systems():
    out = []
    p, prm = disc_case(n=300, phi=0.80, seed=2)
    out.append((p, prm))
    p, prm = ellipse_case(n=250, seed=9, kind=abi.WORLD_PERIODIC, compress=1.3)
    out.append((p, prm))
    p, prm = clump_case(nfree=80, nclump=20, seed=5, phi=0.6)
    out.append((p, prm))
    p, prm = disc_case(n=500, phi=0.75, seed=7)
    out.append((p, prm))
    return out


def _box(prm):
    return [prm.xmin, prm.xmax, prm.ymin, prm.ymax]


def _split_contacts(c, first, k):
    lo, hi = first[k], first[k + 1]
    sel = (c["id_i"] >= lo) & (c["id_i"] < hi)
    out = {key: v[sel] for key, v in c.items()}
    out["id_i"] = out["id_i"] - lo
    out["id_j"] = out["id_j"] - lo
    return out


@pytest.mark.parametrize("precision", [abi.PRECISION_FP64, abi.PRECISION_MIXED])
def test_batch_equals_separate_worlds(precision):
    systems = _systems()
    prm0 = systems[0][1]
    bprm = make_params(abi.WORLD_PERIODIC, prm0.dt, _box(prm0), inputs.KN, inputs.KT,
                       inputs.RESTITUTION, inputs.FRICTION, precision=precision)
    batch = World(bprm)
    batch.set_batch([p for p, _ in systems], [_box(prm) for _, prm in systems],
                    [prm.dt for _, prm in systems])
    nsys, first = batch.batch_info()
    assert nsys == len(systems)
    assert first[-1] == sum(len(p["x"]) for p, _ in systems)
    singles = []
    for p, prm in systems:
        prm.precision = precision
        w = World(prm)
        w.set_particles(p)
        singles.append(w)
    ctl = make_control(update_stress=True)
    for chunk in (1, 40, 80):  # direct steps, then captured chunks with re-sorts
        batch.run(chunk, ctl)
        for w in singles:
            w.run(chunk, ctl)
    sb = batch.get_state()
    cb = batch.get_contacts()
    stress = batch.batch_stress()
    counts = batch.batch_count_contacts()
    boxes = batch.batch_boundaries()
    for k, w in enumerate(singles):
        lo, hi = first[k], first[k + 1]
        ss = w.get_state()
        for key in ("x", "y", "vx", "vy", "rot", "rot_vel"):
            np.testing.assert_array_equal(sb[key][lo:hi], ss[key], err_msg=f"system {k} {key}")
        cs = w.get_contacts()
        cbk = _split_contacts(cb, first, k)
        for key in cs:
            np.testing.assert_array_equal(cbk[key], cs[key], err_msg=f"system {k} {key}")
        assert counts[k] == w.count_contacts() == len(cs["id_i"])
        ref = np.asarray(w.getStress())
        assert np.max(np.abs(stress[k] - ref)) <= 1e-12 * np.max(np.abs(ref)), k
        np.testing.assert_array_equal(boxes[k], np.asarray(w.getBoundary()))
    assert counts.sum() > 0


def test_batch_rejects_stop_on_pressure_and_box_setters():
    systems = _systems()[:2]
    prm0 = systems[0][1]
    batch = World(prm0)
    batch.set_batch([p for p, _ in systems], [_box(prm) for _, prm in systems])
    import ctypes as C
    box = (C.c_double * 4)(*_box(prm0))
    assert batch.lib.xdem_set_boundary(batch.h, box) == abi.ERR_ARGUMENT
    ctl = make_control(stop_pressure=1.0)
    done = C.c_int32(0)
    assert batch.lib.xdem_run(batch.h, 5, C.byref(ctl), C.byref(done)) == abi.ERR_ARGUMENT


def test_launch_config_leaves_results_unchanged():
    """Pair-kernel grid and cell size change the speed only: the contact set
    of any cell size >= 2 r_max is the same and force sums run in id order."""
    p, prm = ellipse_case(n=800, seed=12, kind=abi.WORLD_LEES_EDWARDS, compress=1.3)
    a, b = World(prm), World(prm)
    for w in (a, b):
        w.raise_mask = ~abi.ERR_NEWTON
        w.set_particles(p)
    b.set_launch_config(4, 1.5)
    assert b.launch_config() == (4, 1.5)
    for w in (a, b):
        w.run(70, make_control(update_stress=True))
    sa, sb = a.get_state(), b.get_state()
    for key in ("x", "y", "vx", "vy", "rot", "rot_vel"):
        np.testing.assert_array_equal(sa[key], sb[key], err_msg=key)
    ca, cb = a.get_contacts(), b.get_contacts()
    for key in ca:
        np.testing.assert_array_equal(ca[key], cb[key], err_msg=key)
    ra, rb = np.asarray(a.getStress()), np.asarray(b.getStress())
    assert np.max(np.abs(ra - rb)) <= 1e-12 * np.max(np.abs(ra))


def test_autotune_picks_a_timed_configuration():
    systems = _systems()
    prm0 = systems[0][1]
    batch = World(prm0)
    batch.set_batch([p for p, _ in systems], [_box(prm) for _, prm in systems],
                    [prm.dt for _, prm in systems])
    blocks, factor, ms = batch.autotune(make_control(), steps_per_trial=5)
    assert blocks in (4, 8, 16, 32) and factor in (1.0, 1.2, 1.5)
    assert all(t > 0 for t in ms)
    k = [1.0, 1.2, 1.5].index(factor) * 4 + [4, 8, 16, 32].index(blocks)
    assert ms[k] == min(ms)
