"""Parity against golden fixtures recorded from the compiled reference
(tests/golden/make_golden.py).  These run wherever the reference sources are
absent (the GPU box): the C restatement on the CPU, the CUDA path on the GPU.

Tolerances: single-pair geometry bit-exact for the restatement and for
circles on the GPU; ellipse geometry on the GPU within 1e-11 relative (CUDA's
cos/sin/atan2/pow differ from glibc's in the last bits).  Worlds after 20-25
steps: identical contact pairs, every field within 1e-9 relative (particle
sums differ in order from the reference's unordered_map order).
"""
import ctypes as C
import glob
import os

import numpy as np
import pytest

import oracle
from xdem_b200 import abi

from helpers import CONTACT_KEYS, STATE_KEYS, compare_pair_geometry, rel_err, same_pairs

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
PAIRS = sorted(glob.glob(os.path.join(HERE, "pairs_*.npz")))
WORLDS = sorted(glob.glob(os.path.join(HERE, "world_*.npz")))


def _load_world(path):
    z = np.load(path)
    p = {k[2:]: z[k] for k in z.files if k.startswith("p_")}
    prm = abi.Params()
    C.memmove(C.byref(prm), z["params"].tobytes(), C.sizeof(abi.Params))
    ctl = abi.Control()
    C.memmove(C.byref(ctl), z["control"].tobytes(), C.sizeof(abi.Control))
    ref = {
        "state": {k[2:]: z[k] for k in z.files if k.startswith("s_")},
        "contacts": {k[2:]: z[k] for k in z.files if k.startswith("c_")},
        "forces": {k[2:]: z[k] for k in z.files if k.startswith("f_")},
        "stress": z["stress"], "boundary": z["boundary"], "le": z["lees_edwards"],
        "z_phi": z["z_phi"], "nsteps": int(z["nsteps"]),
    }
    return p, prm, ctl, ref


def _check_world(w, ref, tol):
    assert same_pairs(w.get_contacts(), ref["contacts"])
    c = w.get_contacts()
    for k in CONTACT_KEYS:
        assert rel_err(c[k], ref["contacts"][k]) <= tol, k
    s = w.get_state()
    for k in STATE_KEYS:
        assert rel_err(s[k], ref["state"][k]) <= tol, k
    f = w.get_force_and_torque()
    for k in ("fx", "fy", "torque"):
        assert rel_err(f[k], ref["forces"][k]) <= tol, k
    assert np.array_equal(f["num_contacts"], ref["forces"]["num_contacts"])
    assert rel_err(w.getStress(), ref["stress"]) <= tol
    assert rel_err(w.getBoundary(), ref["boundary"]) <= tol
    assert rel_err(w.getLeesEdwards(), ref["le"]) <= tol


def test_fixtures_present():
    assert len(PAIRS) == 3 and len(WORLDS) >= 5


@pytest.mark.parametrize("path", PAIRS, ids=lambda p: os.path.basename(p))
def test_pairs_restatement_bit_exact(path):
    z = np.load(path)
    out, _ = oracle.pair_geometry(z["pi"], z["pj"], z["off"], int(z["method"]), "port")
    np.testing.assert_array_equal(out[:, :16], z["out"][:, :16])


@pytest.mark.parametrize("path", WORLDS, ids=lambda p: os.path.basename(p))
def test_worlds_restatement(path):
    p, prm, ctl, ref = _load_world(path)
    w = oracle.PortWorld(prm)
    w.set_particles(p)
    if prm.world_kind == abi.WORLD_PERIODIC_CONTROL:
        w.setVirtualBoundaryMass()
    assert w.run(ref["nsteps"], ctl) == ref["nsteps"]
    _check_world(w, ref, 1e-9)
    np.testing.assert_allclose(w.quadron_z_phi(), ref["z_phi"], rtol=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("path", PAIRS, ids=lambda p: os.path.basename(p))
def test_pairs_gpu(path):
    from xdem_b200.world import pair_geometry
    z = np.load(path)
    out, _ = pair_geometry(z["pi"], z["pj"], z["off"], int(z["method"]))
    ref = z["out"]
    assert np.array_equal(out[:, 0], ref[:, 0])
    if "circle" in path:
        np.testing.assert_array_equal(out[:, :16], ref[:, :16])
    else:
        compare_pair_geometry(out, ref, z["pi"], z["pj"], z["off"], int(z["method"]))


@pytest.mark.gpu
@pytest.mark.parametrize("path", WORLDS, ids=lambda p: os.path.basename(p))
def test_worlds_gpu(path):
    from xdem_b200.world import World
    p, prm, ctl, ref = _load_world(path)
    w = World(prm)
    w.set_particles(p)
    if prm.world_kind == abi.WORLD_PERIODIC_CONTROL:
        w.setVirtualBoundaryMass()
    assert w.run(ref["nsteps"], ctl) == ref["nsteps"]
    _check_world(w, ref, 1e-9)
