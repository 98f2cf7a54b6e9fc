"""The C-ABI boundary, checked without a GPU: the library loads, exports every
function include/xdem_gpu.h declares, its structs have the layout the ctypes
mirror assumes, the host-only helpers work, and there is no CPU fallback."""
import ctypes as C
import os
import subprocess
import tempfile

import numpy as np
import pytest

from xdem_b200 import abi, inputs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_declared_symbol():
    lib = abi.load_library()
    names = abi.exported_symbols()
    assert len(names) >= 50
    missing = [s for s in names if not hasattr(lib, s)]
    assert not missing, missing
    assert lib.xdem_abi_version() == 1


def test_struct_layout_matches_header():
    """Compile a probe against include/xdem_gpu.h and compare sizes/offsets."""
    structs = {"xdem_params": abi.Params, "xdem_control": abi.Control,
               "xdem_particles": abi.Particles, "xdem_contacts": abi.Contacts}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "xdem_gpu.h"', "int main(void){"]
    for cname, py in structs.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'printf("{cname}.{f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("return 0;}")
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "probe.c")
        exe = os.path.join(d, "probe")
        open(src, "w").write("\n".join(lines))
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), src, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout
    got = dict(line.rsplit(" ", 1) for line in out.strip().splitlines())
    for cname, py in structs.items():
        assert int(got[f"{cname} size"]) == C.sizeof(py), cname
        for f, _ in py._fields_:
            assert int(got[f"{cname}.{f}"]) == getattr(py, f).offset, (cname, f)


def test_status_strings():
    lib = abi.load_library()
    for bit in abi.STATUS_NAMES:
        assert lib.xdem_status_string(bit) != b"unknown status"


def test_no_cpu_fallback_without_device():
    """Without a CUDA device the product path fails loudly (no silent CPU path)."""
    lib = abi.load_library()
    n = C.c_int32(0)
    if lib.xdem_device_count(C.byref(n)) == 0:
        pytest.skip("a CUDA device is present")
    from xdem_b200.world import World, make_params
    with pytest.raises(abi.XdemError) as e:
        World(make_params(abi.WORLD_PERIODIC, 1e-4, (-5, 5, -5, 5), 1e4, 5e3, 0.5, 0.5))
    assert e.value.status & abi.ERR_CUDA


def test_create_rejects_bad_arguments():
    lib = abi.load_library()
    from xdem_b200.world import make_params
    h = C.c_void_p()
    bad = make_params(7, 1e-4, (-5, 5, -5, 5), 1e4, 5e3, 0.5, 0.5)
    assert lib.xdem_create(C.byref(bad), C.byref(h)) == abi.ERR_ARGUMENT
    bad = make_params(0, -1.0, (-5, 5, -5, 5), 1e4, 5e3, 0.5, 0.5)
    assert lib.xdem_create(C.byref(bad), C.byref(h)) == abi.ERR_ARGUMENT
    bad = make_params(0, 1e-4, (-5, 5, -5, 5), 1e4, 5e3, 0.5, 0.5, max_contacts=64)
    assert lib.xdem_create(C.byref(bad), C.byref(h)) == abi.ERR_ARGUMENT


def test_rsa_no_overlap_and_deterministic():
    r = np.where(np.arange(2000) % 2 == 0, 0.5, 0.7)
    box = inputs.box_for(float(np.sum(np.pi * r * r)), 0.45)
    x1, y1 = inputs.rsa_positions(r, box, 17)
    x2, y2 = inputs.rsa_positions(r, box, 17)
    assert np.array_equal(x1, x2) and np.array_equal(y1, y2)
    L = box[1] - box[0]
    dx = x1[:, None] - x1[None, :]
    dy = y1[:, None] - y1[None, :]
    dx -= L * np.round(dx / L)
    dy -= L * np.round(dy / L)
    d = np.hypot(dx, dy) + np.eye(len(r)) * 1e9
    assert np.all(d >= (r[:, None] + r[None, :]) * (1 - 1e-12))
    assert np.all((x1 >= box[0]) & (x1 < box[1]) & (y1 >= box[2]) & (y1 < box[3]))


def test_particle_properties_formulas():
    """CircularParticle.cpp:16-23 and EllipticParticle.cpp:7-14."""
    shape = np.array([0, 1], np.int32)
    out = inputs.particle_properties(shape, np.array([0.5, 1.2]), np.array([1.0, 2.0]), 2.0)
    assert out["volume"][0] == np.pi * 0.5 * 0.5
    assert out["mass"][0] == out["volume"][0] * 2.0
    assert out["inertia"][0] == out["mass"][0] * 0.5 * 0.5 / 2.0
    assert out["volume"][1] == np.pi * 1.2 * 1.2 / 2.0
    assert out["inertia"][1] == out["mass"][1] * (1.2 * 1.2 + 1.2 * 1.2 / 2.0 / 2.0) / 4.0
    assert out["inv_mass"][1] == 1.0 / out["mass"][1]
