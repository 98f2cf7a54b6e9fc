"""The allocation-free stress entry point (xdem_total_stress_noalloc).

It exists for callers that cannot allocate device memory: code inside a CUDA
graph being captured, host programs that own a fixed device budget and every
buffer in it, real-time loops that must not take the allocator's locks.  The
caller passes device arrays of per-contact forces and branch vectors and a
device output; the library keeps its partial sums in a fixed array of its own.

The test checks it, through the C-ABI, against the existing entry point
(xdem_update_total_stress on a world) within the FP64 tolerance the other
parity tests use, on two calls in a row (the second call finds the first
call's partial sums in the shared array).  Inputs and outputs live in device
memory that the test allocates with torch.  This file is collected last so
that a stop at the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from xdem_b200 import abi
from xdem_b200.world import World, make_control

from helpers import disc_case, rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _world_stress_and_contacts(n, seed):
    p, prm = disc_case(n=n, phi=0.82, seed=seed)
    w = World(prm)
    w.set_particles(p)
    w.run(25, make_control())
    ref = w.updateTotalStress()  # the existing entry point
    c = w.get_contacts()
    box = w.getBoundary()
    area = (box[1] - box[0]) * (box[3] - box[2])
    w.close()
    return ref, c, area


def _noalloc(lib, torch, fx, fy, bx, by, area):
    dev = [torch.tensor(a, dtype=torch.float64, device="cuda") for a in (fx, fy, bx, by)]
    out = torch.full((4,), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    st = lib.xdem_total_stress_noalloc(len(fx), *[C.c_void_p(t.data_ptr()) for t in dev], area,
                                       C.c_void_p(out.data_ptr()), None)
    torch.cuda.synchronize()
    return st, out.cpu().numpy()


def test_noalloc_stress_matches_world_stress_twice():
    torch = pytest.importorskip("torch")
    lib = abi.load_library()
    ref, c, area = _world_stress_and_contacts(3000, 41)
    fx = c["fn_x"] + c["ft_x"]  # ContactInformation.h:63
    fy = c["fn_y"] + c["ft_y"]
    assert len(fx) > 1000
    st1, s1 = _noalloc(lib, torch, fx, fy, c["branch_x"], c["branch_y"], area)
    assert st1 == abi.OK
    assert rel_err(s1, ref) <= TOL, (s1, ref)
    # a second call over a different, smaller contact set, then the first set
    # again: stale partial sums from the earlier calls must not leak in
    ref2, c2, area2 = _world_stress_and_contacts(700, 42)
    st2, s2 = _noalloc(lib, torch, c2["fn_x"] + c2["ft_x"], c2["fn_y"] + c2["ft_y"],
                       c2["branch_x"], c2["branch_y"], area2)
    assert st2 == abi.OK
    assert rel_err(s2, ref2) <= TOL, (s2, ref2)
    st3, s3 = _noalloc(lib, torch, fx, fy, c["branch_x"], c["branch_y"], area)
    assert st3 == abi.OK
    np.testing.assert_array_equal(s3, s1)


def test_noalloc_limits():
    torch = pytest.importorskip("torch")
    lib = abi.load_library()
    cap = lib.xdem_total_stress_noalloc_max_contacts()
    assert cap == 4 * 1024 * 1024
    out = torch.zeros(4, dtype=torch.float64, device="cuda")
    dummy = torch.zeros(1, dtype=torch.float64, device="cuda")
    ptr = C.c_void_p(dummy.data_ptr())
    # beyond the stated maximum: rejected before any work is queued
    assert lib.xdem_total_stress_noalloc(cap + 1, ptr, ptr, ptr, ptr, 1.0,
                                         C.c_void_p(out.data_ptr()), None) == abi.ERR_CAPACITY
    # no contacts: zero stress
    out.fill_(7.0)
    torch.cuda.synchronize()
    assert lib.xdem_total_stress_noalloc(0, None, None, None, None, 2.0,
                                         C.c_void_p(out.data_ptr()), None) == abi.OK
    torch.cuda.synchronize()
    assert np.all(out.cpu().numpy() == 0.0)


def _stress_sum_bound(fx, fy, bx, by, area):
    """numpy's sum and the sum of |terms| that bounds any summation order's
    rounding (relative 1e-12 of it is far above 4M terms times one ulp)."""
    terms = [fx * bx, fx * by, fy * bx, fy * by]
    ref = np.array([t.sum() for t in terms]) / area
    mag = np.array([np.abs(t).sum() for t in terms]) / area
    return ref, mag


@pytest.mark.parametrize("ncontacts", [300_000, 4 * 1024 * 1024])
def test_noalloc_many_blocks_and_the_cap_on_a_stream(ncontacts):
    """Synthetic contacts: about 300k (the final pass loops over more than
    256 block partials) and exactly the stated maximum, queued on a torch
    stream rather than the default one; each compared with numpy's sum."""
    torch = pytest.importorskip("torch")
    lib = abi.load_library()
    assert ncontacts <= lib.xdem_total_stress_noalloc_max_contacts()
    rng = np.random.default_rng(ncontacts)
    fx, fy, bx, by = (rng.normal(0.0, 1.0, ncontacts) for _ in range(4))
    area = 1234.5
    ref, mag = _stress_sum_bound(fx, fy, bx, by, area)
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        dev = [torch.tensor(a, dtype=torch.float64, device="cuda") for a in (fx, fy, bx, by)]
        out = torch.full((4,), float("nan"), dtype=torch.float64, device="cuda")
    stream.synchronize()
    for _ in range(2):
        st = lib.xdem_total_stress_noalloc(ncontacts, *[C.c_void_p(t.data_ptr()) for t in dev], area,
                                           C.c_void_p(out.data_ptr()), C.c_void_p(stream.cuda_stream))
        assert st == abi.OK
        stream.synchronize()
        s = out.cpu().numpy()
        assert np.all(np.abs(s - ref) <= 1e-12 * mag), (s, ref)
