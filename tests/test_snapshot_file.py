"""Snapshot files are checked in full on the host before any of their
contents reaches the device (xdem_snapshot_info runs the same reader as
xdem_load_snapshot, and needs no GPU): a truncated or padded file, systems
that do not cover the ids [0, n) in order, a saved memory order that is not a
permutation within each system, and contact ids outside the world are all
rejected with XDEM_ERR_ARGUMENT.  The files here are written byte by byte
from the layout the library reports (xdem_snapshot_layout)."""
import ctypes as C
import os

import numpy as np
import pytest

from xdem_b200 import abi


class SnapHeader(C.Structure):
    _fields_ = [("magic", C.c_char * 8), ("version", C.c_uint32), ("nsys", C.c_uint32),
                ("n", C.c_int32), ("K", C.c_int32), ("ncontacts", C.c_int64),
                ("scalars_bytes", C.c_uint32), ("params_bytes", C.c_uint32),
                ("since_resort", C.c_int32), ("has_seg", C.c_int32), ("prm", abi.Params)]


def _layout():
    lib = abi.load_library()
    out = (C.c_int64 * 4)()
    assert lib.xdem_snapshot_layout(out) == 0
    return [int(v) for v in out]


def _info(path):
    lib = abi.load_library()
    out = (C.c_int64 * 4)()
    st = lib.xdem_snapshot_info(str(path).encode(), out)
    return st, [int(v) for v in out]


def _write(path, systems, mem_id=None, contacts=((0, 1),), nsys_header=None, n_header=None,
           tail=b"", cut=0):
    """A snapshot of n = sum(counts) particles; systems = [(first, count)]."""
    hsize, ssize, off_first, off_count = _layout()
    n = sum(c for _, c in systems)
    h = SnapHeader()
    h.magic = b"XDEMSNP1"
    h.version = 1
    h.nsys = len(systems) if nsys_header is None else nsys_header
    h.n = n if n_header is None else n_header
    h.K = 24
    h.ncontacts = len(contacts)
    h.scalars_bytes = ssize
    h.params_bytes = C.sizeof(abi.Params)
    h.since_resort = 0
    h.has_seg = 0
    h.prm.world_kind = abi.WORLD_PERIODIC
    assert C.sizeof(SnapHeader) == hsize
    blob = bytearray(bytes(h))
    for first, count in systems:
        rec = bytearray(ssize)
        rec[off_first:off_first + 4] = np.int32(first).tobytes()
        rec[off_count:off_count + 4] = np.int32(count).tobytes()
        blob += rec
    blob += np.zeros(5 * n, np.int32).tobytes()
    blob += np.ones(16 * n, np.float64).tobytes()
    blob += np.asarray(np.arange(n) if mem_id is None else mem_id, np.int32).tobytes()
    ci = np.array([c[0] for c in contacts], np.int32)
    cj = np.array([c[1] for c in contacts], np.int32)
    blob += ci.tobytes() + cj.tobytes()
    blob += np.zeros(19 * len(contacts), np.float64).tobytes()
    blob += tail
    if cut:
        blob = blob[:-cut]
    with open(path, "wb") as f:
        f.write(bytes(blob))
    return path


def test_valid_file_reads(tmp_path):
    st, out = _info(_write(tmp_path / "ok.snap", [(0, 5), (5, 3)], mem_id=[4, 3, 2, 1, 0, 7, 5, 6]))
    assert st == 0
    assert out == [8, 2, 1, abi.WORLD_PERIODIC]


@pytest.mark.parametrize("case", [
    "missing", "bad_magic", "truncated", "padded", "gap", "overlap", "empty_system",
    "short_cover", "mem_dup", "mem_outside_system", "contact_id", "nsys_above_n", "huge_n"])
def test_corrupt_file_rejected(tmp_path, case):
    p = tmp_path / f"{case}.snap"
    if case == "missing":
        pass
    elif case == "bad_magic":
        _write(p, [(0, 4)])
        b = bytearray(open(p, "rb").read())
        b[0] = ord("Y")
        open(p, "wb").write(bytes(b))
    elif case == "truncated":
        _write(p, [(0, 4)], cut=3)
    elif case == "padded":
        _write(p, [(0, 4)], tail=b"\0")
    elif case == "gap":
        _write(p, [(1, 4)], n_header=4)
    elif case == "overlap":
        _write(p, [(0, 3), (2, 2)], n_header=5)
    elif case == "empty_system":
        _write(p, [(0, 4), (4, 0)])
    elif case == "short_cover":
        _write(p, [(0, 3)], n_header=4, tail=b"\0" * (5 * 4 + 16 * 8 + 4))
    elif case == "mem_dup":
        _write(p, [(0, 4)], mem_id=[0, 1, 1, 3])
    elif case == "mem_outside_system":
        _write(p, [(0, 2), (2, 2)], mem_id=[0, 2, 1, 3])
    elif case == "contact_id":
        _write(p, [(0, 4)], contacts=((0, 4),))
    elif case == "nsys_above_n":
        _write(p, [(0, 1), (1, 1)], nsys_header=3)
    elif case == "huge_n":
        _write(p, [(0, 4)], n_header=1 << 30)
    st, _ = _info(p)
    assert st == abi.ERR_ARGUMENT, case


def test_reader_never_follows_a_bad_order_into_the_device():
    """The loader's permutation is built from ids the reader already checked:
    a missing file is rejected before any world is touched."""
    st, _ = _info(os.path.join(os.sep, "nonexistent", "x.snap"))
    assert st == abi.ERR_ARGUMENT
