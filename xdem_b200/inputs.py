"""Seeded synthetic inputs with the shapes, sizes and distributions of the
benchmark configurations (there is no dataset: every input is generated).

Positions come from random sequential addition (RSA) of bounding discs
without overlap; a packing denser than RSA can reach is then made by the
reference's own recipe, an affine scale of box and positions
(scaleBoundarySizeToGivenSolidFraction, PeriodicBoundaryWorld.cpp:276-284),
optionally followed by relaxation or controlled compression on the GPU.
"""
import ctypes as C
import math

import numpy as np

from . import abi

KN = 1.0e4
KT = 0.5 * KN
FRICTION = 0.5
DAMPING_RATIO = 0.3
# restitution coefficient with normal damping ratio 0.3:
# e = exp(-zeta*pi/sqrt(1-zeta^2)); the reference's damping factor is then 2*sqrt(kn)*zeta
RESTITUTION = math.exp(-DAMPING_RATIO * math.pi / math.sqrt(1.0 - DAMPING_RATIO ** 2))


def particle_properties(shape, radius, aspect, density=1.0):
    lib = abi.load_library()
    n = len(radius)
    shape = np.ascontiguousarray(shape, np.int32)
    radius = np.ascontiguousarray(radius, np.float64)
    aspect = np.ascontiguousarray(aspect, np.float64)
    out = {k: np.zeros(n) for k in ("volume", "mass", "inv_mass", "inertia", "inv_inertia")}
    d = C.POINTER(C.c_double)
    st = lib.xdem_particle_properties(
        n, shape.ctypes.data_as(C.POINTER(C.c_int32)), radius.ctypes.data_as(d),
        aspect.ctypes.data_as(d), density, *[out[k].ctypes.data_as(d) for k in
                                             ("volume", "mass", "inv_mass", "inertia", "inv_inertia")])
    if st:
        raise abi.XdemError(st, "xdem_particle_properties")
    return out


def rsa_positions(bound_radius, box, seed, max_attempts=100000, largest_first=True):
    """RSA of discs; with largest_first the discs are added in decreasing size
    (the usual order for polydisperse RSA), positions returned in input order."""
    if largest_first:
        order = np.argsort(-np.asarray(bound_radius), kind="stable")
        xs, ys = rsa_positions(np.asarray(bound_radius)[order], box, seed, max_attempts, False)
        x = np.empty_like(xs)
        y = np.empty_like(ys)
        x[order] = xs
        y[order] = ys
        return x, y
    lib = abi.load_library()
    n = len(bound_radius)
    r = np.ascontiguousarray(bound_radius, np.float64)
    b = np.ascontiguousarray(box, np.float64)
    x = np.zeros(n)
    y = np.zeros(n)
    d = C.POINTER(C.c_double)
    st = lib.xdem_rsa_positions(n, r.ctypes.data_as(d), b.ctypes.data_as(d), C.c_uint64(seed),
                                max_attempts, x.ctypes.data_as(d), y.ctypes.data_as(d))
    if st:
        raise abi.XdemError(st, "xdem_rsa_positions")
    return x, y


def assemble(shape, radius, aspect, x, y, vx, vy, rot, rot_vel, density=1.0):
    n = len(radius)
    props = particle_properties(shape, radius, aspect, density)
    p = {
        "shape": np.ascontiguousarray(shape, np.int32),
        "up_level": np.arange(n, dtype=np.int32),
        "setting": np.zeros(n, np.int32),
        "is_rattler": np.zeros(n, np.int32),
        "outer_radius": np.ascontiguousarray(radius, np.float64),
        "radius": np.ascontiguousarray(radius, np.float64),
        "aspect_ratio": np.ascontiguousarray(aspect, np.float64),
        "x": np.ascontiguousarray(x, np.float64), "y": np.ascontiguousarray(y, np.float64),
        "vx": np.ascontiguousarray(vx, np.float64), "vy": np.ascontiguousarray(vy, np.float64),
        "rot": np.ascontiguousarray(rot, np.float64),
        "rot_vel": np.ascontiguousarray(rot_vel, np.float64),
        "num_sub": np.zeros(n, np.int32),
        "branch_x": np.zeros(n), "branch_y": np.zeros(n),
    }
    p.update(props)
    return p


def segments(x1, y1, x2, y2, vx=0.0, vy=0.0, rot_vel=0.0, density=1.0):
    """Fixed wall segments from their vertices, with the fields the reference
    constructor derives (SegmentObject.h:24-40): radius = outer radius = half
    the vertex distance, position = the midpoint, rotation = the direction's
    angle, SKIP_TIME_INTEGRAL set; volume, mass and inertia as
    SegmentObject::calculateParticleProperties gives them."""
    x1, y1, x2, y2 = (np.ascontiguousarray(np.atleast_1d(v), np.float64) for v in (x1, y1, x2, y2))
    n = len(x1)
    half = np.sqrt((x1 - x2) * (x1 - x2) + (y1 - y2) * (y1 - y2)) / 2.0
    shape = np.full(n, abi.SHAPE_SEGMENT, np.int32)
    p = assemble(shape, half, np.ones(n), (x1 + x2) / 2.0, (y1 + y2) / 2.0,
                 np.broadcast_to(vx, (n,)).copy(), np.broadcast_to(vy, (n,)).copy(),
                 np.arctan2(y2 - y1, x2 - x1), np.broadcast_to(rot_vel, (n,)).copy(), density)
    p["setting"][:] = abi.SKIP_TIME_INTEGRAL
    p["seg_x1"], p["seg_y1"], p["seg_x2"], p["seg_y2"] = x1.copy(), y1.copy(), x2.copy(), y2.copy()
    return p


def concatenate(*parts):
    """One particle dict from several, ids in the order given (clump
    sub-particle ids must stay right after their clump, so a part holding
    clumps goes in whole)."""
    n = [len(q["x"]) for q in parts]
    out = {}
    keys = set().union(*[q.keys() for q in parts])
    for k in keys:
        arrs = []
        for q, m in zip(parts, n):
            if k in q and q[k] is not None:
                arrs.append(np.asarray(q[k]))
            else:
                dt = np.int32 if k in ("shape", "up_level", "setting", "is_rattler", "num_sub") \
                    else np.float64
                arrs.append(np.zeros(m, dt))
        out[k] = np.ascontiguousarray(np.concatenate(arrs))
    # up levels point at ids: shift them with their part
    first = np.cumsum([0] + n[:-1])
    out["up_level"] = np.ascontiguousarray(np.concatenate(
        [np.asarray(q["up_level"], np.int32) + f for q, f in zip(parts, first)]).astype(np.int32))
    return out


def box_for(area, phi):
    half = 0.5 * math.sqrt(area / phi)
    return np.array([-half, half, -half, half])


def scale_to_fraction(p, box, volume_sum, phi):
    """scaleBoundarySizeToGivenSolidFraction (PeriodicBoundaryWorld.cpp:276-284)"""
    cur = volume_sum / ((box[1] - box[0]) * (box[3] - box[2]))
    s = math.sqrt(cur / phi)
    p["x"] = p["x"] * s
    p["y"] = p["y"] * s
    return box * s


def disc_system(n, radii=(0.5, 0.7), phi_rsa=0.45, phi=0.70, seed=0, vel_sigma=0.01,
                density=1.0):
    """Bidisperse discs, 50:50 (config: 1,024 discs, r 0.5/0.7, phi 0.70)."""
    rng = np.random.default_rng(seed)
    r = np.where(rng.permutation(n) < n // 2, radii[0], radii[1]).astype(np.float64)
    area = float(np.sum(np.pi * r * r))
    box = box_for(area, phi_rsa)
    x, y = rsa_positions(r, box, seed + 1)
    vx = rng.normal(0.0, vel_sigma, n)
    vy = rng.normal(0.0, vel_sigma, n)
    p = assemble(np.zeros(n, np.int32), r, np.ones(n), x, y, vx, vy, np.zeros(n), np.zeros(n),
                 density)
    if phi is not None and phi != phi_rsa:
        box = scale_to_fraction(p, box, float(np.sum(p["volume"])), phi)
    return p, box


def ellipse_system(n, b=None, aspect=None, phi_rsa_circle=0.45, phi=None, seed=0, vel_sigma=0.0,
                   density=1.0, rng_kind="bidisperse"):
    """Ellipses with semi-axes (a, b), a = aspect*b, orientations U[0, pi).
    `b` and `aspect` are arrays, or callables rng -> array."""
    rng = np.random.default_rng(seed)
    bb = b(rng, n) if callable(b) else np.asarray(b, np.float64)
    asp = aspect(rng, n) if callable(aspect) else np.asarray(aspect, np.float64)
    a = asp * bb
    area_circle = float(np.sum(np.pi * a * a))
    box = box_for(area_circle, phi_rsa_circle)
    x, y = rsa_positions(a, box, seed + 1)
    rot = rng.uniform(0.0, np.pi, n)
    vx = rng.normal(0.0, vel_sigma, n) if vel_sigma > 0 else np.zeros(n)
    vy = rng.normal(0.0, vel_sigma, n) if vel_sigma > 0 else np.zeros(n)
    p = assemble(np.ones(n, np.int32), a, asp, x, y, vx, vy, rot, np.zeros(n), density)
    if phi is not None:
        box = scale_to_fraction(p, box, float(np.sum(p["volume"])), phi)
    return p, box


def time_step(p, kn=KN, factor=0.02):
    """dt = 0.02 * sqrt(m_min / kn)"""
    return factor * math.sqrt(float(np.min(p["mass"][p["shape"] != abi.SHAPE_CLUMP])) / kn)


# ---- configuration-shaped generators ------------------------------------------

def c1_b(rng, n):
    return rng.uniform(0.4, 0.6, n)


def c1_aspect(rng, n):
    return np.full(n, 1.5)


def c2_b(rng, n):
    return np.where(rng.permutation(n) < n // 2, 0.5, 0.7).astype(np.float64)


def c2_aspect(rng, n):
    return rng.uniform(1.0, 2.0, n)


def c4_aspect(rng, n):
    return rng.uniform(1.0, 3.0, n)


def clump_system(nclump, phi_rsa=0.42, seed=0, vel_sigma=0.01, density=1.0):
    """GluedParticle clumps of 2-5 circular sub-discs (radii U[0.3,0.6], offsets
    uniform within radius 0.8 of the clump centre), placed by RSA of their
    bounding discs at fraction phi_rsa.  Each clump is a row of shape CLUMP
    (SKIP_CONTACT_DETECTION, the GluedParticle) followed by its sub-discs
    (SKIP_TIME_INTEGRAL | SKIP_MACRO_SUM, up_level = the clump's id), whose
    branch vectors and the clump's mass and inertia come from
    xdem_clump_properties (GluedParticle::calculateParticleProperties)."""
    rng = np.random.default_rng(seed)
    k = rng.integers(2, 6, nclump)
    sub_r = [rng.uniform(0.3, 0.6, kk) for kk in k]
    sub_off = []
    bound = np.zeros(nclump)
    for c in range(nclump):
        ang = rng.uniform(0.0, 2.0 * np.pi, k[c])
        rad = 0.8 * np.sqrt(rng.uniform(0.0, 1.0, k[c]))
        off = np.stack([rad * np.cos(ang), rad * np.sin(ang)], 1)
        sub_off.append(off)
        bound[c] = float(np.max(np.hypot(off[:, 0], off[:, 1]) + sub_r[c]))
    box = box_for(float(np.sum(np.pi * bound ** 2)), phi_rsa)
    cx, cy = rsa_positions(bound, box, seed + 1)
    n = int(nclump + k.sum())
    shape = np.zeros(n, np.int32)
    radius = np.zeros(n)
    x = np.zeros(n)
    y = np.zeros(n)
    up = np.arange(n, dtype=np.int32)
    setting = np.zeros(n, np.int32)
    num_sub = np.zeros(n, np.int32)
    parent = np.zeros(nclump, np.int64)
    i = 0
    for c in range(nclump):
        parent[c] = i
        shape[i] = abi.SHAPE_CLUMP
        radius[i] = 1.0
        setting[i] = abi.SKIP_CONTACT_DETECTION
        num_sub[i] = k[c]
        s = slice(i + 1, i + 1 + k[c])
        radius[s] = sub_r[c]
        x[s] = cx[c] + sub_off[c][:, 0]
        y[s] = cy[c] + sub_off[c][:, 1]
        up[s] = i
        setting[s] = abi.SKIP_TIME_INTEGRAL | abi.SKIP_MACRO_SUM
        i += 1 + k[c]
    prop_shape = np.where(shape == abi.SHAPE_CLUMP, abi.SHAPE_CIRCLE, shape).astype(np.int32)
    vx = rng.normal(0.0, vel_sigma, n)
    vy = rng.normal(0.0, vel_sigma, n)
    p = assemble(prop_shape, radius, np.ones(n), x, y, vx, vy, np.zeros(n), np.zeros(n), density)
    p["shape"] = shape
    p["up_level"] = up
    p["setting"] = setting
    p["num_sub"] = num_sub
    lib = abi.load_library()
    d = C.POINTER(C.c_double)
    for c in range(nclump):
        i = int(parent[c])
        kk = int(k[c])
        s = np.arange(i + 1, i + 1 + kk)
        out = np.zeros(7)
        brx = np.zeros(kk)
        bry = np.zeros(kk)
        st = lib.xdem_clump_properties(
            kk, np.ascontiguousarray(shape[s]).ctypes.data_as(C.POINTER(C.c_int32)),
            np.ascontiguousarray(radius[s]).ctypes.data_as(d), np.ones(kk).ctypes.data_as(d),
            np.ascontiguousarray(x[s]).ctypes.data_as(d), np.ascontiguousarray(y[s]).ctypes.data_as(d),
            np.zeros(kk).ctypes.data_as(d), density, out.ctypes.data_as(d), brx.ctypes.data_as(d),
            bry.ctypes.data_as(d))
        if st:
            raise abi.XdemError(st, "xdem_clump_properties")
        p["x"][i], p["y"][i] = out[0], out[1]
        p["volume"][i], p["mass"][i], p["inv_mass"][i] = out[2], out[3], out[4]
        p["inertia"][i], p["inv_inertia"][i] = out[5], out[6]
        # GluedParticle.cpp:71-75: each sub-particle takes the clump's mass and inertia
        p["mass"][s], p["inv_mass"][s] = out[3], out[4]
        p["inertia"][s], p["inv_inertia"][s] = out[5], out[6]
        p["branch_x"][s], p["branch_y"][s] = brx, bry
        p["vx"][s] = p["vx"][i]
        p["vy"][s] = p["vy"][i]
    p["radius"][shape == abi.SHAPE_CLUMP] = -1.0
    p["outer_radius"] = p["radius"].copy()
    return p, box
