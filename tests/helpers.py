"""Shared builders and comparisons for the parity tests."""
import numpy as np

from xdem_b200 import abi, inputs
from xdem_b200.world import make_control, make_params

STATE_KEYS = ("x", "y", "vx", "vy", "rot", "rot_vel")
CONTACT_KEYS = ("normal_x", "normal_y", "point_x", "point_y", "branch_x", "branch_y", "bv1_x",
                "bv1_y", "bv2_x", "bv2_y", "shear_x", "shear_y", "fn_x", "fn_y", "ft_x", "ft_y",
                "torque_i", "torque_j", "damping")


def disc_case(n=256, phi=0.80, seed=3, kind=abi.WORLD_PERIODIC, vel_sigma=0.01, **kw):
    p, box = inputs.disc_system(n, phi=phi, seed=seed, vel_sigma=vel_sigma)
    dt = inputs.time_step(p)
    prm = make_params(kind, dt, box, inputs.KN, inputs.KT, inputs.RESTITUTION, inputs.FRICTION, **kw)
    return p, prm


def ellipse_case(n=400, seed=5, kind=abi.WORLD_PERIODIC, method=abi.ELLIPSE_CLOSEST_APPROACH,
                 compress=1.25, b=inputs.c2_b, aspect=inputs.c2_aspect, phi_rsa_circle=0.42,
                 vel_sigma=0.01, shift_rate=0.1, **kw):
    """RSA of bounding circles, then a mild affine compression (by `compress` in
    solid fraction) that makes contacts without deep overlaps."""
    p, box = inputs.ellipse_system(n, b=b, aspect=aspect, phi_rsa_circle=phi_rsa_circle, phi=None,
                                   seed=seed, vel_sigma=vel_sigma)
    area = (box[1] - box[0]) * (box[3] - box[2])
    phi0 = p["volume"].sum() / area
    box = inputs.scale_to_fraction(p, box, p["volume"].sum(), phi0 * compress)
    dt = inputs.time_step(p)
    prm = make_params(kind, dt, box, inputs.KN, inputs.KT, inputs.RESTITUTION, inputs.FRICTION,
                      ellipse_method=method,
                      shift_strain_rate=shift_rate if kind == abi.WORLD_LEES_EDWARDS else 0.0, **kw)
    return p, prm


def clump_case(nfree=120, nclump=30, seed=11, phi=0.55):
    """Discs plus clumps of 2-5 circular sub-discs (radii U[0.3,0.6], offsets
    within 0.8 of the clump centre); sub-particle ids follow the clump id."""
    rng = np.random.default_rng(seed)
    # bounding radius of each body for RSA
    bodies = []
    for _ in range(nfree):
        bodies.append(("disc", rng.choice([0.5, 0.7])))
    for _ in range(nclump):
        k = int(rng.integers(2, 6))
        r = rng.uniform(0.3, 0.6, k)
        ang = rng.uniform(0, 2 * np.pi, k)
        rad = 0.8 * np.sqrt(rng.uniform(0, 1, k))
        off = np.stack([rad * np.cos(ang), rad * np.sin(ang)], 1)
        bodies.append(("clump", (r, off)))
    order = rng.permutation(len(bodies))
    bodies = [bodies[i] for i in order]
    bound = np.array([b[1] if b[0] == "disc" else float(np.max(np.hypot(b[1][1][:, 0], b[1][1][:, 1]) + b[1][0]))
                      for b in bodies])
    area = float(np.sum(np.pi * bound ** 2))
    box = inputs.box_for(area, 0.42)
    bx, by = inputs.rsa_positions(bound, box, seed + 7)
    # bring the body centres closer (bounding-disc fraction 0.42 -> phi); the
    # clump shapes are built afterwards, so they keep their size
    s = np.sqrt(0.42 / phi)
    bx, by, box = bx * s, by * s, box * s
    rows = []
    for (kind, data), cx, cy in zip(bodies, bx, by):
        if kind == "disc":
            rows.append(dict(shape=0, r=data, x=cx, y=cy, up=-1, setting=0, nsub=0))
        else:
            r, off = data
            rows.append(dict(shape=2, r=-1.0, x=cx, y=cy, up=-1, setting=abi.SKIP_CONTACT_DETECTION,
                             nsub=len(r)))
            for k in range(len(r)):
                rows.append(dict(shape=0, r=r[k], x=cx + off[k, 0], y=cy + off[k, 1], up=-2,
                                 setting=abi.SKIP_TIME_INTEGRAL | abi.SKIP_MACRO_SUM, nsub=0))
    n = len(rows)
    shape = np.array([r["shape"] for r in rows], np.int32)
    rad = np.array([r["r"] for r in rows])
    x = np.array([r["x"] for r in rows])
    y = np.array([r["y"] for r in rows])
    nsub = np.array([r["nsub"] for r in rows], np.int32)
    setting = np.array([r["setting"] for r in rows], np.int32)
    up = np.arange(n, dtype=np.int32)
    cur = -1
    for i, r in enumerate(rows):
        if r["shape"] == 2:
            cur = i
        elif r["up"] == -2:
            up[i] = cur
    prop_shape = np.where(shape == 2, 0, shape).astype(np.int32)
    prop_r = np.where(shape == 2, 1.0, rad)
    p = inputs.assemble(prop_shape, prop_r, np.ones(n), x, y, rng.normal(0, 0.01, n),
                        rng.normal(0, 0.01, n), np.zeros(n), np.zeros(n))
    p["shape"] = shape
    p["radius"] = rad.copy()
    p["outer_radius"] = rad.copy()
    p["up_level"] = up
    p["setting"] = setting
    p["num_sub"] = nsub
    bxv = np.zeros(n)
    byv = np.zeros(n)
    from xdem_b200 import abi as A
    import ctypes as C
    lib = A.load_library()
    d = C.POINTER(C.c_double)
    for i in np.where(shape == 2)[0]:
        k = nsub[i]
        s = np.arange(i + 1, i + 1 + k)
        out = np.zeros(7)
        brx = np.zeros(k)
        bry = np.zeros(k)
        sub_shape = np.ascontiguousarray(shape[s])
        st = lib.xdem_clump_properties(
            int(k), sub_shape.ctypes.data_as(C.POINTER(C.c_int32)),
            np.ascontiguousarray(rad[s]).ctypes.data_as(d), np.ones(k).ctypes.data_as(d),
            np.ascontiguousarray(x[s]).ctypes.data_as(d), np.ascontiguousarray(y[s]).ctypes.data_as(d),
            np.zeros(k).ctypes.data_as(d), 1.0, out.ctypes.data_as(d), brx.ctypes.data_as(d),
            bry.ctypes.data_as(d))
        assert st == 0
        p["x"][i], p["y"][i] = out[0], out[1]
        p["volume"][i], p["mass"][i], p["inv_mass"][i] = out[2], out[3], out[4]
        p["inertia"][i], p["inv_inertia"][i] = out[5], out[6]
        p["vx"][s] = p["vx"][i]
        p["vy"][s] = p["vy"][i]
        for q, sp in enumerate(s):
            # GluedParticle.cpp:71-75: each sub-particle takes the clump's mass and inertia
            p["mass"][sp], p["inv_mass"][sp] = out[3], out[4]
            p["inertia"][sp], p["inv_inertia"][sp] = out[5], out[6]
            bxv[sp], byv[sp] = brx[q], bry[q]
            p["vx"][sp] = p["vx"][i]
            p["vy"][sp] = p["vy"][i]
    p["branch_x"] = bxv
    p["branch_y"] = byv
    p["outer_radius"][shape == 2] = -1.0
    dt = inputs.time_step(p)
    prm = make_params(abi.WORLD_PERIODIC, dt, box, inputs.KN, inputs.KT, inputs.RESTITUTION,
                      inputs.FRICTION)
    return p, prm


def same_pairs(ca, cb):
    return (len(ca["id_i"]) == len(cb["id_i"]) and np.array_equal(ca["id_i"], cb["id_i"])
            and np.array_equal(ca["id_j"], cb["id_j"]))


def rel_err(a, b, floor=1e-300):
    """Largest |a-b| relative to the largest finite magnitude; NaN must sit at
    the same places in both (the reference itself yields NaN fields for some
    degenerate ellipse pairs), inf likewise."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    if len(a) == 0:
        return 0.0
    if not np.array_equal(np.isnan(a), np.isnan(b)):
        return float("inf")
    fin = np.isfinite(a) & np.isfinite(b)
    if not np.array_equal(a[~fin & ~np.isnan(a)], b[~fin & ~np.isnan(b)]):
        return float("inf")
    if not fin.any():
        return 0.0
    a, b = a[fin], b[fin]
    scale = max(np.max(np.abs(a)), np.max(np.abs(b)), floor)
    return float(np.max(np.abs(a - b)) / scale)


def compare_pair_geometry(og, oc, pi, pj, off, method, tol=1e-10):
    """GPU pair geometry `og` against the checker's `oc` (rows as
    xdem_pair_geometry).  Conditioning: the orientations are perturbed by one
    ulp (the size of the cos/sin differences between CUDA and glibc) and the
    checker's own outputs move by `spread`; the GPU may differ by a few times
    that, and by at most `tol` of the field's scale on the well-conditioned
    pairs (all but the near-tangent ones of the intersection quartic, whose
    near-double root turns an ulp into ~sqrt(ulp))."""
    import oracle
    hit = oc[:, 0] == 1
    spread = np.zeros_like(oc)
    for sgn in (-1.0, 1.0):
        qi, qj = pi.copy(), pj.copy()
        qi[:, 7] = np.nextafter(pi[:, 7], sgn * np.inf)
        qj[:, 7] = np.nextafter(pj[:, 7], -sgn * np.inf)
        op, _ = oracle.pair_geometry(qi, qj, off, method, "port")
        both = (op[:, 0] == 1) & hit
        d = np.where(both[:, None], np.abs(np.nan_to_num(op - oc)), 0.0)
        spread = np.maximum(spread, d)
    for col in range(1, 16):
        a, b = og[hit, col], oc[hit, col]
        assert np.array_equal(np.isnan(a), np.isnan(b)), col
        fin = np.isfinite(a)
        if not fin.any():
            continue
        scale = np.max(np.abs(b[fin]))
        err = np.abs(a[fin] - b[fin])
        allowed = tol * scale + 8.0 * spread[hit, col][fin]
        assert np.all(err <= allowed), (col, float(np.max(err / allowed)))
    # pairs whose outputs move by at most 1e-12 of scale under a 1-ulp
    # perturbation (condition number below ~5e3) must also meet `tol` alone
    well = hit & (spread[:, 9] <= 1e-12 * np.nanmax(np.abs(oc[hit, 9])))
    assert well.sum() >= 0.75 * hit.sum(), (well.sum(), hit.sum())
    for col in range(1, 16):
        assert rel_err(og[well, col], oc[well, col]) <= tol, col
    return int(hit.sum() - well.sum())


def compare_contacts(ca, cb, tol, keys=CONTACT_KEYS):
    assert same_pairs(ca, cb), (len(ca["id_i"]), len(cb["id_i"]))
    worst = {k: rel_err(ca[k], cb[k]) for k in keys}
    bad = {k: v for k, v in worst.items() if v > tol}
    assert not bad, bad
    return worst


def compare_states(sa, sb, tol, keys=STATE_KEYS):
    worst = {k: rel_err(sa[k], sb[k]) for k in keys}
    bad = {k: v for k, v in worst.items() if v > tol}
    assert not bad, bad
    return worst


def controls():
    return {
        "plain": make_control(),
        "stress": make_control(update_stress=True),
        "strain": make_control(update_stress=True, box_law=abi.BOX_STRAIN, p0=-2e-3, p1=-2e-3),
        "stress_xy": make_control(update_stress=True, box_law=abi.BOX_STRESS_XY, p0=5.0,
                                  scale_rattlers=0.99, sequence=abi.SEQ_SUBSTEPS),
        "uniform": make_control(update_stress=True, box_law=abi.BOX_STRESS_UNIFORM, p0=5.0,
                                reset_rattlers=True),
        # updatePeriodicBoundary_stressControlUniform_strainLimit
        # (PeriodicControlWorld.cpp:215-237); needs setup_control (max strain rate)
        "uniform_limit": make_control(update_stress=True, box_law=abi.BOX_STRESS_UNIFORM_LIMIT,
                                      p0=5.0, reset_rattlers=True),
    }


# max strain rate of the "uniform_limit" control: the box velocity grows by
# (p0 - p) L dt per step, so the limit (rate * L / 2) binds after a few tens of
# steps and the law runs both branches within a short trajectory
UNIFORM_LIMIT_MAX_STRAIN_RATE = 0.05


def setup_control(name, *worlds):
    """World settings a control of controls() needs (setMaxStrainRate,
    PeriodicControlWorld.cpp:69-71, for the strain-limited law)."""
    if name == "uniform_limit":
        for w in worlds:
            w.setMaxStrainRate(UNIFORM_LIMIT_MAX_STRAIN_RATE)


def dense_ellipse_case(n=3000, seed=21, kind=abi.WORLD_LEES_EDWARDS, phi=0.85, aspect=inputs.c4_aspect,
                       shift_rate=0.1, steps=1500, relax=300):
    """An ellipse packing compressed on the GPU (FP64) to solid fraction phi;
    returns (particles, contacts, params) for a world of the given kind."""
    from xdem_b200 import packing
    p, box = inputs.ellipse_system(n, b=inputs.c2_b, aspect=aspect, phi_rsa_circle=0.40, phi=None,
                                   seed=seed, vel_sigma=0.01)
    dt = inputs.time_step(p)
    q, contacts, b, _ = packing.compress(p, box, phi, dt, steps=steps, relax=relax)
    prm = make_params(kind, dt, b, inputs.KN, inputs.KT, inputs.RESTITUTION, inputs.FRICTION,
                      shift_strain_rate=shift_rate if kind == abi.WORLD_LEES_EDWARDS else 0.0)
    return q, contacts, prm


def _point_segment_nearest(px, py, x1, y1, x2, y2):
    dx, dy = x2 - x1, y2 - y1
    t = np.clip(((px - x1) * dx + (py - y1) * dy) / (dx * dx + dy * dy), 0.0, 1.0)
    qx, qy = x1 + t * dx, y1 + t * dy
    return np.hypot(px - qx, py - qy), qx, qy


def _point_segment_distance(px, py, x1, y1, x2, y2):
    return _point_segment_nearest(px, py, x1, y1, x2, y2)[0]


def segment_case(n=400, phi=0.80, seed=31, kind=abi.WORLD_PERIODIC, nfront=3, vel_sigma=0.05,
                 long_walls=False, **kw):
    """Bidisperse discs with fixed wall segments: a horizontal chain inside the
    box, a tilted chain, and single segments next to the periodic edges (their
    pairs with discs across the edge are image pairs).  Discs near a segment
    are moved out to an overlap of 10% of their radius, so that the first
    steps start with many mild wall contacts.  The first `nfront` segments take the
    lowest ids (they own their contacts, SegmentObject.cpp:45-80), the others
    the highest (the discs own theirs, CircularParticle.cpp:94-129)."""
    p, box = inputs.disc_system(n, phi=phi, seed=seed, vel_sigma=vel_sigma)
    L = box[1] - box[0]
    piece = 3.0 if long_walls else 1.2
    xs = np.arange(-0.35 * L, 0.35 * L - piece, piece)
    x1 = list(xs)
    y1 = [0.1 * L] * len(xs)
    x2 = list(xs + piece)
    y2 = [0.1 * L] * len(xs)
    ang = 0.6
    for k in range(4):  # tilted chain
        sx = -0.2 * L + k * piece * np.cos(ang)
        sy = -0.3 * L + k * piece * np.sin(ang)
        x1.append(sx)
        y1.append(sy)
        x2.append(sx + piece * np.cos(ang))
        y2.append(sy + piece * np.sin(ang))
    for (cx, cy, a) in ((box[1] - 0.3, 0.0, 1.4), (box[0] + 0.2, -0.25 * L, 0.3),
                        (0.3 * L, box[3] - 0.25, 0.05), (-0.1 * L, box[2] + 0.3, 2.0)):
        x1.append(cx - 0.5 * piece * np.cos(a))
        y1.append(cy - 0.5 * piece * np.sin(a))
        x2.append(cx + 0.5 * piece * np.cos(a))
        y2.append(cy + 0.5 * piece * np.sin(a))
    x1, y1, x2, y2 = (np.asarray(v, np.float64) for v in (x1, y1, x2, y2))
    # discs closer than 0.9 r to a segment move out to 0.9 r (along the
    # segment's normal when the centre lies on it); those still closer than
    # 0.75 r to some segment afterwards are removed
    for k in range(len(x1)):
        d, qx, qy = _point_segment_nearest(p["x"], p["y"], x1[k], y1[k], x2[k], y2[k])
        near = d < 0.9 * p["radius"]
        ux, uy = p["x"] - qx, p["y"] - qy
        nx, ny = -(y2[k] - y1[k]), x2[k] - x1[k]
        nn = np.hypot(nx, ny)
        tiny = d < 1e-9
        ux = np.where(tiny, nx / nn, ux / np.maximum(d, 1e-300))
        uy = np.where(tiny, ny / nn, uy / np.maximum(d, 1e-300))
        p["x"] = np.where(near, qx + ux * 0.9 * p["radius"], p["x"])
        p["y"] = np.where(near, qy + uy * 0.9 * p["radius"], p["y"])
    keep = np.ones(len(p["x"]), bool)
    for k in range(len(x1)):
        d = _point_segment_distance(p["x"], p["y"], x1[k], y1[k], x2[k], y2[k])
        keep &= d >= 0.75 * p["radius"]
    discs = {k: np.ascontiguousarray(v[keep]) for k, v in p.items()}
    discs["up_level"] = np.arange(int(keep.sum()), dtype=np.int32)
    dt = inputs.time_step(discs)
    seg = inputs.segments(x1, y1, x2, y2)
    front = {k: v[:nfront] for k, v in seg.items()}
    back = {k: v[nfront:] for k, v in seg.items()}
    for part in (front, back):
        part["up_level"] = np.arange(len(part["x"]), dtype=np.int32)
    q = inputs.concatenate(front, discs, back)
    prm = make_params(kind, dt, box, inputs.KN, inputs.KT, inputs.RESTITUTION, inputs.FRICTION, **kw)
    return q, prm
