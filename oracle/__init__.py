"""TEST INFRASTRUCTURE ONLY — the CPU checkers of the CUDA path.

Two checkers share the reference-named interface of xdem_b200.world.WorldBase:
  PortWorld  the C restatement in oracle/xdem_oracle.c (liboracle.so), built
             by `make -C oracle` (and by __graft_entry__.build());
  RefWorld   the unmodified reference sources compiled with
             oracle/ref_harness.cpp into oracle/_ref/libxdem_ref.so.  It is only
             present where the reference sources were available at build time.
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use
this package; the product never imports it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from xdem_b200 import abi
from xdem_b200.world import WorldBase

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libxdem_ref.so")

_d = C.POINTER(C.c_double)
_i = C.POINTER(C.c_int32)
_port = None
_ref = None


def build(ref_src=None):
    """make -C oracle (the restatement always; the reference when its sources
    exist).  ref_src: the reference's src/ folder; default the environment
    variable XDEM_REFERENCE_SRC, else the Makefile's own default."""
    ref_src = ref_src or os.environ.get("XDEM_REFERENCE_SRC")
    cmd = ["make", "-s", "-C", HERE]
    if ref_src:
        cmd.append(f"REF_SRC={ref_src}")
    subprocess.run(cmd, check=True)


def ref_available():
    return os.path.exists(REF_LIB)


def _bind(lib, prefix):
    P = C.POINTER
    V = C.c_void_p
    sig = {
        "create": (V, [P(abi.Params), C.c_int32]),
        "destroy": (None, [V]),
        "set_particles": (C.c_int32, [V, P(abi.Particles)]),
        "get_particles": (C.c_int32, [V, P(abi.Particles)]),
        "set_contacts": (C.c_int32, [V, P(abi.Contacts)]),
        "get_contacts": (C.c_int32, [V, P(abi.Contacts)]),
        "get_force_and_torque": (C.c_int32, [V, _d, _d, _d, _i]),
        "get_boundary": (None, [V, _d]),
        "get_stress": (None, [V, _d]),
        "get_lees_edwards": (None, [V, _d]),
        "set_lees_edwards": (None, [V, _d]),
        "set_virtual_boundary_mass": (None, [V, C.c_double]),
        "set_max_strain_rate": (None, [V, C.c_double]),
        "kinetic_energy": (C.c_double, [V]),
        "count_contacts": (C.c_int64, [V]),
        "call": (C.c_int32, [V, C.c_int32, C.c_double, C.c_double, C.c_double]),
        "run": (C.c_int32, [V, C.c_int32, P(abi.Control), P(C.c_int32)]),
        "quadron_z_phi": (None, [V, _d]),
        "pair_geometry": (C.c_int32, [C.c_int32, C.c_int32, _d, _d, _d, _d]),
    }
    fns = {}
    for name, (res, args) in sig.items():
        fn = getattr(lib, prefix + name)
        fn.restype = res
        fn.argtypes = args
        fns[name] = fn
    return fns


def port_lib():
    global _port
    if _port is None:
        if not os.path.exists(PORT_LIB):
            raise ImportError(f"{PORT_LIB} missing: run `make -C oracle`")
        lib = C.CDLL(PORT_LIB)
        _port = _bind(lib, "xo_")
        lib.xo_status.restype = C.c_uint32
        lib.xo_status.argtypes = [C.c_void_p]
        lib.xo_newton_quartic.restype = C.c_double
        lib.xo_newton_quartic.argtypes = [C.c_double] * 6 + [_i, _i]
        lib.xo_bisect_quartic.restype = C.c_double
        lib.xo_bisect_quartic.argtypes = [C.c_double] * 7
        _port["bisect_quartic"] = lib.xo_bisect_quartic
        _port["status"] = lib.xo_status
        _port["newton_quartic"] = lib.xo_newton_quartic
        lib.xo_closest_quartic.restype = C.c_int32
        lib.xo_closest_quartic.argtypes = [C.c_int32, _d, _d, _d, _d]
        _port["closest_quartic"] = lib.xo_closest_quartic
    return _port


def ref_lib():
    global _ref
    if _ref is None:
        if not ref_available():
            raise ImportError(f"{REF_LIB} missing: the reference was not compiled here")
        lib = C.CDLL(REF_LIB)
        _ref = _bind(lib, "refh_")
        lib.refh_particle_properties.restype = None
        lib.refh_particle_properties.argtypes = [C.c_int32, _i, _d, _d, C.c_double] + [_d] * 5
        lib.refh_clump_properties.restype = None
        lib.refh_clump_properties.argtypes = [C.c_int32, _i, _d, _d, _d, _d, _d, C.c_double, _d,
                                              _d, _d]
        lib.refh_set_threads.restype = None
        lib.refh_set_threads.argtypes = [C.c_void_p, C.c_int32]
        lib.refh_get_control_mass.restype = C.c_double
        lib.refh_get_control_mass.argtypes = [C.c_void_p]
        _ref["particle_properties"] = lib.refh_particle_properties
        _ref["clump_properties"] = lib.refh_clump_properties
        _ref["set_threads"] = lib.refh_set_threads
        _ref["control_mass"] = lib.refh_get_control_mass
    return _ref


class _CpuWorld(WorldBase):
    def __init__(self, fns, params, threads=1):
        self.f = fns
        self.params = params
        self.h = fns["create"](C.byref(params), threads)
        self.n = 0

    def close(self):
        if self.h:
            self.f["destroy"](self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _set_particles(self, s):
        return self.f["set_particles"](self.h, C.byref(s))

    def _get_state(self, s):
        return self.f["get_particles"](self.h, C.byref(s))

    def _set_contacts(self, s):
        return self.f["set_contacts"](self.h, C.byref(s))

    def _get_contacts(self, s):
        return self.f["get_contacts"](self.h, C.byref(s))

    def _forces(self, fx, fy, t, nc):
        return self.f["get_force_and_torque"](self.h, fx, fy, t, nc)

    def count_contacts(self):
        return int(self.f["count_contacts"](self.h))

    def _call(self, which, a=0.0, b=0.0, c=0.0):
        return self._status(self.f["call"](self.h, which, a, b, c))

    def _run(self, nsteps, ctl, done):
        return self._status(self.f["run"](self.h, nsteps, C.byref(ctl), C.byref(done)))

    def _status(self, st):
        return st

    def _boundary(self, p):
        self.f["get_boundary"](self.h, p)

    def _stress(self, p):
        self.f["get_stress"](self.h, p)

    def _le(self, p):
        self.f["get_lees_edwards"](self.h, p)

    def _set_le(self, p):
        self.f["set_lees_edwards"](self.h, p)

    def _ke(self):
        return float(self.f["kinetic_energy"](self.h))

    def setVirtualBoundaryMass(self, mass=-1.0):
        self.f["set_virtual_boundary_mass"](self.h, mass)

    def setMaxStrainRate(self, rate):
        self.f["set_max_strain_rate"](self.h, rate)

    def quadron_z_phi(self):
        out = np.zeros(2)
        self.f["quadron_z_phi"](self.h, out.ctypes.data_as(_d))
        return out


class PortWorld(_CpuWorld):
    """The C restatement."""

    def __init__(self, params, threads=1):
        super().__init__(port_lib(), params, threads)

    def _status(self, st):
        # status bits accumulate in the world; read and clear them
        return int(self.f["status"](self.h))


class RefWorld(_CpuWorld):
    """The compiled reference."""

    def __init__(self, params, threads=1):
        super().__init__(ref_lib(), params, threads)

    def set_threads(self, threads):
        self.f["set_threads"](self.h, threads)

    def control_mass(self):
        return float(self.f["control_mass"](self.h))


def pair_geometry(pi, pj, off, method=abi.ELLIPSE_CLOSEST_APPROACH, which="port"):
    fns = port_lib() if which == "port" else ref_lib()
    pi = np.ascontiguousarray(pi, np.float64)
    pj = np.ascontiguousarray(pj, np.float64)
    off = np.ascontiguousarray(off, np.float64)
    out = np.zeros((pi.shape[0], 17))
    st = fns["pair_geometry"](pi.shape[0], method, pi.ctypes.data_as(_d), pj.ctypes.data_as(_d),
                              off.ctypes.data_as(_d), out.ctypes.data_as(_d))
    return out, st


def ref_particle_properties(shape, radius, aspect, density=1.0):
    fns = ref_lib()
    n = len(radius)
    shape = np.ascontiguousarray(shape, np.int32)
    radius = np.ascontiguousarray(radius, np.float64)
    aspect = np.ascontiguousarray(aspect, np.float64)
    out = {k: np.zeros(n) for k in ("volume", "mass", "inv_mass", "inertia", "inv_inertia")}
    fns["particle_properties"](n, shape.ctypes.data_as(_i), radius.ctypes.data_as(_d),
                               aspect.ctypes.data_as(_d), density,
                               *[out[k].ctypes.data_as(_d) for k in
                                 ("volume", "mass", "inv_mass", "inertia", "inv_inertia")])
    return out


def closest_quartic(pi, pj, off):
    """Per ellipse pair (pair_geometry's input layout), the checker's
    closest-approach quartic: columns A, B, C, D, E, the analytic start
    s = sqrt(delta+1), the root q, Newton's iterations, 1 where Newton did not
    terminate, contacted; zeros where the pair is rejected before the quartic
    is formed."""
    pi = np.ascontiguousarray(pi, np.float64)
    pj = np.ascontiguousarray(pj, np.float64)
    off = np.ascontiguousarray(off, np.float64)
    out = np.zeros((pi.shape[0], 10))
    st = port_lib()["closest_quartic"](pi.shape[0], pi.ctypes.data_as(_d), pj.ctypes.data_as(_d),
                                       off.ctypes.data_as(_d), out.ctypes.data_as(_d))
    return out, st


def newton_quartic(A, B, Cc, D, E, init):
    """(iterate, iterations, stuck) of the checker's Newton iteration."""
    it = C.c_int32(0)
    stuck = C.c_int32(0)
    r = port_lib()["newton_quartic"](A, B, Cc, D, E, init, C.byref(it), C.byref(stuck))
    return r, it.value, bool(stuck.value)


def bisect_quartic(A, B, Cc, D, E, s, q):
    return port_lib()["bisect_quartic"](A, B, Cc, D, E, s, q)


# ---- CPU-only inputs (no product library): the reference arm of bench.py ----

def particle_properties(shape, radius, aspect, density=1.0):
    """calculateParticleProperties of circles and ellipses: the compiled
    reference's own when it is built here, else its formulas
    (CircularParticle.cpp:16-23, EllipticParticle.cpp:7-14) in numpy."""
    if ref_available():
        return ref_particle_properties(shape, radius, aspect, density)
    r = np.asarray(radius, np.float64)
    k = np.asarray(aspect, np.float64)
    ell = np.asarray(shape) == abi.SHAPE_ELLIPSE
    vol = np.where(ell, np.pi * r * r / k, np.pi * r * r)
    mass = vol * density
    inertia = np.where(ell, mass * (r * r + r * r / k / k) / 4.0, mass * r * r / 2.0)
    return {"volume": vol, "mass": mass, "inv_mass": 1.0 / mass, "inertia": inertia,
            "inv_inertia": 1.0 / inertia}


def rsa_discs(radius, box, seed, max_attempts=100000):
    """Random sequential addition of discs (largest first) into the periodic
    box without overlap, with a cell grid; numpy only, seeded."""
    rng = np.random.default_rng(seed)
    r = np.asarray(radius, np.float64)
    n = len(r)
    L = box[1] - box[0]
    H = box[3] - box[2]
    cell = 2.0 * float(r.max())
    nx, ny = max(1, int(L // cell)), max(1, int(H // cell))
    grid = {}
    x = np.zeros(n)
    y = np.zeros(n)
    for i in np.argsort(-r, kind="stable"):
        for _ in range(max_attempts):
            px, py = rng.uniform(box[0], box[1]), rng.uniform(box[2], box[3])
            cx, cy = int((px - box[0]) / L * nx) % nx, int((py - box[2]) / H * ny) % ny
            ok = True
            for dx in (-1, 0, 1):
                for dy in (-1, 0, 1):
                    for j in grid.get(((cx + dx) % nx, (cy + dy) % ny), ()):
                        ddx = px - x[j]
                        ddy = py - y[j]
                        ddx -= L * round(ddx / L)
                        ddy -= H * round(ddy / H)
                        if ddx * ddx + ddy * ddy < (r[i] + r[j]) ** 2:
                            ok = False
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if ok:
                x[i], y[i] = px, py
                grid.setdefault((cx, cy), []).append(i)
                break
        else:
            raise RuntimeError("RSA did not place every disc")
    return x, y


def strain_compress(world_cls, p, box, dt, phi_target, steps, relax, damping=0.1,
                    method=abi.ELLIPSE_CLOSEST_APPROACH, threads=1):
    """Strain-controlled compression (updatePeriodicBoundary_strainControl,
    PeriodicControlWorld.cpp:124-135) of the particle dict p to phi_target in
    about `steps` steps, then `relax` steps at the final box, by a CPU world;
    returns (particles with the new state, contacts, box)."""
    import math
    from xdem_b200 import inputs
    from xdem_b200.world import make_control, make_params
    prm = make_params(abi.WORLD_PERIODIC_CONTROL, dt, box, inputs.KN, inputs.KT,
                      inputs.RESTITUTION, inputs.FRICTION, global_damping=damping,
                      ellipse_method=method)
    w = world_cls(prm, threads)
    w.raise_mask = ~abi.ERR_NEWTON
    w.set_particles(p)
    vol = float(p["volume"].sum())
    phi0 = vol / ((box[1] - box[0]) * (box[3] - box[2]))
    s_step = math.sqrt(phi0 / phi_target) ** (1.0 / steps)
    ctl = make_control(box_law=abi.BOX_STRAIN, reset_rattlers=False)
    done = 0
    while done < 3 * steps:
        b = w.getBoundary()
        L = b[1] - b[0]
        s_rem = math.sqrt(vol / (L * (b[3] - b[2])) / phi_target)
        if s_rem >= 1.0 - 1e-12:
            break
        left = max(1, int(math.ceil(math.log(s_rem) / math.log(s_step))))
        chunk = min(200, left)
        per = s_rem ** (1.0 / chunk) if chunk == left else s_step
        ctl.p0 = ctl.p1 = (per - 1.0) / (L * dt)
        w.run(chunk, ctl)
        done += chunk
    if relax:
        w.run(relax, make_control())
    st = w.get_state()
    q = dict(p)
    for k in ("x", "y", "vx", "vy", "rot", "rot_vel"):
        q[k] = st[k].copy()
    contacts = w.get_contacts()
    b = np.array(w.getBoundary())
    w.close()
    return q, contacts, b


def ellipse_sample(n, seed, aspect_hi=3.0, phi=0.85, threads=1, steps=3000, relax=1000):
    """A CPU-made sample of the ellipse shear workloads: n ellipses with
    b in {0.5, 0.7} (50:50) and a/b ~ U[1, aspect_hi], orientations U[0, pi),
    RSA of their bounding discs at fraction 0.40, then the C restatement's
    strain-controlled compression to solid fraction phi and a relaxation.
    Returns (particles, contacts, box, dt)."""
    from xdem_b200 import inputs
    rng = np.random.default_rng(seed)
    b = np.where(rng.permutation(n) < n // 2, 0.5, 0.7).astype(np.float64)
    k = rng.uniform(1.0, aspect_hi, n)
    a = k * b
    box = inputs.box_for(float(np.sum(np.pi * a * a)), 0.40)
    x, y = rsa_discs(a, box, seed + 1)
    rot = rng.uniform(0.0, np.pi, n)
    shape = np.ones(n, np.int32)
    props = particle_properties(shape, a, k)
    zero = np.zeros(n)
    p = {"shape": shape, "up_level": np.arange(n, dtype=np.int32), "setting": np.zeros(n, np.int32),
         "is_rattler": np.zeros(n, np.int32), "outer_radius": a, "radius": a.copy(),
         "aspect_ratio": k, "x": x, "y": y, "vx": zero.copy(), "vy": zero.copy(), "rot": rot,
         "rot_vel": zero.copy()}
    p.update(props)
    dt = 0.02 * float(np.sqrt(np.min(p["mass"]) / inputs.KN))
    q, contacts, box = strain_compress(PortWorld, p, box, dt, phi, steps, relax, threads=threads)
    return q, contacts, box, dt
