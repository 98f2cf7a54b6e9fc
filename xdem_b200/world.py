"""Host-side mirror of the reference's world interface over the C-ABI.

`WorldBase` carries the method names of the reference's BaseWorld,
PeriodicBoundaryWorld, PeriodicControlWorld and LeesEdwardsBoundaryWorld
(BaseWorld.h:59-105, PeriodicControlWorld.h:23-39,
LeesEdwardsBoundaryWorld.h:29-47) so that a driver written against the
reference reads the same.  A subclass supplies the primitive calls; `World`
runs them on the GPU through libxdem_b200.so.  Where the reference exits, the
methods raise XdemError carrying the status bits.
"""
import ctypes as C

import numpy as np

from . import abi

# sub-step codes shared with the CPU checkers
MODIFY, APPLY_BG, REMOVE_BG, FIND, UPDATE, COLLECT, INTEGRATE = 0, 1, 2, 3, 4, 5, 6
RESET_RATTLERS, SCALE_RATTLERS, STRESS, BOX_LAW, LE_BOUNDARY, TAKE_STEP, SCALE_TO_FRACTION = (
    7, 8, 9, 10, 11, 12, 13)


def make_params(kind, dt, box, kn, kt, restitution, friction, global_damping=0.0,
                shift_strain_rate=0.0, ellipse_method=abi.ELLIPSE_CLOSEST_APPROACH,
                precision=abi.PRECISION_FP64, max_contacts=0, max_particle_size=0.0):
    p = abi.Params()
    p.world_kind = kind
    p.ellipse_method = ellipse_method
    p.precision = precision
    p.max_contacts = max_contacts
    p.dt = dt
    p.xmin, p.xmax, p.ymin, p.ymax = box
    p.normal_stiffness = kn
    p.shear_stiffness = kt
    p.restitution_coeff = restitution
    p.frictional_coeff = friction
    p.global_damping = global_damping
    p.shift_strain_rate = shift_strain_rate
    p.max_particle_size = max_particle_size
    return p


def make_control(sequence=abi.SEQ_TAKE_TIME_STEP, scale_rattlers=None, reset_rattlers=False,
                 update_stress=False, box_law=abi.BOX_NONE, p0=0.0, p1=0.0, stop_pressure=None):
    c = abi.Control()
    c.sequence = sequence
    c.scale_rattlers = 0 if scale_rattlers is None else 1
    c.rattler_scale = 0.0 if scale_rattlers is None else scale_rattlers
    c.reset_rattlers = int(bool(reset_rattlers))
    c.update_stress = int(bool(update_stress))
    c.box_law = box_law
    c.p0, c.p1 = p0, p1
    c.stop_on_pressure = 0 if stop_pressure is None else 1
    c.stop_pressure = 0.0 if stop_pressure is None else stop_pressure
    return c


class WorldBase:
    """Reference-named methods over primitive calls supplied by a subclass."""

    raise_mask = 0xFFFFFFFF

    def _check(self, st, where):
        self.last_status = st
        if st & self.raise_mask:
            raise abi.XdemError(st, where)
        return st

    # ---- particles and contacts ----------------------------------------
    def set_particles(self, p):
        self.n = len(p["x"])
        self._pstruct_arrays = p
        self._check(self._set_particles(abi.particles_struct(p)), "set_particles")

    def get_state(self):
        out = abi.empty_state(self.n)
        self._check(self._get_state(abi.state_struct(out)), "get_state")
        return out

    def set_contacts(self, c):
        n = len(c["id_i"])
        arrs = {k: np.ascontiguousarray(v) for k, v in c.items()}
        self._check(self._set_contacts(abi.contacts_struct(arrs, n)), "set_contacts")

    def get_contacts(self):
        cap = max(16, self.count_contacts())
        arrs = abi.contact_arrays(cap)
        s = abi.contacts_struct(arrs)
        st = self._get_contacts(s)
        if st == abi.ERR_CAPACITY:
            arrs = abi.contact_arrays(int(s.count))
            s = abi.contacts_struct(arrs)
            st = self._get_contacts(s)
        self._check(st, "get_contacts")
        return abi.trim_contacts(arrs, int(s.count))

    def get_force_and_torque(self):
        fx = np.zeros(self.n)
        fy = np.zeros(self.n)
        t = np.zeros(self.n)
        nc = np.zeros(self.n, np.int32)
        d = C.POINTER(C.c_double)
        self._check(self._forces(fx.ctypes.data_as(d), fy.ctypes.data_as(d), t.ctypes.data_as(d),
                                 nc.ctypes.data_as(C.POINTER(C.c_int32))), "get_force_and_torque")
        return {"fx": fx, "fy": fy, "torque": t, "num_contacts": nc}

    # ---- reference sub-steps ------------------------------------------------
    def modifyParticlePosition(self):
        return self._check(self._call(MODIFY), "modifyParticlePosition")

    def applyBackgroudVelocity(self):
        return self._check(self._call(APPLY_BG), "applyBackgroudVelocity")

    def removeBackgroudVelocity(self):
        return self._check(self._call(REMOVE_BG), "removeBackgroudVelocity")

    def findPossibleContacts(self):
        return self._check(self._call(FIND), "findPossibleContacts")

    def updateContacts(self):
        return self._check(self._call(UPDATE), "updateContacts")

    def collectForceAndTorque(self):
        return self._check(self._call(COLLECT), "collectForceAndTorque")

    def takeTimeIntegral(self):
        return self._check(self._call(INTEGRATE), "takeTimeIntegral")

    def resetVelocityOfRattlers(self):
        return self._check(self._call(RESET_RATTLERS), "resetVelocityOfRattlers")

    def scaleVelocityOfRattlers(self, scale):
        return self._check(self._call(SCALE_RATTLERS, scale), "scaleVelocityOfRattlers")

    def updateTotalStress(self):
        self._check(self._call(STRESS), "updateTotalStress")
        return self.getStress()

    def updatePeriodicBoundary_strainControl(self, rx, ry):
        return self._check(self._call(BOX_LAW, abi.BOX_STRAIN, rx, ry), "strainControl")

    def updatePeriodicBoundary_stressControlXY(self, stress):
        return self._check(self._call(BOX_LAW, abi.BOX_STRESS_XY, stress), "stressControlXY")

    def updatePeriodicBoundary_stressControlUniform(self, stress):
        return self._check(self._call(BOX_LAW, abi.BOX_STRESS_UNIFORM, stress),
                           "stressControlUniform")

    def updatePeriodicBoundary_stressControlUniform_strainLimit(self, stress):
        return self._check(self._call(BOX_LAW, abi.BOX_STRESS_UNIFORM_LIMIT, stress),
                           "stressControlUniform_strainLimit")

    def updateLeesEdwardBoundary(self):
        return self._check(self._call(LE_BOUNDARY), "updateLeesEdwardBoundary")

    def scaleBoundarySizeToGivenSolidFraction(self, phi):
        return self._check(self._call(SCALE_TO_FRACTION, phi), "scaleBoundarySizeToGivenSolidFraction")

    def takeTimeStep(self):
        return self._check(self._call(TAKE_STEP), "takeTimeStep")

    def run(self, nsteps, control=None):
        ctl = control if control is not None else make_control()
        done = C.c_int32(0)
        self._check(self._run(nsteps, ctl, done), "run")
        return done.value

    # ---- getters -----------------------------------------------------------
    def getBoundary(self):
        b = np.zeros(4)
        self._boundary(b.ctypes.data_as(C.POINTER(C.c_double)))
        return b

    def getStress(self):
        s = np.zeros(4)
        self._stress(s.ctypes.data_as(C.POINTER(C.c_double)))
        return s

    def getLeesEdwards(self):
        s = np.zeros(4)
        self._le(s.ctypes.data_as(C.POINTER(C.c_double)))
        return s

    def setLeesEdwards(self, vals):
        s = np.ascontiguousarray(vals, np.float64)
        self._set_le(s.ctypes.data_as(C.POINTER(C.c_double)))

    def getKineticEnergy(self):
        return self._ke()

    def countActucalContacts(self):
        return self.count_contacts()


class World(WorldBase):
    """A world on the GPU (the product path)."""

    def __init__(self, params):
        self.lib = abi.load_library()
        self.params = params
        self.h = C.c_void_p()
        st = self.lib.xdem_create(C.byref(params), C.byref(self.h))
        if st:
            raise abi.XdemError(st, "xdem_create")
        self.n = 0

    def close(self):
        if self.h:
            self.lib.xdem_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _set_particles(self, s):
        return self.lib.xdem_set_particles(self.h, C.byref(s))

    # ---- batched systems (one handle, many independent systems) ------------
    def set_batch(self, systems, boxes, dts=None):
        """Places the systems (particle dicts with local ids) side by side in
        this world: system s takes the ids first_s + id (xdem_batch_set_particles)."""
        nsys = len(systems)
        arr = (abi.Particles * nsys)()
        for k, p in enumerate(systems):
            arr[k] = abi.particles_struct(p)
        self._batch_keep = (systems, arr)
        boxes = np.ascontiguousarray(np.asarray(boxes, np.float64).reshape(nsys, 4))
        d = C.POINTER(C.c_double)
        dts_p = None
        if dts is not None:
            dts = np.ascontiguousarray(np.asarray(dts, np.float64))
            dts_p = dts.ctypes.data_as(d)
        self.n = int(sum(len(p["x"]) for p in systems))
        self._check(self.lib.xdem_batch_set_particles(self.h, nsys, arr, boxes.ctypes.data_as(d),
                                                      dts_p), "batch_set_particles")

    def save_snapshot(self, path):
        """Writes the whole world (particles, contact history, scalars) to a
        binary file."""
        self._check(self.lib.xdem_save_snapshot(self.h, str(path).encode()), "save_snapshot")

    def load_snapshot(self, path):
        """Replaces this world's state with a saved one (same world kind)."""
        self._check(self.lib.xdem_load_snapshot(self.h, str(path).encode()), "load_snapshot")
        k, first = self.batch_info()
        self.n = int(first[-1])

    def quadron_z_phi(self):
        """Rattler-free (Z, solid fraction) as QuadronAnalysis computes them."""
        out = np.zeros(2)
        self._check(self.lib.xdem_quadron_z_phi(self.h, out.ctypes.data_as(C.POINTER(C.c_double))),
                    "quadron_z_phi")
        return out

    def batch_quadron_z_phi(self):
        k, _ = self.batch_info()
        out = np.zeros((k, 2))
        self._check(self.lib.xdem_batch_quadron_z_phi(
            self.h, out.ctypes.data_as(C.POINTER(C.c_double))), "batch_quadron_z_phi")
        return out

    def batch_info(self):
        """(number of systems, first id of each system followed by n)"""
        k = C.c_int32(0)
        self._check(self.lib.xdem_batch_info(self.h, C.byref(k), None), "batch_info")
        first = np.zeros(k.value + 1, np.int32)
        self._check(self.lib.xdem_batch_info(self.h, C.byref(k),
                                             first.ctypes.data_as(C.POINTER(C.c_int32))), "batch_info")
        return k.value, first

    def batch_stress(self):
        k, _ = self.batch_info()
        out = np.zeros((k, 4))
        self._check(self.lib.xdem_batch_get_stress(self.h, out.ctypes.data_as(C.POINTER(C.c_double))),
                    "batch_get_stress")
        return out

    def batch_boundaries(self):
        k, _ = self.batch_info()
        out = np.zeros((k, 4))
        self._check(self.lib.xdem_batch_get_boundaries(
            self.h, out.ctypes.data_as(C.POINTER(C.c_double))), "batch_get_boundaries")
        return out

    def batch_count_contacts(self):
        k, _ = self.batch_info()
        out = np.zeros(k, np.int64)
        self._check(self.lib.xdem_batch_count_contacts(
            self.h, out.ctypes.data_as(C.POINTER(C.c_int64))), "batch_count_contacts")
        return out

    def _get_state(self, s):
        return self.lib.xdem_get_particles(self.h, C.byref(s))

    def _set_contacts(self, s):
        return self.lib.xdem_set_contacts(self.h, C.byref(s))

    def _get_contacts(self, s):
        return self.lib.xdem_get_contacts(self.h, C.byref(s))

    def _forces(self, fx, fy, t, nc):
        return self.lib.xdem_get_force_and_torque(self.h, fx, fy, t, nc)

    def count_contacts(self):
        v = C.c_int64(0)
        self._check(self.lib.xdem_count_contacts(self.h, C.byref(v)), "count_contacts")
        return int(v.value)

    def _call(self, which, a=0.0, b=0.0, c=0.0):
        L, h = self.lib, self.h
        if which == MODIFY:
            return L.xdem_modify_particle_position(h)
        if which == APPLY_BG:
            return L.xdem_apply_background_velocity(h)
        if which == REMOVE_BG:
            return L.xdem_remove_background_velocity(h)
        if which == FIND:
            return L.xdem_find_possible_contacts(h)
        if which == UPDATE:
            return L.xdem_update_contacts(h)
        if which == COLLECT:
            return L.xdem_collect_force_and_torque(h)
        if which == INTEGRATE:
            return L.xdem_take_time_integral(h)
        if which == RESET_RATTLERS:
            return L.xdem_reset_velocity_of_rattlers(h)
        if which == SCALE_RATTLERS:
            return L.xdem_scale_velocity_of_rattlers(h, a)
        if which == STRESS:
            return L.xdem_update_total_stress(h, None)
        if which == BOX_LAW:
            return L.xdem_update_boundary(h, int(a), b, c)
        if which == LE_BOUNDARY:
            return L.xdem_update_lees_edwards_boundary(h)
        if which == TAKE_STEP:
            return L.xdem_take_time_step(h)
        if which == SCALE_TO_FRACTION:
            return L.xdem_scale_boundary_to_solid_fraction(h, a)
        return abi.ERR_ARGUMENT

    def _run(self, nsteps, ctl, done):
        return self.lib.xdem_run(self.h, nsteps, C.byref(ctl), C.byref(done))

    def _boundary(self, p):
        return self.lib.xdem_get_boundary(self.h, p)

    def _stress(self, p):
        return self.lib.xdem_get_stress(self.h, p)

    def _le(self, p):
        return self.lib.xdem_get_lees_edwards(self.h, p)

    def _set_le(self, p):
        return self.lib.xdem_set_lees_edwards(self.h, p)

    def _ke(self):
        v = C.c_double(0.0)
        self._check(self.lib.xdem_get_kinetic_energy(self.h, C.byref(v)), "getKineticEnergy")
        return v.value

    def setVirtualBoundaryMass(self, mass=-1.0):
        self._check(self.lib.xdem_set_virtual_boundary_mass(self.h, mass), "setVirtualBoundaryMass")

    def setMaxStrainRate(self, rate):
        self._check(self.lib.xdem_set_max_strain_rate(self.h, rate), "setMaxStrainRate")

    def setShiftStrainRate(self, rate):
        self._check(self.lib.xdem_set_shift_strain_rate(self.h, rate), "setShiftStrainRate")

    def setContactModel(self, kn, kt, restitution, friction):
        self._check(self.lib.xdem_set_contact_model(self.h, kn, kt, restitution, friction),
                    "setContactModel")

    def setGlobalDamping(self, g):
        self._check(self.lib.xdem_set_global_damping(self.h, g), "setGlobalDamping")

    def synchronize(self):
        return self.lib.xdem_synchronize(self.h)

    # ---- per-step state exchange and timing ---------------------------------
    def upload_state(self, x, y, vx, vy, rot, rot_vel):
        d = C.POINTER(C.c_double)
        return self._check(self.lib.xdem_upload_state(
            self.h, *[C.cast(a, d) if isinstance(a, int) else a.ctypes.data_as(d)
                      for a in (x, y, vx, vy, rot, rot_vel)]), "upload_state")

    def download_state(self, x, y, vx, vy, rot, rot_vel):
        d = C.POINTER(C.c_double)
        return self._check(self.lib.xdem_download_state(
            self.h, *[C.cast(a, d) if isinstance(a, int) else a.ctypes.data_as(d)
                      for a in (x, y, vx, vy, rot, rot_vel)]), "download_state")

    def set_profiling(self, on):
        self._check(self.lib.xdem_set_profiling(self.h, 1 if on else 0), "set_profiling")

    def profile(self):
        k = self.lib.xdem_profile_kinds()
        launches = (C.c_int64 * k)()
        ms = (C.c_double * k)()
        self._check(self.lib.xdem_get_profile(self.h, k, launches, ms), "get_profile")
        return {self.lib.xdem_profile_name(i).decode(): (int(launches[i]), float(ms[i]))
                for i in range(k) if launches[i]}

    def newton_stats(self):
        """(solves, iterations, capped solves) of the closest-approach Newton
        iteration since creation or the last reset."""
        out = (C.c_int64 * 3)()
        self._check(self.lib.xdem_get_newton_stats(self.h, out), "newton_stats")
        return int(out[0]), int(out[1]), int(out[2])

    def set_launch_config(self, pair_blocks_per_sm, cell_factor):
        self._check(self.lib.xdem_set_launch_config(self.h, pair_blocks_per_sm, cell_factor),
                    "set_launch_config")

    def set_candidate_lists(self, capacity, skin_fraction=0.1):
        """Before set_particles: partners kept per particle (0 = full 3x3 scan
        every step) and the skin as a fraction of the cell size."""
        self._check(self.lib.xdem_set_candidate_lists(self.h, capacity, skin_fraction),
                    "set_candidate_lists")

    def set_memory_order_refresh(self, interval):
        """Steps between re-sorts of the device memory order (odd; 0 = never)."""
        self._check(self.lib.xdem_set_memory_order_refresh(self.h, interval),
                    "set_memory_order_refresh")

    def candidate_list_stats(self):
        """{builds, longest, entries, capacity} of the candidate lists"""
        out = (C.c_int64 * 4)()
        self._check(self.lib.xdem_get_candidate_list_stats(self.h, out), "candidate_list_stats")
        return dict(zip(("builds", "longest", "entries", "capacity"), (int(v) for v in out)))

    def launch_config(self):
        b = C.c_int32(0)
        f = C.c_double(0.0)
        self._check(self.lib.xdem_get_launch_config(self.h, C.byref(b), C.byref(f)), "launch_config")
        return int(b.value), float(f.value)

    def autotune(self, control=None, steps_per_trial=20):
        """Picks the fastest launch configuration by timing real steps (the
        world advances 12 * (steps_per_trial + 1) steps); returns
        (blocks per SM, cell factor, 12 trial times in ms)."""
        ctl = control if control is not None else make_control()
        ms = (C.c_double * 12)()
        self._check(self.lib.xdem_autotune(self.h, C.byref(ctl), steps_per_trial, ms), "autotune")
        b, f = self.launch_config()
        return b, f, [float(v) for v in ms]

    def pair_count(self):
        """Pairs that passed the last candidate scan (geometry evaluated)."""
        v = C.c_int64(0)
        self._check(self.lib.xdem_get_pair_count(self.h, C.byref(v)), "pair_count")
        return int(v.value)

    def reset_newton_stats(self):
        self._check(self.lib.xdem_reset_newton_stats(self.h), "reset_newton_stats")

    def launch_count(self):
        v = C.c_int64(0)
        self._check(self.lib.xdem_launch_count(self.h, C.byref(v)), "launch_count")
        return int(v.value)


def pair_geometry(pi, pj, off, method=abi.ELLIPSE_CLOSEST_APPROACH, precision=abi.PRECISION_FP64):
    """Contact geometry of npairs pairs on the GPU (rows as xdem_pair_geometry)."""
    lib = abi.load_library()
    pi = np.ascontiguousarray(pi, np.float64)
    pj = np.ascontiguousarray(pj, np.float64)
    off = np.ascontiguousarray(off, np.float64)
    npairs = pi.shape[0]
    out = np.zeros((npairs, 17))
    d = C.POINTER(C.c_double)
    st = lib.xdem_pair_geometry(npairs, method, precision, pi.ctypes.data_as(d), pj.ctypes.data_as(d),
                                off.ctypes.data_as(d), out.ctypes.data_as(d))
    return out, st
