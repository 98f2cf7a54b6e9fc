"""ctypes mirror of include/xdem_gpu.h.

The structs here are shared by the CUDA library's wrapper (xdem_b200.world)
and by the CPU checkers under oracle/, which use the same argument structs.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libxdem_b200.so")

# status bits (enum xdem_status_bits)
OK = 0
ERR_CAPACITY = 1 << 0
ERR_NEWTON = 1 << 1
ERR_NONFINITE = 1 << 2
ERR_UNSUPPORTED_PAIR = 1 << 3
ERR_ZERO_VECTOR = 1 << 4
ERR_CUDA = 1 << 5
ERR_ARGUMENT = 1 << 6
ERR_GRID = 1 << 7
ERR_TIMEOUT = 1 << 8
STATUS_NAMES = {
    ERR_CAPACITY: "CAPACITY", ERR_NEWTON: "NEWTON", ERR_NONFINITE: "NONFINITE",
    ERR_UNSUPPORTED_PAIR: "UNSUPPORTED_PAIR", ERR_ZERO_VECTOR: "ZERO_VECTOR",
    ERR_CUDA: "CUDA", ERR_ARGUMENT: "ARGUMENT", ERR_GRID: "GRID", ERR_TIMEOUT: "TIMEOUT",
}

WORLD_PERIODIC, WORLD_PERIODIC_CONTROL, WORLD_LEES_EDWARDS = 0, 1, 2
SHAPE_CIRCLE, SHAPE_ELLIPSE, SHAPE_CLUMP, SHAPE_SEGMENT = 0, 1, 2, 3
SKIP_TIME_INTEGRAL, SKIP_CONTACT_DETECTION, SKIP_MACRO_SUM = 1, 2, 4
ELLIPSE_CLOSEST_APPROACH, ELLIPSE_INTERSECTION = 0, 1
PRECISION_FP64, PRECISION_MIXED = 0, 1
BOX_NONE, BOX_STRAIN, BOX_STRESS_XY, BOX_STRESS_UNIFORM, BOX_STRESS_UNIFORM_LIMIT = 0, 1, 2, 3, 4
SEQ_TAKE_TIME_STEP, SEQ_SUBSTEPS = 0, 1


def status_text(st):
    if st == 0:
        return "OK"
    return "|".join(name for bit, name in STATUS_NAMES.items() if st & bit)


class XdemError(RuntimeError):
    def __init__(self, status, where=""):
        self.status = status
        super().__init__(f"{where}: status {status} ({status_text(status)})")


_d = C.POINTER(C.c_double)
_i = C.POINTER(C.c_int32)
_f = C.POINTER(C.c_float)


class Params(C.Structure):
    _fields_ = [
        ("world_kind", C.c_int32), ("ellipse_method", C.c_int32), ("precision", C.c_int32),
        ("max_contacts", C.c_int32), ("dt", C.c_double),
        ("xmin", C.c_double), ("xmax", C.c_double), ("ymin", C.c_double), ("ymax", C.c_double),
        ("normal_stiffness", C.c_double), ("shear_stiffness", C.c_double),
        ("restitution_coeff", C.c_double), ("frictional_coeff", C.c_double),
        ("global_damping", C.c_double), ("shift_strain_rate", C.c_double),
        ("max_particle_size", C.c_double),
    ]


class Control(C.Structure):
    _fields_ = [
        ("sequence", C.c_int32), ("scale_rattlers", C.c_int32), ("reset_rattlers", C.c_int32),
        ("update_stress", C.c_int32), ("box_law", C.c_int32), ("stop_on_pressure", C.c_int32),
        ("rattler_scale", C.c_double), ("p0", C.c_double), ("p1", C.c_double),
        ("stop_pressure", C.c_double),
    ]


PARTICLE_INT_FIELDS = ("shape", "up_level", "setting", "is_rattler")
PARTICLE_DOUBLE_FIELDS = ("outer_radius", "radius", "aspect_ratio", "x", "y", "vx", "vy", "rot",
                          "rot_vel", "volume", "mass", "inv_mass", "inertia", "inv_inertia")


SEGMENT_FIELDS = ("seg_x1", "seg_y1", "seg_x2", "seg_y2")


class Particles(C.Structure):
    _fields_ = ([("n", C.c_int32)] + [(f, _i) for f in PARTICLE_INT_FIELDS]
                + [(f, _d) for f in PARTICLE_DOUBLE_FIELDS]
                + [("num_sub", _i), ("branch_x", _d), ("branch_y", _d)]
                + [(f, _d) for f in SEGMENT_FIELDS])


CONTACT_DOUBLE_FIELDS = ("normal_x", "normal_y", "point_x", "point_y", "branch_x", "branch_y",
                         "bv1_x", "bv1_y", "bv2_x", "bv2_y", "shear_x", "shear_y",
                         "fn_x", "fn_y", "ft_x", "ft_y", "torque_i", "torque_j", "damping")


class Contacts(C.Structure):
    _fields_ = ([("count", C.c_int64), ("capacity", C.c_int64), ("id_i", _i), ("id_j", _i)]
                + [(f, _d) for f in CONTACT_DOUBLE_FIELDS])


def _ptr(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


def particles_struct(p):
    """Particles struct over a dict of numpy arrays (kept alive by the caller).
    Optional keys: is_rattler, num_sub, branch_x, branch_y, seg_x1, seg_y1,
    seg_x2, seg_y2."""
    s = Particles()
    n = len(p["x"])
    s.n = n
    for f in PARTICLE_INT_FIELDS:
        if f in p and p[f] is not None:
            assert p[f].dtype == np.int32 and p[f].flags.c_contiguous and len(p[f]) == n, f
            setattr(s, f, _ptr(p[f], C.c_int32))
    for f in PARTICLE_DOUBLE_FIELDS:
        if f in p and p[f] is not None:
            assert p[f].dtype == np.float64 and p[f].flags.c_contiguous and len(p[f]) == n, f
            setattr(s, f, _ptr(p[f], C.c_double))
    for f, ct in (("num_sub", C.c_int32), ("branch_x", C.c_double), ("branch_y", C.c_double)):
        if f in p and p[f] is not None:
            setattr(s, f, _ptr(p[f], ct))
    for f in SEGMENT_FIELDS:
        if f in p and p[f] is not None:
            assert p[f].dtype == np.float64 and p[f].flags.c_contiguous and len(p[f]) == n, f
            setattr(s, f, _ptr(p[f], C.c_double))
    return s


def empty_state(n):
    """Arrays for a particle download."""
    out = {f: np.zeros(n, np.float64) for f in ("x", "y", "vx", "vy", "rot", "rot_vel",
                                                 "branch_x", "branch_y")}
    out["is_rattler"] = np.zeros(n, np.int32)
    return out


def state_struct(out):
    s = Particles()
    s.n = len(out["x"])
    for f in ("x", "y", "vx", "vy", "rot", "rot_vel", "branch_x", "branch_y"):
        setattr(s, f, _ptr(out[f], C.c_double))
    s.is_rattler = _ptr(out["is_rattler"], C.c_int32)
    return s


def contact_arrays(cap):
    out = {"id_i": np.zeros(cap, np.int32), "id_j": np.zeros(cap, np.int32)}
    for f in CONTACT_DOUBLE_FIELDS:
        out[f] = np.zeros(cap, np.float64)
    return out


def contacts_struct(arrs, count=None):
    s = Contacts()
    cap = len(arrs["id_i"])
    s.capacity = cap
    s.count = cap if count is None else count
    s.id_i = _ptr(arrs["id_i"], C.c_int32)
    s.id_j = _ptr(arrs["id_j"], C.c_int32)
    for f in CONTACT_DOUBLE_FIELDS:
        setattr(s, f, _ptr(arrs[f], C.c_double))
    return s


def trim_contacts(arrs, count):
    return {k: v[:count].copy() for k, v in arrs.items()}


_lib = None


def load_library(path=LIB_PATH):
    """Loads the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(
            f"{path} is missing: build it with `python -m xdem_b200.build` or "
            "`python -c 'import __graft_entry__ as g; g.build()'`")
    lib = C.CDLL(path)
    P = C.POINTER
    W = C.c_void_p
    sig = {
        "xdem_abi_version": (C.c_int32, []),
        "xdem_status_string": (C.c_char_p, [C.c_int32]),
        "xdem_device_count": (C.c_int32, [P(C.c_int32)]),
        "xdem_create": (C.c_int32, [P(Params), P(W)]),
        "xdem_destroy": (C.c_int32, [W]),
        "xdem_set_stream": (C.c_int32, [W, C.c_void_p]),
        "xdem_get_stream": (C.c_int32, [W, P(C.c_void_p)]),
        "xdem_set_particles": (C.c_int32, [W, P(Particles)]),
        "xdem_batch_set_particles": (C.c_int32, [W, C.c_int32, P(Particles), _d, _d]),
        "xdem_quadron_z_phi": (C.c_int32, [W, _d]),
        "xdem_save_snapshot": (C.c_int32, [W, C.c_char_p]),
        "xdem_load_snapshot": (C.c_int32, [W, C.c_char_p]),
        "xdem_batch_quadron_z_phi": (C.c_int32, [W, _d]),
        "xdem_batch_info": (C.c_int32, [W, P(C.c_int32), P(C.c_int32)]),
        "xdem_batch_get_stress": (C.c_int32, [W, _d]),
        "xdem_batch_get_boundaries": (C.c_int32, [W, _d]),
        "xdem_batch_count_contacts": (C.c_int32, [W, P(C.c_int64)]),
        "xdem_get_particles": (C.c_int32, [W, P(Particles)]),
        "xdem_set_contacts": (C.c_int32, [W, P(Contacts)]),
        "xdem_get_contacts": (C.c_int32, [W, P(Contacts)]),
        "xdem_get_force_and_torque": (C.c_int32, [W, _d, _d, _d, _i]),
        "xdem_count_contacts": (C.c_int32, [W, P(C.c_int64)]),
        "xdem_get_boundary": (C.c_int32, [W, _d]),
        "xdem_set_boundary": (C.c_int32, [W, _d]),
        "xdem_get_stress": (C.c_int32, [W, _d]),
        "xdem_get_lees_edwards": (C.c_int32, [W, _d]),
        "xdem_set_lees_edwards": (C.c_int32, [W, _d]),
        "xdem_set_shift_strain_rate": (C.c_int32, [W, C.c_double]),
        "xdem_set_time_increment": (C.c_int32, [W, C.c_double]),
        "xdem_set_global_damping": (C.c_int32, [W, C.c_double]),
        "xdem_set_contact_model": (C.c_int32, [W, C.c_double, C.c_double, C.c_double, C.c_double]),
        "xdem_set_virtual_boundary_mass": (C.c_int32, [W, C.c_double]),
        "xdem_set_max_strain_rate": (C.c_int32, [W, C.c_double]),
        "xdem_get_kinetic_energy": (C.c_int32, [W, _d]),
        "xdem_get_newton_stats": (C.c_int32, [W, P(C.c_int64)]),
        "xdem_reset_newton_stats": (C.c_int32, [W]),
        "xdem_get_pair_count": (C.c_int32, [W, P(C.c_int64)]),
        "xdem_modify_particle_position": (C.c_int32, [W]),
        "xdem_apply_background_velocity": (C.c_int32, [W]),
        "xdem_remove_background_velocity": (C.c_int32, [W]),
        "xdem_find_possible_contacts": (C.c_int32, [W]),
        "xdem_update_contacts": (C.c_int32, [W]),
        "xdem_collect_force_and_torque": (C.c_int32, [W]),
        "xdem_take_time_integral": (C.c_int32, [W]),
        "xdem_reset_velocity_of_rattlers": (C.c_int32, [W]),
        "xdem_scale_velocity_of_rattlers": (C.c_int32, [W, C.c_double]),
        "xdem_update_total_stress": (C.c_int32, [W, _d]),
        "xdem_update_boundary": (C.c_int32, [W, C.c_int32, C.c_double, C.c_double]),
        "xdem_update_lees_edwards_boundary": (C.c_int32, [W]),
        "xdem_scale_boundary_to_solid_fraction": (C.c_int32, [W, C.c_double]),
        "xdem_take_time_step": (C.c_int32, [W]),
        "xdem_run": (C.c_int32, [W, C.c_int32, P(Control), P(C.c_int32)]),
        "xdem_synchronize": (C.c_int32, [W]),
        "xdem_upload_state": (C.c_int32, [W, _d, _d, _d, _d, _d, _d]),
        "xdem_download_state": (C.c_int32, [W, _d, _d, _d, _d, _d, _d]),
        "xdem_set_profiling": (C.c_int32, [W, C.c_int32]),
        "xdem_profile_kinds": (C.c_int32, []),
        "xdem_profile_name": (C.c_char_p, [C.c_int32]),
        "xdem_get_profile": (C.c_int32, [W, C.c_int32, P(C.c_int64), _d]),
        "xdem_launch_count": (C.c_int32, [W, P(C.c_int64)]),
        "xdem_timer_start": (C.c_int32, [W]),
        "xdem_timer_stop": (C.c_int32, [W, _d]),
        "xdem_total_stress_noalloc": (C.c_int32, [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                                                  C.c_void_p, C.c_double, C.c_void_p, C.c_void_p]),
        "xdem_total_stress_noalloc_max_contacts": (C.c_int64, []),
        "xdem_host_alloc": (C.c_void_p, [C.c_int64]),
        "xdem_range_push": (C.c_int32, [C.c_char_p]),
        "xdem_set_launch_config": (C.c_int32, [W, C.c_int32, C.c_double]),
        "xdem_set_candidate_lists": (C.c_int32, [W, C.c_int32, C.c_double]),
        "xdem_get_candidate_list_stats": (C.c_int32, [W, P(C.c_int64)]),
        "xdem_set_memory_order_refresh": (C.c_int32, [W, C.c_int32]),
        "xdem_snapshot_info": (C.c_int32, [C.c_char_p, P(C.c_int64)]),
        "xdem_snapshot_layout": (C.c_int32, [P(C.c_int64)]),
        "xdem_get_launch_config": (C.c_int32, [W, P(C.c_int32), P(C.c_double)]),
        "xdem_autotune": (C.c_int32, [W, P(Control), C.c_int32, _d]),
        "xdem_mlp_create": (C.c_int32, [C.c_uint64, P(W)]),
        "xdem_mlp_destroy": (C.c_int32, [W]),
        "xdem_mlp_param_count": (C.c_int32, []),
        "xdem_mlp_get_params": (C.c_int32, [W, _f, _f]),
        "xdem_mlp_set_params": (C.c_int32, [W, _f, _f]),
        "xdem_mlp_forward": (C.c_int32, [W, C.c_int64, _f, _f]),
        "xdem_selftest_bounded_wait": (C.c_int32, [_d]),
        "xdem_mlp_gradient": (C.c_int32, [W, C.c_int64, _f, _f, _f, _f, _f]),
        "xdem_mlp_add_samples": (C.c_int32, [W, C.c_int64, _f, _f, _f]),
        "xdem_mlp_dataset": (C.c_int32, [W, P(C.c_int64), _f, _f, _f]),
        "xdem_mlp_clear_dataset": (C.c_int32, [W]),
        "xdem_mlp_train": (C.c_int32, [W, C.c_int32, C.c_int32, C.c_float, C.c_uint64, C.c_int64, _f]),
        "xdem_harvest_pairs": (C.c_int32, [W, W, C.c_int32, C.c_int64, P(C.c_int64)]),
        "xdem_set_warm_start": (C.c_int32, [W, W]),
        "xdem_get_warm_stats": (C.c_int32, [W, P(C.c_int64)]),
        "xdem_range_pop": (C.c_int32, []),
        "xdem_host_free": (None, [C.c_void_p]),
        "xdem_pair_geometry": (C.c_int32, [C.c_int32, C.c_int32, C.c_int32, _d, _d, _d, _d]),
        "xdem_rsa_positions": (C.c_int32, [C.c_int32, _d, _d, C.c_uint64, C.c_int64, _d, _d]),
        "xdem_particle_properties": (C.c_int32, [C.c_int32, _i, _d, _d, C.c_double, _d, _d, _d,
                                                 _d, _d]),
        "xdem_clump_properties": (C.c_int32, [C.c_int32, _i, _d, _d, _d, _d, _d, C.c_double, _d,
                                              _d, _d]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def exported_symbols():
    """Names of the C-ABI functions declared in include/xdem_gpu.h."""
    import re
    hdr = os.path.join(os.path.dirname(HERE), "include", "xdem_gpu.h")
    text = open(hdr).read()
    return sorted(set(re.findall(r"\b(xdem_[a-z0-9_]+)\s*\(", text)))
