"""ctypes binding of the C ABI in include/pmpm.h (libpmpm_b200.so).

This is the thin Python view of the native library used by the tests, the
benchmark and the autograd wrapper; the reference-shaped Python API lives in
the MPM2D / MPM3D extension modules.  Loading fails loudly when the library
has not been built: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import math
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpmpm_b200.so")

MAX_MATERIALS = 16
MAX_BCS = 16

SHAPE = {"linear": 0, "quadratic": 1, "cubic": 2}
MAT_NONE, MAT_LINEAR_ELASTIC, MAT_NEWTON_FLUID, MAT_DRUCKER_PRAGER = 0, 1, 2, 3
BC_GRAVITY, BC_NODEDOMAIN, BC_BODYFORCE, BC_PLANARDOMAIN = 1, 2, 3, 4
FLAG_KEEP_VELOCITY_GRADIENT = 1
FLAG_DETERMINISTIC = 2
FLAG_MUSL = 4

STATUS = {
    0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "out of device memory", 4: "not supported",
    5: "call out of order", 16: "a particle left the background grid", 17: "non-finite particle position",
    18: "too many particles in one cell", 19: "a bounded wait inside a kernel ran out",
}

FIELDS = {
    "positions": 0, "velocities": 1, "stresses": 2, "F": 3, "velocity_gradient": 4, "masses": 5,
    "volumes": 6, "volumes_original": 7, "colors": 8, "is_rigid": 9, "is_active": 10,
    "forces_external": 11, "eps_e": 12, "stress_ref": 13, "youngs_modulus": 14, "friction_angle": 15,
    "acc_eps_p": 16, "alpha": 16, "pc": 17,
    "node_masses": 20, "node_moments": 21, "node_moments_nt": 22, "node_ids": 23, "node_types": 24,
    "bins": 30, "hash_unsorted": 31, "hash_sorted": 32, "sorted_index": 33, "cell_start": 34, "cell_end": 35,
}
_U8 = {"colors", "is_rigid", "is_active"}
_I32 = {"node_ids", "node_types", "bins", "sorted_index", "cell_start", "cell_end"}
_U32 = {"hash_unsorted", "hash_sorted"}


class PmpmError(RuntimeError):
    def __init__(self, status, what=""):
        self.status = status
        super().__init__(f"{what}: {STATUS.get(status, 'status %d' % status)} ({status})")


class Material(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int), ("density", ctypes.c_float), ("params", ctypes.c_float * 12)]


class BC(ctypes.Structure):
    _fields_ = [("type", ctypes.c_int), ("ints", ctypes.c_int * 8), ("reals", ctypes.c_float * 16),
                ("values", ctypes.c_void_p), ("mask", ctypes.c_void_p)]


class Desc(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int), ("origin", ctypes.c_float * 3), ("end", ctypes.c_float * 3),
                ("cell_size", ctypes.c_float), ("shape_function", ctypes.c_int), ("dt", ctypes.c_float),
                ("particles_per_cell", ctypes.c_int), ("alpha", ctypes.c_float),
                ("num_materials", ctypes.c_int), ("materials", ctypes.POINTER(Material)),
                ("num_bcs", ctypes.c_int), ("bcs", ctypes.POINTER(BC)), ("flags", ctypes.c_uint),
                ("device", ctypes.c_int), ("stream", ctypes.c_void_p), ("resort_interval", ctypes.c_int)]


class Instance(ctypes.Structure):
    _fields_ = [("desc", ctypes.POINTER(Desc)), ("num_particles", ctypes.c_int), ("positions", ctypes.c_void_p),
                ("velocities", ctypes.c_void_p), ("colors", ctypes.c_void_p)]


EXPORTS = [
    "pmpm_status_string", "pmpm_material_linear_elastic", "pmpm_material_newton_fluid",
    "pmpm_material_drucker_prager", "pmpm_material_dp_rheo", "pmpm_bc_gravity", "pmpm_bc_nodedomain",
    "pmpm_bc_bodyforce", "pmpm_bc_planardomain", "pmpm_create", "pmpm_destroy", "pmpm_get_grid",
    "pmpm_set_particles", "pmpm_initialize", "pmpm_get_field", "pmpm_set_field", "pmpm_num_particles",
    "pmpm_num_nodes", "pmpm_field_bytes", "pmpm_partition", "pmpm_shape_functions",
    "pmpm_num_surround_nodes", "pmpm_p2g", "pmpm_g2p", "pmpm_stress_update", "pmpm_solve",
    "pmpm_get_step", "pmpm_set_step", "pmpm_synchronize", "pmpm_stream", "pmpm_material_point_update",
    "pmpm_profile_step", "pmpm_active_nodes", "pmpm_launch_count", "pmpm_partition_noalloc",
    "pmpm_bc_rigidbodylevelset", "pmpm_bc_rigid_sdf", "pmpm_calculate_timestep", "pmpm_material_timestep",
    "pmpm_rollout_forward", "pmpm_rollout_reset", "pmpm_rollout_backward", "pmpm_material_point_vjp",
    "pmpm_rollout_set_memory", "pmpm_musl_stage", "pmpm_material_von_mises", "pmpm_autotune",
    "pmpm_material_modified_cam_clay", "pmpm_material_drucker_prager_cap", "pmpm_set_p2g_kernel",
    "pmpm_set_wait_limit", "pmpm_scan_tag", "pmpm_pick_resort_interval", "pmpm_set_p2g_staging", "pmpm_set_resort_interval", "pmpm_get_tuning",
]

EXPORTS += [
    "pmpm_batch_create", "pmpm_batch_destroy", "pmpm_batch_initialize", "pmpm_batch_solve",
    "pmpm_batch_num_instances", "pmpm_batch_num_particles", "pmpm_batch_get_field", "pmpm_batch_set_field",
    "pmpm_batch_synchronize", "pmpm_batch_profile_step", "pmpm_batch_launch_count",
    "pmpm_batch_set_wait_limit",
]

RIGID_MODES = {"static": 0, "loop_rotate": 1}
SDF_SHAPES = {"sphere": 0, "half_cylinder_shell": 1}

_lib = None


def lib():
    """Load libpmpm_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with __graft_entry__.build() "
                          "(python -c 'import __graft_entry__ as g; g.build()')")
    L = ctypes.CDLL(LIB_PATH)
    vp, i, f, sz = ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_size_t
    fp = ctypes.POINTER(ctypes.c_float)
    L.pmpm_status_string.restype = ctypes.c_char_p
    L.pmpm_status_string.argtypes = [i]
    L.pmpm_material_linear_elastic.argtypes = [f, f, f, i, ctypes.POINTER(Material)]
    L.pmpm_material_newton_fluid.argtypes = [f, f, f, f, ctypes.POINTER(Material)]
    L.pmpm_material_drucker_prager.argtypes = [f, f, f, f, f, f, ctypes.POINTER(Material)]
    L.pmpm_material_dp_rheo.argtypes = [f, f, f, f, f, f, ctypes.POINTER(Material)]
    L.pmpm_bc_gravity.argtypes = [fp, i, i, fp, i, ctypes.POINTER(BC)]
    L.pmpm_bc_nodedomain.argtypes = [ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int), i,
                                     ctypes.POINTER(BC)]
    L.pmpm_bc_bodyforce.argtypes = [i, fp, ctypes.POINTER(ctypes.c_ubyte), ctypes.POINTER(BC)]
    L.pmpm_bc_planardomain.argtypes = [fp, fp, i, ctypes.POINTER(BC)]
    L.pmpm_bc_rigidbodylevelset.argtypes = [i, fp, fp, i, i, ctypes.POINTER(BC)]
    L.pmpm_bc_rigid_sdf.argtypes = [i, i, fp, fp, f, f, fp, f, f, i, ctypes.POINTER(BC)]
    L.pmpm_calculate_timestep.argtypes = [f, f, f, f, f, fp]
    L.pmpm_rollout_forward.argtypes = [vp, i, i]
    L.pmpm_rollout_set_memory.argtypes = [vp, ctypes.c_longlong]
    L.pmpm_musl_stage.argtypes = [vp, i]
    L.pmpm_autotune.argtypes = [vp, i, ctypes.POINTER(ctypes.c_int)]
    L.pmpm_set_p2g_kernel.argtypes = [vp, i]
    L.pmpm_material_von_mises.argtypes = [f, f, f, f, f, ctypes.POINTER(Material)]
    L.pmpm_material_modified_cam_clay.argtypes = [f] * 10 + [ctypes.POINTER(Material)]
    L.pmpm_material_drucker_prager_cap.argtypes = [f] * 11 + [ctypes.POINTER(Material)]
    L.pmpm_material_point_vjp.argtypes = [ctypes.POINTER(Material), i, i, f] + [vp] * 11 + [i, i]
    L.pmpm_rollout_reset.argtypes = [vp]
    L.pmpm_rollout_backward.argtypes = [vp, vp, i, vp, vp, vp, vp]
    L.pmpm_batch_create.argtypes = [i, ctypes.POINTER(Instance), i, vp, i, ctypes.POINTER(vp)]
    L.pmpm_batch_destroy.argtypes = [vp]
    L.pmpm_batch_initialize.argtypes = [vp]
    L.pmpm_batch_solve.argtypes = [vp, i]
    L.pmpm_batch_num_instances.argtypes = [vp]
    L.pmpm_batch_num_particles.argtypes = [vp, i]
    L.pmpm_batch_get_field.argtypes = [vp, i, i, vp, sz, i]
    L.pmpm_batch_set_field.argtypes = [vp, i, i, vp, sz, i]
    L.pmpm_batch_synchronize.argtypes = [vp]
    L.pmpm_batch_profile_step.argtypes = [vp, fp, ctypes.POINTER(ctypes.c_int)]
    L.pmpm_batch_launch_count.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
    L.pmpm_material_timestep.argtypes = [ctypes.POINTER(Material), f, f, fp]
    L.pmpm_create.argtypes = [ctypes.POINTER(Desc), ctypes.POINTER(vp)]
    L.pmpm_destroy.argtypes = [vp]
    L.pmpm_get_grid.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int), fp]
    L.pmpm_set_particles.argtypes = [vp, i, vp, vp, vp, i, vp, vp, vp]
    L.pmpm_initialize.argtypes = [vp]
    L.pmpm_get_field.argtypes = [vp, i, vp, sz, i]
    L.pmpm_set_field.argtypes = [vp, i, vp, sz, i]
    L.pmpm_num_particles.argtypes = [vp]
    L.pmpm_num_nodes.argtypes = [vp]
    L.pmpm_field_bytes.argtypes = [vp, i]
    L.pmpm_field_bytes.restype = sz
    L.pmpm_partition.argtypes = [vp]
    L.pmpm_shape_functions.argtypes = [vp, vp, vp, i]
    L.pmpm_num_surround_nodes.argtypes = [vp]
    L.pmpm_p2g.argtypes = [vp, i]
    L.pmpm_g2p.argtypes = [vp, i]
    L.pmpm_stress_update.argtypes = [vp]
    L.pmpm_solve.argtypes = [vp, i]
    L.pmpm_get_step.argtypes = [vp, ctypes.POINTER(ctypes.c_int)]
    L.pmpm_set_step.argtypes = [vp, i]
    L.pmpm_synchronize.argtypes = [vp]
    L.pmpm_stream.argtypes = [vp]
    L.pmpm_stream.restype = vp
    L.pmpm_profile_step.argtypes = [vp, fp, ctypes.POINTER(ctypes.c_int)]
    L.pmpm_active_nodes.argtypes = [vp, ctypes.POINTER(ctypes.c_int)]
    L.pmpm_launch_count.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
    L.pmpm_set_wait_limit.argtypes = [vp, ctypes.c_longlong]
    L.pmpm_set_p2g_staging.argtypes = [vp, i]
    L.pmpm_set_resort_interval.argtypes = [vp, i]
    L.pmpm_get_tuning.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                  ctypes.POINTER(ctypes.c_int)]
    L.pmpm_batch_set_wait_limit.argtypes = [vp, ctypes.c_longlong]
    L.pmpm_scan_tag.argtypes = [ctypes.c_uint, ctypes.POINTER(ctypes.c_uint)]
    L.pmpm_pick_resort_interval.argtypes = [f, fp, i, ctypes.POINTER(ctypes.c_int)]
    L.pmpm_partition_noalloc.argtypes = [i, fp, f, ctypes.POINTER(ctypes.c_int), vp, i, vp, vp, vp, vp, vp]
    L.pmpm_material_point_update.argtypes = [ctypes.POINTER(Material), i, i, f, vp, vp, vp, vp, vp, vp, vp, i, i]
    _lib = L
    return L


def scan_tag(launch):
    """The key scan's look-back tag for launch number `launch` (diagnostic)."""
    t = ctypes.c_uint()
    check(lib().pmpm_scan_tag(ctypes.c_uint(launch & 0xffffffff), ctypes.byref(t)), "pmpm_scan_tag")
    return t.value


def pick_resort_interval(t_sort, step_ms):
    """The autotuner's re-sort interval for a re-sort time and the step times
    after it (ms)."""
    a = np.ascontiguousarray(step_ms, dtype=np.float32)
    k = ctypes.c_int()
    check(lib().pmpm_pick_resort_interval(ctypes.c_float(t_sort), a.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                          len(a), ctypes.byref(k)), "pmpm_pick_resort_interval")
    return k.value


def check(status, what):
    if status != 0:
        raise PmpmError(status, what)


def _f3(vals):
    a = (ctypes.c_float * 3)()
    for k, v in enumerate(list(vals)[:3]):
        a[k] = float(v)
    return a


def make_material(m: dict) -> Material:
    """Material description dict -> pmpm_material (through the C helpers)."""
    L = lib()
    out = Material()
    t = m["type"]
    if t == "Material":
        out.type = MAT_NONE
        out.density = float(m.get("density", 0.0))
    elif t == "LinearElastic":
        check(L.pmpm_material_linear_elastic(m["density"], m["E"], m.get("pois", 0.0),
                                             1 if m.get("corrected") else 0, ctypes.byref(out)), "material")
    elif t == "NewtonFluid":
        check(L.pmpm_material_newton_fluid(m["density"], m["viscosity"], m.get("bulk_modulus", 0.0),
                                           m.get("gamma", 7.0), ctypes.byref(out)), "material")
    elif t == "DruckerPrager":
        check(L.pmpm_material_drucker_prager(m["density"], m["E"], m.get("pois", 0.0),
                                             m.get("friction_angle", 30.0), m.get("dilatancy_angle", 0.0),
                                             m.get("cohesion", 0.0), ctypes.byref(out)), "material")
    elif t == "VonMises":
        check(L.pmpm_material_von_mises(m["density"], m["E"], m.get("pois", 0.0), m["yield_stress"], m.get("H", 0.0),
                                        ctypes.byref(out)), "material")
    elif t == "ModifiedCamClay":
        check(L.pmpm_material_modified_cam_clay(m["density"], m["E"], m.get("pois", 0.0), m["M"], m["lam"], m["kap"],
                                                m["Vs"], m["R"], m.get("Pt", 0.0), m.get("beta", 1.0),
                                                ctypes.byref(out)), "material")
    elif t == "DruckerPragerCap":
        check(L.pmpm_material_drucker_prager_cap(m["density"], m["E"], m.get("pois", 0.0), m["M"], m["lam"],
                                                 m["kap"], m["Vs"], m["R"], m.get("Pt", 0.0), m.get("beta", 1.0),
                                                 m.get("dilatancy_angle", 0.0), ctypes.byref(out)), "material")
    elif t == "DP_rheo":
        check(L.pmpm_material_dp_rheo(m["density"], m["E"], m.get("pois", 0.0), m["M"], m.get("Pt", 0.0),
                                      m.get("dilatancy_angle", 0.0), ctypes.byref(out)), "material")
    else:
        raise ValueError(f"unknown material {t}")
    return out


def make_bc(b: dict, dim: int, num_nodes: int, keep: list) -> BC:
    L = lib()
    out = BC()
    t = b["type"]
    if t == "Gravity":
        g = _f3(b["gravity"])
        ge = _f3(b.get("gravity_end", [0.0] * dim))
        check(L.pmpm_bc_gravity(g, 1 if b.get("is_ramp") else 0, int(b.get("ramp_step", 0)), ge, dim,
                                ctypes.byref(out)), "bc")
    elif t == "NodeDomain":
        f0 = (ctypes.c_int * 3)(*(list(b.get("face0_mode", [0] * dim)) + [0] * 3)[:3])
        f1 = (ctypes.c_int * 3)(*(list(b.get("face1_mode", [0] * dim)) + [0] * 3)[:3])
        check(L.pmpm_bc_nodedomain(f0, f1, dim, ctypes.byref(out)), "bc")
    elif t == "BodyForce":
        vals = np.ascontiguousarray(np.asarray(b["values"], np.float32).reshape(num_nodes, dim))
        mask = np.ascontiguousarray(np.asarray(b["mask"]).astype(np.uint8).reshape(num_nodes))
        keep += [vals, mask]
        mode = {"forces": 0, "moments": 1, "fixed": 2}[b["mode"]]
        check(L.pmpm_bc_bodyforce(mode, vals.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                  mask.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)), ctypes.byref(out)), "bc")
        if not b.get("is_active", True):
            out.ints[1] = 0
    elif t == "PlanarDomain":
        check(L.pmpm_bc_planardomain(_f3(b.get("face0_friction", [0.0] * dim)),
                                     _f3(b.get("face1_friction", [0.0] * dim)), dim, ctypes.byref(out)), "bc")
    elif t == "RigidBodyLevelSet" and "shape" not in b:
        check(L.pmpm_bc_rigidbodylevelset(RIGID_MODES[b.get("mode", "static")],
                                          _f3(b.get("euler_angles_per_second", [0.0] * dim)),
                                          _f3(b.get("COM", [0.0] * dim)),
                                          1 if b.get("corrected_rotation", False) else 0, dim,
                                          ctypes.byref(out)), "bc")
    elif t == "RigidBodyLevelSet":
        check(L.pmpm_bc_rigid_sdf(SDF_SHAPES[b["shape"]], int(b.get("axis", 2)), _f3(b["center"]),
                                  _f3(b.get("velocity", [0.0] * dim)), float(b.get("angular_velocity", 0.0)),
                                  float(b.get("angle", 0.0)), _f3(b["dims"]), float(b.get("friction", 0.0)),
                                  float(b.get("contact_distance", 0.0)), dim, ctypes.byref(out)), "bc")
    else:
        raise ValueError(f"unknown boundary condition {t}")
    return out


def material_point_vjp(material: dict, dim, dt, L, eps_e, stress_ref, grad_stress, grad_eps_e, youngs=None,
                       friction=None, method=0, device=0):
    """Vector-Jacobian product of the single-point Drucker-Prager update:
    returns (dL, d eps_e, dE, dphi) for the adjoints of the new stress and
    elastic strain.  method 0 reverse mode, 1 forward-mode dual numbers."""
    m = make_material(material)
    a = lambda x, shape: np.ascontiguousarray(np.asarray(x, np.float32).reshape(shape))
    L = a(L, (-1, dim, dim))
    n = L.shape[0]
    eps = a(eps_e, (n, dim, dim))
    sref = a(stress_ref, (n, 3, 3))
    gS = a(grad_stress, (n, 3, 3))
    gEo = a(grad_eps_e, (n, dim, dim))
    Y = None if youngs is None else a(youngs, (n,))
    Fr = None if friction is None else a(friction, (n,))
    oL = np.empty((n, dim, dim), np.float32)
    oE = np.empty((n, dim, dim), np.float32)
    oY = np.empty(n, np.float32)
    oF = np.empty(n, np.float32)
    p = lambda x: None if x is None else x.ctypes.data_as(ctypes.c_void_p)
    check(lib().pmpm_material_point_vjp(ctypes.byref(m), dim, n, float(dt), p(L), p(eps), p(sref), p(Y), p(Fr),
                                        p(gS), p(gEo), p(oL), p(oE), p(oY), p(oF), int(method), int(device)),
          "pmpm_material_point_vjp")
    return oL, oE, oY, oF


def calculate_timestep(cell_size, factor, bulk_modulus, shear_modulus, density):
    """tools::calculate_timestep (src/common/tools.cpp:373-380)."""
    out = ctypes.c_float()
    check(lib().pmpm_calculate_timestep(float(cell_size), float(factor), float(bulk_modulus),
                                        float(shear_modulus), float(density), ctypes.byref(out)),
          "pmpm_calculate_timestep")
    return out.value


def material_timestep(material: dict, cell_size, factor):
    """<Material>::calculate_timestep (src/materials/linearelastic.cpp:96-105) for a material dict."""
    out = ctypes.c_float()
    m = make_material(material)
    check(lib().pmpm_material_timestep(ctypes.byref(m), float(cell_size), float(factor), ctypes.byref(out)),
          "pmpm_material_timestep")
    return out.value


def field_shape(name, dim, n, num_nodes, nsn=None):
    return {
        "positions": (n, dim), "velocities": (n, dim), "forces_external": (n, dim),
        "stresses": (n, 3, 3), "stress_ref": (n, 3, 3), "F": (n, dim, dim), "velocity_gradient": (n, dim, dim),
        "eps_e": (n, dim, dim), "masses": (n,), "volumes": (n,), "volumes_original": (n,),
        "youngs_modulus": (n,), "friction_angle": (n,), "acc_eps_p": (n,),
        "alpha": (n,), "pc": (n,), "colors": (n,), "is_rigid": (n,), "is_active": (n,),
        "node_masses": (num_nodes,), "node_moments": (num_nodes, dim), "node_moments_nt": (num_nodes, dim),
        "node_ids": (num_nodes, 3), "node_types": (num_nodes, 3), "bins": (n, dim),
        "hash_unsorted": (n,), "hash_sorted": (n,), "sorted_index": (n,),
        "cell_start": (num_nodes,), "cell_end": (num_nodes,),
    }[name]


def field_dtype(name):
    if name in _U8:
        return np.uint8
    if name in _I32:
        return np.int32
    if name in _U32:
        return np.uint32
    return np.float32


def make_desc(dim, origin, end, cell_size, shape_function="linear", dt=1e-3, particles_per_cell=1, alpha=0.99,
              materials=(), bcs=(), flags=0, device=0, stream=None, resort_interval=32, keep=None):
    """pmpm_desc of a simulation; the arrays it points to are appended to `keep`."""
    keep = [] if keep is None else keep
    mats = list(materials)
    bcl = list(bcs)
    if len(mats) > MAX_MATERIALS or len(bcl) > MAX_BCS:
        raise ValueError("too many materials or boundary conditions")
    marr = (Material * max(1, len(mats)))(*[make_material(m) for m in mats]) if mats else (Material * 1)()
    # node count is needed for BodyForce arrays; compute it the reference way
    num_nodes = 1
    for a in range(dim):
        num_nodes *= int(np.float32(np.float32(end[a]) - np.float32(origin[a])) / np.float32(cell_size)) + 1
    barr = (BC * max(1, len(bcl)))(*[make_bc(b, dim, num_nodes, keep) for b in bcl]) if bcl else (BC * 1)()
    keep += [marr, barr]
    d = Desc()
    d.dim = dim
    d.origin = _f3(list(origin) + [0.0] * 3)
    d.end = _f3(list(end) + [0.0] * 3)
    d.cell_size = float(cell_size)
    d.shape_function = SHAPE[shape_function] if isinstance(shape_function, str) else int(shape_function)
    d.dt = float(dt)
    d.particles_per_cell = int(particles_per_cell)
    d.alpha = float(alpha)
    d.num_materials = len(mats)
    d.materials = ctypes.cast(marr, ctypes.POINTER(Material))
    d.num_bcs = len(bcl)
    d.bcs = ctypes.cast(barr, ctypes.POINTER(BC))
    d.flags = int(flags)
    d.device = int(device)
    d.stream = stream
    d.resort_interval = int(resort_interval)
    return d


class Simulation:
    """One simulation handle (pmpm_sim) of the C ABI."""

    def __init__(self, dim, origin, end, cell_size, shape_function="linear", dt=1e-3, particles_per_cell=1,
                 alpha=0.99, materials=(), bcs=(), flags=0, device=0, stream=None, resort_interval=32):
        L = lib()
        self.dim = dim
        self._keep = []
        d = make_desc(dim, origin, end, cell_size, shape_function, dt, particles_per_cell, alpha, materials, bcs,
                      flags, device, stream, resort_interval, self._keep)
        h = ctypes.c_void_p()
        check(L.pmpm_create(ctypes.byref(d), ctypes.byref(h)), "pmpm_create")
        self._h = h
        self._desc = d
        nc = (ctypes.c_int * 3)()
        nt = ctypes.c_int()
        inv = ctypes.c_float()
        check(L.pmpm_get_grid(h, nc, ctypes.byref(nt), ctypes.byref(inv)), "pmpm_get_grid")
        self.num_cells = [nc[0], nc[1], nc[2]]
        self.num_nodes = nt.value
        self.inv_cell_size = inv.value
        self.n = 0

    def close(self):
        if getattr(self, "_h", None):
            lib().pmpm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def set_particles(self, positions, velocities=None, colors=None, rigid_positions=None,
                      rigid_velocities=None, rigid_colors=None):
        d = self.dim

        def arr(a, dt, shape=None):
            if a is None:
                return None
            a = np.ascontiguousarray(np.asarray(a, dt))
            return a.reshape(shape) if shape else a

        x = arr(positions, np.float32, (-1, d))
        v = arr(velocities, np.float32, (-1, d))
        c = arr(colors, np.uint8)
        rx = arr(rigid_positions, np.float32, (-1, d))
        rv = arr(rigid_velocities, np.float32, (-1, d))
        rc = arr(rigid_colors, np.uint8)
        n = 0 if x is None else x.shape[0]
        nr = 0 if rx is None else rx.shape[0]
        ptr = lambda a: None if a is None or a.size == 0 else a.ctypes.data_as(ctypes.c_void_p)
        check(lib().pmpm_set_particles(self._h, n, ptr(x), ptr(v), ptr(c), nr, ptr(rx), ptr(rv), ptr(rc)),
              "pmpm_set_particles")
        self.n = n + nr
        return self

    def initialize(self):
        check(lib().pmpm_initialize(self._h), "pmpm_initialize")
        return self

    def get(self, name, out=None):
        shape = field_shape(name, self.dim, self.n, self.num_nodes)
        dt = field_dtype(name)
        if out is None:
            out = np.empty(shape, dt)
        check(lib().pmpm_get_field(self._h, FIELDS[name], out.ctypes.data_as(ctypes.c_void_p), out.nbytes, 0),
              f"get {name}")
        return out

    def get_device(self, name, ptr, nbytes):
        check(lib().pmpm_get_field(self._h, FIELDS[name], ctypes.c_void_p(ptr), nbytes, 1), f"get {name}")

    def set(self, name, values):
        shape = field_shape(name, self.dim, self.n, self.num_nodes)
        a = np.ascontiguousarray(np.asarray(values, field_dtype(name)).reshape(shape))
        check(lib().pmpm_set_field(self._h, FIELDS[name], a.ctypes.data_as(ctypes.c_void_p), a.nbytes, 0),
              f"set {name}")

    def get_ptr(self, name, ptr, nbytes, on_device=False):
        """Copy a field to raw memory (host pointer, e.g. pinned, or device pointer)."""
        check(lib().pmpm_get_field(self._h, FIELDS[name], ctypes.c_void_p(ptr), nbytes, 1 if on_device else 0),
              f"get {name}")

    def set_ptr(self, name, ptr, nbytes, on_device=False):
        """Copy a field from raw memory (host pointer, e.g. pinned, or device pointer)."""
        check(lib().pmpm_set_field(self._h, FIELDS[name], ctypes.c_void_p(ptr), nbytes, 1 if on_device else 0),
              f"set {name}")

    def set_device(self, name, ptr, nbytes):
        check(lib().pmpm_set_field(self._h, FIELDS[name], ctypes.c_void_p(ptr), nbytes, 1), f"set {name}")

    def partition(self):
        check(lib().pmpm_partition(self._h), "pmpm_partition")

    def shape_functions(self):
        L = lib()
        nsn = L.pmpm_num_surround_nodes(self._h)
        psi = np.empty((self.n, nsn), np.float32)
        dpsi = np.empty((self.n, nsn, self.dim), np.float32)
        check(L.pmpm_shape_functions(self._h, psi.ctypes.data_as(ctypes.c_void_p),
                                     dpsi.ctypes.data_as(ctypes.c_void_p), 0), "pmpm_shape_functions")
        return psi, dpsi

    def p2g(self, apply_bcs=False):
        check(lib().pmpm_p2g(self._h, 1 if apply_bcs else 0), "pmpm_p2g")

    def g2p(self, stress_update=False):
        check(lib().pmpm_g2p(self._h, 1 if stress_update else 0), "pmpm_g2p")

    def stress_update(self):
        check(lib().pmpm_stress_update(self._h), "pmpm_stress_update")

    def solve(self, nsteps=1):
        check(lib().pmpm_solve(self._h, int(nsteps)), "pmpm_solve")

    def synchronize(self):
        return lib().pmpm_synchronize(self._h)

    @property
    def step(self):
        s = ctypes.c_int()
        check(lib().pmpm_get_step(self._h, ctypes.byref(s)), "pmpm_get_step")
        return s.value

    @step.setter
    def step(self, v):
        check(lib().pmpm_set_step(self._h, int(v)), "pmpm_set_step")

    def profile_step(self):
        """One step with per-phase CUDA-event times (ms): partition, P2G, G2P."""
        ms = (ctypes.c_float * 3)()
        nl = ctypes.c_int()
        check(lib().pmpm_profile_step(self._h, ms, ctypes.byref(nl)), "pmpm_profile_step")
        return [ms[0], ms[1], ms[2]], nl.value

    def launch_count(self):
        c = ctypes.c_longlong()
        check(lib().pmpm_launch_count(self._h, ctypes.byref(c)), "pmpm_launch_count")
        return c.value

    def set_wait_limit(self, spins):
        """Bound on the key scan's look-back polls (default 2**22)."""
        check(lib().pmpm_set_wait_limit(self._h, int(spins)), "pmpm_set_wait_limit")

    def set_p2g_staging(self, mode):
        """3D sweeps: 1 bulk copies of sorted records, 0 gather through the sorted order."""
        check(lib().pmpm_set_p2g_staging(self._h, int(mode)), "pmpm_set_p2g_staging")

    def set_resort_interval(self, steps):
        check(lib().pmpm_set_resort_interval(self._h, int(steps)), "pmpm_set_resort_interval")

    def tuning(self):
        """The handle's choices: {"p2g_kernel", "staging", "resort_interval"}."""
        k, g, r = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(lib().pmpm_get_tuning(self._h, ctypes.byref(k), ctypes.byref(g), ctypes.byref(r)), "pmpm_get_tuning")
        return {"p2g_kernel": k.value, "staging": g.value, "resort_interval": r.value}

    def autotune(self, steps=5):
        """Time each P2G kernel this configuration has on `steps` steps, keep
        the fastest, restore the state; returns the chosen variant."""
        c = ctypes.c_int()
        check(lib().pmpm_autotune(self._h, int(steps), ctypes.byref(c)), "pmpm_autotune")
        return c.value

    def set_p2g_kernel(self, variant):
        """Select the P2G kernel (1 sweep, 0 cell scatter; 3D quadratic)."""
        check(lib().pmpm_set_p2g_kernel(self._h, int(variant)), "pmpm_set_p2g_kernel")

    # ---- differentiable rollouts ----
    def rollout_forward(self, nsteps, checkpoint_every=25):
        check(lib().pmpm_rollout_forward(self._h, int(nsteps), int(checkpoint_every)), "pmpm_rollout_forward")
        return self

    def rollout_set_memory(self, nbytes):
        """Memory for segments kept whole from the forward pass (< 0 automatic, 0 checkpoints only)."""
        check(lib().pmpm_rollout_set_memory(self._h, int(nbytes)), "pmpm_rollout_set_memory")
        return self

    def rollout_reset(self):
        check(lib().pmpm_rollout_reset(self._h), "pmpm_rollout_reset")
        return self

    def rollout_backward(self, grad_positions):
        """Host arrays: returns (dL/dE, dL/dphi, dL/dx0, dL/dv0) for a loss
        gradient dL/dx of the final positions."""
        g = np.ascontiguousarray(np.asarray(grad_positions, np.float32).reshape(self.n, self.dim))
        gE = np.empty(self.n, np.float32)
        gp = np.empty(self.n, np.float32)
        gx = np.empty((self.n, self.dim), np.float32)
        gv = np.empty((self.n, self.dim), np.float32)
        ptr = lambda a: a.ctypes.data_as(ctypes.c_void_p)
        check(lib().pmpm_rollout_backward(self._h, ptr(g), 0, ptr(gE), ptr(gp), ptr(gx), ptr(gv)),
              "pmpm_rollout_backward")
        return gE, gp, gx, gv

    def rollout_backward_ptr(self, grad_positions, grad_youngs, grad_friction, grad_positions0=0,
                             grad_velocities0=0):
        """Device pointers (integers; 0 for an output not wanted)."""
        vp = lambda p: ctypes.c_void_p(p) if p else None
        check(lib().pmpm_rollout_backward(self._h, vp(grad_positions), 1, vp(grad_youngs), vp(grad_friction),
                                          vp(grad_positions0), vp(grad_velocities0)), "pmpm_rollout_backward")

    def active_nodes(self):
        c = ctypes.c_int()
        check(lib().pmpm_active_nodes(self._h, ctypes.byref(c)), "pmpm_active_nodes")
        return c.value

    @property
    def stream(self):
        return lib().pmpm_stream(self._h)


def material_point_update(mat: dict, dim, L, stress, eps_e=None, stress_ref=None, dt=1.0, masses=None,
                          volumes=None, volumes_original=None, velgrad_is_strain_increment=False, device=0):
    """Material update of independent points on the GPU (host arrays in, host arrays out)."""
    m = make_material(mat)
    Lh = np.ascontiguousarray(np.asarray(L, np.float32).reshape(-1, dim, dim))
    n = Lh.shape[0]
    S = np.ascontiguousarray(np.asarray(stress, np.float32).reshape(n, 3, 3).copy())
    E = None if eps_e is None else np.ascontiguousarray(np.asarray(eps_e, np.float32).reshape(n, dim, dim).copy())
    R = None if stress_ref is None else np.ascontiguousarray(np.asarray(stress_ref, np.float32).reshape(n, 3, 3))
    mm = None if masses is None else np.ascontiguousarray(np.asarray(masses, np.float32))
    vv = None if volumes is None else np.ascontiguousarray(np.asarray(volumes, np.float32))
    v0 = None if volumes_original is None else np.ascontiguousarray(np.asarray(volumes_original, np.float32))
    p = lambda a: None if a is None else a.ctypes.data_as(ctypes.c_void_p)
    check(lib().pmpm_material_point_update(ctypes.byref(m), dim, n, float(dt), p(Lh), p(S), p(E), p(R), p(mm),
                                           p(vv), p(v0), 1 if velgrad_is_strain_increment else 0, device),
          "pmpm_material_point_update")
    return S, E


class Batch:
    """A batched ensemble (pmpm_batch): independent simulations stepped with
    one launch per phase.  `instances` are dicts with the Simulation keyword
    arguments (dim, origin, end, cell_size, shape_function, dt,
    particles_per_cell, alpha, materials, bcs) plus positions, velocities and
    colors."""

    KEYS = ("dim", "origin", "end", "cell_size", "shape_function", "dt", "particles_per_cell", "alpha",
            "materials", "bcs")

    def __init__(self, instances, flags=0, device=0, stream=None, resort_interval=32):
        L = lib()
        self._keep = []
        insts = list(instances)
        arr = (Instance * len(insts))()
        self.dims, self.n, self.num_nodes = [], [], []
        for k, sc in enumerate(insts):
            kw = {key: sc[key] for key in self.KEYS if key in sc}
            d = make_desc(**kw, flags=flags, device=device, keep=self._keep)
            self._keep.append(d)
            dim = kw["dim"]
            x = np.ascontiguousarray(np.asarray(sc["positions"], np.float32).reshape(-1, dim))
            v = sc.get("velocities")
            v = None if v is None else np.ascontiguousarray(np.asarray(v, np.float32).reshape(-1, dim))
            c = sc.get("colors")
            c = None if c is None else np.ascontiguousarray(np.asarray(c).astype(np.uint8))
            self._keep += [x, v, c]
            arr[k].desc = ctypes.pointer(d)
            arr[k].num_particles = x.shape[0]
            arr[k].positions = x.ctypes.data_as(ctypes.c_void_p)
            arr[k].velocities = None if v is None else v.ctypes.data_as(ctypes.c_void_p)
            arr[k].colors = None if c is None else c.ctypes.data_as(ctypes.c_void_p)
            nn = 1
            for a in range(dim):
                nn *= int(np.float32(np.float32(kw["end"][a]) - np.float32(kw["origin"][a]))
                          / np.float32(kw["cell_size"])) + 1
            self.dims.append(dim)
            self.n.append(x.shape[0])
            self.num_nodes.append(nn)
        h = ctypes.c_void_p()
        check(L.pmpm_batch_create(len(insts), arr, int(device), stream, int(resort_interval), ctypes.byref(h)),
              "pmpm_batch_create")
        self._h = h
        self._keep = None  # the batch copied everything it needs

    def close(self):
        if getattr(self, "_h", None):
            lib().pmpm_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self):
        return len(self.n)

    def initialize(self):
        check(lib().pmpm_batch_initialize(self._h), "pmpm_batch_initialize")
        return self

    def solve(self, nsteps=1):
        check(lib().pmpm_batch_solve(self._h, int(nsteps)), "pmpm_batch_solve")
        return self

    def synchronize(self):
        return lib().pmpm_batch_synchronize(self._h)

    def get(self, instance, name, out=None):
        shape = field_shape(name, self.dims[instance], self.n[instance], self.num_nodes[instance])
        if out is None:
            out = np.empty(shape, field_dtype(name))
        check(lib().pmpm_batch_get_field(self._h, int(instance), FIELDS[name], out.ctypes.data_as(ctypes.c_void_p),
                                         out.nbytes, 0), f"get {name}")
        return out

    def set(self, instance, name, values):
        shape = field_shape(name, self.dims[instance], self.n[instance], self.num_nodes[instance])
        a = np.ascontiguousarray(np.asarray(values, field_dtype(name)).reshape(shape))
        check(lib().pmpm_batch_set_field(self._h, int(instance), FIELDS[name], a.ctypes.data_as(ctypes.c_void_p),
                                         a.nbytes, 0), f"set {name}")

    def get_ptr(self, instance, name, ptr, nbytes, on_device=False):
        check(lib().pmpm_batch_get_field(self._h, int(instance), FIELDS[name], ctypes.c_void_p(ptr), nbytes,
                                         1 if on_device else 0), f"get {name}")

    def set_ptr(self, instance, name, ptr, nbytes, on_device=False):
        check(lib().pmpm_batch_set_field(self._h, int(instance), FIELDS[name], ctypes.c_void_p(ptr), nbytes,
                                         1 if on_device else 0), f"set {name}")

    def profile_step(self):
        ms = (ctypes.c_float * 3)()
        nl = ctypes.c_int()
        check(lib().pmpm_batch_profile_step(self._h, ms, ctypes.byref(nl)), "pmpm_batch_profile_step")
        return [ms[0], ms[1], ms[2]], nl.value

    def launch_count(self):
        c = ctypes.c_longlong()
        check(lib().pmpm_batch_launch_count(self._h, ctypes.byref(c)), "pmpm_batch_launch_count")
        return c.value

    def set_wait_limit(self, spins):
        check(lib().pmpm_batch_set_wait_limit(self._h, int(spins)), "pmpm_batch_set_wait_limit")
