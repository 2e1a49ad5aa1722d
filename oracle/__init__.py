"""CPU oracle of the PyroclastMPM update-stress-last step (ctypes wrapper).

TEST INFRASTRUCTURE ONLY.  The oracle is the checker for the CUDA path: only
``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``
import it.  The product library never links or calls it.

The C restatement (``oracle.c``) is compiled twice, in FP32 (the reference's
``DOUBLE_PRECISION=OFF`` build) and in FP64 (the drift oracle).  Arrays use the
reference container layouts (AoS, row-major), see ``oracle.h``.

Material and boundary-condition descriptions are plain dicts shared with the
product-side tests, e.g. ``{"type": "LinearElastic", "density": 1000.0,
"E": 1000.0, "pois": 0.3}``; ``material_params`` turns them into the
parameter vectors both implementations use.
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS = {}

LINEAR, QUADRATIC, CUBIC = 0, 1, 2
SHAPE_FUNCTIONS = {"linear": LINEAR, "quadratic": QUADRATIC, "cubic": CUBIC}

MAT_NONE, MAT_LINEAR_ELASTIC, MAT_NEWTON_FLUID, MAT_DRUCKER_PRAGER, MAT_VON_MISES = 0, 1, 2, 3, 4
MAT_MODIFIED_CAM_CLAY, MAT_DRUCKER_PRAGER_CAP = 5, 6
BC_GRAVITY, BC_NODEDOMAIN, BC_BODYFORCE, BC_PLANARDOMAIN = 1, 2, 3, 4
BC_RIGIDBODY_LEVELSET, BC_RIGID_SDF = 5, 6
RIGID_MODES = {"static": 0, "loop_rotate": 1}
SDF_SHAPES = {"sphere": 0, "half_cylinder_shell": 1}


def build() -> None:
    """Compile liboracle_f32.so / liboracle_f64.so (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _lib(precision: str):
    if precision not in _LIBS:
        path = os.path.join(_HERE, "_build", f"liboracle_{precision}.so")
        if not os.path.exists(path):
            build()
        _LIBS[precision] = ctypes.CDLL(path)
    return _LIBS[precision]


def _real(precision):
    return (ctypes.c_float, np.float32) if precision == "f32" else (ctypes.c_double, np.float64)


def _structs(precision):
    creal, _ = _real(precision)

    class Grid(ctypes.Structure):
        _fields_ = [("dim", ctypes.c_int), ("origin", creal * 3), ("end", creal * 3),
                    ("cell_size", creal), ("inv_cell_size", creal),
                    ("num_cells", ctypes.c_int * 3), ("num_cells_total", ctypes.c_int)]

    class Material(ctypes.Structure):
        _fields_ = [("type", ctypes.c_int), ("density", creal), ("p", creal * 12)]

    class BC(ctypes.Structure):
        _fields_ = [("type", ctypes.c_int), ("i", ctypes.c_int * 8), ("r", creal * 16),
                    ("values", ctypes.c_void_p), ("mask", ctypes.c_void_p)]

    P = ctypes.c_void_p

    class Sim(ctypes.Structure):
        _fields_ = [("grid", Grid), ("shape_function", ctypes.c_int), ("nsn", ctypes.c_int),
                    ("dt", creal), ("alpha", creal), ("small_mass_cutoff", creal),
                    ("global_step", ctypes.c_int), ("particles_per_cell", ctypes.c_int),
                    ("num_particles", ctypes.c_int),
                    ("positions", P), ("velocities", P), ("stresses", P), ("F", P),
                    ("velocity_gradient", P), ("masses", P), ("volumes", P),
                    ("volumes_original", P), ("forces_external", P),
                    ("colors", P), ("is_rigid", P), ("is_active", P), ("psi", P), ("dpsi", P),
                    ("bins", P), ("hash_unsorted", P), ("hash_sorted", P), ("sorted_index", P),
                    ("cell_start", P), ("cell_end", P),
                    ("node_masses", P), ("node_moments", P), ("node_moments_nt", P),
                    ("node_ids", P), ("node_types", P),
                    ("num_materials", ctypes.c_int), ("materials", P),
                    ("num_bcs", ctypes.c_int), ("bcs", P),
                    ("eps_e", P), ("stress_ref", P), ("youngs", P), ("friction", P), ("musl", ctypes.c_int), ("acc_eps_p", P),
                    ("pc", P)]

    return Grid, Material, BC, Sim


def grid_dims(dim, origin, end, cell_size, precision="f32"):
    """Reference Grid node counts (types_common.h:260-272) in the given precision."""
    _, npr = _real(precision)
    h = npr(cell_size)
    n = [1, 1, 1]
    for a in range(dim):
        n[a] = int(npr(npr(end[a]) - npr(origin[a])) / h) + 1
    return n


def material_params(mat: dict, precision: str = "f32"):
    """(type id, density, 8 parameters) computed in the working precision."""
    _, npr = _real(precision)
    t = mat["type"]
    dens = npr(mat.get("density", 0.0))
    if t == "Material":
        return MAT_NONE, dens, [0.0] * 8
    if t == "LinearElastic":
        E, nu = npr(mat["E"]), npr(mat.get("pois", 0.0))
        one, two, three = npr(1), npr(2), npr(3)
        bulk = E / (three * (one - two * nu))
        shear = E / (two * (one + nu))
        lame = E * nu / ((one + nu) * (one - two * nu))
        return MAT_LINEAR_ELASTIC, dens, [E, nu, lame, shear, bulk, 1.0 if mat.get("corrected") else 0.0, 0, 0]
    if t == "NewtonFluid":
        return MAT_NEWTON_FLUID, dens, [npr(mat["viscosity"]), npr(mat.get("bulk_modulus", 0.0)),
                                        npr(mat.get("gamma", 7.0)), 0, 0, 0, 0, 0]
    if t == "DruckerPrager":
        E, nu = npr(mat["E"]), npr(mat.get("pois", 0.0))
        one, two, three = npr(1), npr(2), npr(3)
        bulk = E / (three * (one - two * nu))
        shear = E / (two * (one + nu))
        phi = math.radians(float(mat.get("friction_angle", 30.0)))
        psi = math.radians(float(mat.get("dilatancy_angle", 0.0)))
        c = float(mat.get("cohesion", 0.0))
        s3 = math.sqrt(3.0)
        eta = 6.0 * math.sin(phi) / (s3 * (3.0 - math.sin(phi)))
        xi = 6.0 * math.cos(phi) / (s3 * (3.0 - math.sin(phi)))
        eta_bar = 6.0 * math.sin(psi) / (s3 * (3.0 - math.sin(psi)))
        kc = xi * c
        has_apex = 1.0 if eta > 0 else 0.0
        p_apex = kc / eta if eta > 0 else 0.0
        return MAT_DRUCKER_PRAGER, dens, [bulk, shear, npr(eta), npr(eta_bar), npr(kc), npr(p_apex), has_apex,
                                          float(nu)]
    if t == "VonMises":
        E, nu = npr(mat["E"]), npr(mat.get("pois", 0.0))
        one, two, three = npr(1), npr(2), npr(3)
        bulk = E / (three * (one - two * nu))
        shear = E / (two * (one + nu))
        return MAT_VON_MISES, dens, [bulk, shear, npr(mat["yield_stress"]), npr(mat.get("H", 0.0)), 0, 0, 0, 0]
    if t == "ModifiedCamClay":
        # ModifiedCamClay::ModifiedCamClay (src/materials/modifiedcamclay.cpp:47-63)
        E, nu = npr(mat["E"]), npr(mat.get("pois", 0.0))
        one, two, three = npr(1), npr(2), npr(3)
        bulk = E / (three * (one - two * nu))
        shear = E / (two * (one + nu))
        return MAT_MODIFIED_CAM_CLAY, dens, [bulk, shear, npr(mat["M"]), npr(mat["lam"]), npr(mat["kap"]),
                                             npr(mat["Vs"]), npr(mat.get("Pt", 0.0)), npr(mat["R"])]
    if t == "DruckerPragerCap":
        # DruckerPragerCap::DruckerPragerCap (src/materials/druckerprager_cap.cpp:43-67)
        E, nu = npr(mat["E"]), npr(mat.get("pois", 0.0))
        one, two, three = npr(1), npr(2), npr(3)
        bulk = E / (three * (one - two * nu))
        shear = E / (two * (one + nu))
        psi = math.radians(float(mat.get("dilatancy_angle", 0.0)))
        eta_bar = 6.0 * math.sin(psi) / (math.sqrt(3.0) * (3.0 + math.sin(psi)))
        return MAT_DRUCKER_PRAGER_CAP, dens, [bulk, shear, npr(mat["M"]), npr(mat["lam"]), npr(mat["kap"]),
                                              npr(mat["Vs"]), npr(mat.get("Pt", 0.0)), npr(mat["R"]),
                                              npr(mat.get("beta", 1.0)), npr(eta_bar)]
    if t == "DP_rheo":
        # the reference's DP_rheo parameters (src/materials/dp_rheo.cpp:45-70)
        E, nu = npr(mat["E"]), npr(mat.get("pois", 0.0))
        one, two, three = npr(1), npr(2), npr(3)
        bulk = E / (three * (one - two * nu))
        shear = E / (two * (one + nu))
        M, Pt = npr(mat["M"]), npr(mat.get("Pt", 0.0))
        psi = npr(npr(mat.get("dilatancy_angle", 0.0)) * npr(math.pi / 180.0))
        eta_bar = npr(6.0 * math.sin(float(psi)) / (math.sqrt(3.0) * (3.0 + math.sin(float(psi)))))
        eta = npr(math.sqrt(1.0 / 3.0) * float(M))
        return MAT_DRUCKER_PRAGER, dens, [bulk, shear, eta, eta_bar, npr(eta * Pt), Pt, 1.0, -1.0]
    raise ValueError(f"unknown material {t}")


class OracleSim:
    """One USL simulation held in numpy arrays, stepped by the C oracle."""

    def __init__(self, dim, origin, end, cell_size, positions, velocities=None, colors=None,
                 shape_function="linear", dt=1e-3, particles_per_cell=1, alpha=0.99,
                 materials=(), bcs=(), precision="f32", global_step=0,
                 stresses=None, volumes=None, masses=None, volumes_original=None,
                 rigid_positions=None, rigid_velocities=None, rigid_colors=None,
                 youngs_modulus=None, friction_angle=None, musl=False):
        self.precision = precision
        self.lib = _lib(precision)
        Grid, Material, BC, Sim = _structs(precision)
        creal, npr = _real(precision)
        self.npr = npr
        self.dim = d = dim
        self.sf = SHAPE_FUNCTIONS[shape_function] if isinstance(shape_function, str) else int(shape_function)
        # inputs are always copied: the simulation advances its arrays in place.
        # Rigid particles follow the others (ParticlesContainer ctor,
        # src/particles/particles.cpp:51-149).
        x = np.array(positions, dtype=npr, copy=True).reshape(-1, d)
        nr = 0 if rigid_positions is None else len(np.asarray(rigid_positions).reshape(-1, d))
        n0 = x.shape[0]
        if nr:
            x = np.concatenate([x, np.asarray(rigid_positions, npr).reshape(nr, d)])
            rv = np.zeros((nr, d), npr) if rigid_velocities is None else np.asarray(rigid_velocities, npr)
            v0 = np.zeros((n0, d), npr) if velocities is None else np.asarray(velocities, npr).reshape(n0, d)
            velocities = np.concatenate([v0, rv.reshape(nr, d)])
            c0 = np.zeros(n0, np.uint8) if colors is None else np.asarray(colors).astype(np.uint8)
            rc = np.zeros(nr, np.uint8) if rigid_colors is None else np.asarray(rigid_colors).astype(np.uint8)
            colors = np.concatenate([c0, rc])
        n = x.shape[0]
        self.n = n
        g = Grid()
        o3 = (creal * 3)(*[float(origin[a]) if a < d else 0.0 for a in range(3)])
        e3 = (creal * 3)(*[float(end[a]) if a < d else 0.0 for a in range(3)])
        self.lib.or_grid_init(ctypes.byref(g), d, o3, e3, creal(cell_size))
        self.grid = g
        nn = g.num_cells_total
        self.num_nodes = nn
        self.nsn = self.lib.or_num_surround_nodes(d, self.sf)
        z = lambda *shape: np.zeros(shape, dtype=npr)
        self.a = a = {}
        a["positions"] = x
        a["velocities"] = z(n, d) if velocities is None else np.array(velocities, npr, copy=True).reshape(n, d)
        a["stresses"] = z(n, 3, 3) if stresses is None else np.array(stresses, npr, copy=True).reshape(n, 3, 3)
        a["F"] = np.ascontiguousarray(np.broadcast_to(np.eye(d, dtype=npr), (n, d, d)))
        a["velocity_gradient"] = z(n, d, d)
        a["masses"] = np.full(n, -1.0, npr) if masses is None else np.asarray(masses, npr).copy()
        a["volumes"] = np.full(n, -1.0, npr) if volumes is None else np.asarray(volumes, npr).copy()
        a["volumes_original"] = (np.full(n, -1.0, npr) if volumes_original is None
                                 else np.asarray(volumes_original, npr).copy())
        a["forces_external"] = z(n, d)
        a["colors"] = (np.zeros(n, np.uint8) if colors is None else np.asarray(colors).astype(np.uint8))
        a["is_rigid"] = np.zeros(n, np.uint8)
        a["is_rigid"][n0:] = 1
        a["is_active"] = np.ones(n, np.uint8)
        a["psi"] = z(n * self.nsn)
        a["dpsi"] = z(n * self.nsn * d)
        a["bins"] = np.zeros((n, d), np.int32)
        a["hash_unsorted"] = np.zeros(n, np.uint32)
        a["hash_sorted"] = np.zeros(n, np.uint32)
        a["sorted_index"] = np.arange(n, dtype=np.int32)
        a["cell_start"] = np.zeros(nn, np.int32)
        a["cell_end"] = np.zeros(nn, np.int32)
        a["node_masses"] = z(nn)
        a["node_moments"] = z(nn, d)
        a["node_moments_nt"] = z(nn, d)
        a["node_ids"] = np.zeros((nn, 3), np.int32)
        a["node_types"] = np.zeros((nn, 3), np.int32)
        a["eps_e"] = z(n, d, d)
        a["stress_ref"] = z(n, 3, 3)
        a["acc_eps_p"] = z(n)
        a["pc"] = z(n)
        if youngs_modulus is not None:
            a["youngs"] = np.array(youngs_modulus, npr, copy=True).reshape(n)
            a["friction"] = np.array(friction_angle, npr, copy=True).reshape(n)
        self.lib.or_node_ids(ctypes.byref(g), a["node_ids"].ctypes.data_as(ctypes.c_void_p))
        self.lib.or_node_types(ctypes.byref(g), self.sf, a["node_ids"].ctypes.data_as(ctypes.c_void_p),
                               a["node_types"].ctypes.data_as(ctypes.c_void_p))

        self.materials = list(materials)
        mats = (Material * max(1, len(self.materials)))()
        for k, m in enumerate(self.materials):
            t, dens, p = material_params(m, precision)
            mats[k].type = t
            mats[k].density = float(dens)
            for j in range(len(p)):
                mats[k].p[j] = float(p[j])
        self._mats = mats
        self.bc_list = list(bcs)
        bcarr = (BC * max(1, len(self.bc_list)))()
        self._bc_keep = []
        for k, bc in enumerate(self.bc_list):
            self._fill_bc(bcarr[k], bc, d, nn, npr)
        self._bcs = bcarr

        s = Sim()
        s.grid = g
        s.shape_function = self.sf
        s.nsn = self.nsn
        s.dt = float(npr(dt))
        s.alpha = float(npr(alpha))
        s.small_mass_cutoff = float(npr(1e-9))
        s.global_step = int(global_step)
        s.particles_per_cell = int(particles_per_cell)
        s.num_particles = n
        for k, v in a.items():
            setattr(s, k, v.ctypes.data_as(ctypes.c_void_p))
        s.num_materials = len(self.materials)
        s.materials = ctypes.cast(mats, ctypes.c_void_p)
        s.num_bcs = len(self.bc_list)
        s.bcs = ctypes.cast(bcarr, ctypes.c_void_p)
        s.musl = 1 if musl else 0
        self.s = s

    def _fill_bc(self, c, bc, d, nn, npr):
        t = bc["type"]
        if t == "Gravity":
            c.type = BC_GRAVITY
            g = list(bc["gravity"]) + [0.0] * 3
            ge = list(bc.get("gravity_end", [0.0] * d)) + [0.0] * 3
            for a in range(3):
                c.r[a] = float(npr(g[a]))
                c.r[3 + a] = float(npr(ge[a]))
            c.i[0] = 1 if bc.get("is_ramp", False) else 0
            c.i[1] = int(bc.get("ramp_step", 0))
        elif t == "NodeDomain":
            c.type = BC_NODEDOMAIN
            f0 = list(bc.get("face0_mode", [0] * d)) + [0] * 3
            f1 = list(bc.get("face1_mode", [0] * d)) + [0] * 3
            for a in range(3):
                c.i[a] = int(f0[a])
                c.i[3 + a] = int(f1[a])
        elif t == "BodyForce":
            c.type = BC_BODYFORCE
            c.i[0] = {"forces": 0, "moments": 1, "fixed": 2}[bc["mode"]]
            c.i[1] = 1 if bc.get("is_active", True) else 0
            vals = np.ascontiguousarray(np.asarray(bc["values"], npr).reshape(nn, d))
            mask = np.ascontiguousarray(np.asarray(bc["mask"]).astype(np.uint8).reshape(nn))
            self._bc_keep += [vals, mask]
            c.values = vals.ctypes.data_as(ctypes.c_void_p)
            c.mask = mask.ctypes.data_as(ctypes.c_void_p)
        elif t == "PlanarDomain":
            c.type = BC_PLANARDOMAIN
            f0 = list(bc.get("face0_friction", [0.0] * d)) + [0.0] * 3
            f1 = list(bc.get("face1_friction", [0.0] * d)) + [0.0] * 3
            deg = npr(math.pi / 180.0)
            for a in range(3):
                c.r[a] = float(npr(npr(f0[a]) * deg))
                c.r[3 + a] = float(npr(npr(f1[a]) * deg))
        elif t == "RigidBodyLevelSet" and "shape" not in bc:
            c.type = BC_RIGIDBODY_LEVELSET
            c.i[0] = RIGID_MODES[bc.get("mode", "static")]
            c.i[1] = 1 if bc.get("corrected_rotation", False) else 0
            rate = list(bc.get("euler_angles_per_second", [0.0] * d)) + [0.0] * 3
            com = list(bc.get("COM", [0.0] * d)) + [0.0] * 3
            for a in range(3):
                c.r[a] = float(npr(rate[a])) if a < d else 0.0
                c.r[3 + a] = float(npr(com[a])) if a < d else 0.0
        elif t == "RigidBodyLevelSet":
            c.type = BC_RIGID_SDF
            c.i[0] = SDF_SHAPES[bc["shape"]]
            c.i[1] = int(bc.get("axis", 2)) if d == 3 else 2
            cen = list(bc["center"]) + [0.0] * 3
            vel = list(bc.get("velocity", [0.0] * d)) + [0.0] * 3
            dims = list(bc["dims"]) + [0.0] * 3
            for a in range(3):
                c.r[a] = float(npr(cen[a])) if a < d else 0.0
                c.r[3 + a] = float(npr(vel[a])) if a < d else 0.0
                c.r[8 + a] = float(npr(dims[a])) if (c.i[0] == 1 or a == 0) else 0.0
            c.r[6] = float(npr(bc.get("angular_velocity", 0.0)))
            c.r[7] = float(npr(bc.get("friction", 0.0)))
            c.r[11] = float(npr(bc.get("contact_distance", 0.0)))
            c.r[12] = float(npr(bc.get("angle", 0.0)))
        else:
            raise ValueError(f"unknown boundary condition {t}")

    # --- Solver::Solver set-up (src/solver/solver.cpp:69-104) -------------
    def initialize(self):
        L = self.lib
        L.or_partition(ctypes.byref(self.s))
        L.or_initial_volumes(ctypes.byref(self.s))
        for k, m in enumerate(self.materials):
            _, dens, _ = material_params(m, self.precision)
            L.or_initial_masses(ctypes.byref(self.s), k, self._creal(dens))
        # Drucker-Prager history starts from the current stresses
        self.a["stress_ref"][:] = self.a["stresses"]
        self.a["eps_e"][:] = 0
        # ModifiedCamClay::initialize (src/materials/modifiedcamclay.cpp:68-108),
        # DruckerPragerCap::initialize (src/materials/druckerprager_cap.cpp:72-108):
        # alpha = 0, pc = R p0 with p0 = -tr(sigma)/3, per particle of the colour
        npr = self.npr
        self.a["acc_eps_p"][:] = 0
        for k, m in enumerate(self.materials):
            if m["type"] not in ("ModifiedCamClay", "DruckerPragerCap"):
                continue
            sel = self.a["colors"] == k
            tr = np.trace(self.a["stresses"][sel], axis1=1, axis2=2).astype(np.float64)
            p0 = (-tr / 3.0).astype(npr)
            self.a["pc"][sel] = p0 * npr(m["R"])
        return self

    def _creal(self, v):
        return (ctypes.c_float if self.precision == "f32" else ctypes.c_double)(float(v))

    def call(self, name):
        getattr(self.lib, name)(ctypes.byref(self.s))

    def solve(self, nsteps=1):
        self.lib.or_solve_nsteps(ctypes.byref(self.s), int(nsteps))

    def run(self, total_steps):
        """Solver::run (src/solver/solver.cpp:140-174): total_steps + 1 solves."""
        self.solve(total_steps + 1)

    @property
    def global_step(self):
        return self.s.global_step

    def __getitem__(self, k):
        return self.a[k]


def mcc_point(dim, L, stress, eps_e, stress_ref, alpha, pc, volume, dt, mat, precision="f32"):
    """One Modified Cam Clay (or, for a DruckerPragerCap material, Drucker-
    Prager cap, volume = the original volume) update of a single material
    point: returns the new (stress, eps_e, alpha, pc)."""
    lib = _lib(precision)
    creal, npr = _real(precision)
    _, Material, _, _ = _structs(precision)
    t, dens, p = material_params(mat, precision)
    m = Material()
    m.type = t
    m.density = float(dens)
    for j in range(len(p)):
        m.p[j] = float(p[j])
    Lc = np.ascontiguousarray(np.asarray(L, npr).reshape(dim, dim))
    sig = np.ascontiguousarray(np.asarray(stress, npr).reshape(3, 3).copy())
    eps = np.ascontiguousarray(np.asarray(eps_e, npr).reshape(dim, dim).copy())
    sref = np.ascontiguousarray(np.asarray(stress_ref, npr).reshape(3, 3))
    a = np.array([alpha], npr)
    c = np.array([pc], npr)
    vp = ctypes.c_void_p
    fn = lib.or_dpc_point if mat["type"] == "DruckerPragerCap" else lib.or_mcc_point
    fn(dim, Lc.ctypes.data_as(vp), sig.ctypes.data_as(vp), eps.ctypes.data_as(vp), sref.ctypes.data_as(vp),
       a.ctypes.data_as(vp), c.ctypes.data_as(vp), creal(volume), creal(dt), ctypes.byref(m))
    return sig, eps, a[0], c[0]


def dp_point(dim, L, stress, eps_e, stress_ref, dt, mat, precision="f32", velgrad_is_strain_increment=False):
    """One Drucker-Prager stress update of a single material point."""
    lib = _lib(precision)
    creal, npr = _real(precision)
    _, _, p = material_params(mat, precision)
    Lc = np.ascontiguousarray(np.asarray(L, npr).reshape(dim, dim))
    sig = np.ascontiguousarray(np.asarray(stress, npr).reshape(3, 3).copy())
    eps = np.ascontiguousarray(np.asarray(eps_e, npr).reshape(dim, dim).copy())
    sref = np.ascontiguousarray(np.asarray(stress_ref, npr).reshape(3, 3))
    pa = np.asarray(p, npr)
    vp = ctypes.c_void_p
    lib.or_dp_point(dim, Lc.ctypes.data_as(vp), sig.ctypes.data_as(vp), eps.ctypes.data_as(vp),
                    sref.ctypes.data_as(vp), creal(dt), pa.ctypes.data_as(vp),
                    1 if velgrad_is_strain_increment else 0)
    return sig, eps
