"""Synthetic particle sets of the benchmark configurations (seeded, no data files).

Each builder returns a dict with the grid, the particles and the solver
settings, in the form both the C ABI ``Simulation`` and the oracle take.
Sizes follow the configuration descriptions; ``scale`` shrinks the particle
region (same cell size, same particle spacing) for quick parity runs.
"""
from __future__ import annotations

import numpy as np


def _lattice(lo, hi, spacing):
    """Points at (i + 1/2) * spacing inside [lo, hi) per axis (x fastest)."""
    axes = []
    for a in range(len(lo)):
        n = int(np.floor((hi[a] - lo[a]) / spacing + 1e-9))
        axes.append(lo[a] + (np.arange(n) + 0.5) * spacing)
    mesh = np.meshgrid(*axes[::-1], indexing="ij")
    pts = np.stack([m.ravel() for m in mesh[::-1]], axis=1)
    return pts


def two_discs(cell_size=0.02, radius=0.2, centers=((0.25, 0.25), (0.75, 0.75)), ppc_1d=2, speed=0.1,
              E=1000.0, pois=0.3, density=1000.0, dt=1e-3, alpha=0.99):
    """Two elastic discs moving toward each other on [0,1]^2 (linear shape
    functions): 2x2 particles per cell on the sub-cell lattice."""
    spacing = cell_size / ppc_1d
    pos, vel = [], []
    for k, c in enumerate(centers):
        c = np.asarray(c, np.float64)
        lo = np.floor((c - radius) / spacing) * spacing
        hi = np.ceil((c + radius) / spacing) * spacing
        pts = _lattice(lo, hi, spacing)
        inside = ((pts - c) ** 2).sum(axis=1) < radius ** 2
        pts = pts[inside]
        pos.append(pts)
        vel.append(np.full_like(pts, speed if k == 0 else -speed))
    return dict(dim=2, origin=[0.0, 0.0], end=[1.0, 1.0], cell_size=cell_size, shape_function="linear",
                dt=dt, particles_per_cell=ppc_1d ** 2, alpha=alpha,
                materials=[{"type": "LinearElastic", "density": density, "E": E, "pois": pois}], bcs=[],
                positions=np.concatenate(pos), velocities=np.concatenate(vel))


def water_column(cell_size=0.02, block=(0.4, 0.6), domain=(1.0, 1.0), ppc_1d=2, dt=1e-4, viscosity=1e-3,
                 bulk_modulus=2e6, gamma=7.0, density=1000.0, shape_function="quadratic"):
    """2D water block in the corner of a box (Newtonian fluid, gravity, slip
    walls), as the reference's water example sets it up."""
    spacing = cell_size / ppc_1d
    pts = _lattice(np.zeros(2), np.asarray(block, np.float64), spacing)
    return dict(dim=2, origin=[0.0, 0.0], end=list(domain), cell_size=cell_size, shape_function=shape_function,
                dt=dt, particles_per_cell=ppc_1d ** 2, alpha=0.99,
                materials=[{"type": "NewtonFluid", "density": density, "viscosity": viscosity,
                            "bulk_modulus": bulk_modulus, "gamma": gamma}],
                bcs=[{"type": "Gravity", "gravity": [0.0, -9.81]},
                     {"type": "NodeDomain", "face0_mode": [1, 1], "face1_mode": [1, 1]}],
                positions=pts, velocities=np.zeros_like(pts))


def granular_column(domain=(1.0, 0.25, 0.5), cell_size=1.0 / 256, column=(0.2, 0.25, 0.2), ppc_1d=2,
                    jitter=0.25, seed=0, shape_function="quadratic", dt=1e-5, scale=1.0,
                    density=1500.0, E=1.0e7, pois=0.3, friction_angle=30.0, dilatancy_angle=0.0, cohesion=0.0):
    """3D granular column against the x = 0 wall, Drucker-Prager, gravity,
    slip walls on all faces.  Particles on a (ppc_1d)^3 lattice per cell,
    each coordinate jittered uniformly by +-jitter * spacing (numpy PCG64)."""
    spacing = cell_size / ppc_1d
    col = np.asarray(column, np.float64) * scale
    pts = _lattice(np.zeros(3), col, spacing)
    rng = np.random.Generator(np.random.PCG64(seed))
    pts = pts + rng.uniform(-jitter * spacing, jitter * spacing, size=pts.shape)
    return dict(dim=3, origin=[0.0, 0.0, 0.0], end=list(domain), cell_size=cell_size,
                shape_function=shape_function, dt=dt, particles_per_cell=ppc_1d ** 3, alpha=0.99,
                materials=[{"type": "DruckerPrager", "density": density, "E": E, "pois": pois,
                            "friction_angle": friction_angle, "dilatancy_angle": dilatancy_angle,
                            "cohesion": cohesion}],
                bcs=[{"type": "Gravity", "gravity": [0.0, 0.0, -9.81]},
                     {"type": "NodeDomain", "face0_mode": [1, 1, 1], "face1_mode": [1, 1, 1]}],
                positions=pts, velocities=np.zeros_like(pts))


def scoop(center=(0.15, 0.25, 0.3), radius=0.15, thickness=0.01, length=0.4, velocity=(0.5, 0.0, 0.0),
          angular_velocity=1.0, friction=0.3, angle=0.0, axis=1):
    """Half-cylinder shell rigid body (RigidBodyLevelSet with an analytic
    signed distance): axis along y, the shell on the -x side of its axis at
    angle 0 (open towards +x), translating and turning about its axis."""
    return {"type": "RigidBodyLevelSet", "shape": "half_cylinder_shell", "axis": axis, "center": list(center),
            "velocity": list(velocity), "angular_velocity": angular_velocity, "angle": angle,
            "dims": [radius, thickness, length], "friction": friction, "contact_distance": 0.0}


def granular_bed(domain=(1.5, 0.6, 0.8), cell_size=1.0 / 160, bed=(1.0, 0.5, 0.3), ppc_1d=2, jitter=0.25,
                 seed=1, shape_function="cubic", dt=8e-6, scale=1.0, with_scoop=True, **kw):
    """3D granular bed dug by a translating, turning half-cylinder scoop
    (R 0.15, t 0.01, L 0.4, 0.5 m/s in x, 1 rad/s, Coulomb 0.3); Drucker-Prager,
    gravity, slip walls.  The scoop's axis sits at the bed's top, offset from
    the node lattice by (0.37, 0.21, 0.43) cells: on a node line, nodes would
    lie exactly on the shell's mid-surface and its end caps' centre lines,
    where the contact normal flips direction with the last bit of rounding."""
    spacing = cell_size / ppc_1d
    b = np.asarray(bed, np.float64) * scale
    pts = _lattice(np.zeros(3), b, spacing)
    rng = np.random.Generator(np.random.PCG64(seed))
    pts = pts + rng.uniform(-jitter * spacing, jitter * spacing, size=pts.shape)
    d = granular_column(domain=domain, cell_size=cell_size, shape_function=shape_function, dt=dt, **kw)
    d.update(positions=pts, velocities=np.zeros_like(pts))
    if with_scoop:
        top = float(b[2])
        off = np.array([0.37, 0.21, 0.43]) * cell_size
        body = scoop(center=tuple(np.array([0.15 * scale, 0.5 * float(b[1]), top]) + off), radius=0.15 * scale,
                     thickness=max(0.01 * scale, 1.5 * cell_size), length=0.8 * float(b[1]))
        d["bcs"] = [d["bcs"][0], body, d["bcs"][1]]
    return d


def _wave_timestep(mat, h, cfl):
    """cfl * h / c with the p-wave speed c = sqrt((K + 4G/3) / rho), K and G in
    FP32 as the material constructors, the root in double (tools.cpp:373-380);
    a Newtonian fluid has G = 0."""
    f = np.float32
    rho = float(mat["density"])
    if mat["type"] == "NewtonFluid":
        K, G = f(mat["bulk_modulus"]), f(0.0)
    else:
        E, nu = f(mat["E"]), f(mat.get("pois", 0.0))
        K = E / (f(3) * (f(1) - f(2) * nu))
        G = E / (f(2) * (f(1) + nu))
    c = f(np.sqrt((float(K) + 4.0 * float(G) / 3.0) / rho))
    return float(f(cfl) * (f(h) / c))


def ensemble(num=256, seed=3, shape_function="quadratic", np_range=(2000, 64000), grid_range=(64, 512), cfl=0.3):
    """Batched-ensemble instances: 2D column collapses (even instances) and
    disc impacts (odd), particle counts log-uniform in np_range, grids of
    G x G nodes on [0,1]^2 with G log-uniform in grid_range, materials cycled
    linear elastic (E ~ U[1, 20] MPa, nu 0.3) / Newtonian fluid (mu 1e-3,
    K 2e6) / Drucker-Prager (E ~ U[1, 20] MPa, phi ~ U[20, 40] deg), dt from
    each instance's CFL number.  Particles sit on a regular sub-cell lattice
    of 2x2 to 4x4 per cell; where the grid cannot hold the drawn count with
    at most 4x4 per cell over the scene's region, the count is the most it
    holds."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for i in range(num):
        target = float(np.exp(rng.uniform(np.log(np_range[0]), np.log(np_range[1]))))
        G = int(round(np.exp(rng.uniform(np.log(grid_range[0]), np.log(grid_range[1])))))
        h = 1.0 / (G - 1)
        E = float(rng.uniform(1e6, 20e6))
        phi = float(rng.uniform(20.0, 40.0))
        kind = i % 3
        if kind == 0:
            mat = {"type": "LinearElastic", "density": 1000.0, "E": E, "pois": 0.3}
        elif kind == 1:
            mat = {"type": "NewtonFluid", "density": 1000.0, "viscosity": 1e-3, "bulk_modulus": 2e6, "gamma": 7.0}
        else:
            mat = {"type": "DruckerPrager", "density": 1500.0, "E": E, "pois": 0.3, "friction_angle": phi,
                   "dilatancy_angle": 0.0, "cohesion": 0.0}
        column = i % 2 == 0
        region = 0.18 if column else 0.2  # area the scene's bodies may cover
        ppc_1d = 2
        while ppc_1d < 4 and target * (h / ppc_1d) ** 2 > region:
            ppc_1d += 1
        sp = h / ppc_1d
        area = min(target * sp * sp, region)
        if column:
            w = float(np.sqrt(area / 2.0))
            pts = _lattice(np.array([h, h]), np.array([h + w, h + 2.0 * w]), sp)
            vel = np.zeros_like(pts)
            bcs = [{"type": "Gravity", "gravity": [0.0, -9.81]},
                   {"type": "NodeDomain", "face0_mode": [1, 1], "face1_mode": [1, 1]}]
        else:
            r = float(np.sqrt(area / (2.0 * np.pi)))
            pts, vel = [], []
            for k, c in enumerate(((0.3, 0.3), (0.7, 0.7))):
                c = np.asarray(c)
                lo = np.floor((c - r) / sp) * sp
                p = _lattice(lo, lo + 2 * r + 2 * sp, sp)
                p = p[((p - c) ** 2).sum(axis=1) < r * r]
                pts.append(p)
                vel.append(np.full_like(p, 0.5 if k == 0 else -0.5))
            pts, vel = np.concatenate(pts), np.concatenate(vel)
            bcs = [{"type": "NodeDomain", "face0_mode": [1, 1], "face1_mode": [1, 1]}]
        out.append(dict(dim=2, origin=[0.0, 0.0], end=[1.0, 1.0], cell_size=h, shape_function=shape_function,
                        dt=_wave_timestep(mat, h, cfl), particles_per_cell=ppc_1d * ppc_1d, alpha=0.99,
                        materials=[mat], bcs=bcs, positions=pts, velocities=vel))
    return out


def calibration_cube(n_side=64, cell_size=1.0 / 128, domain=0.5, seed=2, dt=2e-5, E_median=5e6, E_sigma=0.2,
                     phi_mean=25.0, phi_std=3.0, target_E=1e7, target_phi=30.0):
    """Differentiable-calibration cube: n_side^3 particles on a 2x2x2 lattice
    per cell (side n_side/2 cells) standing on the floor of a domain^3 box,
    Drucker-Prager (rho 1500, nu 0.3, psi 0, c 0), quadratic B-splines,
    gravity, slip walls.  Returns the scene with the initial per-particle
    parameters (E log-normal around E_median, phi normal, numpy PCG64 `seed`)
    and the target parameters."""
    spacing = cell_size / 2
    side = n_side * spacing
    lo = np.array([0.5 * (domain - side), 0.5 * (domain - side), 0.0])
    pts = _lattice(lo, lo + side, spacing)
    rng = np.random.Generator(np.random.PCG64(seed))
    E = E_median * np.exp(rng.normal(0.0, E_sigma, len(pts)))
    phi = rng.normal(phi_mean, phi_std, len(pts))
    scene = dict(dim=3, origin=[0.0, 0.0, 0.0], end=[domain] * 3, cell_size=cell_size,
                 shape_function="quadratic", dt=dt, particles_per_cell=8, alpha=0.99,
                 materials=[{"type": "DruckerPrager", "density": 1500.0, "E": target_E, "pois": 0.3,
                             "friction_angle": target_phi, "dilatancy_angle": 0.0, "cohesion": 0.0}],
                 bcs=[{"type": "Gravity", "gravity": [0.0, 0.0, -9.81]},
                      {"type": "NodeDomain", "face0_mode": [1, 1, 1], "face1_mode": [1, 1, 1]}],
                 positions=pts, velocities=np.zeros_like(pts))
    return scene, E.astype(np.float32), phi.astype(np.float32), (target_E, target_phi)


def sim_kwargs(scene):
    """Keyword arguments of Simulation / OracleSim from a scene dict."""
    keys = ["dim", "origin", "end", "cell_size", "shape_function", "dt", "particles_per_cell", "alpha",
            "materials", "bcs"]
    return {k: scene[k] for k in keys}
