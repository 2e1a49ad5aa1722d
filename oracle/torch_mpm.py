"""Plain-PyTorch restatement of the USL step for gradient checks (test
infrastructure, like the C oracle: only tests import it).

A small FP64 MPM whose torch.autograd gradient is the reference the CUDA
adjoint (pmpm_rollout_backward) is checked against: 3D, quadratic B-splines
with the 4-wide window and the boundary fold of the C oracle
(oracle.c: window_offset, slot_target, sf_quadratic / sf_dquadratic), P2G
with the 1e-9 node-mass cutoff (usl_inline.h:82-180 as oracle.c: or_p2g),
gravity and NodeDomain in list order (gravity.cpp:65-88,
nodedomain_inline.h:40-87), G2P with the FLIP/PIC blend, x += dt v_pic,
F = (I + L dt) F and V = det(F) V0 (usl_inline.h:245-332), then the
Drucker-Prager cone / apex return mapping of update_dp_rheo
(dp_rheo_inline.h:123-246 as oracle.c: or_dp_point) with per-particle
Young's modulus and friction angle (oracle.c: dp_particle_params).
Every particle-node pair is a dense tensor entry, so only small particle
sets (hundreds to a few thousand) are practical.
"""
from __future__ import annotations

import math

import numpy as np
import torch

CUTOFF = 1e-9      # NodesContainer small_mass_cutoff
SLIP_CUTOFF = 1e-5  # apply_nodedomain skips lighter nodes


def _quadratic(r, inv_h):
    """sf_quadratic and sf_dquadratic (uniform C1 quadratic B-spline)."""
    ar = r.abs()
    inner = ar < 0.5
    outer = (ar >= 0.5) & (ar < 1.5)
    t = 1.5 - ar
    N = torch.where(inner, 0.75 - r * r, torch.where(outer, 0.5 * t * t, torch.zeros_like(r)))
    dN = torch.where(inner, -2.0 * r, torch.where(outer, torch.where(r > 0, -t, t), torch.zeros_like(r))) * inv_h
    return N, dN


class TorchMPM:
    """One 3D quadratic USL simulation with per-particle Drucker-Prager
    parameters.  scene: the dict of pyroclastmpm_b200.scenes (origin, end,
    cell_size, dt, particles_per_cell, alpha, materials[0] Drucker-Prager,
    bcs: Gravity / NodeDomain)."""

    def __init__(self, scene):
        assert scene["dim"] == 3 and scene["shape_function"] == "quadratic"
        self.dt = float(scene["dt"])
        self.alpha = float(scene["alpha"])
        self.h = float(scene["cell_size"])
        self.inv_h = float(np.float32(1.0) / np.float32(self.h))  # Grid::inv_cell_size, FP32 as the step
        self.origin = torch.tensor(scene["origin"], dtype=torch.float64)
        self.n = [int(np.float32(np.float32(scene["end"][a]) - np.float32(scene["origin"][a])) / np.float32(self.h))
                  + 1 for a in range(3)]
        self.nn = self.n[0] * self.n[1] * self.n[2]
        self.ppc = int(scene["particles_per_cell"])
        mat = scene["materials"][0]
        assert mat["type"] == "DruckerPrager"
        self.density = float(mat["density"])
        self.nu = float(mat["pois"])
        self.cohesion = float(mat.get("cohesion", 0.0))
        psi = math.radians(float(mat.get("dilatancy_angle", 0.0)))
        self.eta_bar = 6.0 * math.sin(psi) / (math.sqrt(3.0) * (3.0 + math.sin(psi)))
        self.gravity = None
        self.walls = None
        for bc in scene["bcs"]:
            if bc["type"] == "Gravity":
                self.gravity = torch.tensor(bc["gravity"], dtype=torch.float64)
            elif bc["type"] == "NodeDomain":
                self.walls = (list(bc["face0_mode"]), list(bc["face1_mode"]))
            else:
                raise ValueError(bc["type"])
        self.bc_order = [bc["type"] for bc in scene["bcs"]]
        w = torch.arange(-1, 3)
        wz, wx, wy = torch.meshgrid(w, w, w, indexing="ij")  # slot order: z fastest, then x, then y
        self.win = torch.stack([wx.reshape(-1), wy.reshape(-1), wz.reshape(-1)], dim=1)  # [64, 3]

    def initial_state(self, x0, v0):
        """Particle state after Solver set-up: V = h^3 / ppc, m = rho V,
        F = I, zero stress and elastic strain."""
        n = x0.shape[0]
        vol = self.h ** 3 / self.ppc
        V0 = torch.full((n,), vol, dtype=torch.float64)
        return {"x": x0, "v": v0, "F": torch.eye(3, dtype=torch.float64).expand(n, 3, 3).clone(),
                "sig": torch.zeros(n, 3, 3, dtype=torch.float64), "eps": torch.zeros(n, 3, 3, dtype=torch.float64),
                "V": V0.clone(), "V0": V0, "m": self.density * V0}

    def _weights(self, x):
        u = (x - self.origin) * self.inv_h
        b = torch.floor(u.detach()).long()  # positive coordinates: truncation = floor
        sel = b[:, None, :] + self.win[None, :, :]                     # [n, 64, 3]
        hi = torch.tensor(self.n) - 1
        tgt = torch.minimum(torch.clamp(sel, min=0), hi)               # the fold onto the grid
        r = u[:, None, :] - sel.double()
        N, dN = _quadratic(r, self.inv_h)
        psi = N[..., 0] * N[..., 1] * N[..., 2]
        dpsi = torch.stack([dN[..., 0] * N[..., 1] * N[..., 2], dN[..., 1] * N[..., 0] * N[..., 2],
                            dN[..., 2] * N[..., 0] * N[..., 1]], dim=-1)
        node = tgt[..., 0] + tgt[..., 1] * self.n[0] + tgt[..., 2] * self.n[0] * self.n[1]
        return psi, dpsi, node, tgt

    def _dp(self, L, eps, E, phi_deg):
        """Drucker-Prager cone / apex return (reference stress zero: the
        history starts from an unstressed state)."""
        dt = self.dt
        nu = self.nu
        K = E / (3.0 * (1.0 - 2.0 * nu))
        G = E / (2.0 * (1.0 + nu))
        phi = phi_deg * (math.pi / 180.0)
        sn, cs = torch.sin(phi), torch.cos(phi)
        eta = 6.0 * sn / (math.sqrt(3.0) * (3.0 - sn))
        xi = 6.0 * cs / (math.sqrt(3.0) * (3.0 - sn))
        kc = xi * self.cohesion
        p_apex = torch.where(eta > 0, kc / torch.where(eta > 0, eta, torch.ones_like(eta)), torch.zeros_like(eta))
        Lt = L.transpose(1, 2)
        deps = 0.5 * (L + Lt) * dt
        W = 0.5 * (L - Lt) * dt
        deps = deps - W @ eps + eps @ W
        eps_tr = eps + deps
        ev = eps_tr.diagonal(dim1=1, dim2=2).sum(-1)
        I = torch.eye(3, dtype=torch.float64)
        p_tr = K * ev
        s_tr = 2.0 * G[:, None, None] * (eps_tr - (ev / 3.0)[:, None, None] * I)
        J2 = 0.5 * (s_tr * s_tr).sum((1, 2))
        sqrtJ2 = torch.sqrt(torch.clamp(J2, min=1e-300))
        Phi = sqrtJ2 + eta * p_tr - kc
        plastic = Phi > 0
        dgamma = torch.where(plastic, Phi, torch.zeros_like(Phi)) / (K * eta * self.eta_bar + G)
        p_pl = p_tr - K * self.eta_bar * dgamma
        apex = plastic & (eta > 0) & (sqrtJ2 - G * dgamma < 0)
        scale = torch.where(plastic & ~apex, 1.0 - G * dgamma / sqrtJ2, torch.ones_like(sqrtJ2))
        s_new = torch.where(apex[:, None, None], torch.zeros_like(s_tr), scale[:, None, None] * s_tr)
        p_new = torch.where(apex, p_apex, torch.where(plastic, p_pl, p_tr))
        sig = s_new + p_new[:, None, None] * I
        eps_new = torch.where(plastic[:, None, None],
                              s_new / (2.0 * G[:, None, None]) + (p_new / (3.0 * K))[:, None, None] * I, eps_tr)
        return sig, eps_new

    def step(self, st, E, phi_deg):
        x, v, F, sig, eps, V, V0, m = (st[k] for k in ("x", "v", "F", "sig", "eps", "V", "V0", "m"))
        n = x.shape[0]
        dt = self.dt
        psi, dpsi, node, tgt = self._weights(x)
        flat = node.reshape(-1)
        # ---- P2G ----
        sm = psi * m[:, None]
        mass = torch.zeros(self.nn, dtype=torch.float64).index_add(0, flat, sm.reshape(-1))
        mom = torch.zeros(self.nn, 3, dtype=torch.float64).index_add(
            0, flat, (sm[..., None] * v[:, None, :]).reshape(-1, 3))
        f = -V[:, None, None] * torch.einsum("pab,psb->psa", sig, dpsi)
        force = torch.zeros(self.nn, 3, dtype=torch.float64).index_add(0, flat, f.reshape(-1, 3))
        live = mass > CUTOFF
        mass = torch.where(live, mass, torch.zeros_like(mass))
        mom = torch.where(live[:, None], mom, torch.zeros_like(mom))
        mnt = torch.where(live[:, None], mom + force * dt, torch.zeros_like(mom))
        # ---- node conditions in list order ----
        ids = torch.stack(torch.meshgrid(torch.arange(self.n[0]), torch.arange(self.n[1]), torch.arange(self.n[2]),
                                         indexing="ij"), dim=-1).permute(2, 1, 0, 3).reshape(-1, 3)
        for kind in self.bc_order:
            if kind == "Gravity":
                mnt = mnt + torch.where(live[:, None], self.gravity[None, :] * mass[:, None] * dt, torch.zeros_like(mnt))
            else:
                heavy = mass > SLIP_CUTOFF
                f0, f1 = self.walls
                for a in range(3):
                    lo = heavy & (ids[:, a] < 1)
                    hi = heavy & (ids[:, a] >= self.n[a] - 1)
                    for arr_name in ("mom", "mnt"):
                        arr = mom if arr_name == "mom" else mnt
                        col = arr[:, a]
                        if f0[a] == 1:
                            col = torch.where(lo, torch.clamp(col, min=0.0), col)
                        if f1[a] == 1:
                            col = torch.where(hi, torch.clamp(col, max=0.0), col)
                        arr = torch.cat([arr[:, :a], col[:, None], arr[:, a + 1:]], dim=1)
                        if f0[a] == 0:
                            arr = torch.where(lo[:, None], torch.zeros_like(arr), arr)
                        if f1[a] == 0:
                            arr = torch.where(hi[:, None], torch.zeros_like(arr), arr)
                        if arr_name == "mom":
                            mom = arr
                        else:
                            mnt = arr
        # ---- G2P ----
        mg = mass[node]                                           # [n, 64]
        ok = mg > CUTOFF
        safe = torch.where(ok, mg, torch.ones_like(mg))
        vn = mom[node] / safe[..., None]
        vnt = mnt[node] / safe[..., None]
        w = torch.where(ok, psi, torch.zeros_like(psi))
        wd = torch.where(ok[..., None], dpsi, torch.zeros_like(dpsi))
        dv = (w[..., None] * (vnt - vn)).sum(1)
        vpic = (w[..., None] * vnt).sum(1)
        L = torch.einsum("psa,psc->pac", wd, vnt)
        v_new = (1.0 - self.alpha) * vpic + self.alpha * (v + dv)
        x_new = x + dt * vpic
        I = torch.eye(3, dtype=torch.float64)
        F_new = (I + L * dt) @ F
        V_new = torch.linalg.det(F_new) * V0
        sig_new, eps_new = self._dp(L, eps, E, phi_deg)
        return {"x": x_new, "v": v_new, "F": F_new, "sig": sig_new, "eps": eps_new, "V": V_new, "V0": V0, "m": m}

    def rollout(self, x0, v0, E, phi_deg, steps):
        st = self.initial_state(x0, v0)
        for _ in range(steps):
            st = self.step(st, E, phi_deg)
        return st
