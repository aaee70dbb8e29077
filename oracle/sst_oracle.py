"""ORACLE — test infrastructure only. Never imported by the product (``gputest_b200``).

A CPU restatement, in NumPy/SciPy, of the k-omega SST model (Menter, Kuntz & Langtry 2003)
of FlowTrace's unstructured solver (``flowtrace/unstructured/turbulence.py:65-438``), as
``OracleSimple`` (``oracle/simplec_oracle.py``) drives it: the effective face viscosities of
the momentum equations (mu + mu_t inside, Spalding's law-of-the-wall viscosity on walls), the
explicit transpose-stress source, the turbulent energy diffusivity, and after the energy
equation one transport solve each of k and omega followed by the mu_t update.

Operations follow the reference's NumPy path in the same order, so results agree with it to
round-off. Pinned against the reference itself: ``tests/golden/make_sst_golden.py`` runs the
reference's SST solver on the cases of ``tests/golden/sst_cases.py`` and stores its fields,
residuals, wall distances and face viscosities; ``tests/test_oracle_sst.py`` re-checks this
restatement against them.
"""

from __future__ import annotations

import math
from typing import Dict

import numpy as np

KAPPA = 0.41          # turbulence.py:51 (SST and Spalding's law)
E_WALL = 9.793        # turbulence.py:55
B_SPALDING = 5.2      # turbulence.py:56
CMU = 0.09            # turbulence.py:57
PR_T = 0.85           # turbulence.py:59


def spalding_uplus(re_y, iters: int = 30):
    """u+ from Spalding's law y+ = u+ + e^{-kB}(e^{ku+} - 1 - ku+ - (ku+)^2/2 - (ku+)^3/6) with
    y+ = Re_y / u+, by Newton's method on f(u+) = Re_y/u+ - y+(u+) (``turbulence.py:65-87``):
    start at sqrt(Re_y) below Re_y = 120, else at the log law; each step at most halves u+; stop
    when every face's step is below 1e-10 u+."""
    ry = np.maximum(np.asarray(re_y, dtype=float), 0.0)
    kap, eb = KAPPA, math.exp(-KAPPA * B_SPALDING)
    u = np.where(ry < 120.0, np.sqrt(np.maximum(ry, 1e-300)),
                 np.log(np.maximum(E_WALL * np.sqrt(np.maximum(ry, 1.0)), 1.0)) / kap + 1.0)
    for _ in range(iters):
        x = np.minimum(kap * u, 60.0)
        ex = np.exp(x)
        yplus = u + eb * (ex - 1 - x - x ** 2 / 2 - x ** 3 / 6)
        dyplus = 1 + eb * kap * (ex - 1 - x - x ** 2 / 2)
        uc = np.maximum(u, 1e-300)
        f = ry / uc - yplus
        df = -ry / uc ** 2 - dyplus
        du = f / df
        u = np.maximum(u - du, 0.5 * u)
        if np.all(np.abs(du) <= 1e-10 * np.maximum(u, 1e-12)):
            break
    return np.where(ry > 0, u, 0.0)


def strain_rate(gU, dim):
    """|S| = sqrt(2 S_ij S_ij), S_ij = (du_i/dx_j + du_j/dx_i)/2 (``turbulence.py:99-113``)."""
    acc = 0.0
    for i in range(dim):
        for j in range(dim):
            acc = acc + (0.5 * (gU[i][:, j] + gU[j][:, i])) ** 2
    return np.sqrt(2.0 * acc)


def wall_distance(solver):
    """Distance of every cell centre to the nearest wall face (``turbulence.py:191-229``): the
    eight nearest wall-face centres (k-d tree) are the candidates; in 2-D the exact distance to
    each candidate segment, in 3-D the distance to a disc of 1.2 x the face's equal-area radius
    in the face plane. 1e30 everywhere when the mesh has no wall."""
    from scipy.spatial import cKDTree

    mesh, fv = solver.mesh, solver.fv
    xc = fv.cell_centre
    wall_ids = [z.id for z in mesh.boundary_zones() if solver.zone_specs[z.name].kind == "wall"]
    wf = np.nonzero(np.isin(mesh.face_zone, wall_ids))[0]
    if wf.size == 0:
        return np.full(solver.nc, 1e30)
    fc_all, S_all = fv.face_centre, fv.face_area_vec
    fc = fc_all[wf]
    kq = min(8, wf.size)
    _, near = cKDTree(fc).query(xc, k=kq)
    near = np.atleast_2d(near).reshape(xc.shape[0], kq)
    best = np.full(xc.shape[0], np.inf)
    if mesh.dim == 2:
        a = mesh.nodes[mesh.face_nodes[mesh.face_ptr[wf]]]
        b = mesh.nodes[mesh.face_nodes[mesh.face_ptr[wf] + 1]]
        for j in range(kq):
            f = near[:, j]
            seg = b[f] - a[f]
            t = np.clip(np.einsum("cd,cd->c", xc - a[f], seg) / np.maximum(np.einsum("cd,cd->c", seg, seg), 1e-300), 0, 1)
            best = np.minimum(best, np.linalg.norm(xc - (a[f] + t[:, None] * seg), axis=1))
    else:
        nrm = S_all[wf]
        area = np.linalg.norm(nrm, axis=1)
        nrm = nrm / area[:, None]
        rad = np.sqrt(area / np.pi) * 1.2
        for j in range(kq):
            f = near[:, j]
            v = xc - fc[f]
            along = np.einsum("cd,cd->c", v, nrm[f])
            dn = np.abs(along)
            dt = np.linalg.norm(v - along[:, None] * nrm[f], axis=1)
            best = np.minimum(best, np.where(dt <= rad[f], dn, np.sqrt(dn ** 2 + (dt - rad[f]) ** 2)))
    return np.maximum(best, 1e-300)


class OracleSST:
    """k-omega SST state and equations of one ``OracleSimple`` (``turbulence.py:116-438``)."""

    sk1, sw1, b1 = 0.85, 0.5, 0.075                                                 # turbulence.py:356-359
    sk2, sw2, b2 = 1.0, 0.856, 0.0828
    bstar, a1 = 0.09, 0.31
    g1 = b1 / bstar - sw1 * KAPPA ** 2 / math.sqrt(bstar)
    g2 = b2 / bstar - sw2 * KAPPA ** 2 / math.sqrt(bstar)
    relax_default = 0.8
    field_name = "specific-diss-rate"

    def __init__(self, s):
        """``turbulence.py:123-186``."""
        from .simplec_oracle import INLET, OUTLET, PRESSURE, WALL

        self.s = s
        fv, c = s.fv, s.case
        self.rho, self.mu = c.density, c.viscosity
        self.nu = self.mu / self.rho
        self.wall_b = s.bkind == WALL
        self.inlet_b = s.bkind == INLET
        self.open_b = (s.bkind == OUTLET) | (s.bkind == PRESSURE)
        self.yb = np.abs(np.einsum("fd,fd->f", fv.db, fv.nb))      # owner centre to wall face, normal
        self.y = wall_distance(s)
        wf = np.nonzero(self.wall_b)[0]
        self.wall_faces = wf
        self.wall_cells = np.unique(fv.Pb[wf])
        ywc = np.full(s.nc, np.inf)
        np.minimum.at(ywc, fv.Pb[wf], self.yb[wf])
        self.y_wall_cell = ywc
        if self.wall_cells.size:
            self.y[self.wall_cells] = ywc[self.wall_cells]
        speed = np.linalg.norm(s.ub_fixed, axis=1)
        u_ref = float(speed[self.inlet_b].max()) if self.inlet_b.any() else float(c.turb_reference_velocity or 1.0)
        self.u_ref = max(u_ref, 1e-6)
        kin, win = np.zeros(fv.n_bf), np.zeros(fv.n_bf)
        for z in s.mesh.boundary_zones():
            spec = s.zone_specs[z.name]
            m = fv.bzone == z.id
            inten = spec.turb_intensity if spec.turb_intensity is not None else c.turb_intensity
            ratio = spec.turb_viscosity_ratio if spec.turb_viscosity_ratio is not None else c.turb_viscosity_ratio
            U = np.where(speed[m] > 0, speed[m], self.u_ref)
            kz = 1.5 * (inten * U) ** 2 if spec.k is None else np.full(m.sum(), spec.k)
            kin[m] = np.maximum(kz, 1e-12 * self.u_ref ** 2)
            win[m] = self._omega_from(kin[m], ratio, spec.omega)
        self.kb_in, self.sb_in = kin, win
        init = c.turb_init or {}
        k0 = init.get("k", 1.5 * (c.turb_intensity * self.u_ref) ** 2)
        w0 = init.get("omega", float(self._omega_from(np.array([k0]), c.turb_viscosity_ratio, None)[0]))
        self.k = np.full(s.nc, k0, dtype=np.float64)
        self.w = np.full(s.nc, w0, dtype=np.float64)
        self.k_min = 1e-14 * self.u_ref ** 2
        self.w_min = 1e-14
        self.relax_k = c.relax_k if c.relax_k is not None else self.relax_default
        self.relax_w = c.relax_w if c.relax_w is not None else self.relax_default
        self.yplus = np.zeros(fv.n_bf)
        self.mut = self.rho * self.k / self.w

    def _omega_from(self, k, ratio, explicit):
        """omega = rho k / (mu ratio), or the explicit value (``turbulence.py:362-365``)."""
        if explicit is not None:
            return np.full(np.shape(k), float(explicit))
        return self.rho * np.asarray(k) / (self.mu * ratio)

    # ---- what the flow equations take from the model ------------------------------------------
    def wall_viscosity(self, U):
        """Per boundary face: on walls mu Re_y / u+^2 from Spalding's law with the owner cell's
        wall-parallel speed relative to the wall (so that tau_w = mu_w u_t / y); records y+
        (``turbulence.py:399-417``)."""
        fv = self.s.fv
        rel = U[fv.Pb] - self.s.ub_fixed
        ut = np.linalg.norm(rel - np.einsum("fd,fd->f", rel, fv.nb)[:, None] * fv.nb, axis=1)
        re_y = ut * self.yb / self.nu
        up = spalding_uplus(re_y)
        ok = (re_y > 1e-12) & (up > 0)
        mu_w = np.full(re_y.shape, self.mu)
        mu_w[ok] = self.mu * re_y[ok] / up[ok] ** 2
        yp = np.zeros(re_y.shape)
        yp[ok] = re_y[ok] / up[ok]
        self.yplus = np.where(self.wall_b, yp, 0.0)
        return np.where(self.wall_b, mu_w, self.mu)

    def momentum_viscosity(self, U):
        """(interior faces: mu + interpolated mu_t, boundary faces: mu + mu_t of the owner, the
        wall viscosity on walls) (``turbulence.py:235-243``)."""
        fv = self.s.fv
        mut_f = fv.face_interp(self.mut)
        mub = self.mu + self.mut[fv.Pb]
        mub = np.where(self.wall_b, self.wall_viscosity(U), mub)
        return self.mu + mut_f, mub

    def energy_diffusivity(self, k_over_cp):
        """k/cp + mu_t/Pr_t on faces; walls keep k/cp (``turbulence.py:245-249``)."""
        fv = self.s.fv
        mut_f = fv.face_interp(self.mut)
        gb = k_over_cp + np.where(self.wall_b, 0.0, self.mut[fv.Pb] / PR_T)
        return k_over_cp + mut_f / PR_T, gb

    def transpose_stress(self, gU):
        """div(mu_t (grad U)^T) per cell, explicit: for component k the face flux
        mu_t,f (grad u_j . e_k)_f . S_f summed over the cell (``turbulence.py:251-261``)."""
        s, fv = self.s, self.s.fv
        mut_f = fv.face_interp(self.mut)
        out = np.zeros((s.nc, s.dim))
        for k in range(s.dim):
            gT = np.stack([gU[j][:, k] for j in range(s.dim)], axis=1)
            out[:, k] = fv.Cdiff @ (mut_f * np.sum(fv.face_interp_vec(gT) * fv.S, axis=1))
        return out

    # ---- transport -------------------------------------------------------------------------------
    def _bvals(self, phi, inflow):
        """Fixed at inlets and at outlet faces with inflow, zero-gradient elsewhere
        (``turbulence.py:263-269``)."""
        s = self.s
        fixed = self.inlet_b | (self.open_b & (s.Fb < 0))
        return np.where(fixed, inflow, phi[s.fv.Pb]), fixed.astype(np.float64)

    def _transport(self, phi, inflow, sigma, Sc, Sp, relax, fixed_cells=None, fixed_vals=None, floor=0.0):
        """One relaxed implicit solve of div(F phi) - div((mu + sigma mu_t) grad phi) = Sc - Sp phi,
        cells in ``fixed_cells`` pinned to ``fixed_vals`` by a 1e10 x max(diag) penalty; the
        residual is taken over the cells above the floor and not pinned (``turbulence.py:271-304``)."""
        s, fv = self.s, self.s.fv
        phib, fixed = self._bvals(phi, inflow)
        grad = fv.gradient(phi, phib)
        gam = self.mu + sigma * self.mut
        gf, gb = fv.face_interp(gam), gam[fv.Pb]
        diag, aPN, aNP, Db = s._coefficients((gf, gb), fixed)
        rhs = s._rhs((gf, gb), phi, grad, phib, Db, Sc * fv.vol, scheme=s.case.turb_scheme)
        diag = diag + Sp * fv.vol
        pinned = fixed_cells is not None and fixed_cells.size
        if pinned:
            big = 1e10 * float(np.max(diag))
            diag[fixed_cells] = diag[fixed_cells] + big
            rhs[fixed_cells] = rhs[fixed_cells] + big * fixed_vals
        A = fv.matrix(diag, aPN, aNP)
        live = phi > floor * (1.0 + 1e-9)
        if pinned:
            live[fixed_cells] = False
        r = np.abs(rhs - A @ phi)[live]
        den = np.abs(diag * phi)[live]
        res = float(np.sum(r)) / max(float(np.sum(den)), 1e-300)
        dr = diag / relax
        Ar = fv.matrix(dr, aPN, aNP)
        b = rhs + ((1.0 - relax) / relax) * diag * phi
        new, info = s._solve(Ar, b, phi, dr, tol=1e-3, maxiter=60)
        self.last_iters.append(info.iterations)
        return np.maximum(new, floor), res

    def _gradient(self, phi, inflow):
        return self.s.fv.gradient(phi, self._bvals(phi, inflow)[0])

    def _blend(self):
        """F1, F2 and grad k . grad omega (``turbulence.py:367-380``)."""
        k, w, y, rho, nu = self.k, self.w, self.y, self.rho, self.nu
        kw = np.sum(self._gradient(k, self.kb_in) * self._gradient(w, self.sb_in), axis=1)
        cd = np.maximum(2.0 * rho * self.sw2 * kw / w, 1e-10)
        sk = np.sqrt(k)
        visc = 500.0 * nu / (y * y * w)
        arg1 = np.minimum(np.maximum(sk / (self.bstar * w * y), visc), 4.0 * rho * self.sw2 * k / (cd * y * y))
        arg2 = np.maximum(2.0 * sk / (self.bstar * w * y), visc)
        return np.tanh(arg1 ** 4), np.tanh(arg2 ** 2), kw

    def _omega_wall(self):
        """Wall-cell omega sqrt(w_vis^2 + w_log^2), w_vis = 6 nu / (beta1 y^2), w_log =
        sqrt(k) / (Cmu^0.25 kappa y) (``turbulence.py:390-397``)."""
        yc = self.y_wall_cell[self.wall_cells]
        k = self.k[self.wall_cells]
        w_vis = 6.0 * self.nu / (self.b1 * yc ** 2)
        w_log = np.sqrt(np.maximum(k, 0.0)) / (CMU ** 0.25 * KAPPA * yc)
        return np.sqrt(w_vis ** 2 + w_log ** 2)

    def solve(self, gU) -> Dict[str, float]:
        """k then omega, then mu_t = rho a1 k / max(a1 omega, |S| F2) (``turbulence.py:382-438``)."""
        self.last_iters = []
        rho, k, w = self.rho, self.k, self.w
        S = strain_rate(gU, self.s.dim)
        S2 = S * S
        F1, _, kw = self._blend()

        def bl(a, b):
            return F1 * a + (1.0 - F1) * b

        Pk = np.minimum(self.mut * S2, 10.0 * self.bstar * rho * k * w)
        knew, rk = self._transport(k, self.kb_in, bl(self.sk1, self.sk2), Pk, self.bstar * rho * w,
                                   self.relax_k, floor=self.k_min)
        cross = (1.0 - F1) * 2.0 * rho * self.sw2 * kw / w
        Sc = bl(self.g1, self.g2) * rho * S2 + np.maximum(cross, 0.0)
        Sp = bl(self.b1, self.b2) * rho * w + np.maximum(-cross, 0.0) / w
        wnew, rw = self._transport(w, self.sb_in, bl(self.sw1, self.sw2), Sc, Sp, self.relax_w,
                                   fixed_cells=self.wall_cells, fixed_vals=self._omega_wall(), floor=self.w_min)
        self.k, self.w = knew, wnew
        _, F2, _ = self._blend()
        self.mut = self.rho * self.a1 * self.k / np.maximum(self.a1 * self.w, S * F2)
        return {"k": rk, "omega": rw}

    # ---- fields and state --------------------------------------------------------------------------
    def fields(self):
        """``turbulence.py:311-323``."""
        out = {"turb-kinetic-energy": self.k.copy(), self.field_name: self.w.copy(),
               "viscosity-turb": self.mut.copy(), "viscosity-ratio": self.mut / self.mu,
               "wall-distance": self.y.copy()}
        yp = np.zeros(self.s.nc)
        if self.wall_faces.size:
            np.maximum.at(yp, self.s.fv.Pb[self.wall_faces], self.yplus[self.wall_faces])
        out["y-plus"] = yp
        return out

    def state(self):
        return {"k": self.k.copy(), "w": self.w.copy(), "mut": self.mut.copy()}

    def load(self, st):
        if "k" in st:
            self.k = np.array(st["k"], dtype=np.float64)
            self.w = np.array(st["w"], dtype=np.float64)
            self.mut = np.array(st["mut"], dtype=np.float64)
