"""ORACLE — test infrastructure only. Never imported by the product (``gputest_b200``).

A CPU restatement of FlowTrace's conjugate heat transfer solver
(``flowtrace/unstructured/conjugate.py:46-318``) on top of ``OracleSimple``: the flow is solved
on the fluid cells only (the sub-mesh of ``extract_cells``, whose fluid-solid interfaces become
no-slip walls), and one energy equation on every cell of the full mesh, with harmonic-mean face
diffusivities, the fluid's mass fluxes (zero on solid faces) and the solids' volumetric sources.

The sub-mesh comes from the package's ``extract_cells``, itself pinned to the reference's by
``tests/golden/extract_digests.json``. Pinned against the reference's solver by
``tests/golden/make_conjugate_golden.py`` (fixtures) and ``tests/test_oracle_conjugate.py``.
"""

from __future__ import annotations

import copy

import numpy as np

from .simplec_oracle import T_FIXED, T_FLUX, FLUENT_TO_KIND, OracleFV, OracleSimple, _Spec


class _EnergyOps:
    """The discretisation routines of ``OracleSimple`` on the full mesh (``conjugate.py:29-43``)."""

    _split_gamma = staticmethod(OracleSimple._split_gamma)
    _coefficients = OracleSimple._coefficients
    _rhs = OracleSimple._rhs
    _residual = OracleSimple._residual
    _solve = OracleSimple._solve

    def __init__(self, fv, case):
        self.fv, self.case, self.native = fv, case, None
        self.F = self.Fb = None


class OracleConjugate:
    """``ConjugateSolver`` (``conjugate.py:46-318``), laminar or with the k-omega SST model."""

    def __init__(self, mesh, case):
        from gputest_b200.mesh.unstructured import extract_cells
        from gputest_b200.unstructured.case import BoundarySpec

        if not case.energy:
            raise ValueError("conjugate heat transfer needs the energy equation (case.energy = True)")
        self.case, self.mesh = case, mesh
        solid_ids = {}
        for name, spec in case.solids.items():                                      # conjugate.py:55-64
            z = mesh.zone_by_name(name)
            if z is None or z.kind != "cell":
                raise ValueError(f"solid zone {name!r} is not a cell zone of this mesh")
            solid_ids[z.id] = spec
        for z in mesh.cell_zones():
            if z.type == "solid" and z.id not in solid_ids:
                raise ValueError(f"cell zone {z.name!r} is a solid: give its conductivity in case.solids")
        solid = np.isin(mesh.cell_zone, list(solid_ids))
        if solid.all():
            raise ValueError("no fluid cells")
        sub, fmap, cmap = extract_cells(mesh, ~solid)
        self.cell_map = cmap
        fcase = copy.deepcopy(case)                                                # conjugate.py:67-73
        fcase.solids = {}
        fcase.energy = False  # the flow's own energy equation is replaced by the one below
        for z in sub.boundary_zones():
            if z.name.startswith("interface-"):
                fcase.boundaries[z.name] = BoundarySpec("wall")
        self.flow = OracleSimple(sub, fcase)
        self.flow.guard_enabled = False  # simple.py:733: no divergence guard under a conjugate solver
        self.fv = fv = OracleFV(mesh)
        self.nc, self.dim = mesh.n_cells, mesh.dim
        self.solid = solid
        gam = np.full(mesh.n_cells, case.conductivity / case.cp)                   # conjugate.py:79-87
        q = np.zeros(mesh.n_cells)
        for zid, spec in solid_ids.items():
            m = mesh.cell_zone == zid
            gam[m] = float(spec["conductivity"]) / case.cp
            q[m] = float(spec.get("source", 0.0)) / case.cp
        self.gam_cell = gam
        self.q_cell = q * fv.vol
        pos_if = -np.ones(mesh.n_faces, dtype=np.int64)                           # conjugate.py:89-100
        pos_if[fv.if_idx] = np.arange(fv.n_if)
        pos_bf = -np.ones(mesh.n_faces, dtype=np.int64)
        pos_bf[fv.bf_idx] = np.arange(fv.n_bf)
        sfv = self.flow.fv
        full_of_sub = np.where(fmap >= 0, fmap, -fmap - 1)
        self._if_dst = pos_if[full_of_sub[sfv.if_idx]]
        bsub = sfv.bf_idx
        keep = pos_bf[full_of_sub[bsub]] >= 0
        self._bf_src = np.nonzero(keep)[0]
        self._bf_dst = pos_bf[full_of_sub[bsub[keep]]]
        self._build_thermal_bcs(_Spec, FLUENT_TO_KIND)
        self.ops = _EnergyOps(fv, case)
        self.T = np.full(self.nc, case.init_T, dtype=np.float64)
        self._gT = None
        self.last_linear = {}
        self._res_energy = 1.0

    def _build_thermal_bcs(self, spec_cls, kinds):
        """``conjugate.py:112-134``."""
        fv = self.fv
        n = fv.n_bf
        tk, tv, out = np.zeros(n, dtype=np.int64), np.zeros(n), np.zeros(n, dtype=bool)
        for z in self.mesh.boundary_zones():
            spec = self.case.boundaries.get(z.name) or spec_cls(kinds.get(z.type, "wall"))
            m = fv.bzone == z.id
            if spec.kind == "wall":
                tk[m] = {"adiabatic": 0, "temperature": T_FIXED, "flux": T_FLUX}[spec.thermal]
            elif spec.kind in ("inlet", "pressure"):
                tk[m] = T_FIXED
            out[m] = spec.kind == "outlet"
            tv[m] = spec.value
        self.tkind, self.tval, self.is_outlet = tk, tv, out

    def _full_fluxes(self):
        """Fluid fluxes on the full mesh, zero on solid faces (``conjugate.py:136-144``)."""
        F = np.zeros(self.fv.n_if)
        Fb = np.zeros(self.fv.n_bf)
        F[self._if_dst] = self.flow.F[np.arange(self.flow.F.shape[0])]
        Fb[self._bf_dst] = self.flow.Fb[self._bf_src]
        return F, Fb

    def face_gamma(self):
        """Harmonic mean of the two cells' diffusivities, weighted by the distances to the face;
        with the SST model the fluid cells add mu_t / Pr_t (``conjugate.py:146-159``)."""
        fv = self.fv
        g = self.gam_cell.copy()
        if self.flow.turb is not None:
            from .sst_oracle import PR_T

            g[self.cell_map] += self.flow.turb.mut / PR_T
        gP, gN = g[fv.P], g[fv.N]
        w = fv.w
        return 1.0 / ((1.0 - w) / gP + w / gN), g[fv.Pb]

    def _energy(self):
        """``conjugate.py:161-187``."""
        fv, ops, c = self.fv, self.ops, self.case
        ops.F, ops.Fb = self._full_fluxes()
        T = self.T
        TP = T[fv.Pb]
        if self._gT is not None:
            TP = TP + np.sum(self._gT[fv.Pb] * fv.db_t, axis=1)
        fixed = self.tkind == T_FIXED
        flux = self.tkind == T_FLUX
        Tb = np.where(fixed, self.tval, TP)
        Tb = np.where(self.is_outlet & (ops.Fb < 0), self.tval, Tb)
        gT = fv.gradient(T, Tb)
        self._gT = gT
        gam = self.face_gamma()
        q_in = fv.Cb @ (flux * self.tval * fv.Sb_mag / c.cp) + self.q_cell
        diag, aPN, aNP, Db = ops._coefficients(gam, fixed.astype(np.float64))
        rhs = ops._rhs(gam, T, gT, Tb, Db, q_in)
        A = fv.matrix(diag, aPN, aNP)
        r = ops._residual(A, diag, T, rhs)
        aT = c.relax_T
        dr = diag / aT
        Ar = fv.matrix(dr, aPN, aNP)
        b = rhs + ((1.0 - aT) / aT) * diag * T
        self.T, info = ops._solve(Ar, b, T, dr, tol=1e-4, maxiter=200)
        self.energy_iters = info.iterations
        return r

    @property
    def iteration(self):
        return self.flow.iteration

    @property
    def finished(self):
        return (self.flow.converged and self._res_energy < self.case.tol) or self.flow.iteration >= self.case.max_iter

    def step(self):
        """``conjugate.py:189-199``."""
        if self.finished:
            return 0.0
        self.flow.step()
        self._res_energy = self._energy()
        self.last_linear = self.flow.last_linear
        if self.flow.iteration > 5 and self._res_energy >= self.case.tol:
            self.flow.converged = False
        return 1.0

    def residuals(self):
        """``conjugate.py:217-221``."""
        r = self.flow.residuals()
        return {k: dict(v, energy=self._res_energy) for k, v in r.items()}

    def fields(self):
        """``conjugate.py:235-245``: fluid fields on the full mesh (zero in the solids)."""
        out = {}
        for k, v in self.flow.fields().items():
            a = np.zeros(self.nc)
            a[self.cell_map] = v
            out[k] = a
        out["temperature"] = self.T.copy()
        return out

    def heat_flow(self):
        """``conjugate.py:254-284``."""
        fv, c = self.fv, self.case
        T = self.T
        TP = T[fv.Pb]
        _, Fb = self._full_fluxes()
        tk, tv = self.tkind, self.tval
        Tb = np.where(tk == T_FIXED, tv, TP)
        Tb = np.where(self.is_outlet & (Fb < 0), tv, Tb)
        g = self.gam_cell[fv.Pb] * c.cp
        cond = g * fv.alpha_b * (Tb - TP) * (tk == T_FIXED) + np.where(tk == T_FLUX, tv * fv.Sb_mag, 0.0)
        q = cond - c.cp * Fb * Tb
        res = {z.name: float(q[fv.bzone == z.id].sum()) for z in self.mesh.boundary_zones()}
        gf = self.face_gamma()[0] * c.cp
        sP, sN = self.solid[fv.P], self.solid[fv.N]
        iface = sP != sN
        flux = gf * fv.alpha * (T[fv.N] - T[fv.P])
        into_fluid = np.where(sN & ~sP, flux, -flux)
        res["fluid-solid interfaces"] = float(into_fluid[iface].sum())
        res["volumetric sources"] = float(self.q_cell.sum() * c.cp)
        return res
