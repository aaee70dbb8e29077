"""Conjugate heat transfer on the B200 path (``flowtrace/unstructured/conjugate.py:46-325``).

As the reference's ``ConjugateSolver``: the momentum and pressure equations are solved on the
fluid cells only (the sub-mesh of ``extract_cells``, whose fluid-solid interfaces become no-slip
walls) by a ``SimpleSolver``, and one energy equation on every cell of the full mesh, with
face diffusivities from the distance-weighted harmonic mean of the two cells' conductivities
(heat flux continuous across an interface, exact for a 1-D composite wall), the fluid's mass
fluxes (zero on solid faces) and the solids' volumetric sources.

On the device the energy equation runs on the full mesh's own ``FVMesh`` through the same
kernels as the solver's energy stage: ``b2s_energy_bvals_d``, ``b2s_ls_gradient_d``,
``b2s_energy_assemble_turb_d`` (per-face diffusivities), ``b2s_bicgstab_jacobi_d`` (tolerance
1e-4, 200 iterations, as the reference) and ``b2s_sum_partials_d``; the fluid's fluxes are
scattered into the full mesh's face order by index maps built once. What runs on the host is
set-up (``conjugate_setup``: solid zones, the sub-mesh, conductivities, sources, the face maps)
and the reports.

With the k-omega SST model the fluid cells' diffusivity is k/cp + mu_t/Pr_t, so the face
diffusivities are rebuilt on the device every iteration from the flow's mu_t
(``harmonic_face_gamma``).
"""

from __future__ import annotations

import copy
import ctypes
from typing import Dict

import numpy as np

from .. import _lib
from ..linalg.krylov import INFO_DTYPE, read_info
from ..mesh.unstructured import UnstructuredMesh, extract_cells
from .case import FLUENT_TO_KIND, BoundarySpec, UnstructuredCase
from .fvmesh import FVMesh, HostFV
from .simple import T_FIXED, T_FLUX, SimpleSolver

__all__ = ["ConjugateSolver", "conjugate_setup", "device_flux_maps", "harmonic_face_gamma", "make_solver"]

PR_T = 0.85  # turbulent Prandtl number of the energy equation (flowtrace/unstructured/turbulence.py:59)


def harmonic_face_gamma(g, w, fP, fN, bP):
    """Face diffusivities from the cell diffusivities ``g`` (``conjugate.py:146-159``): inside,
    1 / ((1 - w) / g_P + w / g_N), the owner side holding (1 - w) of the distance; on boundary
    faces the owner's value. Tensors on any device (index tensors of dtype long)."""
    gP, gN = g[fP], g[fN]
    return 1.0 / ((1.0 - w) / gP + w / gN), g[bP]


def conjugate_setup(mesh: UnstructuredMesh, case: UnstructuredCase, hfv: HostFV = None,
                    sub_hfv: HostFV = None) -> dict:
    """Host set-up of a conjugate case, in the reference's numbering (``conjugate.py:47-134``):
    the solid mask, the fluid sub-mesh with its face and cell maps, the flow case (no solids, no
    energy equation, interfaces as walls), the diffusivity k/cp per cell, the source per cell
    (source/cp x volume), the harmonic face diffusivities ``gamma_face`` / ``gamma_bface``, the
    positions of the sub-mesh's interior faces among the full mesh's interior faces (``if_dst``),
    the sub-mesh boundary faces that are full-mesh boundary faces (``bf_src`` -> ``bf_dst``),
    and the thermal boundary arrays of the full mesh (kind, value, outlet mask)."""
    if not case.energy:
        raise ValueError("conjugate heat transfer needs the energy equation (case.energy = True)")
    solid_ids = {}
    for name, spec in case.solids.items():
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
    fcase = copy.deepcopy(case)
    fcase.solids = {}
    fcase.energy = False  # the conjugate energy equation below replaces the flow's own
    for z in sub.boundary_zones():
        if z.name.startswith("interface-"):
            fcase.boundaries[z.name] = BoundarySpec("wall")
    hfv = hfv if hfv is not None else HostFV(mesh)
    sub_hfv = sub_hfv if sub_hfv is not None else HostFV(sub)
    gam = np.full(mesh.n_cells, case.conductivity / case.cp)
    q = np.zeros(mesh.n_cells)
    for zid, spec in solid_ids.items():
        m = mesh.cell_zone == zid
        gam[m] = float(spec["conductivity"]) / case.cp
        q[m] = float(spec.get("source", 0.0)) / case.cp
    gP, gN, w = gam[hfv.P], gam[hfv.N], hfv.w
    gamma_face = 1.0 / ((1.0 - w) / gP + w / gN)  # the owner side holds (1 - w) of d
    pos_if = -np.ones(mesh.n_faces, dtype=np.int64)
    pos_if[hfv.if_idx] = np.arange(hfv.n_if)
    pos_bf = -np.ones(mesh.n_faces, dtype=np.int64)
    pos_bf[hfv.bf_idx] = np.arange(hfv.n_bf)
    full_of_sub = np.where(fmap >= 0, fmap, -fmap - 1)
    if_dst = pos_if[full_of_sub[sub_hfv.if_idx]]
    keep = pos_bf[full_of_sub[sub_hfv.bf_idx]] >= 0
    bf_src = np.nonzero(keep)[0]
    bf_dst = pos_bf[full_of_sub[sub_hfv.bf_idx[keep]]]
    n = hfv.n_bf
    tk, tv, out = np.zeros(n, dtype=np.int64), np.zeros(n), np.zeros(n, dtype=bool)
    for z in mesh.boundary_zones():
        spec = case.boundaries.get(z.name) or BoundarySpec(kind=FLUENT_TO_KIND.get(z.type, "wall"))
        m = hfv.bzone == z.id
        if spec.kind == "wall":
            tk[m] = {"adiabatic": 0, "temperature": T_FIXED, "flux": T_FLUX}[spec.thermal]
        elif spec.kind in ("inlet", "pressure"):
            tk[m] = T_FIXED
        out[m] = spec.kind == "outlet"
        tv[m] = spec.value
    return {"solid": solid, "sub": sub, "face_map": fmap, "cell_map": cmap, "flow_case": fcase, "gam_cell": gam,
            "q_cell": q * hfv.vol, "gamma_face": gamma_face, "gamma_bface": gam[hfv.Pb], "if_dst": if_dst,
            "bf_src": bf_src, "bf_dst": bf_dst, "tkind": tk, "tval": tv, "is_outlet": out}


def device_flux_maps(hs: dict, fv, sfv):
    """Index maps from the fluid sub-mesh's device face order (``sfv``) to the full mesh's
    (``fv``): interior face i of the fluid goes to full interior face ``if_dst[i]``; fluid
    boundary face ``bf_src[k]`` to full boundary face ``bf_dst[k]`` (``hs`` from
    ``conjugate_setup``)."""
    full_if, full_bf, sub_bf = np.argsort(fv.face_ref), np.argsort(fv.bface_ref), np.argsort(sfv.bface_ref)
    return full_if[hs["if_dst"][sfv.face_ref]], sub_bf[hs["bf_src"]], full_bf[hs["bf_dst"]]


class ConjugateSolver:
    """Drop-in for ``flowtrace.unstructured.conjugate.ConjugateSolver`` on one B200."""

    ENERGY_TOL, ENERGY_MAXITER = 1e-4, 200  # conjugate.py:184

    def __init__(self, mesh: UnstructuredMesh, case: UnstructuredCase, backend=None, **flow_kwargs):
        import torch

        self.case, self.mesh = case, mesh
        hfv = HostFV(mesh)
        hs = conjugate_setup(mesh, case, hfv=hfv)
        self.solid, self.cell_map = hs["solid"], hs["cell_map"]
        self.gam_cell, self.tkind_h = hs["gam_cell"], hs["tkind"]
        self.tval_h, self.is_outlet_h = hs["tval"], hs["is_outlet"]
        self._gamma_face_h, self._q_cell_h = hs["gamma_face"], hs["q_cell"]
        self.flow = SimpleSolver(hs["sub"], hs["flow_case"], **flow_kwargs)
        self.flow.external_energy = True  # no divergence guard under a conjugate solver (simple.py:733)
        self.torch_device = dev = self.flow.torch_device
        self.fv = fv = FVMesh(mesh, dev)
        self.nc, self.dim = mesh.n_cells, mesh.dim
        self.energy = True
        sfv = self.flow.fv
        as_idx = lambda a: torch.as_tensor(np.asarray(a, dtype=np.int64), device=dev)  # noqa: E731
        self._if_dst, self._bf_src, self._bf_dst = (as_idx(a) for a in device_flux_maps(hs, fv, sfv))
        z = lambda *shape: torch.zeros(*shape, dtype=torch.float64, device=dev)  # noqa: E731
        nc, nf, nb, dim = fv.nc, max(fv.n_if, 1), max(fv.n_bf, 1), fv.dim
        one = lambda t, n=1: t if t.numel() else z(n)  # noqa: E731
        self.gamma_f = one(fv.faces_to_device(hs["gamma_face"]))
        self.gamma_b = one(fv.bfaces_to_device(hs["gamma_bface"]))
        self.q_cell = fv.cells_to_device(hs["q_cell"])
        self.F, self.Fb = z(nf), z(nb)
        self.T = z(nc) + float(case.init_T)
        self.Tn, self.gT, self.Tb = z(nc), z(dim, nc), z(nb)
        nnz = fv.nnz
        self.val, self.diag, self.inv, self.b, self.br = z(nnz), z(nc), z(nc), z(nc), z(nc)
        L = _lib.lib()
        self.nblk = L.b2s_mesh_part_blocks(fv.cmesh_ref)
        self.part = z(2 * self.nblk)
        self.q_of = torch.arange(2, dtype=torch.int32, device=dev)
        self.report = torch.zeros(16 + INFO_DTYPE.itemsize, dtype=torch.uint8, device=dev)
        self.scal = self.report[:16].view(torch.float64)
        wb = L.b2s_bicgstab_workspace_bytes(nc, 1)
        self.work = torch.empty(wb // 8 + 1, dtype=torch.float64, device=dev)
        # boundary conditions of the full mesh: only the thermal masks are read by the energy kernels
        zb = z(nb)
        bfd = lambda a: one(fv.bfaces_to_device(np.asarray(a, dtype=np.float64)))  # noqa: E731
        tk = hs["tkind"]
        self._bc_t = {"m_wall": zb, "m_inlet": zb, "m_pres": zb, "m_sym": zb, "m_dirvel": zb, "ub_fixed": z(dim, nb),
                      "pb_fixed": zb, "m_tfix": bfd(tk == T_FIXED), "m_tflux": bfd(tk == T_FLUX),
                      "m_out": bfd(hs["is_outlet"]), "tval": bfd(hs["tval"])}
        self.cbc = _lib.BC(**{k: v.data_ptr() for k, v in self._bc_t.items()})
        self._turb_idx = None
        if self.flow.turb is not None:  # mu_t / Pr_t joins the fluid cells' diffusivity every iteration
            self._turb_idx = as_idx(fv.iperm[hs["cell_map"][sfv.perm]])  # fluid device cell -> full device cell
            self._gam_cell = fv.cells_to_device(hs["gam_cell"])
            self._mut_full = z(nc)
            self._face_idx = (fv.t["fP"].long(), fv.t["fN"].long(), fv.t["bP"].long())
            self._update_gamma()
        self._lagT = False
        self._res_energy = 1.0
        self.last_linear = {}
        self.energy_info = None
        self.kernel_launches = 0

    # ------------------------------------------------------------------ the energy equation
    def _update_gamma(self):
        """Face diffusivities with the flow's current mu_t (``conjugate.py:146-159``)."""
        fl, fv = self.flow, self.fv
        self._mut_full.index_copy_(0, self._turb_idx, fl.turb._mut[fl._cur])
        gf, gb = harmonic_face_gamma(self._gam_cell + self._mut_full / PR_T, fv.t["w"], *self._face_idx)
        self.gamma_f[: gf.numel()].copy_(gf)
        self.gamma_b[: gb.numel()].copy_(gb)

    def _full_fluxes(self):
        """The fluid's current mass fluxes on the full mesh's faces, zero on solid faces
        (``conjugate.py:136-144``)."""
        fl = self.flow
        sF, sFb = fl._F[fl._cur], fl._Fb[fl._cur]
        self.F.zero_()
        self.Fb.zero_()
        if self._if_dst.numel():
            self.F.index_copy_(0, self._if_dst, sF[: self._if_dst.numel()])
        if self._bf_dst.numel():
            self.Fb.index_copy_(0, self._bf_dst, sFb.index_select(0, self._bf_src))

    def _energy(self) -> float:
        """``conjugate.py:161-187`` on the device; returns the scaled residual of the system
        before the solve."""
        L, fv, c = _lib.lib(), self.fv, self.case
        s = _lib.stream_ptr()
        m, bc = fv.cmesh_ref, ctypes.byref(self.cbc)
        self._full_fluxes()
        if self._turb_idx is not None:
            self._update_gamma()
        _lib.check(L.b2s_energy_bvals_d(m, bc, self.T.data_ptr(), self.gT.data_ptr() if self._lagT else None,
                                        self.Fb.data_ptr(), self.Tb.data_ptr(), s), "b2s_energy_bvals_d")
        _lib.check(L.b2s_ls_gradient_d(m, 1, self.T.data_ptr(), self.Tb.data_ptr(), self.gT.data_ptr(), s),
                   "b2s_ls_gradient_d")
        self._lagT = True
        _lib.check(L.b2s_energy_assemble_turb_d(m, bc, self.gamma_f.data_ptr(), self.gamma_b.data_ptr(), c.cp,
                                                c.relax_T, int(c.scheme == "second-order"), self.T.data_ptr(),
                                                self.gT.data_ptr(), self.Tb.data_ptr(), self.F.data_ptr(),
                                                self.Fb.data_ptr(), self.q_cell.data_ptr(), self.val.data_ptr(),
                                                self.diag.data_ptr(), self.inv.data_ptr(), self.b.data_ptr(),
                                                self.br.data_ptr(), self.part.data_ptr(), s),
                   "b2s_energy_assemble_turb_d")
        self.Tn.copy_(self.T)
        _lib.check(L.b2s_bicgstab_jacobi_d(fv.nc, 1, fv.rowptr.data_ptr(), fv.col.data_ptr(), self.val.data_ptr(),
                                           self.br.data_ptr(), self.inv.data_ptr(), self.Tn.data_ptr(),
                                           self.ENERGY_TOL, self.ENERGY_MAXITER, 1, self.work.data_ptr(),
                                           self.work.numel() * 8, self.report.data_ptr() + 16, s),
                   "b2s_bicgstab_jacobi_d")
        _lib.check(L.b2s_sum_partials_d(self.part.data_ptr(), self.nblk, 2, 2, self.q_of.data_ptr(),
                                        self.scal.data_ptr(), s), "b2s_sum_partials_d")
        self.kernel_launches += 5
        self.T, self.Tn = self.Tn, self.T
        raw = self.report.cpu().numpy()
        num, den = raw[:16].view(np.float64)
        self.energy_info = read_info(raw[16:])[0]
        return float(num) / float(den) if den > 0 else float(num)

    # ------------------------------------------------------------------ solver API
    @property
    def iteration(self):
        return self.flow.iteration

    @property
    def step_count(self):
        return self.flow.iteration

    @property
    def converged(self):
        return self.flow.converged and self._res_energy < self.case.tol

    @property
    def finished(self):
        return self.converged or self.flow.iteration >= self.case.max_iter

    def step(self) -> float:
        """One outer iteration: the flow on the fluid cells, then the energy equation on all cells
        (``conjugate.py:189-199``)."""
        if self.finished:
            return 0.0
        self.flow.step()
        self._res_energy = self._energy()
        self.last_linear = self.flow.last_linear
        if self.flow.iteration > 5 and self._res_energy >= self.case.tol:
            self.flow.converged = False
        return 1.0

    def run(self, max_steps=None) -> int:
        n = 0
        while not self.finished and (max_steps is None or n < max_steps):
            self.step()
            n += 1
        return n

    def residuals(self) -> dict:
        """``conjugate.py:217-221``."""
        r = self.flow.residuals()
        return {k: dict(v, energy=self._res_energy) for k, v in r.items()}

    def diagnostics(self) -> dict:
        d = self.flow.diagnostics()
        if d.get("available"):
            d["scope"] = "fluid cells (flow sub-mesh); conjugate energy reported by residuals()"
        return d

    def cell_centres(self) -> np.ndarray:
        return self.fv.geometry.cell_centre

    @property
    def temperature(self) -> np.ndarray:
        return self.fv.cells_to_host(self.T)

    def fields(self, names=None) -> Dict[str, np.ndarray]:
        """Fluid fields on the full mesh (zero in the solids) and the temperature everywhere
        (``conjugate.py:235-245``)."""
        out = {}
        for k, v in self.flow.fields().items():
            a = np.zeros(self.nc)
            a[self.cell_map] = v
            out[k] = a
        out["temperature"] = self.temperature
        if names:
            out = {k: v for k, v in out.items() if k in names}
        return out

    def mass_balance(self) -> dict:
        return self.flow.mass_balance()

    def wall_forces(self) -> dict:
        """Fluid forces on the walls (fluid-solid interfaces appear as ``interface-*`` zones)."""
        return self.flow.wall_forces()

    def heat_flow(self) -> dict:
        """Heat flow into the domain per full-mesh boundary zone, the heat crossing every
        fluid-solid interface (positive from solid into fluid) and the solids' sources
        (``conjugate.py:254-284``)."""
        fv, c, h = self.fv, self.case, self.fv.host
        T = self.temperature
        TP = T[h.Pb]
        self._full_fluxes()
        Fb = fv.bfaces_to_host(self.Fb[: h.n_bf])
        tk, tv = self.tkind_h, self.tval_h
        Tb = np.where(tk == T_FIXED, tv, TP)
        Tb = np.where(self.is_outlet_h & (Fb < 0), tv, Tb)
        g = self.gam_cell[h.Pb] * c.cp
        cond = g * h.alpha_b * (Tb - TP) * (tk == T_FIXED) + np.where(tk == T_FLUX, tv * h.Sb_mag, 0.0)
        q = cond - c.cp * Fb * Tb
        res = {z.name: float(q[h.bzone == z.id].sum()) for z in self.mesh.boundary_zones()}
        if self._turb_idx is not None:
            self._update_gamma()
        gf = (fv.faces_to_host(self.gamma_f[: h.n_if]) if self._turb_idx is not None else self._gamma_face_h) * c.cp
        sP, sN = self.solid[h.P], self.solid[h.N]
        iface = sP != sN
        flux = gf * h.alpha * (T[h.N] - T[h.P])
        into_fluid = np.where(sN & ~sP, flux, -flux)
        res["fluid-solid interfaces"] = float(into_fluid[iface].sum())
        res["volumetric sources"] = float(self._q_cell_h.sum() * c.cp)
        return res

    def describe(self) -> dict:
        d = self.flow.describe()
        d.update({"solver": d["solver"] + " + conjugate heat transfer", "cells": self.nc,
                  "solid_cells": int(self.solid.sum()), "solid_zones": list(self.case.solids)})
        return d

    @property
    def zone_specs_flow(self):
        return self.flow.zone_specs

    def state_dict(self) -> dict:
        st = self.flow.state_dict()
        st["T_full"] = self.temperature
        return st

    def load_state(self, st: dict) -> None:
        self.flow.load_state(st)
        if "T_full" in st:
            self.T.copy_(self.fv.cells_to_device(np.asarray(st["T_full"], dtype=np.float64)))
            self._lagT = False

    def initialize(self, fields: dict) -> None:
        sub = {k: np.asarray(v)[self.cell_map] for k, v in fields.items() if k != "temperature"}
        self.flow.initialize(sub)
        if "temperature" in fields:
            self.T.copy_(self.fv.cells_to_device(np.asarray(fields["temperature"], dtype=np.float64)))
            self._lagT = False

    @property
    def guard_events(self):
        return self.flow.guard_events

    @property
    def U(self):
        return self.flow.U

    @property
    def turb(self):
        return self.flow.turb


def make_solver(mesh: UnstructuredMesh, case: UnstructuredCase, backend=None):
    """``SimpleSolver``, or ``ConjugateSolver`` when the case has solid zones (``conjugate.py:321-325``)."""
    if case.solids or any(z.type == "solid" for z in mesh.cell_zones()):
        return ConjugateSolver(mesh, case, backend)
    return SimpleSolver(mesh, case, backend)
