"""The k-omega SST model on the B200 path (``flowtrace/unstructured/turbulence.py:116-438``).

``DeviceSST`` holds the model's state on the device (k and omega as one [2][nc] array, mu_t),
triple-buffered like the flow state so that the pipelined ``SimpleSolver.run`` can discard a
speculative iteration, and enqueues the model's stages (``csrc/b2s_sst.cu``) inside the
solver's outer iteration:

* before the momentum assembly, the face viscosities mu + mu_t (Spalding's law-of-the-wall
  viscosity on walls), the turbulent heat diffusivity and the transpose-stress source;
* after the energy equation, k and then omega (boundary values, gradients, blending, sources,
  assembly, the near-wall omega pin, a relaxed Jacobi-BiCGSTAB solve each) and mu_t.

What runs on the host is the set-up the reference also does on the host (``host_setup``): the
wall distance (a k-d tree of the wall-face centres, the eight nearest faces of every cell as
candidates, exact distances to those), the inflow values of k and omega per boundary zone and
the initial field.
"""

from __future__ import annotations

import ctypes
import math

import numpy as np

from .. import _lib

KAPPA = 0.41        # von Karman constant of the SST model and of Spalding's law
B_SPALDING = 5.2
CMU = 0.09
SIGMA_W1, BETA_1 = 0.5, 0.075
SIGMA_W2, BETA_2 = 0.856, 0.0828
BETA_STAR = 0.09
RELAX_DEFAULT = 0.8


def wall_distance(mesh, geometry, wall_zone_ids, n_cells) -> np.ndarray:
    """Distance of every cell centre to the nearest wall face (``turbulence.py:191-229``): the
    eight nearest wall-face centres are the candidates; in 2-D the exact distance to each
    candidate segment, in 3-D to a disc of 1.2 x the face's equal-area radius in the face's
    plane. 1e30 everywhere without walls."""
    xc = geometry.cell_centre
    wf = np.nonzero(np.isin(mesh.face_zone, wall_zone_ids))[0]
    if wf.size == 0:
        return np.full(n_cells, 1e30)
    from scipy.spatial import cKDTree

    fc = geometry.face_centre[wf]
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
        nrm = geometry.face_area_vec[wf]
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


def _omega_from(rho, mu, k, ratio, explicit):
    """omega = rho k / (mu ratio), or the explicit value (``turbulence.py:362-365``)."""
    if explicit is not None:
        return np.full(np.shape(k), float(explicit))
    return rho * np.asarray(k) / (mu * ratio)


def host_setup(mesh, hfv, bkind, zone_specs, ub_fixed, case) -> dict:
    """The model's set-up arrays in the reference's numbering (``turbulence.py:123-186``): the
    wall distance ``y`` (wall cells: the normal distance to their wall face), ``y_wall`` (wall
    cells: the smallest normal distance to one of their wall faces, +inf elsewhere), ``yb``
    (|db . n| per boundary face), the inflow values ``kb_in`` / ``wb_in`` per boundary face
    from each zone's intensity and viscosity ratio (or explicit k / omega), the initial ``k0`` /
    ``w0``, the reference speed and the floors. ``hfv`` is the host finite-volume data
    (``fvmesh.HostFV``), ``bkind`` the boundary kind codes per boundary face."""
    from .simple import INLET, WALL

    rho, mu = float(case.density), float(case.viscosity)
    nc, nb = hfv.nc, hfv.n_bf
    wall_b = bkind == WALL
    inlet_b = bkind == INLET
    yb = np.abs(np.einsum("fd,fd->f", hfv.db, hfv.nb))
    wall_ids = [z.id for z in mesh.boundary_zones() if zone_specs[z.name].kind == "wall"]
    y = wall_distance(mesh, hfv.geometry, wall_ids, nc)
    wf = np.nonzero(wall_b)[0]
    wall_cells = np.unique(hfv.Pb[wf])
    ywc = np.full(nc, np.inf)
    np.minimum.at(ywc, hfv.Pb[wf], yb[wf])
    if wall_cells.size:
        y[wall_cells] = ywc[wall_cells]
    speed = np.linalg.norm(ub_fixed, axis=1)
    u_ref = float(speed[inlet_b].max()) if inlet_b.any() else float(case.turb_reference_velocity or 1.0)
    u_ref = max(u_ref, 1e-6)
    kin, win = np.zeros(nb), np.zeros(nb)
    for z in mesh.boundary_zones():
        spec = zone_specs[z.name]
        m = hfv.bzone == z.id
        inten = spec.turb_intensity if spec.turb_intensity is not None else case.turb_intensity
        ratio = spec.turb_viscosity_ratio if spec.turb_viscosity_ratio is not None else case.turb_viscosity_ratio
        U = np.where(speed[m] > 0, speed[m], u_ref)
        kz = 1.5 * (inten * U) ** 2 if spec.k is None else np.full(m.sum(), spec.k)
        kin[m] = np.maximum(kz, 1e-12 * u_ref ** 2)
        win[m] = _omega_from(rho, mu, kin[m], ratio, spec.omega)
    init = case.turb_init or {}
    k0 = init.get("k", 1.5 * (case.turb_intensity * u_ref) ** 2)
    w0 = init.get("omega", float(_omega_from(rho, mu, np.array([k0]), case.turb_viscosity_ratio, None)[0]))
    return {"y": y, "y_wall": ywc, "yb": yb, "kb_in": kin, "wb_in": win, "k0": k0, "w0": w0, "u_ref": u_ref,
            "k_min": 1e-14 * u_ref ** 2, "w_min": 1e-14, "wall_faces": wf, "wall_cells": wall_cells}


class DeviceSST:
    """k-omega SST state and stages of one ``SimpleSolver`` (``turbulence.py:123-186`` set-up)."""

    field_name = "specific-diss-rate"

    def __init__(self, solver):
        import torch

        s = self.s = solver
        fv, c = s.fv, s.case
        dev = s.torch_device
        self.rho, self.mu = float(c.density), float(c.viscosity)
        self.nu = self.mu / self.rho
        nc, nb, dim = s.nc, fv.host.n_bf, s.dim
        hs = host_setup(s.mesh, fv.host, s.bkind_h, s.zone_specs, s._ub_fixed_h, c)
        self.wall_faces_h, self.wall_cells_h, self.y_h = hs["wall_faces"], hs["wall_cells"], hs["y"]
        self.u_ref, self.k_min, self.w_min = hs["u_ref"], hs["k_min"], hs["w_min"]
        self.relax_k = c.relax_k if c.relax_k is not None else RELAX_DEFAULT
        self.relax_w = c.relax_w if c.relax_w is not None else RELAX_DEFAULT
        y, ywc, yb, kin, win, k0, w0 = (hs[k] for k in ("y", "y_wall", "yb", "kb_in", "wb_in", "k0", "w0"))
        # device arrays
        z = lambda *shape: torch.zeros(*shape, dtype=torch.float64, device=dev)  # noqa: E731
        one = lambda t: t if t.numel() else z(1)  # noqa: E731
        self._t = {"y": fv.cells_to_device(y), "y_wall": fv.cells_to_device(ywc),
                   "yb": one(fv.bfaces_to_device(yb)), "kb_in": one(fv.bfaces_to_device(kin)),
                   "wb_in": one(fv.bfaces_to_device(win))}
        g1 = BETA_1 / BETA_STAR - SIGMA_W1 * KAPPA ** 2 / math.sqrt(BETA_STAR)
        g2 = BETA_2 / BETA_STAR - SIGMA_W2 * KAPPA ** 2 / math.sqrt(BETA_STAR)
        self.params = _lib.SST(
            rho=self.rho, mu=self.mu, nu=self.nu, k_min=self.k_min, w_min=self.w_min, relax_k=float(self.relax_k),
            relax_w=float(self.relax_w), k_over_cp=float(c.conductivity / c.cp) if s.energy else 0.0,
            eb=math.exp(-KAPPA * B_SPALDING), cmu25=CMU ** 0.25, g1=g1, g2=g2,
            second_order=int(c.turb_scheme == "second-order"), pad_=0,
            **{k: v.data_ptr() for k, v in self._t.items()})
        self.pref = ctypes.byref(self.params)
        nf, nbb, nnz = max(fv.n_if, 1), max(nb, 1), fv.nnz
        self._KW = [z(2, nc) for _ in range(3)]
        self._mut = [z(nc) for _ in range(3)]
        for KW in self._KW:
            KW[0].fill_(k0)
            KW[1].fill_(w0)
        for i in range(3):
            self._mut[i].copy_(self.rho * self._KW[i][0] / self._KW[i][1])  # turbulence.py:384-386
        self.mu_f, self.mu_b, self.yplus = z(nf), z(nbb), z(nbb)
        self.tsrc = z(dim, nc)
        self.kT_f, self.kT_b = (z(nf), z(nbb)) if s.energy else (None, None)
        self.bUc, self.gUc = z(1 + dim, nbb), z(dim, dim, nc)
        self.KWb, self.fixed, self.gKW = z(2, nbb), z(nbb), z(2, dim, nc)
        self.coef = z(8, nc)
        self.KWn = z(2, nc)
        self.val = [z(nnz) for _ in range(2)]
        self.diag = [z(nc) for _ in range(2)]
        self.b = [z(nc) for _ in range(2)]
        self.inv = [z(nc) for _ in range(2)]
        self.br = [z(nc) for _ in range(2)]
        if _lib.lib().b2s_sst_part_blocks(fv.cmesh_ref) != s.nblk:
            raise RuntimeError("SST partial-sum blocks differ from the solver's")

    # ---- stages -------------------------------------------------------------------------------
    def launch_momentum_terms(self, Up, gUp, slot, s, mu_b=None):
        """Face viscosities, heat diffusivity and transpose stress of the state in ``slot``;
        with ``mu_b`` the boundary viscosities go there and y+ is left as it is."""
        L, fv = _lib.lib(), self.s.fv
        _lib.check(L.b2s_sst_momentum_terms_d(
            fv.cmesh_ref, ctypes.byref(self.s.cbc), self.pref, Up.data_ptr(), gUp.data_ptr(),
            self._mut[slot].data_ptr(), self.mu_f.data_ptr(), (mu_b if mu_b is not None else self.mu_b).data_ptr(),
            self.yplus.data_ptr() if mu_b is None else None, self.tsrc.data_ptr(),
            self.kT_f.data_ptr() if self.kT_f is not None else None,
            self.kT_b.data_ptr() if self.kT_b is not None else None, s), "b2s_sst_momentum_terms_d")
        return 1

    def launch_transport(self, old, new, Upn, Fn, Fbn, pt, q_max, q_res, info, s):
        """k and omega of the new flow state, then mu_t (``simple.py:662-669``,
        ``turbulence.py:419-438``); returns the number of kernels launched."""
        sv = self.s
        L, fv = _lib.lib(), sv.fv
        m, bc, t = fv.cmesh_ref, ctypes.byref(sv.cbc), self.pref
        nc, nb, dim = sv.nc, max(fv.n_bf, 1), sv.dim
        KW, mut = self._KW[old], self._mut[old]
        # gradient of the corrected velocity, boundary values reconstructed with this
        # iteration's starting gradients
        gp = sv.gpf if sv.case.pressure_gradient == "green-gauss" else sv.gUp[0]
        _lib.check(L.b2s_flow_bvals_d(m, bc, Upn.data_ptr(), sv.gUp.data_ptr(), gp.data_ptr(), self.bUc.data_ptr(), s),
                   "b2s_flow_bvals_d")
        _lib.check(L.b2s_ls_gradient_d(m, dim, Upn.data_ptr() + 8 * nc, self.bUc.data_ptr() + 8 * nb,
                                       self.gUc.data_ptr(), s), "b2s_ls_gradient_d")
        _lib.check(L.b2s_sst_bvals_d(m, bc, t, KW.data_ptr(), Fbn.data_ptr(), self.KWb.data_ptr(),
                                     self.fixed.data_ptr(), s), "b2s_sst_bvals_d")
        _lib.check(L.b2s_ls_gradient_d(m, 2, KW.data_ptr(), self.KWb.data_ptr(), self.gKW.data_ptr(), s),
                   "b2s_ls_gradient_d")
        _lib.check(L.b2s_sst_sources_d(m, t, self.gUc.data_ptr(), KW.data_ptr(), self.gKW.data_ptr(), mut.data_ptr(),
                                       self.coef.data_ptr(), s), "b2s_sst_sources_d")
        self.KWn.copy_(KW)
        for q in (0, 1):
            _lib.check(L.b2s_sst_transport_assemble_d(
                m, t, q, KW.data_ptr(), self.KWb.data_ptr(), self.fixed.data_ptr(), self.gKW.data_ptr(),
                Fn.data_ptr(), Fbn.data_ptr(), self.coef.data_ptr(), self.val[q].data_ptr(), self.diag[q].data_ptr(),
                self.b[q].data_ptr(), pt(q_max[q]), s), "b2s_sst_transport_assemble_d")
            _lib.check(L.b2s_sst_transport_finish_d(
                m, t, q, KW.data_ptr(), self.coef.data_ptr(), pt(q_max[q]), self.val[q].data_ptr(),
                self.diag[q].data_ptr(), self.b[q].data_ptr(), self.inv[q].data_ptr(), self.br[q].data_ptr(),
                pt(q_res[q]), s), "b2s_sst_transport_finish_d")
            _lib.check(L.b2s_bicgstab_jacobi_d(nc, 1, fv.rowptr.data_ptr(), fv.col.data_ptr(), self.val[q].data_ptr(),
                                               self.br[q].data_ptr(), self.inv[q].data_ptr(),
                                               self.KWn.data_ptr() + 8 * q * nc, 1e-3, 60, 1, sv.work_bicg.data_ptr(),
                                               sv.work_bicg.numel() * 8, info[q], s), "b2s_bicgstab_jacobi_d")
        _lib.check(L.b2s_sst_update_d(m, t, self.KWn.data_ptr(), self.coef.data_ptr(), self._KW[new].data_ptr(),
                                      self._mut[new].data_ptr(), s), "b2s_sst_update_d")
        return 12

    # ---- state and fields --------------------------------------------------------------------
    def snapshot(self, slot):
        return {"KW": self._KW[slot].clone(), "mut": self._mut[slot].clone()}

    def restore(self, snap, slot):
        self._KW[slot].copy_(snap["KW"])
        self._mut[slot].copy_(snap["mut"])

    def state(self, slot):
        fv = self.s.fv
        return {"k": fv.cells_to_host(self._KW[slot][0]), "w": fv.cells_to_host(self._KW[slot][1]),
                "mut": fv.cells_to_host(self._mut[slot])}

    def load(self, st, slot):
        fv = self.s.fv
        if "k" in st:
            self._KW[slot][0].copy_(fv.cells_to_device(np.asarray(st["k"], dtype=np.float64)))
            self._KW[slot][1].copy_(fv.cells_to_device(np.asarray(st["w"], dtype=np.float64)))
            self._mut[slot].copy_(fv.cells_to_device(np.asarray(st["mut"], dtype=np.float64)))

    def fields(self, slot):
        """``turbulence.py:311-323``."""
        fv, h = self.s.fv, self.s.fv.host
        st = self.state(slot)
        out = {"turb-kinetic-energy": st["k"], self.field_name: st["w"], "viscosity-turb": st["mut"],
               "viscosity-ratio": st["mut"] / self.mu, "wall-distance": self.y_h.copy()}
        yp = np.zeros(self.s.nc)
        if self.wall_faces_h.size:
            ypb = fv.bfaces_to_host(self.yplus[: h.n_bf])
            np.maximum.at(yp, h.Pb[self.wall_faces_h], ypb[self.wall_faces_h])
        out["y-plus"] = yp
        return out

    def wall_viscosity(self, Up, gUp, slot):
        """Boundary-face viscosity of the momentum equations at the state in ``slot`` (reference
        numbering): mu + mu_t, on walls the wall-function value (``simple.py:900-904``)."""
        import torch

        fv = self.s.fv
        mu_b = torch.zeros_like(self.mu_b)
        self.launch_momentum_terms(Up, gUp, slot, _lib.stream_ptr(), mu_b=mu_b)
        return fv.bfaces_to_host(mu_b[: fv.n_bf])
