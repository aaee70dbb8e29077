"""Batches of independent SIMPLEC cases on one device: ``BatchSimpleSolver``.

The reference runs a sweep of cases one after another, each through its own solver
(``flowtrace/runtime/batch.py:142-222`` calling ``SimpleSolver.step``). Here the cases of a batch
are one block-diagonal problem: their meshes are joined into a disjoint union
(``union_mesh``, each case's cells contiguous on the device), every finite-volume stage is one
launch for all of them, and the linear solves are per case inside persistent launches that
deal whole cases to blocks (``b2s_bicgstab_groups_f32_d``, ``b2s_pcg_groups_mixed_d``). Every
case keeps its own Krylov scalars and stopping tests, its own residual normalisation and
convergence test (``simple.py:675-703``), its own pressure level when it is closed, and its own
viscosity (the diffusion coefficients of the momentum assembly are scaled per face). The
arithmetic is the mixed-precision iteration of ``MixedSimpleSolver``; with no AMG rebuild due,
a whole outer iteration of all cases is one CUDA graph replay.

Differences from running the cases one by one: the AMG hierarchy is set up for the union
(aggregates never cross cases; coarsening stops when every case has at most ``max_coarse``
rows - a case already that small is carried to the next level unchanged - and each case's
coarsest block gets its own dense inverse). This changes the preconditioner, not the converged
fields. The stability guard of the single-case
solver runs per case (its rollback and relaxation ladder, with per-case relaxation factors).
Cases keep iterating until every case has converged (a converged case's residuals keep
falling), and ``case_converged_at`` records when each one first passed.
"""

from __future__ import annotations

import copy
import ctypes
from typing import List, Sequence

import numpy as np

from .. import _lib
from ..linalg.amg import AMGHierarchy
from ..linalg.krylov import INFO_DTYPE
from ..mesh.unstructured import UnstructuredMesh, union_groups, union_mesh
from .case import UnstructuredCase
from .mixed import MixedSimpleSolver
from .simple import COMPONENTS

_SHARED = ("density", "scheme", "relax_u", "relax_p", "pressure_tol", "algorithm", "pressure_gradient",
           "init_velocity", "body_force", "tol", "max_iter")


def _union_case(cases: Sequence[UnstructuredCase], meshes: Sequence[UnstructuredMesh]) -> UnstructuredCase:
    base = cases[0]
    for c in cases[1:]:
        for k in _SHARED:
            if getattr(c, k) != getattr(base, k):
                raise ValueError(f"cases of a batch must share {k!r}")
    if any(c.energy for c in cases):
        raise NotImplementedError("batches without the energy equation only")
    u = copy.deepcopy(base)
    u.boundaries = {}
    for i, (c, m) in enumerate(zip(cases, meshes)):
        for z in m.boundary_zones():
            if z.name in c.boundaries:
                u.boundaries[f"c{i}/{z.name}"] = copy.deepcopy(c.boundaries[z.name])
    u.viscosity = 1.0  # the per-case viscosity scales the momentum diffusion coefficients
    return u


class BatchSimpleSolver(MixedSimpleSolver):
    """Many independent cases (list of meshes and cases of one dimension) solved together."""

    TURBULENCE = ("laminar",)

    # team shapes of the per-case Krylov solves (``b2s_team_config``: blocks per cluster, threads
    # per block, rows-per-warp switch), one per solve; ``autotune`` picks among TEAM_CANDIDATES on
    # the batch itself
    DEFAULT_TEAM = (4, 1024, 24)
    TEAM_CANDIDATES = tuple((cb, bt, wr) for cb in (2, 4, 8) for bt in (512, 1024) for wr in (16, 24, 48))

    def __init__(self, meshes: List[UnstructuredMesh], cases: List[UnstructuredCase], max_coarse: int = 150,
                 amg_theta: float = 0.08):
        if len(meshes) != len(cases) or not meshes:
            raise ValueError("one case per mesh")
        self.meshes, self.cases = list(meshes), list(cases)
        self.ncase = len(meshes)
        self.case_cells = np.array([m.n_cells for m in meshes], dtype=np.int64)
        self.case_offsets = np.concatenate([[0], np.cumsum(self.case_cells)])
        self._cell_groups = union_groups(meshes)  # reference (union) numbering
        self.mu_case = np.array([float(c.viscosity) for c in cases])
        super().__init__(union_mesh(self.meshes), _union_case(cases, meshes), max_coarse=max_coarse,
                         amg_theta=amg_theta)
        self.reaggregate = False  # the batch hierarchy is set up once (aggregates per case)
        self.team = _lib.TeamConfig(*self.DEFAULT_TEAM, 0)  # pressure-correction solve
        self.team_momentum = _lib.TeamConfig(*self.DEFAULT_TEAM, 0)
        self.tuning = None
        self.case_iteration = 0
        self.case_converged_at = np.full(self.ncase, -1, dtype=np.int64)
        self._res_max5_case = np.zeros(self.ncase)

    # ------------------------------------------------------------------ set-up
    def _prepare_mesh(self):
        import torch

        fv = self.fv
        dev = self.torch_device
        g_dev = self._cell_groups[fv.perm]  # case of every device cell
        if np.any(np.diff(g_dev) < 0):
            raise RuntimeError("cases are not contiguous on the device")
        cells = np.concatenate([[0], np.cumsum(np.bincount(g_dev, minlength=self.ncase))])
        # tiles of at most 256 cells inside each case
        tiles, tile_group = [0], []
        for g in range(self.ncase):
            a, b = int(cells[g]), int(cells[g + 1])
            cuts = list(range(a + 256, b, 256)) + [b]
            tiles += cuts
            tile_group += [g] * len(cuts)
        fv.set_tiling(np.array(tiles))
        group_tiles = np.concatenate([[0], np.cumsum(np.bincount(tile_group, minlength=self.ncase))])
        i32 = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.int32), device=dev)  # noqa: E731
        self.g_cells, self.g_tiles, self.g_tile_group = i32(cells), i32(group_tiles), i32(tile_group)
        self.g_cells_h = cells
        self.g_order = i32(np.argsort(-np.diff(cells), kind="stable"))  # largest case first
        # momentum diffusion scaled by each case's viscosity (owner's case for faces)
        t = fv.t
        mu_f = self.mu_case[g_dev[t["fP"].cpu().numpy()]] if fv.n_if else np.zeros(0)
        mu_b = self.mu_case[g_dev[t["bP"].cpu().numpy()]] if fv.n_bf else np.zeros(0)
        f64 = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=dev)  # noqa: E731
        self._mom_t = {
            "alpha": f64(mu_f * t["alpha"].cpu().numpy()) if fv.n_if else t["alpha"],
            "alpha_b": f64(mu_b * t["alpha_b"].cpu().numpy()) if fv.n_bf else t["alpha_b"],
            "Tv": f64(mu_f[None, :] * t["Tv"].cpu().numpy().reshape(fv.dim, -1)) if fv.n_if else t["Tv"],
        }
        mm = _lib.Mesh()
        ctypes.memmove(ctypes.byref(mm), ctypes.byref(fv.cmesh), ctypes.sizeof(mm))
        mm.alpha, mm.alpha_b, mm.Tv = (self._mom_t[k].data_ptr() for k in ("alpha", "alpha_b", "Tv"))
        self._mesh_mom = mm
        self._m_mom = ctypes.byref(mm)

    def _build_boundaries(self):
        import torch

        super()._build_boundaries()
        fv = self.fv
        g_dev = self._cell_groups[fv.perm]
        bP = fv.t["bP"].cpu().numpy() if fv.n_bf else np.zeros(0, dtype=np.int64)
        m_pres_dev = self._bc_t["m_pres"].cpu().numpy()[: fv.n_bf]  # device boundary-face order
        open_ = np.zeros(self.ncase, dtype=bool)
        if fv.n_bf:
            np.logical_or.at(open_, g_dev[bP], m_pres_dev > 0)
        self.case_singular = ~open_
        self.g_singular = torch.as_tensor(self.case_singular.astype(np.int32), device=self.torch_device)

    def _allocate(self):
        import torch

        super()._allocate()
        dev, nc, dim, ng = self.torch_device, self.nc, self.dim, self.ncase
        L = _lib.lib()
        wb = L.b2s_bicgstab_groups_workspace_bytes(nc, dim, 1)
        self.work_bicg_g = torch.empty(wb // 8 + 1, dtype=torch.float64, device=dev)
        nrec = ng * (dim + 1)
        self.report_g = torch.zeros(ng * self.NQ * 8 + nrec * INFO_DTYPE.itemsize, dtype=torch.uint8, device=dev)
        self.report_g_host = torch.zeros_like(self.report_g, device="cpu").pin_memory()
        self.gscal = self.report_g[: ng * self.NQ * 8].view(torch.float64)
        base = self.report_g.data_ptr() + ng * self.NQ * 8
        self.info_mom_g = base
        self.info_p_g = base + ng * dim * INFO_DTYPE.itemsize
        # per-case relaxation (lowered per case by the stability guard), expanded per cell
        self.case_relax_u = np.full(ng, float(self.case.relax_u))
        self.case_relax_p = np.full(ng, float(self.relax_p))
        self.case_algo = [self.case.algorithm] * ng
        self.relax_u_c = torch.empty(nc, dtype=torch.float64, device=dev)
        self.relax_p_c = torch.empty(nc, dtype=torch.float64, device=dev)
        self.simplec_c = torch.empty(nc, dtype=torch.int32, device=dev)
        for g in range(ng):
            self._set_case_relax(g)

    def _setup_amg(self, start=0):
        """Host set-up of the batch hierarchy (aggregates numbered case by case; never
        re-aggregated, so ``start`` is always 0)."""
        import torch

        torch.cuda.current_stream().synchronize()
        self._graphs.clear()  # captured iterations reference the old hierarchy's buffers
        self.val_P.copy_(self.val_P32)
        A_host = self.fv.matrix_to_host(self.val_P)
        self._amg = AMGHierarchy(A_host, self.fv.perm, self.fv.rowptr, self.fv.col, self.fv.t["slot_diag"],
                                 self.val_P, self.fv.slot_ref, singular=False, max_coarse=self.max_coarse,
                                 theta=self.amg_theta, groups=self._cell_groups,
                                 group_singular=self.case_singular.astype(np.int32))
        self.amg_setups += 1
        self._amg_fresh = False
        self._amg.enable_mixed(self.val_P32)

    def _params(self):
        prm = super()._params()
        prm.relax_u_cell = self.relax_u_c.data_ptr()
        prm.relax_p_cell = self.relax_p_c.data_ptr()
        prm.simplec_cell = self.simplec_c.data_ptr()
        return prm

    def _set_case_relax(self, g):
        a, b = int(self.g_cells_h[g]), int(self.g_cells_h[g + 1])
        self.relax_u_c[a:b] = float(self.case_relax_u[g])
        self.relax_p_c[a:b] = float(self.case_relax_p[g])
        self.simplec_c[a:b] = int(self.case_algo[g] == "SIMPLEC")

    # ------------------------------------------------------------------ stability guard per case
    def _case_slices(self, g):
        """Device index ranges of case g: cells, owned interior faces, boundary faces."""
        a, b = int(self.g_cells_h[g]), int(self.g_cells_h[g + 1])
        return (a, b), (int(self._own_ptr_h[a]), int(self._own_ptr_h[b])), (int(self._bptr_h[a]), int(self._bptr_h[b]))

    def _snapshot_cases(self, cases):
        c = self._cur
        self._snap_it[cases] = self.iteration
        if len(cases) == self.ncase:  # every case: whole-array copies
            self._snap_Up.copy_(self._Up[c])
            self._snap_F.copy_(self._F[c])
            self._snap_Fb.copy_(self._Fb[c])
            return
        for g in cases:
            (a, b), (fa, fb), (ba, bb) = self._case_slices(g)
            self._snap_Up[:, a:b] = self._Up[c][:, a:b]
            self._snap_F[fa:fb] = self._F[c][fa:fb]
            self._snap_Fb[ba:bb] = self._Fb[c][ba:bb]

    def _restore_case(self, g):
        c = self._cur
        (a, b), (fa, fb), (ba, bb) = self._case_slices(g)
        self._Up[c][:, a:b] = self._snap_Up[:, a:b]
        self._F[c][fa:fb] = self._snap_F[fa:fb]
        self._Fb[c][ba:bb] = self._snap_Fb[ba:bb]
        # no lagged gradients for the restored case (the single-case rollback drops them too)
        self.gUp[:, :, a:b] = 0.0
        self.gpf[:, a:b] = 0.0

    def _reset_guard(self):
        super()._reset_guard()
        if not hasattr(self, "g_cells_h"):
            return
        ng = self.ncase
        self._own_ptr_h = self.fv.t["own_ptr"].cpu().numpy()
        self._bptr_h = self.fv.t["bptr"].cpu().numpy()
        c = self._cur
        self._snap_Up, self._snap_F, self._snap_Fb = self._Up[c].clone(), self._F[c].clone(), self._Fb[c].clone()
        self._snap_it = np.zeros(ng, dtype=np.int64)
        self._snap_r = np.full(ng, np.inf)
        self._case_guard_min = np.full(ng, np.inf)
        self.case_guard_events = [[] for _ in range(ng)]

    def _case_guard(self, r, flux):
        """``SimpleSolver._stability_guard`` per case (``simple.py:722-776``): a case whose raw
        continuity residual is not finite or grew GUARD_GROWTH-fold over its best goes back to
        its last snapshot with lower relaxation (pressure first, then SIMPLE with 0.3 / 0.3)."""
        rolled = np.zeros(self.ncase, dtype=bool)
        if not self.guard_enabled:
            return rolled
        ref = np.maximum(self._case_guard_min, self.GUARD_ROUNDOFF * flux)
        bad = ~np.isfinite(r) | ((self.iteration > 10) & (r > self.GUARD_GROWTH * ref))
        for g in np.flatnonzero(bad):
            if self.case_relax_p[g] * self.GUARD_FACTOR >= self.GUARD_MIN_RELAX:
                self.case_relax_p[g] *= self.GUARD_FACTOR
            elif self.case_algo[g] == "SIMPLEC" or self.case_relax_u[g] * 0.7 >= self.GUARD_MIN_RELAX_U - 1e-12:
                if self.case_algo[g] == "SIMPLEC":
                    self.case_algo[g] = "SIMPLE"
                    self.case_relax_u[g], self.case_relax_p[g] = min(self.case_relax_u[g], 0.3), 0.3
                else:
                    self.case_relax_u[g] *= 0.7
            else:
                continue
            self._restore_case(int(g))
            self._set_case_relax(int(g))
            self._case_guard_min[g] = self._snap_r[g]
            self.case_guard_events[g].append({"detected_at": self.iteration, "restored_to": int(self._snap_it[g]),
                                              "relax_p": round(float(self.case_relax_p[g]), 4),
                                              "relax_u": round(float(self.case_relax_u[g]), 4),
                                              "algorithm": self.case_algo[g], "continuity": float(r[g])})
            rolled[g] = True
        if rolled.any():
            self._amg_age = 10 ** 9  # a new preconditioner, as after the single-case rollback
        ok = np.isfinite(r) & ~rolled & (self.iteration > 5)
        self._case_guard_min[ok] = np.minimum(self._case_guard_min[ok], r[ok])
        if self.iteration % self.GUARD_EVERY == 0:
            snap = np.flatnonzero(ok & (r <= 2.0 * self._case_guard_min))
            self._snapshot_cases(snap)
            self._snap_r[snap] = r[snap]
        return rolled

    # ------------------------------------------------------------------ iteration
    def _launch(self, amg_ready=False):
        L, fv = _lib.lib(), self.fv
        self._mark("start")
        s = _lib.stream_ptr()
        m, bc = fv.cmesh_ref, ctypes.byref(self.cbc)
        prm = self._params()
        pr = ctypes.byref(prm)
        dim, nc, ng = self.dim, self.nc, self.ncase
        old = self._cur
        new = next(i for i in range(3) if i != old)
        Up, F, Fb = self._Up[old], self._F[old], self._Fb[old]
        lag = self._lag
        gg = self.case.pressure_gradient == "green-gauss"
        gp_force_prev = self.gpf if gg else self.gUp[0]
        _lib.check(L.b2s_flow_bvals_d(m, bc, Up.data_ptr(), self.gUp.data_ptr() if lag else None,
                                      gp_force_prev.data_ptr() if lag else None, self.bUp.data_ptr(), s),
                   "b2s_flow_bvals_d")
        _lib.check(L.b2s_ls_gradient_d(m, 1 + dim, Up.data_ptr(), self.bUp.data_ptr(), self.gUp.data_ptr(), s),
                   "b2s_ls_gradient_d")
        if gg:
            _lib.check(L.b2s_gg_gradient_d(m, Up.data_ptr(), self.bUp.data_ptr(), self.gUp.data_ptr(),
                                           self.gpf.data_ptr(), s), "b2s_gg_gradient_d")
            gp = self.gpf
        else:
            gp = self.gUp[0]
        self._lag = True
        self.kernel_launches += 3 if gg else 2
        self._mark("gradients")
        part = self.part
        pt = lambda q: part.data_ptr() + 8 * q * self.nblk  # noqa: E731
        _lib.check(L.b2s_momentum_assemble_mixed_d(self._m_mom, bc, pr, Up.data_ptr(), self.gUp.data_ptr(),
                                                   gp.data_ptr(), self.bUp.data_ptr(), F.data_ptr(), Fb.data_ptr(),
                                                   None, None, self.val_A32.data_ptr(), self.inv32.data_ptr(),
                                                   self.dP.data_ptr(), self.r32.data_ptr(), pt(self.Q_MOM), s),
                   "b2s_momentum_assemble_mixed_d")
        self._mark("momentum_assembly")
        _lib.check(L.b2s_bicgstab_groups_f32_d(ng, self.g_cells.data_ptr(), self.g_order.data_ptr(), nc, dim,
                                               fv.rowptr.data_ptr(), fv.col.data_ptr(), self.val_A32.data_ptr(),
                                               self.r32.data_ptr(), self.inv32.data_ptr(), self.dU32.data_ptr(), 0.1,
                                               30, 1, 1, self.Ustar.data_ptr(), Up[1:].data_ptr(),
                                               self.work_bicg_g.data_ptr(), self.work_bicg_g.numel() * 8,
                                               self.info_mom_g, ctypes.byref(self.team_momentum), s),
                   "b2s_bicgstab_groups_f32_d")
        self._mark("momentum_solve")
        _lib.check(L.b2s_pressure_assemble_mixed_d(m, bc, pr, self.Ustar.data_ptr(), Up.data_ptr(), gp.data_ptr(),
                                                   self.dP.data_ptr(), self.Fst.data_ptr(), self.cf.data_ptr(),
                                                   self.Fbst.data_ptr(), self.cb.data_ptr(), self.val_P32.data_ptr(),
                                                   self.rhs_p.data_ptr(), pt(self.Q_CONT), s),
                   "b2s_pressure_assemble_mixed_d")
        self.kernel_launches += 3
        self._mark("pressure_assembly")
        if not amg_ready:
            self._ensure_amg(s)
        self._mark("amg_rebuild")
        self._amg.pcg_groups_mixed(m, self.g_order, self.g_singular, self.cf, self.cb, self.rhs_p, self.pp,
                                   self.case.pressure_tol, 200, self.info_p_g, maxpass=self.REFINE_PASSES,
                                   min_inner_tol=self.INNER_TOL_FLOOR, team=self.team)
        self.kernel_launches += 1
        self._mark("pressure_solve")
        Upn, Fn, Fbn = self._Up[new], self._F[new], self._Fb[new]
        _lib.check(L.b2s_correct_d(m, bc, pr, self.Fst.data_ptr(), self.cf.data_ptr(), self.Fbst.data_ptr(),
                                   self.cb.data_ptr(), self.pp.data_ptr(), Up.data_ptr(), self.Ustar.data_ptr(),
                                   self.dP.data_ptr(), Fn.data_ptr(), Fbn.data_ptr(), Upn.data_ptr(),
                                   pt(self.Q_SUMP), s), "b2s_correct_d")
        self.kernel_launches += 1
        if self.case_singular.any():
            _lib.check(L.b2s_remove_group_means_d(m, Upn.data_ptr(), part.data_ptr(), self.nblk, self.Q_SUMP,
                                                  self.g_tiles.data_ptr(), self.g_tile_group.data_ptr(),
                                                  self.g_cells.data_ptr(), self.g_singular.data_ptr(), s),
                       "b2s_remove_group_means_d")
            self.kernel_launches += 1
        self._mark("corrections")
        _lib.check(L.b2s_group_sums_d(part.data_ptr(), self.nblk, self.NQ, ng, self.g_tiles.data_ptr(),
                                      self.gscal.data_ptr(), s), "b2s_group_sums_d")
        self.kernel_launches += 1
        self._mark("residuals")
        return old, new

    def _read_report(self):
        import torch

        self.report_g_host.copy_(self.report_g, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        if self._events:
            self._resolve_stage_events()
        raw = self.report_g_host.numpy()
        ng = self.ncase
        scal = raw[: ng * self.NQ * 8].view(np.float64).reshape(ng, self.NQ).copy()
        # the solve records as one structured array (one Python object per record would cost
        # milliseconds per iteration for hundreds of cases)
        infos = raw[ng * self.NQ * 8:].view(INFO_DTYPE).copy()
        return scal, infos

    def step(self) -> float:
        """One outer iteration of every case (``simple.py:500-703`` per case)."""
        if self.finished:
            return 0.0
        self._capture = None
        c, dim, ng = self.case, self.dim, self.ncase
        rebuild_due = self._amg is None or self._amg_age >= self.amg_rebuild
        if self.use_graphs and not rebuild_due and self._lag and not self.profile_stages:
            try:
                old, new = self._launch_graph()
            except RuntimeError:
                self.use_graphs = False
                self._graphs.clear()
                old, new = self._launch()
        else:
            old, new = self._launch()
        scal, infos = self._read_report()
        self._cur = new
        self.iteration += 1
        self.step_count = self.iteration
        num = scal[:, self.Q_MOM:self.Q_MOM + dim]
        den = scal[:, self.Q_MOM + dim:self.Q_MOM + 2 * dim]
        floor = 1e-3 * np.maximum(den.max(axis=1), 1e-300)
        res = {name: num[:, k] / np.maximum(den[:, k], floor) for k, name in enumerate(COMPONENTS[:dim])}
        cont = scal[:, self.Q_CONT].copy()
        if self.iteration <= 5:
            self._res_max5_case = np.maximum(self._res_max5_case, np.maximum(cont, 1e-300))
        flux = scal[:, self.Q_SUMF] + scal[:, self.Q_SUMFB]
        res["continuity"] = cont / np.maximum(self._res_max5_case, 1e-3 * flux)
        self._case_res = res
        rolled = self._case_guard(cont, flux)
        it = infos["iterations"].astype(np.int64)
        self.last_linear = {"momentum_iters": it[: ng * dim].reshape(ng, dim),
                            "pressure_iters": it[ng * dim: ng * (dim + 1)],
                            "pressure_residual": infos["residual"][ng * dim: ng * (dim + 1)].astype(np.float64)}
        worst = np.max(np.stack(list(res.values())), axis=0)
        done = (worst < c.tol) & (self.iteration > 5) & ~rolled
        newly = done & (self.case_converged_at < 0)
        self.case_converged_at[newly] = self.iteration
        self.converged = bool(np.all(self.case_converged_at >= 0))
        return 1.0

    def autotune(self, candidates=None, reps=5, margin=0.05) -> dict:
        """Pick the team shapes of the per-case Krylov solves (``b2s_team_config``: blocks per
        thread-block cluster, threads per block, the mean row length from which rows are walked
        one warp per row), one for the momentum Jacobi-BiCGSTAB and one for the refined
        pressure-correction AMG-PCG, by timing every candidate on this batch's current systems
        (those of the last outer iteration; one is run first if none has): each solve ``reps``
        times after one untimed call, CUDA events, median. A candidate replaces the current shape
        only when it is faster by more than ``margin`` (timing noise must not pick a shape). The
        timed solves write scratch copies, so the solver's state is unchanged; captured graphs
        are dropped (they hold the previous shapes). A candidate the device cannot launch is
        skipped. Returns {"momentum": shape, "pressure": shape, "ms": {candidate: (momentum ms,
        pressure ms) or None}}."""
        import torch

        if self._amg is None or self.iteration == 0:
            self.step()
        L, fv, ng, dim, nc = _lib.lib(), self.fv, self.ncase, self.dim, self.nc
        s = _lib.stream_ptr()
        dev = self.torch_device
        dU = torch.empty_like(self.dU32)
        Ust = torch.empty_like(self.Ustar)
        pp = torch.empty_like(self.pp)
        info = torch.zeros(ng * max(dim, 1) * INFO_DTYPE.itemsize, dtype=torch.uint8, device=dev)
        base = self._Up[self._cur][1:]
        m = fv.cmesh_ref

        def momentum(team):
            _lib.check(L.b2s_bicgstab_groups_f32_d(ng, self.g_cells.data_ptr(), self.g_order.data_ptr(), nc, dim,
                                                   fv.rowptr.data_ptr(), fv.col.data_ptr(), self.val_A32.data_ptr(),
                                                   self.r32.data_ptr(), self.inv32.data_ptr(), dU.data_ptr(), 0.1, 30,
                                                   1, 1, Ust.data_ptr(), base.data_ptr(), self.work_bicg_g.data_ptr(),
                                                   self.work_bicg_g.numel() * 8, info.data_ptr(), ctypes.byref(team),
                                                   s), "b2s_bicgstab_groups_f32_d")

        def pressure(team):
            self._amg.pcg_groups_mixed(m, self.g_order, self.g_singular, self.cf, self.cb, self.rhs_p, pp,
                                       self.case.pressure_tol, 200, info.data_ptr(), maxpass=self.REFINE_PASSES,
                                       min_inner_tol=self.INNER_TOL_FLOOR, team=team)

        def timed(fn, team):
            fn(team)
            torch.cuda.synchronize()
            ms = []
            for _ in range(reps):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                fn(team)
                e1.record()
                torch.cuda.synchronize()
                ms.append(e0.elapsed_time(e1))
            return float(np.median(ms))

        cur_m = (self.team_momentum.cluster_blocks, self.team_momentum.block_threads, self.team_momentum.wide_row)
        cur_p = (self.team.cluster_blocks, self.team.block_threads, self.team.wide_row)
        cands = [tuple(c) for c in (candidates or self.TEAM_CANDIDATES)]
        times = {}
        for cand in dict.fromkeys(cands + [cur_m, cur_p]):
            team = _lib.TeamConfig(*cand, 0)
            try:
                times[cand] = (timed(momentum, team), timed(pressure, team))
            except RuntimeError:
                times[cand] = None
        ok = {k: v for k, v in times.items() if v is not None}
        if not ok:
            raise RuntimeError("no team shape could be launched")
        choice = []
        for q, cur in ((0, cur_m), (1, cur_p)):
            best = min(ok, key=lambda k: ok[k][q])
            keep = cur in ok and ok[best][q] > (1.0 - margin) * ok[cur][q]
            choice.append(cur if keep else best)
        self.team_momentum = _lib.TeamConfig(*choice[0], 0)
        self.team = _lib.TeamConfig(*choice[1], 0)
        self._graphs.clear()
        self.tuning = {"momentum": choice[0], "pressure": choice[1], "ms": times}
        return self.tuning

    def run(self, max_steps=None, hooks=None) -> int:
        """Step until every case converged or ``max_iter`` (or ``max_steps``), one iteration at a
        time (the per-case guard reads each iteration's report before the next one starts).
        ``hooks`` as ``SimpleSolver.run``."""
        before, after, done = (tuple(hooks) + (None,) * 3)[:3] if hooks is not None else (None, None, None)
        n = 0
        while not self.finished and (max_steps is None or n < max_steps):
            if before:
                before()
            self.step()
            if after:
                after()
            if done:
                done()
            n += 1
        return n

    @property
    def finished(self) -> bool:
        return self.converged or self.iteration >= self.case.max_iter

    def case_residuals(self, i: int) -> dict:
        """Scaled residuals of case i after the last iteration (``simple.py:675-703``)."""
        return {k: float(v[i]) for k, v in self._case_res.items()}

    def case_fields(self, i: int) -> dict:
        """``fields()`` of case i (host arrays in its own cell numbering)."""
        f = self.fields()
        a, b = int(self.case_offsets[i]), int(self.case_offsets[i + 1])
        return {k: v[a:b] for k, v in f.items()}

    def residuals(self) -> dict:
        return {"scaled": {k: float(np.max(v)) for k, v in self._case_res.items()}}

    def diagnostics(self) -> dict:
        raise NotImplementedError("diagnostics() is per case: solve the case with SimpleSolver")
