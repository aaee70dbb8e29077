"""Pressure-based SIMPLE/SIMPLEC solver on unstructured meshes, on one B200.

Drop-in for ``flowtrace.unstructured.simple.SimpleSolver`` (``flowtrace/unstructured/
simple.py:71-1072``) on its steady path, laminar or with the k-omega SST model: same
constructor, ``step()``, ``finished``, ``converged``, ``residuals()``, ``diagnostics()``,
``fields()``, ``state_dict()`` / ``load_state()``, ``initialize()``, ``set_sources()``,
``describe()``, ``mass_balance()``, ``wall_forces()``, ``wall_report()``, ``wall_profile()``,
``heat_flow()``, ``cell_centres()``, ``last_linear``, ``guard_events``, the relaxation
attributes and the divergence guard, with the same algorithm.

One outer iteration is a fixed sequence of CUDA stages from ``libb2simplec.so`` on the
current stream, with no host synchronisation until its end, where one device->host copy
brings back the residual sums and the linear-solver records:

  1. boundary values of p and U with the lagged gradients          b2s_flow_bvals_d
  2. least-squares gradients of p and every U component, fused     b2s_ls_gradient_d
  3. Green-Gauss pressure-force gradient                           b2s_gg_gradient_d
  4. momentum coefficients, right-hand sides, relaxed CSR values,
     Jacobi inverse, SIMPLEC d and scaled-residual sums, fused     b2s_momentum_assemble_d
  5. Jacobi-BiCGSTAB of all velocity components, one launch        b2s_bicgstab_jacobi_d
  6. Rhie-Chow fluxes, p' system and continuity sum, fused         b2s_pressure_assemble_d
  7. AMG numeric rebuild every ``amg_rebuild`` iterations          b2s_amg_rebuild_d
  8. AMG-PCG of the pressure correction, one launch                b2s_pcg_amg_d
  9. flux, pressure and velocity corrections with grad(p'), fused  b2s_correct_d (+ mean removal)
 10. energy: boundary values, gradient, assembly, BiCGSTAB         b2s_energy_*_d
 11. k-omega SST: k and omega, mu_t (``turbulence.DeviceSST``)     b2s_sst_*_d
 12. residual sums                                                 b2s_sum_partials_d

With the SST model, stage 4 takes per-face viscosities (mu + mu_t, Spalding's wall-function
viscosity on walls) and the transpose-stress source from b2s_sst_momentum_terms_d, run between
stages 3 and 4, and the energy equation the turbulent diffusivity k/cp + mu_t/Pr_t.

Fields live on the device in the mesh's device numbering, component-major. The public
attributes ``U``, ``p``, ``T``, ``F``, ``Fb`` and every report return host arrays in the
reference's numbering. There is no CPU fallback: without a CUDA device the constructor
raises.

Not implemented (the constructor raises ``NotImplementedError``): the k-epsilon models,
radiation, species, moving reference frames, periodic pairs and transient runs (and the SST
model in the batched form). Cases with solid zones go to ``conjugate.make_solver``.
Additions over the reference: ``set_porosity`` (implicit Brinkman drag alpha V on the momentum
diagonal) and ``set_boundary_velocity`` (a per-face velocity profile on a wall or inlet zone).
"""

from __future__ import annotations

import ctypes
import math
import time
from collections import defaultdict
from typing import Dict

import numpy as np

from .. import _lib
from ..linalg.amg import AMGHierarchy
from ..linalg.krylov import INFO_DTYPE, read_info
from ..mesh.unstructured import UnstructuredMesh
from .case import FLUENT_TO_KIND, BoundarySpec, UnstructuredCase
from .fvmesh import FVMesh

WALL, INLET, OUTLET, PRESSURE, SYMMETRY = range(5)
T_ADIABATIC, T_FIXED, T_FLUX = range(3)
_KIND_CODE = {"wall": WALL, "inlet": INLET, "outlet": OUTLET, "pressure": PRESSURE, "symmetry": SYMMETRY}
COMPONENTS = ("x-velocity", "y-velocity", "z-velocity")


def auto_relax_p(non_orthogonality_deg: float) -> float:
    """Initial SIMPLEC pressure relaxation (``flowtrace/unstructured/simple.py:53-64``)."""
    return 1.0 if non_orthogonality_deg <= 5.0 else 0.8


class DeviceBackend:
    """The ``backend`` attribute callers of the reference use (``be.to_numpy``, ``be.name``)."""

    name = "b200"
    device = "gpu"
    is_gpu = True

    def __init__(self, torch_device):
        self.torch_device = torch_device

    @staticmethod
    def to_numpy(a):
        if hasattr(a, "detach"):
            return a.detach().cpu().numpy()
        return np.asarray(a)

    def synchronize(self):
        import torch

        torch.cuda.synchronize(self.torch_device)


def _check_scope(case: UnstructuredCase, precisions=("fp64",), turbulence=("laminar",)):
    unsupported = []
    if case.turbulence not in turbulence:
        unsupported.append(f"turbulence={case.turbulence!r}")
    if case.radiation != "off":
        unsupported.append("radiation")
    if case.species:
        unsupported.append("species")
    if case.mrf:
        unsupported.append("moving reference frames")
    if case.solids:
        unsupported.append("solid zones")
    if case.periodic:
        unsupported.append("periodic pairs")
    if case.unsteady:
        unsupported.append("transient runs")
    if any(case.buoyancy[:3]):
        unsupported.append("buoyancy")
    if case.precision not in precisions:
        unsupported.append(f"precision={case.precision!r} in SimpleSolver (use MixedSimpleSolver)")
    if unsupported:
        raise NotImplementedError("the B200 SIMPLEC path does not implement: " + ", ".join(unsupported))


class SimpleSolver:
    GUARD_GROWTH = 20.0
    GUARD_ROUNDOFF = 1e-6
    GUARD_EVERY = 20
    GUARD_FACTOR = 0.6
    GUARD_MIN_RELAX = 0.1
    GUARD_FALLBACK = True
    GUARD_MIN_RELAX_U = 0.2
    PRECISIONS = ("fp64",)
    TURBULENCE = ("laminar", "k-omega-sst")

    def __init__(self, mesh: UnstructuredMesh, case: UnstructuredCase, backend=None, max_coarse: int = 150,
                 amg_theta: float = 0.08):
        """``max_coarse``: rows at which the AMG hierarchy stops coarsening (the reference uses 300;
        150 keeps the coarse inverse in shared memory). ``amg_theta``: strength-of-connection
        threshold of the aggregation; 0.08 is the reference's own smoothed aggregation
        (``flowtrace/linalg/amg.py:80-101``, its preconditioner on GPU backends), 0.0 the strength
        rule of pyamg's ``smoothed_aggregation_solver`` defaults that its CPU backend calls
        (``amg.py:149-168``), far better conditioned on anisotropic 3-D meshes."""
        import torch

        _check_scope(case, self.PRECISIONS, self.TURBULENCE)
        self.case, self.mesh = case, mesh
        self.torch_device = _lib.require_device()
        self.be = DeviceBackend(self.torch_device)
        self.dtype = np.dtype(np.float64)
        t0 = time.perf_counter()
        self.fv = fv = FVMesh(mesh, self.torch_device, groups=getattr(self, "_cell_groups", None))
        self._prepare_mesh()
        self.dim = dim = mesh.dim
        self.nc = nc = mesh.n_cells
        self.energy = bool(case.energy)
        self.timers: Dict[str, float] = defaultdict(float)
        self.iteration = 0
        self.step_count = 0
        self.converged = False
        self._res_max5: Dict[str, float] = {}
        self.history = []
        self._amg = None
        self._amg_age = 10 ** 9
        self.amg_rebuild = 10
        self.amg_setups = 0
        # False: aggregates fixed at the first set-up, every numeric quantity rebuilt on the device
        # (no host work after the first iteration). True: the reference's behaviour (it
        # re-aggregates at every rebuild) - the device set-up is redone whenever the strength
        # graph of some level changed (a device check; unchanged graphs give the same
        # aggregates). Fixed aggregates give a preconditioner the reference never builds; on
        # strongly varying coefficients (Brinkman porosity) that can stall the outer iteration,
        # so porous problems (``adjoint.PorousChannel``) turn re-aggregation on.
        self.reaggregate = False
        self.host_amg_setup = False  # True: the host set-up (SciPy) instead of the device set-up
        # the last rebuild re-aggregated: the next one likely will too, so the iterations in
        # between are enqueued stage by stage rather than captured into a CUDA graph that the
        # next set-up would drop (a capture costs more than the replays it saves over 10
        # iterations: 1.25 against 1.10 ms per iteration with re-aggregation on the 131k cavity)
        self._reaggregated = False
        self._perm_dev = None
        self.max_coarse = int(max_coarse)
        self.amg_theta = float(amg_theta)
        self.last_linear = {}
        self.external_energy = False
        self.relax_p = float(case.relax_p) if case.relax_p is not None else auto_relax_p(fv.non_orthogonality_deg)
        self.kernel_launches = 0  # launches of libb2simplec kernels so far
        self.stage_times = defaultdict(float)  # device milliseconds per stage when profile_stages is on
        self.profile_stages = False
        self._events = []
        self.use_graphs = True  # replay the stage sequence as a CUDA graph when no AMG rebuild is due
        self._graphs = {}
        self._lag = False  # lagged gradients available for the boundary reconstruction
        self._lagT = False
        self.porosity = None
        self.mom_source = None
        self.energy_source = None
        self.turb = None
        self._build_boundaries()
        self._allocate()
        if case.turbulence == "k-omega-sst":
            from .turbulence import DeviceSST

            self.turb = DeviceSST(self)
        U0 = np.zeros((nc, dim))
        U0[:] = (list(case.init_velocity) + [0.0] * 3)[:dim]
        T0 = np.full(nc, float(case.init_T)) if self.energy else None
        self._set_fields_host(U0, np.zeros(nc), T0)
        self.guard_enabled = case.relax_p is None and not case.unsteady
        self._capture = None
        self._reset_guard()
        torch.cuda.synchronize(self.torch_device)
        self.setup_seconds = time.perf_counter() - t0

    # ------------------------------------------------------------------ set-up
    def _prepare_mesh(self):
        """Hook run right after the device mesh is built (batches tile it here)."""
        self._m_mom = self.fv.cmesh_ref  # mesh of the momentum assembly (batches scale its diffusion)
    def _build_boundaries(self):
        """Boundary kinds, fixed values and masks (``flowtrace/unstructured/simple.py:185-240``)."""
        fv, case, dim = self.fv, self.case, self.dim
        n = fv.n_bf
        normals = None
        kind = np.zeros(n, dtype=np.int64)
        ub = np.zeros((n, dim))
        pb = np.zeros(n)
        tk = np.zeros(n, dtype=np.int64)
        tv = np.zeros(n)
        self.zone_specs = {}
        for z in self.mesh.boundary_zones():
            spec = case.boundaries.get(z.name)
            if spec is None:
                spec = BoundarySpec(kind=FLUENT_TO_KIND.get(z.type, "wall"))
                if spec.kind == "inlet":
                    spec.normal_speed = 1.0
            self.zone_specs[z.name] = spec
            m = fv.bzone == z.id
            if spec.kind == "periodic" or z.type in ("periodic", "periodic-shadow"):
                if m.any():
                    raise ValueError(f"zone {z.name!r} is periodic but not paired")
                continue
            if spec.rotation is not None:
                raise NotImplementedError("rotating walls are not implemented on the B200 path")
            kind[m] = _KIND_CODE[spec.kind]
            if spec.kind in ("wall", "inlet"):
                if spec.velocity is not None:
                    ub[m] = (list(spec.velocity) + [0.0, 0.0, 0.0])[:dim]
                elif spec.normal_speed is not None:
                    if normals is None:
                        normals = fv.boundary_normals_host()
                    ub[m] = -spec.normal_speed * normals[m]
            pb[m] = spec.pressure
            if spec.kind == "wall":
                tk[m] = {"adiabatic": T_ADIABATIC, "temperature": T_FIXED, "flux": T_FLUX}[spec.thermal]
            elif spec.kind in ("inlet", "pressure"):
                tk[m] = T_FIXED
            tv[m] = spec.value
        self.bkind_h, self.tkind_h = kind, tk
        self._ub_fixed_h, self._pb_fixed_h, self._tval_h = ub, pb, tv
        self.m_wall_h = (kind == WALL).astype(np.float64)
        self.m_inlet_h = (kind == INLET).astype(np.float64)
        self.m_pres_h = ((kind == OUTLET) | (kind == PRESSURE)).astype(np.float64)
        self.m_sym_h = (kind == SYMMETRY).astype(np.float64)
        self.m_dirvel_h = ((kind == WALL) | (kind == INLET) | (kind == SYMMETRY)).astype(np.float64)
        self.singular_p = not bool(((kind == OUTLET) | (kind == PRESSURE)).any())
        up = fv.bfaces_to_device
        self._bc_t = {
            "m_wall": up(self.m_wall_h), "m_inlet": up(self.m_inlet_h), "m_pres": up(self.m_pres_h),
            "m_sym": up(self.m_sym_h), "m_dirvel": up(self.m_dirvel_h), "ub_fixed": up(ub), "pb_fixed": up(pb),
            "m_tfix": up((tk == T_FIXED).astype(np.float64)), "m_tflux": up((tk == T_FLUX).astype(np.float64)),
            "m_out": up((kind == OUTLET).astype(np.float64)), "tval": up(tv),
        }
        if n == 0:
            import torch

            self._bc_t = {k: torch.zeros(1, dtype=torch.float64, device=self.torch_device) for k in self._bc_t}
        self.cbc = _lib.BC(**{k: v.data_ptr() for k, v in self._bc_t.items()})

    def _params(self):
        c = self.case
        body = (list(c.body_force) + [0.0, 0.0, 0.0])[:3]
        return _lib.FlowParams(rho=float(c.density), mu=float(c.viscosity), relax_u=float(self.relax_u),
                               relax_p=float(self.relax_p), body=(ctypes.c_double * 3)(*body),
                               simplec=int(self.algo == "SIMPLEC"), second_order=int(c.scheme == "second-order"),
                               singular_p=int(self.singular_p), pad=0)

    def _allocate(self):
        import torch

        dev, fv = self.torch_device, self.fv
        nc, nf, nb, dim, nnz = fv.nc, fv.n_if, max(fv.n_bf, 1), fv.dim, fv.nnz
        z = lambda *s: torch.zeros(*s, dtype=torch.float64, device=dev)  # noqa: E731
        self._Up = [z(1 + dim, nc) for _ in range(3)]
        self._F = [z(max(nf, 1)) for _ in range(3)]
        self._Fb = [z(nb) for _ in range(3)]
        self._T = [z(nc) for _ in range(3)] if self.energy else None
        self._cur = 0
        self.bUp, self.gUp, self.gpf = z(1 + dim, nb), z(1 + dim, dim, nc), z(dim, nc)
        self.val_A, self.diag, self.inv, self.dP = z(nnz), z(nc), z(nc), z(nc)
        self.bmom, self.brmom, self.Ustar = z(dim, nc), z(dim, nc), z(dim, nc)
        self.Fst, self.cf, self.Fbst, self.cb = z(max(nf, 1)), z(max(nf, 1)), z(nb), z(nb)
        self.val_P, self.rhs_p, self.pp = z(nnz), z(nc), z(nc)
        if self.energy:
            self.Tb, self.gT = z(nb), z(dim, nc)
            self.val_T, self.diagT, self.invT, self.bT, self.brT = z(nnz), z(nc), z(nc), z(nc), z(nc)
        L = _lib.lib()
        self.nblk = L.b2s_mesh_part_blocks(fv.cmesh_ref)
        self.Q_MOM, self.Q_CONT, self.Q_SUMP = 0, 2 * dim, 2 * dim + 1
        self.Q_SUMF, self.Q_SUMFB, self.Q_ENUM, self.Q_EDEN = 2 * dim + 2, 2 * dim + 3, 2 * dim + 4, 2 * dim + 5
        self.NQ = 2 * dim + 6
        ninfo = dim + 2
        if self.case.turbulence != "laminar":
            # per field (k, omega): the blocks' maximum diagonal, then the two residual sums
            self.Q_TMAX, self.Q_TRES = (self.NQ, self.NQ + 3), (self.NQ + 1, self.NQ + 4)
            self.NQ += 6
            ninfo += 2
        self.part = z(self.NQ * self.nblk)
        self.q_of = torch.arange(self.NQ, dtype=torch.int32, device=dev)
        self.report = torch.zeros(self.NQ * 8 + ninfo * INFO_DTYPE.itemsize, dtype=torch.uint8, device=dev)
        # two pinned host copies of the report, each with the event that marks its copy done, so
        # that run() can enqueue the next iteration while the host reads this one's report
        self.report_hosts = [torch.zeros_like(self.report, device="cpu").pin_memory() for _ in range(2)]
        self.report_host = self.report_hosts[0]
        self._rep_events = [torch.cuda.Event() for _ in range(2)]
        self._rep_slot = 0
        self.scal = self.report[: self.NQ * 8].view(torch.float64)
        base = self.report.data_ptr() + self.NQ * 8
        self.info_mom = base
        self.info_p = base + dim * INFO_DTYPE.itemsize
        self.info_T = base + (dim + 1) * INFO_DTYPE.itemsize
        self.info_turb = (base + (dim + 2) * INFO_DTYPE.itemsize, base + (dim + 3) * INFO_DTYPE.itemsize)
        wb = max(L.b2s_bicgstab_workspace_bytes(nc, dim), L.b2s_bicgstab_workspace_bytes(nc, 1))
        self.work_bicg = torch.empty(wb // 8 + 1, dtype=torch.float64, device=dev)

    def _set_fields_host(self, U, p, T):
        """Fields from host arrays (reference numbering); face fluxes rebuilt from U
        (``flowtrace/unstructured/simple.py:110-112,157-159``) on the device, with the
        reference's operations in its order: F = rho sum_k (w U_P + (1 - w) U_N)_k S_k,
        Fb = rho sum_k ub_k Sb_k on inlets and outlets, ub the velocity boundary values
        (fixed on walls and inlets, the tangential part of U_P on symmetry planes, U_P on
        outlets)."""
        import torch

        fv = self.fv
        c = self._cur
        self._Up[c][0].copy_(fv.cells_to_device(p))
        self._Up[c][1:].copy_(fv.cells_to_device(U))
        if self.energy and T is not None:
            self._T[c].copy_(fv.cells_to_device(T))
        Ud = self._Up[c][1:]
        t, rho, dim = fv.t, self.case.density, self.dim
        if fv.n_if:
            w, fP, fN = t["w"], t["fP"].long(), t["fN"].long()
            acc = None
            for k in range(dim):
                uf = w * Ud[k][fP] + (1.0 - w) * Ud[k][fN]
                term = uf * t["S"][k]
                acc = term if acc is None else acc + term
            self._F[c][: fv.n_if].copy_(rho * acc)
        if fv.n_bf:
            bc, bP = self._bc_t, t["bP"].long()
            UP = [Ud[k][bP] for k in range(dim)]
            nb = t["nbv"]
            un = None
            for k in range(dim):
                term = UP[k] * nb[k]
                un = term if un is None else un + term
            fixed = bc["m_wall"] + bc["m_inlet"]
            flux = None
            for k in range(dim):
                ubk = (fixed * bc["ub_fixed"][k] + bc["m_sym"] * (UP[k] - un * nb[k])) + bc["m_pres"] * UP[k]
                term = ubk * t["Sb"][k]
                flux = term if flux is None else flux + term
            self._Fb[c][: fv.n_bf].copy_((rho * flux) * (bc["m_inlet"] + bc["m_pres"]))
        self._lag = self._lagT = False
        torch.cuda.current_stream().synchronize()

    # ------------------------------------------------------------------ public state
    @property
    def U(self):
        return self.fv.cells_to_host(self._Up[self._cur][1:])

    @property
    def p(self):
        return self.fv.cells_to_host(self._Up[self._cur][0])

    @property
    def T(self):
        return self.fv.cells_to_host(self._T[self._cur]) if self.energy else None

    @property
    def F(self):
        return self.fv.faces_to_host(self._F[self._cur][: self.fv.n_if])

    @property
    def Fb(self):
        return self.fv.bfaces_to_host(self._Fb[self._cur][: self.fv.n_bf])

    @property
    def ub_fixed(self):
        """Fixed boundary velocities (n_bf, dim), reference numbering (a copy)."""
        return self._ub_fixed_h.copy()

    @ub_fixed.setter
    def ub_fixed(self, value):
        v = np.asarray(value, dtype=np.float64).reshape(self.fv.n_bf, self.dim)
        self._ub_fixed_h = v.copy()
        self._bc_t["ub_fixed"].copy_(self.fv.bfaces_to_device(v))

    def set_boundary_velocity(self, zone: str, values) -> None:
        """Per-face velocities (n_zone_faces, dim) on a wall or inlet zone, in the zone's face
        order; call ``initialize({})`` afterwards to rebuild the face fluxes."""
        z = self.mesh.zone_by_name(zone)
        if z is None:
            raise ValueError(f"unknown zone {zone!r}")
        m = self.fv.bzone == z.id
        if not np.all((self.bkind_h[m] == WALL) | (self.bkind_h[m] == INLET)):
            raise ValueError(f"zone {zone!r} is not a wall or an inlet")
        ub = self._ub_fixed_h.copy()
        ub[m] = np.asarray(values, dtype=np.float64).reshape(int(m.sum()), self.dim)
        self.ub_fixed = ub

    def set_porosity(self, alpha) -> None:
        """Implicit Brinkman drag: alpha_i V_i added to the momentum diagonal (None removes it)."""
        if alpha is not None and self.porosity is not None:
            self.porosity.copy_(self.fv.cells_to_device(np.asarray(alpha, dtype=np.float64)))
            return
        self._graphs.clear()  # captured iterations hold the previous buffer's address
        self.porosity = None if alpha is None else self.fv.cells_to_device(np.asarray(alpha, dtype=np.float64))

    def initialize(self, fields: dict) -> None:
        """``flowtrace/unstructured/simple.py:140-162``."""
        U = self.U
        for k, name in enumerate(COMPONENTS[: self.dim]):
            if name in fields:
                U[:, k] = np.asarray(fields[name], dtype=np.float64)
        p = self.p
        if "pressure" in fields:
            p = np.asarray(fields["pressure"], dtype=np.float64)
            if self.singular_p:
                p = p - p.mean()
        T = self.T
        if self.energy and "temperature" in fields:
            T = np.asarray(fields["temperature"], dtype=np.float64)
        self._set_fields_host(U, p, T)
        self._capture = None
        self._reset_guard()

    def set_sources(self, momentum=None, energy=None) -> None:
        """Volumetric sources (``flowtrace/unstructured/simple.py:164-182``)."""
        self._graphs.clear()  # captured iterations hold the previous buffers' addresses
        vol = self.fv.host.vol
        self.mom_source = None if momentum is None else self.fv.cells_to_device(
            np.asarray(momentum, dtype=np.float64).reshape(self.nc, self.dim) * vol[:, None])
        if energy is not None:
            if not self.energy:
                raise ValueError("energy source given but the energy equation is off")
            self.energy_source = self.fv.cells_to_device(
                np.asarray(energy, dtype=np.float64).reshape(self.nc) * vol / self.case.cp)
        else:
            self.energy_source = None

    # ------------------------------------------------------------------ the outer iteration
    @property
    def finished(self) -> bool:
        return self.converged or self.iteration >= self.case.max_iter

    def _setup_amg(self, start=0):
        """Set-up of the hierarchy from the current pressure-correction matrix, on the device
        (``AMGHierarchy.on_device``: the reference's aggregation and patterns without a host copy
        of the matrix; from level ``start`` on when re-aggregating, the levels above it shared
        with the current hierarchy); ``host_amg_setup`` selects the host set-up instead. Sets
        ``_amg_fresh``: every numeric quantity already computed from the current matrix."""
        import torch

        # captured iterations reference the old hierarchy's buffers, which are freed with it
        self._graphs.clear()
        if self.host_amg_setup:
            torch.cuda.current_stream().synchronize()
            A_host = self.fv.matrix_to_host(self.val_P)
            self._amg = AMGHierarchy(A_host, self.fv.perm, self.fv.rowptr, self.fv.col, self.fv.t["slot_diag"],
                                     self.val_P, self.fv.slot_ref, singular=self.singular_p,
                                     max_coarse=self.max_coarse, theta=self.amg_theta)
            self._amg_fresh = False
        else:
            if self._perm_dev is None:
                self._perm_dev = torch.as_tensor(self.fv.perm, dtype=torch.int64, device=self.val_P.device)
            self._amg = AMGHierarchy.on_device(self._perm_dev, self.fv.rowptr, self.fv.col, self.fv.t["slot_diag"],
                                               self.val_P, singular=self.singular_p, max_coarse=self.max_coarse,
                                               theta=self.amg_theta, prev=self._amg if start > 0 else None,
                                               start=start)
            self._amg_fresh = True
        self.amg_setups += 1

    def _ensure_amg(self, s):
        """Rebuild policy of ``simple.py:624-628``: a new preconditioner every ``amg_rebuild``
        iterations. The numeric rebuild runs on the device; with ``reaggregate``, when the
        strength graph of some level changed since the set-up (the reference would aggregate
        differently) the set-up is redone from that level on, so the hierarchy is always the
        reference's."""
        levels = lambda: self._amg.n_levels - 1  # noqa: E731
        if self._amg is None:
            self._setup_amg()
            if not self._amg_fresh:
                self._amg.rebuild()
            self.kernel_launches += 6 * levels() + 1
            self._amg_age = 0
        elif self._amg_age >= self.amg_rebuild:
            self._amg.rebuild()
            self.kernel_launches += 6 * levels() + 1
            if self.reaggregate:
                first = self._amg.first_strength_change()
                self.kernel_launches += levels()
                self._reaggregated = first >= 0
                if first >= 0:
                    self._setup_amg(start=first)
                    if not self._amg_fresh:
                        self._amg.rebuild()
                    self.kernel_launches += 6 * levels() + 1
            self._amg_age = 0
        self._amg_age += 1

    def _mark(self, name):
        """Record a CUDA event at a stage boundary (profile_stages only)."""
        if self.profile_stages:
            import torch

            ev = torch.cuda.Event(enable_timing=True)
            ev.record()
            self._events.append((name, ev))

    def _resolve_stage_events(self):
        ev = self._events
        for (_, a), (name, b) in zip(ev[:-1], ev[1:]):
            self.stage_times[name] += a.elapsed_time(b)
        self._events = []

    def _launch(self, amg_ready=False):
        """Enqueue one outer iteration's stages on the current stream (no synchronisation).
        With ``amg_ready`` the AMG hierarchy is current and no host work is done: the sequence
        can be captured into a CUDA graph."""
        L, fv = _lib.lib(), self.fv
        self._mark("start")
        s = _lib.stream_ptr()
        m, bc = fv.cmesh_ref, ctypes.byref(self.cbc)
        prm = self._params()
        pr = ctypes.byref(prm)
        dim, nc = self.dim, self.nc
        old = self._cur
        new = next(i for i in range(3) if i != old)
        Up, F, Fb = self._Up[old], self._F[old], self._Fb[old]
        lag = self._lag
        gp_force_prev = self.gpf if self.case.pressure_gradient == "green-gauss" else self.gUp[0]
        _lib.check(L.b2s_flow_bvals_d(m, bc, Up.data_ptr(), self.gUp.data_ptr() if lag else None,
                                      gp_force_prev.data_ptr() if lag else None, self.bUp.data_ptr(), s),
                   "b2s_flow_bvals_d")
        _lib.check(L.b2s_ls_gradient_d(m, 1 + dim, Up.data_ptr(), self.bUp.data_ptr(), self.gUp.data_ptr(), s),
                   "b2s_ls_gradient_d")
        if self.case.pressure_gradient == "green-gauss":
            _lib.check(L.b2s_gg_gradient_d(m, Up.data_ptr(), self.bUp.data_ptr(), self.gUp.data_ptr(),
                                           self.gpf.data_ptr(), s), "b2s_gg_gradient_d")
            gp = self.gpf
        else:
            gp = self.gUp[0]
        self._lag = True
        self.kernel_launches += 3 if self.case.pressure_gradient == "green-gauss" else 2
        self._mark("gradients")
        part = self.part
        pt = lambda q: part.data_ptr() + 8 * q * self.nblk  # noqa: E731
        por = None if self.porosity is None else self.porosity.data_ptr()
        msrc = None if self.mom_source is None else self.mom_source.data_ptr()
        if self.turb is None:
            _lib.check(L.b2s_momentum_assemble_d(self._m_mom, bc, pr, Up.data_ptr(), self.gUp.data_ptr(),
                                                 gp.data_ptr(), self.bUp.data_ptr(), F.data_ptr(), Fb.data_ptr(), por,
                                                 msrc, self.val_A.data_ptr(), self.diag.data_ptr(),
                                                 self.inv.data_ptr(), self.dP.data_ptr(), self.bmom.data_ptr(),
                                                 self.brmom.data_ptr(), pt(self.Q_MOM), s), "b2s_momentum_assemble_d")
        else:
            t = self.turb
            self.kernel_launches += t.launch_momentum_terms(Up, self.gUp, old, s)
            self._mark("turbulence_terms")
            _lib.check(L.b2s_momentum_assemble_turb_d(self._m_mom, bc, pr, Up.data_ptr(), self.gUp.data_ptr(),
                                                      gp.data_ptr(), self.bUp.data_ptr(), F.data_ptr(), Fb.data_ptr(),
                                                      por, msrc, t.mu_f.data_ptr(), t.mu_b.data_ptr(),
                                                      t.tsrc.data_ptr(), self.val_A.data_ptr(), self.diag.data_ptr(),
                                                      self.inv.data_ptr(), self.dP.data_ptr(), self.bmom.data_ptr(),
                                                      self.brmom.data_ptr(), pt(self.Q_MOM), s),
                       "b2s_momentum_assemble_turb_d")
        self._mark("momentum_assembly")
        self.Ustar.copy_(Up[1:])
        _lib.check(L.b2s_bicgstab_jacobi_d(nc, dim, fv.rowptr.data_ptr(), fv.col.data_ptr(), self.val_A.data_ptr(),
                                           self.brmom.data_ptr(), self.inv.data_ptr(), self.Ustar.data_ptr(), 0.1, 30,
                                           1, self.work_bicg.data_ptr(), self.work_bicg.numel() * 8, self.info_mom, s),
                   "b2s_bicgstab_jacobi_d")
        self._mark("momentum_solve")
        _lib.check(L.b2s_pressure_assemble_d(m, bc, pr, self.Ustar.data_ptr(), Up.data_ptr(), gp.data_ptr(),
                                             self.dP.data_ptr(), self.Fst.data_ptr(), self.cf.data_ptr(),
                                             self.Fbst.data_ptr(), self.cb.data_ptr(), self.val_P.data_ptr(),
                                             self.rhs_p.data_ptr(), pt(self.Q_CONT), s), "b2s_pressure_assemble_d")
        self.kernel_launches += 3  # momentum assembly, BiCGSTAB, pressure assembly
        self._mark("pressure_assembly")
        if not amg_ready:
            self._ensure_amg(s)
        self._mark("amg_rebuild")
        self._amg.pcg(self.rhs_p, self.pp, self.case.pressure_tol, 200, self.singular_p, self.info_p)
        self.kernel_launches += 1
        self._mark("pressure_solve")
        Upn, Fn, Fbn = self._Up[new], self._F[new], self._Fb[new]
        _lib.check(L.b2s_correct_d(m, bc, pr, self.Fst.data_ptr(), self.cf.data_ptr(), self.Fbst.data_ptr(),
                                   self.cb.data_ptr(), self.pp.data_ptr(), Up.data_ptr(), self.Ustar.data_ptr(),
                                   self.dP.data_ptr(), Fn.data_ptr(), Fbn.data_ptr(), Upn.data_ptr(),
                                   pt(self.Q_SUMP), s), "b2s_correct_d")
        if self.singular_p:
            _lib.check(L.b2s_remove_mean_d(nc, Upn.data_ptr(), part.data_ptr(), self.nblk, self.NQ, self.Q_SUMP, s),
                       "b2s_remove_mean_d")
            self.kernel_launches += 1
        self.kernel_launches += 1
        self._mark("corrections")
        if self.energy and not self.external_energy:
            self._launch_energy(old, new, Fn, Fbn, s)
            self.kernel_launches += 4
            self._mark("energy")
        if self.turb is not None:
            self.kernel_launches += self.turb.launch_transport(old, new, Upn, Fn, Fbn, pt, self.Q_TMAX, self.Q_TRES,
                                                               self.info_turb, s)
            self._mark("turbulence")
        _lib.check(L.b2s_sum_partials_d(part.data_ptr(), self.nblk, self.NQ, self.NQ, self.q_of.data_ptr(),
                                        self.scal.data_ptr(), s), "b2s_sum_partials_d")
        self.kernel_launches += 1
        self._mark("residuals")
        return old, new

    def _launch_energy(self, old, new, Fn, Fbn, s):
        """``flowtrace/unstructured/simple.py:778-813`` (laminar, no radiation)."""
        L, fv, c = _lib.lib(), self.fv, self.case
        m, bc = fv.cmesh_ref, ctypes.byref(self.cbc)
        T, Tn = self._T[old], self._T[new]
        _lib.check(L.b2s_energy_bvals_d(m, bc, T.data_ptr(), self.gT.data_ptr() if self._lagT else None,
                                        Fbn.data_ptr(), self.Tb.data_ptr(), s), "b2s_energy_bvals_d")
        _lib.check(L.b2s_ls_gradient_d(m, 1, T.data_ptr(), self.Tb.data_ptr(), self.gT.data_ptr(), s),
                   "b2s_ls_gradient_d")
        self._lagT = True
        second = (c.scalar_scheme or c.scheme) == "second-order"
        esrc = None if self.energy_source is None else self.energy_source.data_ptr()
        tail = (self.val_T.data_ptr(), self.diagT.data_ptr(), self.invT.data_ptr(), self.bT.data_ptr(),
                self.brT.data_ptr(), self.part.data_ptr() + 8 * self.Q_ENUM * self.nblk, s)
        if self.turb is None:
            _lib.check(L.b2s_energy_assemble_d(m, bc, c.conductivity / c.cp, c.cp, c.relax_T, int(second), T.data_ptr(),
                                               self.gT.data_ptr(), self.Tb.data_ptr(), Fn.data_ptr(), Fbn.data_ptr(),
                                               esrc, *tail), "b2s_energy_assemble_d")
        else:  # k/cp + mu_t/Pr_t per face (simple.py:781-782)
            _lib.check(L.b2s_energy_assemble_turb_d(m, bc, self.turb.kT_f.data_ptr(), self.turb.kT_b.data_ptr(), c.cp,
                                                    c.relax_T, int(second), T.data_ptr(), self.gT.data_ptr(),
                                                    self.Tb.data_ptr(), Fn.data_ptr(), Fbn.data_ptr(), esrc, *tail),
                       "b2s_energy_assemble_turb_d")
        Tn.copy_(T)
        _lib.check(L.b2s_bicgstab_jacobi_d(self.nc, 1, fv.rowptr.data_ptr(), fv.col.data_ptr(), self.val_T.data_ptr(),
                                           self.brT.data_ptr(), self.invT.data_ptr(), Tn.data_ptr(), 1e-3, 60, 1,
                                           self.work_bicg.data_ptr(), self.work_bicg.numel() * 8, self.info_T, s),
                   "b2s_bicgstab_jacobi_d")

    def _queue_report(self) -> int:
        """Enqueue the copy of the report into the next pinned host buffer; returns its slot."""
        slot = self._rep_slot
        self._rep_slot ^= 1
        self.report_host = self.report_hosts[slot]
        self.report_host.copy_(self.report, non_blocking=True)
        self._rep_events[slot].record()
        return slot

    def _read_report(self, slot=None):
        if slot is None:
            slot = self._queue_report()
        self._rep_events[slot].synchronize()
        if self._events:
            self._resolve_stage_events()
        raw = self.report_hosts[slot].numpy()
        scal = raw[: self.NQ * 8].view(np.float64).copy()
        infos = read_info(raw[self.NQ * 8:])
        return scal, infos

    def _graph_key(self):
        return (self._cur, self._lag, self._lagT, self.relax_u, self.relax_p, self.algo,
                None if self.porosity is None else self.porosity.data_ptr(),
                None if self.mom_source is None else self.mom_source.data_ptr(),
                None if self.energy_source is None else self.energy_source.data_ptr(), self.amg_setups)

    def _launch_graph(self):
        """Replay (capturing on first use) the CUDA graph of an outer iteration that needs no
        AMG rebuild: the ~15 launches of the stage sequence become one graph launch."""
        import torch

        key = self._graph_key()
        ent = self._graphs.get(key)
        if ent is None:
            g = torch.cuda.CUDAGraph()
            k0 = self.kernel_launches
            with torch.cuda.graph(g):
                old, new = self._launch(amg_ready=True)
            ent = (g, old, new, self.kernel_launches - k0)
            self.kernel_launches = k0
            self._graphs[key] = ent
        g, old, new, nk = ent
        g.replay()
        self.kernel_launches += nk
        self._amg_age += 1
        return old, new

    def _lagged(self):
        """Buffers an iteration overwrites in place and the next one reads (lagged gradients)."""
        out = [self.gUp]
        if self.case.pressure_gradient == "green-gauss":
            out.append(self.gpf)
        if self.energy and getattr(self, "gT", None) is not None:
            out.append(self.gT)
        if self.turb is not None:
            out.append(self.turb.yplus)
        return out

    def _save_lagged(self):
        if getattr(self, "_lag_bak", None) is None:
            self._lag_bak = [t.clone() for t in self._lagged()]
        else:
            for b, t in zip(self._lag_bak, self._lagged()):
                b.copy_(t)

    def _restore_lagged(self):
        for b, t in zip(self._lag_bak, self._lagged()):
            t.copy_(b)

    def _graph_ready(self) -> bool:
        """The next iteration replays a CUDA graph: no AMG rebuild is due and no host work."""
        rebuild_due = self._amg is None or self._amg_age >= self.amg_rebuild
        return (self.use_graphs and not rebuild_due and self._lag and not self.profile_stages
                and not self._reaggregated)

    def _enqueue_iteration(self):
        """Enqueue one outer iteration and the copy of its report; the state pointer moves to the
        iteration's output. Returns (old, new, report slot)."""
        if self._graph_ready():
            try:
                old, new = self._launch_graph()
            except RuntimeError:
                self.use_graphs = False  # capture unsupported here: enqueue the stages one by one
                self._graphs.clear()
                old, new = self._launch()
        else:
            old, new = self._launch()
        slot = self._queue_report()
        self._cur = new
        return old, new, slot

    def step(self) -> float:
        """One outer iteration (``flowtrace/unstructured/simple.py:500-703``)."""
        if self.finished:
            return 0.0
        self._capture = None
        return self._finish_iteration(self._enqueue_iteration())

    def _finish_iteration(self, ticket) -> float:
        """Read an enqueued iteration's report (waiting for it) and apply the host side of the
        iteration: residuals, the stability guard and the convergence test."""
        old, new, slot = ticket
        c, dim = self.case, self.dim
        scal, infos = self._read_report(slot)
        self._cur = new
        mom_info, p_info = infos[:dim], infos[dim]
        res = {}
        num = [float(scal[self.Q_MOM + k]) for k in range(dim)]
        den = [float(scal[self.Q_MOM + dim + k]) for k in range(dim)]
        floor = 1e-3 * max(max(den), 1e-300)
        for k, name in enumerate(COMPONENTS[:dim]):
            res[name] = num[k] / max(den[k], floor)
        res["continuity"] = float(scal[self.Q_CONT])
        cap = {"old": old, "new": new, "mom_info": mom_info, "alpha_u": self.relax_u, "p_info": p_info}
        if self.energy and not self.external_energy:
            r, s_ = float(scal[self.Q_ENUM]), float(scal[self.Q_EDEN])
            res["energy"] = r / s_ if s_ > 0 else r
            cap["energy"] = {"info": infos[dim + 1], "alpha": c.relax_T}
        if self.turb is not None:  # turbulence.py:297-300
            for q, name in enumerate(("k", "omega")):
                qn = self.Q_TRES[q]
                res[name] = float(scal[qn]) / max(float(scal[qn + 1]), 1e-300)
            cap["turbulence"] = {"k_info": infos[dim + 2], "omega_info": infos[dim + 3]}
        self.iteration += 1
        self.step_count = self.iteration
        self.last_linear = {"momentum_iters": [i.iterations for i in mom_info], "pressure_iters": p_info.iterations,
                            "pressure_residual": p_info.residual}
        prev = getattr(self, "_last_res", {}), getattr(self, "_last_raw", {})
        self._last_raw = dict(res)
        if self.iteration <= 5:
            self._res_max5["continuity"] = max(self._res_max5.get("continuity", 0.0), res["continuity"], 1e-300)
        flux_scale = float(scal[self.Q_SUMF]) + float(scal[self.Q_SUMFB])
        res["continuity"] /= max(self._res_max5["continuity"], 1e-3 * flux_scale)
        self._last_res = res
        cap["iteration"] = self.iteration
        self._capture = cap
        rolled_back = self._stability_guard(self._last_raw["continuity"], flux_scale)
        cap["rolled_back"] = rolled_back
        if rolled_back:
            self._last_res, self._last_raw = prev
            return 1.0
        if self.iteration > 5 and max(res.values()) < c.tol:
            self.converged = True
        return 1.0

    def run(self, max_steps=None, hooks=None) -> int:
        """Step until finished (or ``max_steps``); returns the number of steps taken.

        The same iterates as calling ``step()`` that many times, pipelined: while the host reads
        iteration k's report (residuals, guard, convergence), iteration k+1 is already enqueued
        when it is a graph replay (no AMG rebuild or other host work due). If iteration k ends
        the run (converged, or a guard roll-back) the enqueued k+1 is discarded: its output went
        to a state buffer that is not the current one, and the lagged gradients it overwrote in
        place are put back from a device copy taken before it was enqueued (a guard roll-back
        drops the lagged terms anyway). No iteration past ``max_steps`` or the case's
        ``max_iter`` is enqueued. ``hooks`` = (before, after[, done]): callables run around the
        enqueueing of each iteration (e.g. to record CUDA events) and after the host side of
        each kept iteration."""
        before, after, done = (tuple(hooks) + (None,) * 3)[:3] if hooks is not None else (None, None, None)

        def enqueue():
            if before:
                before()
            self._capture = None
            t = self._enqueue_iteration()
            if after:
                after()
            return t

        n = 0
        ticket = None
        while not self.finished and (max_steps is None or n < max_steps):
            if ticket is None:
                ticket = enqueue()
            nxt = None
            more = (max_steps is None or n + 1 < max_steps) and self.iteration + 1 < self.case.max_iter
            if more and self._graph_ready():
                age = self._amg_age
                self._save_lagged()
                nxt = enqueue()
            guard_before = len(getattr(self, "guard_events", []))
            self._finish_iteration(ticket)
            n += 1
            if done:
                done()
            stop = self.finished or (max_steps is not None and n >= max_steps)
            rolled = len(getattr(self, "guard_events", [])) != guard_before
            if nxt is not None and (stop or rolled):
                # discard the speculative iteration: the state stays where iteration k (or the
                # guard's restore, which drops the lagged terms) left it
                if not rolled:
                    self._amg_age = age
                    self._restore_lagged()
                nxt = None
            elif nxt is not None:
                self._cur = nxt[1]
            ticket = nxt
        return n

    # ------------------------------------------------------------------ guard and state
    def _reset_guard(self):
        """``flowtrace/unstructured/simple.py:714-720``."""
        self.guard_events = []
        self.algo = self.case.algorithm
        self.relax_u = self.case.relax_u
        self.guard_exhausted_at = None
        self._guard_min = float("inf")
        self._guard_snap = (self._snapshot(), float("inf")) if self.guard_enabled else None

    def _snapshot(self):
        """Device copy of the state (what ``state_dict`` holds, without leaving the device)."""
        c = self._cur
        snap = {"Up": self._Up[c].clone(), "F": self._F[c].clone(), "Fb": self._Fb[c].clone(),
                "iteration": self.iteration, "res_continuity_norm": self._res_max5.get("continuity", 0.0)}
        if self.energy:
            snap["T"] = self._T[c].clone()
        if self.turb is not None:
            snap["turb"] = self.turb.snapshot(c)
        return snap

    def _restore(self, snap):
        cap = self._capture
        busy = {self._cur} | ({cap["old"]} if cap else set())
        tgt = next(i for i in range(3) if i not in busy)
        self._Up[tgt].copy_(snap["Up"])
        self._F[tgt].copy_(snap["F"])
        self._Fb[tgt].copy_(snap["Fb"])
        if self.energy and "T" in snap:
            self._T[tgt].copy_(snap["T"])
        if self.turb is not None and "turb" in snap:
            self.turb.restore(snap["turb"], tgt)
        self._cur = tgt
        self.iteration = int(snap.get("iteration", 0))
        self._lag = self._lagT = False
        if float(snap.get("res_continuity_norm", 0.0)) > 0:
            self._res_max5["continuity"] = float(snap["res_continuity_norm"])

    def _stability_guard(self, r: float, flux_scale: float) -> bool:
        """Roll back and lower the relaxation on divergence (``simple.py:722-776``)."""
        if not self.guard_enabled or self.external_energy:
            return False
        ref = max(self._guard_min, self.GUARD_ROUNDOFF * flux_scale)
        bad = not math.isfinite(r) or (self.iteration > 10 and r > self.GUARD_GROWTH * ref)
        if bad and self._guard_snap is not None and self.relax_p * self.GUARD_FACTOR >= self.GUARD_MIN_RELAX:
            snap, snap_r = self._guard_snap
            at = self.iteration
            self._restore(snap)
            self.iteration = self.step_count = at
            self.relax_p *= self.GUARD_FACTOR
            self._amg_age = 10 ** 9
            self._guard_min = snap_r
            self.guard_events.append({"detected_at": at, "restored_to": int(snap["iteration"]),
                                      "relax_p": round(self.relax_p, 4), "continuity": r})
            return True
        stage2 = self.GUARD_FALLBACK and (self.algo == "SIMPLEC" or self.relax_u * 0.7 >= self.GUARD_MIN_RELAX_U - 1e-12)
        if bad and self._guard_snap is not None and stage2:
            snap, snap_r = self._guard_snap
            at = self.iteration
            self._restore(snap)
            self.iteration = self.step_count = at
            if self.algo == "SIMPLEC":
                self.algo, self.relax_u, self.relax_p = "SIMPLE", min(self.relax_u, 0.3), 0.3
            else:
                self.relax_u *= 0.7
            self._amg_age = 10 ** 9
            self._guard_min = snap_r
            self.guard_events.append({"detected_at": at, "restored_to": int(snap["iteration"]), "algorithm": self.algo,
                                      "relax_p": round(self.relax_p, 4), "relax_u": round(self.relax_u, 4),
                                      "continuity": r})
            return True
        if bad and self.guard_exhausted_at is None:
            self.guard_exhausted_at = self.iteration
        if math.isfinite(r) and self.iteration > 5:
            self._guard_min = min(self._guard_min, r)
            if self.iteration % self.GUARD_EVERY == 0 and r <= 2.0 * self._guard_min:
                self._guard_snap = (self._snapshot(), r)
        return False

    def state_dict(self) -> dict:
        """Host copies in the reference's numbering (``simple.py:1033-1046``)."""
        st = {"U": self.U, "p": self.p, "F": self.F, "Fb": self.Fb, "iteration": self.iteration}
        if self.energy:
            st["T"] = self.T
        if self.turb is not None:
            st.update(self.turb.state(self._cur))
        st["time"], st["time_step"] = 0.0, 0
        st["res_continuity_norm"] = self._res_max5.get("continuity", 0.0)
        return st

    def load_state(self, st: dict) -> None:
        """``simple.py:1048-1072``."""
        import torch

        fv, h = self.fv, self.fv.host
        Up = torch.cat([fv.cells_to_device(np.asarray(st["p"], dtype=np.float64))[None],
                        fv.cells_to_device(np.asarray(st["U"], dtype=np.float64).reshape(self.nc, self.dim))])
        snap = {"Up": Up, "F": self._F[self._cur].clone(), "Fb": self._Fb[self._cur].clone(),
                "iteration": int(st.get("iteration", 0)), "res_continuity_norm": st.get("res_continuity_norm", 0.0)}
        if h.n_if:
            snap["F"][: h.n_if] = fv.faces_to_device(st["F"])
        if h.n_bf:
            snap["Fb"][: h.n_bf] = fv.bfaces_to_device(st["Fb"])
        if self.energy and "T" in st:
            snap["T"] = fv.cells_to_device(np.asarray(st["T"], dtype=np.float64))
        if self.turb is not None:
            snap["turb"] = self.turb.snapshot(self._cur)
        self._capture = None
        self._restore(snap)
        if self.turb is not None:
            self.turb.load(st, self._cur)

    # ------------------------------------------------------------------ reports
    def residuals(self) -> dict:
        """``simple.py:822-833``."""
        r = dict(getattr(self, "_last_res", {}))
        raw = dict(getattr(self, "_last_raw", r))
        return {"raw": raw, "scaled": r, "normalized": r}

    def diagnostics(self) -> dict:
        from .diagnostics import evaluate

        return evaluate(self)

    def describe(self) -> dict:
        """``simple.py:845-860``."""
        return {
            "solver": f"pressure-based {self.algo}", "turbulence": self.case.turbulence, "backend": self.be.name,
            "device": self.be.device, "precision": str(self.dtype), "cells": self.nc, "faces": self.mesh.n_faces,
            "dim": self.dim, "convection": self.case.scheme, "relax_p": self.relax_p,
            "stability_rollbacks": list(self.guard_events), "stability_guard_exhausted_at": self.guard_exhausted_at,
            "pressure_solver": "AMG-PCG (B200 SA-AMG, " + (f"{self._amg.n_levels} levels)" if self._amg else "not built)"),
            "max_non_orthogonality_deg": round(self.fv.non_orthogonality_deg, 2),
            "setup_seconds": round(self.setup_seconds, 3),
        }

    def fields(self, names=None) -> Dict[str, np.ndarray]:
        """``simple.py:862-880``."""
        U = self.U
        out = {"x-velocity": U[:, 0], "y-velocity": U[:, 1]}
        if self.dim == 3:
            out["z-velocity"] = U[:, 2]
        out["velocity-magnitude"] = np.linalg.norm(U, axis=1)
        out["pressure"] = self.p
        if self.energy:
            out["temperature"] = self.T
        if self.turb is not None:
            out.update(self.turb.fields(self._cur))
        if names:
            out = {k: v for k, v in out.items() if k in names}
        return out

    def cell_centres(self) -> np.ndarray:
        return self.fv.geometry.cell_centre

    def mass_balance(self) -> dict:
        """``simple.py:885-893``."""
        Fb = self.Fb
        out = {}
        for z in self.mesh.boundary_zones():
            m = self.fv.bzone == z.id
            if m.any():
                out[z.name] = float(Fb[m].sum())
        return out

    def _pressure_bvals_host(self):
        h = self.fv.host
        p = self.p
        pP = p[h.Pb]
        if self._lag:
            gsrc = self.gpf if self.case.pressure_gradient == "green-gauss" else self.gUp[0]
            gp = self.fv.cells_to_host(gsrc)
            pP = pP + np.sum(gp[h.Pb] * h.db, axis=1)
        return self.m_pres_h * self._pb_fixed_h + (1.0 - self.m_pres_h) * pP

    def _wall_viscosity_host(self) -> np.ndarray:
        """Boundary-face viscosity of the momentum equations, reference numbering: mu, or with the
        SST model mu + mu_t and on walls the wall-function value (``simple.py:900-904``)."""
        if self.turb is not None:
            return self.turb.wall_viscosity(self._Up[self._cur], self.gUp, self._cur)
        return np.full(self.fv.host.n_bf, float(self.case.viscosity))

    def _wall_shear_host(self):
        """Wall shear stress vector per boundary face, mu_w (u_P - u_w)_t / y_b, and (u_P - u_w)_t."""
        h = self.fv.host
        rel = self.U[h.Pb] - self._ub_fixed_h
        rel_t = rel - np.sum(rel * h.nb, axis=1)[:, None] * h.nb
        return self._wall_viscosity_host()[:, None] * rel_t / h.yb[:, None], rel_t

    def wall_report(self) -> dict:
        """Per wall zone: area, pressure/viscous/total force, Cd and Cl (``case.ref_velocity``,
        ``case.ref_area``), area-weighted and maximum y+, mean skin friction and, with energy, the
        conducted heat flow (``simple.py:906-950``; no radiation on this path)."""
        h, c = self.fv.host, self.case
        rho, mu = c.density, c.viscosity
        tau_vec, _ = self._wall_shear_host()
        tau = np.sqrt(np.sum(tau_vec * tau_vec, axis=1))
        yplus = h.yb * np.sqrt(tau / rho) * rho / mu
        forces = self.wall_forces()
        qconv = None
        if self.energy:
            TP = self.T[h.Pb]
            Tw = np.where(self.tkind_h == T_FIXED, self._tval_h, TP)
            qconv = (c.conductivity * h.alpha_b * (Tw - TP) * (self.tkind_h == T_FIXED)
                     + np.where(self.tkind_h == T_FLUX, self._tval_h * h.Sb_mag, 0.0))
        qdyn = 0.5 * rho * c.ref_velocity ** 2
        out = {}
        for z in self.mesh.boundary_zones():
            if z.name not in forces:
                continue
            m = h.bzone == z.id
            A = h.Sb_mag[m]
            f = forces[z.name]
            Ft = np.asarray(f["total"])
            rep = {"area": float(A.sum()), "force_pressure": f["pressure"], "force_viscous": f["viscous"],
                   "force_total": f["total"], "cd": float(Ft[0] / (qdyn * c.ref_area)),
                   "cl": float(Ft[1] / (qdyn * c.ref_area)),
                   "yplus_avg": float((yplus[m] * A).sum() / A.sum()), "yplus_max": float(yplus[m].max()),
                   "cf_avg": float((tau[m] * A).sum() / A.sum() / qdyn)}
            if qconv is not None:
                rep["heat_flow_conv"] = float(qconv[m].sum())
            out[z.name] = rep
        return out

    def wall_profile(self, zone: str) -> dict:
        """Face-wise x, y, Cf, Cp and y+ on one wall zone, sorted by x (``simple.py:952-968``)."""
        h, c = self.fv.host, self.case
        m = h.bzone == self.mesh.zone_by_name(zone).id
        rho, mu = c.density, c.viscosity
        _, rel_t = self._wall_shear_host()
        tau = self._wall_viscosity_host() * np.sqrt(np.sum(rel_t * rel_t, axis=1)) / h.yb
        qdyn = 0.5 * rho * c.ref_velocity ** 2
        xfb = h.xfb[m]
        order = np.argsort(xfb[:, 0])
        return {"x": xfb[order, 0], "y": xfb[order, 1], "cf": tau[m][order] / qdyn,
                "cp": self._pressure_bvals_host()[m][order] / qdyn,
                "yplus": (h.yb * np.sqrt(tau / rho) * rho / mu)[m][order]}

    def wall_forces(self) -> dict:
        """Pressure and viscous force on every wall zone (``simple.py:970-1001``)."""
        h = self.fv.host
        pb = self._pressure_bvals_host()
        mu_b = self._wall_viscosity_host()
        du = self.U[h.Pb] - self._ub_fixed_h
        du_t = du - np.einsum("fd,fd->f", du, h.nb)[:, None] * h.nb
        f_p = pb[:, None] * h.Sb
        f_v = (mu_b * h.alpha_b)[:, None] * du_t
        out = {}
        for z in self.mesh.boundary_zones():
            m = (h.bzone == z.id) & (self.bkind_h == WALL)
            if not m.any():
                continue
            fp, fvis = f_p[m].sum(axis=0), f_v[m].sum(axis=0)
            out[z.name] = {"pressure": fp.tolist(), "viscous": fvis.tolist(), "total": (fp + fvis).tolist()}
        return out

    def heat_flow(self) -> dict:
        """Heat flow into the domain per boundary zone (``simple.py:1003-1031``)."""
        if not self.energy:
            return {}
        c, h = self.case, self.fv.host
        T = self.T
        TP = T[h.Pb]
        tk, tv, kind = self.tkind_h, self._tval_h, self.bkind_h
        Fb = self.Fb
        Tb = np.where(tk == T_FIXED, tv, TP)
        Tb = np.where((kind == OUTLET) & (Fb < 0), tv, Tb)
        cond = c.conductivity * h.alpha_b * (Tb - TP) * (tk == T_FIXED)
        cond = cond + np.where(tk == T_FLUX, tv * h.Sb_mag, 0.0)
        q = cond - c.cp * Fb * Tb
        return {z.name: float(q[h.bzone == z.id].sum()) for z in self.mesh.boundary_zones()}

    # ------------------------------------------------------------------ captured systems
    def captured_systems(self) -> dict:
        """The latest iteration's systems in the reference's form and numbering (host NumPy /
        SciPy), with the keys of the reference's ``_capture`` (``simple.py:649-651``)."""
        cap = self._capture
        if cap is None:
            return None
        fv, dim = self.fv, self.dim
        old, new = cap["old"], cap["new"]
        Ar = fv.matrix_to_host(self.val_A)
        A = Ar.copy()
        A.setdiag(fv.cells_to_host(self.diag))
        b = fv.cells_to_host(self.bmom)
        br = fv.cells_to_host(self.brmom)
        out = {"U_old": fv.cells_to_host(self._Up[old][1:]), "p_old": fv.cells_to_host(self._Up[old][0]), "A": A,
               "b": [b[:, k] for k in range(dim)], "Ar": Ar, "br": [br[:, k] for k in range(dim)],
               "U_star": fv.cells_to_host(self.Ustar), "mom_info": cap["mom_info"], "alpha_u": cap["alpha_u"],
               "Fst": fv.faces_to_host(self.Fst[: fv.n_if]), "Fbst": fv.bfaces_to_host(self.Fbst[: fv.n_bf]),
               "mass": -fv.cells_to_host(self.rhs_p), "Ap": fv.matrix_to_host(self.val_P),
               "pp": fv.cells_to_host(self.pp), "p_info": cap["p_info"], "F": fv.faces_to_host(self._F[new][: fv.n_if]),
               "Fb": fv.bfaces_to_host(self._Fb[new][: fv.n_bf]), "U_new": fv.cells_to_host(self._Up[new][1:]),
               "p_new": fv.cells_to_host(self._Up[new][0]), "iteration": cap["iteration"],
               "rolled_back": cap.get("rolled_back", False), "dP": fv.cells_to_host(self.dP)}
        if "energy" in cap:
            AT = fv.matrix_to_host(self.val_T)
            ATu = AT.copy()
            ATu.setdiag(fv.cells_to_host(self.diagT))
            out["energy"] = {"A": ATu, "b": fv.cells_to_host(self.bT), "T_old": fv.cells_to_host(self._T[old]),
                             "Ar": AT, "br": fv.cells_to_host(self.brT), "T_new": fv.cells_to_host(self._T[new]),
                             "alpha": cap["energy"]["alpha"], "info": cap["energy"]["info"]}
        return out
