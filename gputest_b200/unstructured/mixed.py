"""Mixed-precision SIMPLEC on the device: ``MixedSimpleSolver``.

The same outer iteration as ``SimpleSolver`` (``flowtrace/unstructured/simple.py:500-703``) with
the linear algebra moved to float where the fixed point does not depend on it:

* the momentum and energy systems are assembled with their matrices (and Jacobi inverses) in
  float, and with the residual r = b - A phi of the unrelaxed system evaluated in double from
  the coefficients in registers; the relaxed system is solved in correction form
  A_r dphi = r from dphi = 0 by a float Jacobi-BiCGSTAB (double reductions) and phi + dphi is
  formed in double. From x0 = phi the reference's solve A_r x = b_r has the same iterates, and
  a converged outer iteration satisfies the double residual equations;
* the pressure-correction matrix is stored in float and solved by float AMG-PCG passes inside a
  double iterative refinement: the true residual is recomputed in double from the double face
  coefficients after every pass and the reference's stopping test (|r| / |b| < pressure_tol)
  is applied to it; the AMG hierarchy is rebuilt in double and copied to float, its coarsest
  level is solved with the double inverse;
* gradients, fluxes, boundary values, the corrections, the continuity imbalance and every norm
  stay double, and so do the fields;
* with the k-omega SST model, the float momentum and energy rows take the model's per-face
  viscosities and transpose-stress source, and the model's own stages (k, omega, mu_t) run in
  double as in ``SimpleSolver``.

The converged fields therefore agree with the double path's to the tolerance of the outer
convergence test, not to the float rounding of the systems. ``diagnostics()`` and
``captured_systems()`` (which re-evaluate the double systems) are not provided here.
"""

from __future__ import annotations

import ctypes

from .. import _lib
from .simple import SimpleSolver


class MixedSimpleSolver(SimpleSolver):
    """Drop-in ``SimpleSolver`` whose linear systems are stored and solved in float."""

    PRECISIONS = ("mixed", "fp32", "fp64")
    TURBULENCE = ("laminar", "k-omega-sst")  # the SST stages themselves stay in double
    REFINE_PASSES = 8       # double refinement passes of the pressure-correction solve at most
    INNER_TOL_FLOOR = 1e-5  # smallest relative reduction asked of one float pass
    # (relative tolerance, iteration cap) of the float energy solve. The double path keeps the
    # reference's (1e-3, 60). Measured on the 524,288-cell heated duct to the 1e-6 residual, caps
    # of 60, 30, 15 and 8 all take the same 283 outer iterations to states within 3e-7 of each
    # other (the flow is what sets the outer count); 8 is the cheapest
    ENERGY_SOLVE = (1e-3, 8)

    def _allocate(self):
        import torch

        super()._allocate()
        dev, fv = self.torch_device, self.fv
        nc, nnz, dim = fv.nc, fv.nnz, fv.dim
        f32 = lambda *s: torch.zeros(*s, dtype=torch.float32, device=dev)  # noqa: E731
        self.val_A32, self.inv32, self.r32, self.dU32 = f32(nnz), f32(nc), f32(dim, nc), f32(dim, nc)
        self.val_P32 = f32(nnz)
        if self.energy:
            self.val_T32, self.invT32, self.rT32, self.dT32 = f32(nnz), f32(nc), f32(nc), f32(nc)
        L = _lib.lib()
        wb = max(L.b2s_bicgstab_f32_workspace_bytes(nc, dim), L.b2s_bicgstab_f32_workspace_bytes(nc, 1))
        self.work_bicg32 = torch.empty(wb // 8 + 1, dtype=torch.float64, device=dev)

    def _setup_amg(self, start=0):
        """Set-up from the widened float pressure matrix; the V-cycle then reads float copies."""
        self.val_P.copy_(self.val_P32)
        super()._setup_amg(start)
        self._amg.enable_mixed(self.val_P32)
        if self._amg_fresh:
            self._amg.to_f32()

    def _launch(self, amg_ready=False):
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
        por = None if self.porosity is None else self.porosity.data_ptr()
        msrc = None if self.mom_source is None else self.mom_source.data_ptr()
        tail = (self.val_A32.data_ptr(), self.inv32.data_ptr(), self.dP.data_ptr(), self.r32.data_ptr(),
                pt(self.Q_MOM), s)
        if self.turb is None:
            _lib.check(L.b2s_momentum_assemble_mixed_d(self._m_mom, bc, pr, Up.data_ptr(), self.gUp.data_ptr(),
                                                       gp.data_ptr(), self.bUp.data_ptr(), F.data_ptr(), Fb.data_ptr(),
                                                       por, msrc, *tail), "b2s_momentum_assemble_mixed_d")
        else:
            t = self.turb
            self.kernel_launches += t.launch_momentum_terms(Up, self.gUp, old, s)
            self._mark("turbulence_terms")
            _lib.check(L.b2s_momentum_assemble_mixed_turb_d(self._m_mom, bc, pr, Up.data_ptr(), self.gUp.data_ptr(),
                                                            gp.data_ptr(), self.bUp.data_ptr(), F.data_ptr(),
                                                            Fb.data_ptr(), por, msrc, t.mu_f.data_ptr(),
                                                            t.mu_b.data_ptr(), t.tsrc.data_ptr(), *tail),
                       "b2s_momentum_assemble_mixed_turb_d")
        self._mark("momentum_assembly")
        # U* = U + dU, dU from A_r dU = b - A U (float, from zero)
        _lib.check(L.b2s_bicgstab_jacobi_f32_d(nc, dim, fv.rowptr.data_ptr(), fv.col.data_ptr(),
                                               self.val_A32.data_ptr(), self.r32.data_ptr(), self.inv32.data_ptr(),
                                               self.dU32.data_ptr(), 0.1, 30, 1, 1, self.Ustar.data_ptr(),
                                               Up[1:].data_ptr(), self.work_bicg32.data_ptr(),
                                               self.work_bicg32.numel() * 8, self.info_mom, s),
                   "b2s_bicgstab_jacobi_f32_d")
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
        self._amg.pcg_mixed(m, self.cf, self.cb, self.rhs_p, self.pp, self.case.pressure_tol, 200, self.singular_p,
                            self.info_p, maxpass=self.REFINE_PASSES, min_inner_tol=self.INNER_TOL_FLOOR)
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
        tail = (self.val_T32.data_ptr(), self.invT32.data_ptr(), self.rT32.data_ptr(),
                self.part.data_ptr() + 8 * self.Q_ENUM * self.nblk, s)
        if self.turb is None:
            _lib.check(L.b2s_energy_assemble_mixed_d(m, bc, c.conductivity / c.cp, c.cp, c.relax_T, int(second),
                                                     T.data_ptr(), self.gT.data_ptr(), self.Tb.data_ptr(),
                                                     Fn.data_ptr(), Fbn.data_ptr(), esrc, *tail),
                       "b2s_energy_assemble_mixed_d")
        else:  # k/cp + mu_t/Pr_t per face (simple.py:781-782)
            _lib.check(L.b2s_energy_assemble_mixed_turb_d(m, bc, self.turb.kT_f.data_ptr(), self.turb.kT_b.data_ptr(),
                                                          c.cp, c.relax_T, int(second), T.data_ptr(),
                                                          self.gT.data_ptr(), self.Tb.data_ptr(), Fn.data_ptr(),
                                                          Fbn.data_ptr(), esrc, *tail),
                       "b2s_energy_assemble_mixed_turb_d")
        _lib.check(L.b2s_bicgstab_jacobi_f32_d(self.nc, 1, fv.rowptr.data_ptr(), fv.col.data_ptr(),
                                               self.val_T32.data_ptr(), self.rT32.data_ptr(), self.invT32.data_ptr(),
                                               self.dT32.data_ptr(), float(self.ENERGY_SOLVE[0]),
                                               int(self.ENERGY_SOLVE[1]), 1, 1, Tn.data_ptr(), T.data_ptr(),
                                               self.work_bicg32.data_ptr(), self.work_bicg32.numel() * 8, self.info_T,
                                               s), "b2s_bicgstab_jacobi_f32_d")

    def diagnostics(self) -> dict:
        raise NotImplementedError("diagnostics() re-evaluates the double systems; use SimpleSolver for it")

    def captured_systems(self) -> dict:
        raise NotImplementedError("captured_systems() is provided by the double-precision SimpleSolver")
