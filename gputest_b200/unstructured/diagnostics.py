r"""Algebraic, conservation and health diagnostics of one SIMPLE/SIMPLEC outer iteration.

The report of ``flowtrace/unstructured/diagnostics.py`` (``evaluate`` :214-359, ``summary``
:362-381, ``pressure_matrix_properties`` :384-412), with the same keys, definitions and
conventions (Oettli-Prager componentwise backward errors with Higham's gamma_K row exclusion,
true linear reductions, local and global continuity, field change, non-finite counts). The
row residuals and cell flux balances are computed on the device by ``b2s_row_residuals_d`` and
``b2s_flux_balance_d`` from the systems the iteration left on the device, and the pressure
matrix's CG conditions by ``b2s_matrix_properties_d``; all scalars are reduced on the device
and reach the host in one transfer. Cell indices in the report (worst
cells) are in the reference's numbering.
"""

from __future__ import annotations

import math
from typing import Dict, List, Optional

import numpy as np

from .. import _lib

DIAGNOSTICS_VERSION = 1
COMPONENTS = ("x-velocity", "y-velocity", "z-velocity")


def unit_roundoff(dtype) -> float:
    """u = eps/2 of the working precision (``diagnostics.py:107-109``)."""
    return float(np.finfo(np.dtype(dtype)).eps) / 2.0


def gamma(k: int, u: float) -> float:
    """Higham's gamma_k = k u / (1 - k u) (``diagnostics.py:112-115``)."""
    ku = k * u
    return ku / (1.0 - ku) if ku < 1.0 else math.inf


def ratio(num: float, den: float) -> float:
    """num/den with 0/0 = 0 and x/0 = inf (``diagnostics.py:118-124``)."""
    if not (math.isfinite(num) and math.isfinite(den)):
        return math.inf
    if den > 0.0:
        return num / den
    return 0.0 if num == 0.0 else math.inf


class _Scalars:
    """Device scalars collected under names and moved to the host in one transfer."""

    def __init__(self):
        self.names: List[str] = []
        self.vals: list = []

    def add(self, name, v):
        import torch

        self.names.append(name)
        self.vals.append(torch.as_tensor(v, dtype=torch.float64).reshape(()))

    def fetch(self) -> Dict[str, float]:
        import torch

        if not self.vals:
            return {}
        dev = next((v.device for v in self.vals if v.is_cuda), "cpu")
        host = torch.stack([v.to(dev) for v in self.vals]).cpu().numpy()
        return {n: float(v) for n, v in zip(self.names, host)}


def _rows(fv, val, b, x, dval=None):
    """(r, s) per row of a device system; dval replaces the stored diagonal (unrelaxed a_P)."""
    import torch

    r = torch.empty(fv.nc, dtype=torch.float64, device=b.device)
    s = torch.empty_like(r)
    _lib.check(_lib.lib().b2s_row_residuals_d(fv.nc, fv.rowptr.data_ptr(), fv.col.data_ptr(), val.data_ptr(),
                                              fv.t["slot_diag"].data_ptr(), None if dval is None else dval.data_ptr(),
                                              b.contiguous().data_ptr(), x.contiguous().data_ptr(), r.data_ptr(),
                                              s.data_ptr(), _lib.stream_ptr()), "b2s_row_residuals_d")
    return r, s


def _row_set(sc: _Scalars, prefix: str, pairs, K: int, u: float) -> None:
    """Componentwise metrics of several (r, s) row sets sharing one reference scale
    (``diagnostics.py:154-178``)."""
    import torch

    finite_s = [torch.where(torch.isfinite(s), s, torch.zeros_like(s)) for _, _, s in pairs]
    s_ref = finite_s[0].max()
    for fs in finite_s[1:]:
        s_ref = torch.maximum(s_ref, fs.max())
    thr = gamma(K, u) * s_ref
    sc.add(f"{prefix}|s_ref", s_ref)
    for name, r, s in pairs:
        ar = r.abs()
        finite = torch.isfinite(r) & torch.isfinite(s)
        active = finite & (s > thr)
        excluded = finite & ~active
        q = torch.where(active, ar / torch.where(active, s, torch.ones_like(s)), torch.zeros_like(s))
        key = f"{prefix}|{name}"
        sc.add(key + "|row_scaled", q.max())
        sc.add(key + "|worst_row", torch.argmax(q).double())
        sc.add(key + "|active_rows", active.sum().double())
        sc.add(key + "|excluded_rows", excluded.sum().double())
        sc.add(key + "|excluded_abs_max", torch.where(excluded, ar, torch.zeros_like(ar)).max())
        sc.add(key + "|nonfinite_rows", (~finite).sum().double())
        fin_r = torch.where(finite, ar, torch.zeros_like(ar))
        sc.add(key + "|abs_l1", fin_r.sum())
        sc.add(key + "|abs_max", fin_r.max())
        sc.add(key + "|l2", torch.sqrt((fin_r * fin_r).sum()))


def _row_report(vals, prefix, name, centres, perm) -> dict:
    key = f"{prefix}|{name}"
    nonfinite = int(vals[key + "|nonfinite_rows"])
    worst = int(perm[int(vals[key + "|worst_row"])])
    out = {"row_scaled": math.inf if nonfinite else vals[key + "|row_scaled"], "abs_l1": vals[key + "|abs_l1"],
           "abs_max": vals[key + "|abs_max"], "abs_l2": vals[key + "|l2"],
           "active_rows": int(vals[key + "|active_rows"]), "excluded_rows": int(vals[key + "|excluded_rows"]),
           "excluded_abs_max": vals[key + "|excluded_abs_max"], "nonfinite_rows": nonfinite}
    if out["active_rows"] and not nonfinite:
        out["worst_cell"] = worst
        out["worst_cell_centre"] = [float(v) for v in centres[worst]]
    return out


def _linear_info(info) -> Optional[dict]:
    if info is None:
        return None
    res = float(info.residual)
    return {"iterations": int(info.iterations), "reported_residual": res if math.isfinite(res) else None,
            "converged": bool(info.converged)}


def evaluate(solver) -> dict:
    """Diagnostics of the solver's most recent outer iteration (``diagnostics.py:214-359``)."""
    import torch

    cap = getattr(solver, "_capture", None)
    if cap is None:
        return {"available": False, "version": DIAGNOSTICS_VERSION,
                "reason": "no outer iteration has been completed since the solver was created or restored"}
    fv, dim = solver.fv, solver.dim
    u = unit_roundoff(solver.dtype)
    K_rows, K_cont = fv.row_terms_max, fv.cell_faces_max
    sc = _Scalars()
    names = COMPONENTS[:dim]
    old, new = cap["old"], cap["new"]
    U_old, U_new = solver._Up[old][1:], solver._Up[new][1:]
    p_old, p_new = solver._Up[old][0], solver._Up[new][0]
    pre = [(names[k],) + _rows(fv, solver.val_A, solver.bmom[k], U_old[k], dval=solver.diag) for k in range(dim)]
    sol = [(names[k],) + _rows(fv, solver.val_A, solver.brmom[k], solver.Ustar[k]) for k in range(dim)]
    _row_set(sc, "mom_pre", pre, K_rows, u)
    _row_set(sc, "mom_sol", sol, K_rows, u)
    for k in range(dim):
        r0, _ = _rows(fv, solver.val_A, solver.brmom[k], U_old[k])
        sc.add(f"mom_true_r0|{names[k]}", torch.sqrt((r0 * r0).sum()))
    ecap = cap.get("energy")
    if ecap is not None:
        T_old, T_new = solver._T[old], solver._T[new]
        _row_set(sc, "T_pre", [("energy",) + _rows(fv, solver.val_T, solver.bT, T_old, dval=solver.diagT)], K_rows, u)
        _row_set(sc, "T_sol", [("energy",) + _rows(fv, solver.val_T, solver.brT, T_new)], K_rows, u)
        r0, _ = _rows(fv, solver.val_T, solver.brT, T_old)
        sc.add("T_true_r0", torch.sqrt((r0 * r0).sum()))
    _row_set(sc, "pcorr", [("p-correction",) + _rows(fv, solver.val_P, solver.rhs_p, solver.pp)], K_rows, u)
    nf, nb = fv.n_if, fv.n_bf
    for tag, F, Fb in (("pred", solver.Fst, solver.Fbst), ("corr", solver._F[new], solver._Fb[new])):
        m = torch.empty(fv.nc, dtype=torch.float64, device=F.device)
        t = torch.empty_like(m)
        _lib.check(_lib.lib().b2s_flux_balance_d(fv.cmesh_ref, F.data_ptr(), Fb.data_ptr(), m.data_ptr(), t.data_ptr(),
                                                 _lib.stream_ptr()), "b2s_flux_balance_d")
        _row_set(sc, "cont_" + tag, [("cells", m, t)], K_cont, u)
        sc.add(f"cont_{tag}|face_flux_l1", F[:nf].abs().sum() + Fb[:nb].abs().sum())
        sc.add(f"cont_{tag}|signed_sum", m.sum())
    Fb = solver._Fb[new][:nb]
    sc.add("global|signed", Fb.sum())
    sc.add("global|throughflow", Fb.abs().sum())
    sc.add("dU|num", torch.sqrt(((U_new - U_old) ** 2).sum(0)).max())
    vmag = torch.maximum(torch.sqrt((U_new * U_new).sum(0)).max(), torch.sqrt((U_old * U_old).sum(0)).max())
    if nb:
        ub = solver._bc_t["ub_fixed"]
        vmag = torch.maximum(vmag, torch.sqrt((ub * ub).sum(0)).max())
    sc.add("dU|ref", vmag)
    sc.add("dp|num", (p_new - p_old).abs().max())
    sc.add("dp|range", p_new.max() - p_new.min())
    health = {"velocity": U_new, "pressure": p_new, "face_mass_flux": solver._F[new][:nf], "boundary_mass_flux": Fb}
    if ecap is not None:
        sc.add("dT|num", (T_new - T_old).abs().max())
        hi, lo = T_new.max(), T_new.min()
        if nb:
            fixed = solver._bc_t["m_tfix"] > 0
            tval = solver._bc_t["tval"]
            inf = torch.full_like(tval, math.inf)
            hi = torch.maximum(hi, torch.where(fixed, tval, -inf).max())
            lo = torch.minimum(lo, torch.where(fixed, tval, inf).min())
        sc.add("dT|ref", hi - lo)
        health["temperature"] = T_new
    turb = getattr(solver, "turb", None)
    tnames = ("k", "omega") if turb is not None and "turbulence" in cap else ()
    for q, tname in enumerate(tnames):  # diagnostics.py:287-290
        t_old, t_new = turb._KW[old][q], turb._KW[new][q]
        sc.add(f"d{tname}|num", (t_new - t_old).abs().max())
        sc.add(f"d{tname}|ref", t_new.abs().max())
        health[tname] = t_new
    for hname, arr in health.items():
        sc.add(f"health|{hname}", (~torch.isfinite(arr)).sum().double())
    vals = sc.fetch()
    centres, perm = fv.geometry.cell_centre, fv.perm
    out: dict = {"available": True, "version": DIAGNOSTICS_VERSION, "iteration": int(cap["iteration"]),
                 "rolled_back": bool(cap.get("rolled_back", False)), "precision": str(solver.dtype),
                 "unit_roundoff": u, "row_terms_max": K_rows, "cell_faces_max": K_cont}
    mom: dict = {"definition": "pre_solve: b - A U^n (assembled, unrelaxed); solve: b_r - A_r U* (system passed "
                               "to the linear solver)",
                 "relax_u": float(cap["alpha_u"]),
                 "row_scale_reference": {"pre_solve": vals["mom_pre|s_ref"], "solve": vals["mom_sol|s_ref"]},
                 "excluded_row_threshold": {"pre_solve": gamma(K_rows, u) * vals["mom_pre|s_ref"],
                                            "solve": gamma(K_rows, u) * vals["mom_sol|s_ref"]}}
    for k, nm in enumerate(names):
        p_rep = _row_report(vals, "mom_pre", nm, centres, perm)
        s_rep = _row_report(vals, "mom_sol", nm, centres, perm)
        s_rep["linear_solver"] = _linear_info(cap["mom_info"][k])
        s_rep["true_reduction_l2"] = ratio(s_rep["abs_l2"], vals[f"mom_true_r0|{nm}"])
        mom[nm] = {"pre_solve": p_rep, "solve": s_rep}
    out["momentum"] = mom
    if ecap is not None:
        p_rep = _row_report(vals, "T_pre", "energy", centres, perm)
        s_rep = _row_report(vals, "T_sol", "energy", centres, perm)
        s_rep["linear_solver"] = _linear_info(ecap.get("info"))
        s_rep["true_reduction_l2"] = ratio(s_rep["abs_l2"], vals["T_true_r0"])
        out["energy"] = {"pre_solve": p_rep, "solve": s_rep, "relax_T": float(ecap["alpha"])}
    pc = _row_report(vals, "pcorr", "p-correction", centres, perm)
    pc["linear_solver"] = _linear_info(cap.get("p_info"))
    pc["relative_l2"] = ratio(pc["abs_l2"], vals["cont_pred|cells|l2"])
    pc["definition"] = "A_p p' = -m* (rhs = minus the predictor imbalance); residual = -(corrected imbalance)"
    out["pressure_correction"] = pc
    cont: dict = {"units": "kg/s (per unit depth in 2-D), positive = net outflow"}
    for tag, label in (("pred", "predictor"), ("corr", "corrected")):
        rep = _row_report(vals, "cont_" + tag, "cells", centres, perm)
        cont[label] = {"local_max_relative": rep["row_scaled"], "abs_l1": rep["abs_l1"], "abs_max": rep["abs_max"],
                       "abs_l2": rep["abs_l2"],
                       "l1_over_face_flux": ratio(rep["abs_l1"], vals[f"cont_{tag}|face_flux_l1"]),
                       "active_cells": rep["active_rows"], "excluded_cells": rep["excluded_rows"],
                       "excluded_abs_max": rep["excluded_abs_max"], "nonfinite_cells": rep["nonfinite_rows"],
                       "sum_of_cells": vals[f"cont_{tag}|signed_sum"]}
        if "worst_cell" in rep:
            cont[label]["worst_cell"] = rep["worst_cell"]
            cont[label]["worst_cell_centre"] = rep["worst_cell_centre"]
    cont["global_boundary"] = {"signed": vals["global|signed"], "throughflow": vals["global|throughflow"],
                               "relative": ratio(abs(vals["global|signed"]), vals["global|throughflow"])}
    out["continuity"] = cont
    rolled = out["rolled_back"]
    U_ref = vals["dU|ref"]
    change: dict = {"velocity": None if rolled else ratio(vals["dU|num"], U_ref), "velocity_reference": U_ref}
    rho = float(solver.case.density)
    p_ref = max(vals["dp|range"], rho * U_ref * U_ref)
    change["pressure"] = None if rolled else ratio(vals["dp|num"], p_ref)
    change["pressure_reference"] = p_ref
    if ecap is not None:
        change["temperature"] = None if rolled else ratio(vals["dT|num"], vals["dT|ref"])
        change["temperature_reference"] = vals["dT|ref"]
    for tname in tnames:
        change[tname] = None if rolled else ratio(vals[f"d{tname}|num"], vals[f"d{tname}|ref"])
    out["field_change"] = change
    nonfinite = {hname: int(vals[f"health|{hname}"]) for hname in health}
    out["health"] = {"finite": not any(nonfinite.values()), "nonfinite_values": nonfinite}
    return out


def summary(d: dict) -> dict:
    """Flat headline numbers (``diagnostics.py:362-381``)."""
    if not d.get("available"):
        return {}
    mom = d["momentum"]
    comps = [k for k in COMPONENTS if k in mom]
    out = {"iteration": d["iteration"],
           "momentum_pre_row_scaled": max(mom[k]["pre_solve"]["row_scaled"] for k in comps),
           "momentum_solve_row_scaled": max(mom[k]["solve"]["row_scaled"] for k in comps),
           "continuity_predictor_local_max": d["continuity"]["predictor"]["local_max_relative"],
           "continuity_corrected_local_max": d["continuity"]["corrected"]["local_max_relative"],
           "continuity_global_relative": d["continuity"]["global_boundary"]["relative"],
           "velocity_change": d["field_change"]["velocity"], "pressure_change": d["field_change"]["pressure"],
           "finite": d["health"]["finite"]}
    if "energy" in d:
        out["energy_pre_row_scaled"] = d["energy"]["pre_solve"]["row_scaled"]
    return out


def pressure_matrix_properties(solver) -> Optional[dict]:
    """Whether preconditioned CG applies to the latest pressure-correction matrix, with the keys
    of ``flowtrace/unstructured/diagnostics.py:384-412``: it is a symmetric M-matrix (positive
    semi-definite; singular up to a constant when no boundary fixes the pressure) when

    * |A - A^T| is at most 64 u max|A| (u the unit round-off): on the mesh pattern every
      off-diagonal pair is one face's (a_PN, a_NP), so this is the largest |a_PN - a_NP|;
    * no off-diagonal entry exceeds 64 u max|A|;
    * every diagonal entry is positive and every row weakly diagonally dominant: the margin
      (a_ii - sum_{j != i} |a_ij|) / |a_ii| is at least -64 u.

    One device pass over the matrix (``b2s_matrix_properties_d``: exact maxima and minima over
    rows and faces) and a read of five numbers; None before the first iteration."""
    import torch

    if getattr(solver, "_capture", None) is None:
        return None
    L, fv = _lib.lib(), solver.fv
    work = torch.empty(int(L.b2s_matrix_properties_workspace_bytes()) // 8, dtype=torch.float64, device=fv.device)
    res = torch.empty(5, dtype=torch.float64, device=fv.device)
    _lib.check(L.b2s_matrix_properties_d(fv.cmesh_ref, solver.val_P.data_ptr(), work.data_ptr(), work.numel() * 8,
                                         res.data_ptr(), _lib.stream_ptr()), "b2s_matrix_properties_d")
    amax, asym_abs, off_max, margin, dmin = (float(v) for v in res.cpu().numpy())
    scale = amax or 1.0
    asym = asym_abs / scale if fv.nnz else 0.0
    tol = 64 * unit_roundoff(np.float64)
    out = {"symmetric": asym <= tol, "max_relative_asymmetry": asym,
           "offdiagonal_nonpositive": bool(off_max <= tol * scale) if fv.n_if else True,
           "weakly_diagonally_dominant": bool(margin >= -tol) and bool(dmin > 0),
           "min_dominance_margin": margin, "singular": bool(getattr(solver, "singular_p", False))}
    out["cg_applicable"] = out["symmetric"] and out["offdiagonal_nonpositive"] and out["weakly_diagonally_dominant"]
    return out
