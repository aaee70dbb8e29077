"""``SimpleSolver.diagnostics()`` on the device, checked by the algebraic identities of the
reference's own diagnostics tests (``tests/test_diagnostics.py:52-193,287-298``)."""

import math

import numpy as np
import pytest

from gputest_b200.mesh.unstructured import cartesian_mesh_2d
from gputest_b200.unstructured import diagnostics as D
from gputest_b200.unstructured.case import BoundarySpec, UnstructuredCase

pytestmark = pytest.mark.gpu
EPS = np.finfo(np.float64).eps


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _cavity(n=16, warp=0.05, **kw):
    from gputest_b200.unstructured.simple import SimpleSolver

    kw.setdefault("max_iter", 1000)
    case = UnstructuredCase(boundaries={"top": BoundarySpec("wall", velocity=[1.0, 0.0])}, **kw)
    return SimpleSolver(cartesian_mesh_2d(n, n, warp=warp), case)


def _duct(energy=True, **kw):
    from gputest_b200.unstructured.simple import SimpleSolver

    m = cartesian_mesh_2d(24, 8, 3.0, 1.0, names=("in", "out", "bottom", "top"), warp=0.03)
    case = UnstructuredCase(boundaries={"in": BoundarySpec("inlet", velocity=[1.0, 0.0], value=1.0),
                                        "out": BoundarySpec("outlet"),
                                        "bottom": BoundarySpec("wall", thermal="temperature", value=0.0),
                                        "top": BoundarySpec("wall")}, energy=energy, **kw)
    return SimpleSolver(m, case)


def _run(s, n):
    for _ in range(n):
        s.step()
    return s


def test_unavailable_before_the_first_iteration_and_after_a_restore():
    s = _cavity()
    assert s.diagnostics()["available"] is False
    _run(s, 3)
    assert s.diagnostics()["available"] is True
    s.load_state(s.state_dict())
    assert s.diagnostics()["available"] is False


def test_captured_system_reproduces_the_scaled_residual():
    s = _run(_cavity(), 12)
    cap = s.captured_systems()
    A, U = cap["A"], cap["U_old"]
    diag = A.diagonal()
    num = [np.abs(cap["b"][k] - A @ U[:, k]).sum() for k in range(2)]
    den = [np.abs(diag * U[:, k]).sum() for k in range(2)]
    floor = 1e-3 * max(max(den), 1e-300)
    for k, name in enumerate(("x-velocity", "y-velocity")):
        assert num[k] / max(den[k], floor) == pytest.approx(s.residuals()["scaled"][name], rel=1e-12)


def test_relaxed_and_assembled_systems_share_the_presolve_residual():
    s = _run(_cavity(), 8)
    cap = s.captured_systems()
    for k in range(2):
        u0 = cap["U_old"][:, k]
        r_pre = cap["b"][k] - cap["A"] @ u0
        r_rel = cap["br"][k] - cap["Ar"] @ u0
        scale = np.abs(cap["br"][k]).max() + np.abs(cap["Ar"].data).max() * np.abs(u0).max()
        assert np.abs(r_rel - r_pre).max() <= 64 * EPS * scale


def test_solved_system_residual_matches_the_linear_solver():
    s = _run(_cavity(), 20)
    d = s.diagnostics()
    for comp in ("x-velocity", "y-velocity"):
        sol = d["momentum"][comp]["solve"]
        lin = sol["linear_solver"]
        assert sol["true_reduction_l2"] == pytest.approx(lin["reported_residual"], rel=1e-6)
        if lin["converged"]:
            assert sol["true_reduction_l2"] < 0.1 * (1 + 1e-6)


def test_corrected_imbalance_is_the_pressure_correction_residual():
    s = _run(_duct(energy=False), 15)
    cap = s.captured_systems()
    h = s.fv.host
    import scipy.sparse as sp

    faces = np.arange(h.n_if)
    Cdiff = sp.csr_matrix((np.r_[np.ones(h.n_if), -np.ones(h.n_if)], (np.r_[h.P, h.N], np.r_[faces, faces])),
                          shape=(h.nc, h.n_if))
    Cb = sp.csr_matrix((np.ones(h.n_bf), (h.Pb, np.arange(h.n_bf))), shape=(h.nc, h.n_bf))
    corrected = Cdiff @ cap["F"] + Cb @ cap["Fb"]
    residual = -cap["mass"] - cap["Ap"] @ cap["pp"]
    assert np.abs(corrected + residual).max() <= 1e-12 * np.abs(cap["mass"]).max()
    d = s.diagnostics()
    pc = d["pressure_correction"]
    assert d["continuity"]["corrected"]["abs_l2"] == pytest.approx(pc["abs_l2"], rel=1e-9)
    assert pc["relative_l2"] == pytest.approx(pc["linear_solver"]["reported_residual"], rel=1e-6)


def test_global_boundary_imbalance_is_the_sum_of_cell_imbalances():
    s = _run(_duct(energy=False), 30)
    c = s.diagnostics()["continuity"]
    g = c["global_boundary"]
    assert g["throughflow"] > 0 and g["relative"] >= 0
    assert g["signed"] == pytest.approx(c["corrected"]["sum_of_cells"], abs=1e-12 * g["throughflow"])
    assert c["corrected"]["local_max_relative"] > 0


def test_zero_scale_system_reports_zero_not_nan():
    from gputest_b200.unstructured.simple import SimpleSolver

    s = _run(SimpleSolver(cartesian_mesh_2d(6, 6), UnstructuredCase(boundaries={}, max_iter=10)), 2)
    d = s.diagnostics()
    for comp in ("x-velocity", "y-velocity"):
        for stage in ("pre_solve", "solve"):
            rep = d["momentum"][comp][stage]
            assert rep["row_scaled"] == 0.0 and rep["active_rows"] == 0 and rep["excluded_rows"] == s.nc
    assert d["continuity"]["global_boundary"] == {"signed": 0.0, "throughflow": 0.0, "relative": 0.0}
    assert d["field_change"]["velocity"] == 0.0 and d["field_change"]["pressure"] == 0.0
    assert d["health"]["finite"]


def test_nonfinite_values_are_counted_and_fail_thresholds():
    s = _run(_cavity(), 5)
    cap = s._capture
    s.bmom[0][3] = float("nan")  # test-only corruption of the captured right-hand side (device data)
    s._Up[cap["new"]][2][7] = float("inf")
    d = s.diagnostics()
    pre = d["momentum"]["x-velocity"]["pre_solve"]
    assert pre["nonfinite_rows"] == 1 and pre["row_scaled"] == math.inf
    assert d["health"]["finite"] is False and d["health"]["nonfinite_values"]["velocity"] == 1
    assert D.summary(d)["finite"] is False


def test_energy_diagnostics_and_field_change_definition():
    s = _run(_duct(), 10)
    d = s.diagnostics()
    e = d["energy"]
    assert e["pre_solve"]["active_rows"] > 0 and e["solve"]["linear_solver"]["iterations"] >= 0
    cap = s.captured_systems()
    dU = np.linalg.norm(cap["U_new"] - cap["U_old"], axis=1).max()
    U_ref = max(np.linalg.norm(cap["U_new"], axis=1).max(), np.linalg.norm(cap["U_old"], axis=1).max(),
                np.linalg.norm(s.ub_fixed, axis=1).max())
    assert d["field_change"]["velocity"] == pytest.approx(dU / U_ref, rel=1e-12)
    p_ref = max(np.ptp(cap["p_new"]), s.case.density * U_ref ** 2)
    assert d["field_change"]["pressure"] == pytest.approx(np.abs(cap["p_new"] - cap["p_old"]).max() / p_ref, rel=1e-12)
    T_old, T_new = cap["energy"]["T_old"], cap["energy"]["T_new"]
    T_ref = max(T_new.max(), 1.0) - min(T_new.min(), 0.0)
    assert d["field_change"]["temperature"] == pytest.approx(np.abs(T_new - T_old).max() / T_ref, rel=1e-12)


def test_diagnostics_converge_towards_zero():
    s = _cavity(n=12, tol=1e-8)
    _run(s, 5)
    early = D.summary(s.diagnostics())
    s.run()
    late = D.summary(s.diagnostics())
    assert s.converged
    for k in ("momentum_pre_row_scaled", "continuity_predictor_local_max", "velocity_change"):
        assert late[k] < 1e-3 * early[k]


def _host_matrix_properties(A):
    """The definitions of ``flowtrace/unstructured/diagnostics.py:384-412`` evaluated with SciPy
    on a host copy of the matrix (the checker of the device pass)."""
    import scipy.sparse as sp

    A = sp.csr_matrix(A)
    scale = float(abs(A).max()) or 1.0
    diag = A.diagonal()
    off = (A - sp.diags(diag)).tocsr()
    off.eliminate_zeros()
    rowsum = np.asarray(abs(off).sum(axis=1)).ravel()
    return {"asym": float(abs(A - A.T).max()) / scale, "off_max": float(off.data.max()) if off.nnz else -np.inf,
            "margin": float(((diag - rowsum) / np.maximum(np.abs(diag), 1e-300)).min()), "scale": scale,
            "dmin": float(diag.min())}


def test_pressure_matrix_meets_the_conditions_for_cg():
    s = _cavity(n=10)
    assert D.pressure_matrix_properties(s) is None
    _run(s, 3)
    pm = D.pressure_matrix_properties(s)
    assert pm["cg_applicable"] and pm["symmetric"] and pm["singular"]
    d = _run(_duct(energy=False), 3)
    pm = D.pressure_matrix_properties(d)
    assert pm["cg_applicable"] and not pm["singular"] and pm["min_dominance_margin"] >= -64 * D.unit_roundoff(np.float64)
    for solver in (s, d):
        pm = D.pressure_matrix_properties(solver)
        h = _host_matrix_properties(solver.fv.matrix_to_host(solver.val_P))
        assert pm["max_relative_asymmetry"] == h["asym"]
        assert pm["min_dominance_margin"] == pytest.approx(h["margin"], rel=1e-12, abs=1e-15)
        assert pm["offdiagonal_nonpositive"] == (h["off_max"] <= 64 * D.unit_roundoff(np.float64) * h["scale"])


def test_pressure_matrix_properties_flag_a_planted_asymmetry_and_a_positive_offdiagonal():
    """Entries planted in a copy of the matrix on the host side: the device pass reports what the
    host definitions give."""
    s = _cavity(n=10)
    _run(s, 3)
    fv = s.fv
    j = int(fv.t["slot_PN"][5])
    s.val_P[j] = s.val_P[j] * 0.5  # a_PN != a_NP on one face
    pm = D.pressure_matrix_properties(s)
    h = _host_matrix_properties(fv.matrix_to_host(s.val_P))
    assert not pm["symmetric"] and pm["max_relative_asymmetry"] == pytest.approx(h["asym"], rel=1e-15)
    assert not pm["cg_applicable"]
    s.val_P[j] = abs(float(s.val_P[j])) + 1.0  # a positive off-diagonal entry
    pm = D.pressure_matrix_properties(s)
    assert not pm["offdiagonal_nonpositive"]
