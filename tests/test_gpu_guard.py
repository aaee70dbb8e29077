"""The drop-in SimpleSolver's stability guard against the oracle's (``flowtrace/unstructured/
simple.py:705-776``): roll-back to the last healthy snapshot, the relax_p ladder, the
SIMPLEC -> SIMPLE fallback and ``guard_exhausted_at``. The reference's own forced-divergence
test (``tests/test_diagnostics.py:170-193``: a 24 x 24 cavity sheared by x += y, automatic
relaxation) is the model. The divergence is made on the host: by the sheared mesh itself, or by
a NaN written into the solver's state between iterations, never by a device fault."""

import math

import numpy as np
import pytest

from gputest_b200.mesh.unstructured import cartesian_mesh_2d
from gputest_b200.unstructured.case import BoundarySpec, UnstructuredCase
from oracle.simplec_oracle import OracleSimple

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


def _sheared(max_iter=3000):
    mesh = cartesian_mesh_2d(24, 24)
    mesh.nodes[:, 0] = mesh.nodes[:, 0] + mesh.nodes[:, 1]
    case = UnstructuredCase(boundaries={"top": BoundarySpec("wall", velocity=[1.0, 0.0])}, viscosity=0.1,
                            max_iter=max_iter, tol=1e-6, pressure_tol=1e-9)
    return mesh, case


def _pair(mesh, case):
    from gputest_b200.unstructured.simple import SimpleSolver

    s = SimpleSolver(mesh, case, max_coarse=300)
    s.reaggregate = True  # the reference re-aggregates at every rebuild
    return s, OracleSimple(mesh, case)


def _events_equal(ge, go):
    assert len(ge) == len(go)
    for a, b in zip(ge, go):
        assert a["detected_at"] == b["detected_at"] and a["restored_to"] == b["restored_to"]
        assert a["relax_p"] == b["relax_p"] and a.get("algorithm") == b.get("algorithm")
        assert a.get("relax_u") == b.get("relax_u")
        assert math.isfinite(a["continuity"]) == math.isfinite(b["continuity"])
        if math.isfinite(b["continuity"]):
            assert a["continuity"] == pytest.approx(b["continuity"], rel=1e-6)


def test_sheared_cavity_guard_rolls_back_like_the_oracle():
    """The sheared cavity diverges with the automatic relax_p; both solvers roll back at the same
    iterations to the same snapshots, lower relax_p along the same ladder and then converge to
    the same fields in the same number of iterations."""
    mesh, case = _sheared()
    s, o = _pair(mesh, case)
    while not o.finished:
        o.step()
        s.step()
        assert len(s.guard_events) == len(o.guard_events), o.iteration
    assert len(o.guard_events) >= 2  # the oracle rolls back twice on this mesh (relax_p 0.8 -> 0.48 -> 0.288)
    _events_equal(s.guard_events, o.guard_events)
    assert s.relax_p == pytest.approx(o.relax_p, rel=1e-15)
    assert s.guard_exhausted_at == o.guard_exhausted_at
    assert s.iteration == o.iteration and s.converged == o.converged
    fs, fo = s.fields(), o.fields()
    for k in ("x-velocity", "y-velocity", "pressure"):
        assert _rel(fs[k], fo[k]) < 1e-6, k
    d = s.diagnostics()
    assert d["available"]


def test_nan_in_the_state_restores_the_snapshot_like_the_oracle():
    """A NaN planted in the velocity between iterations (host-side injection) makes the
    continuity residual non-finite; both guards restore the same snapshot, lower relax_p, and
    the next iterations equal the oracle's."""
    from gputest_b200.unstructured.simple import SimpleSolver

    mesh = cartesian_mesh_2d(16, 16, triangulate=True, warp=0.05)
    case = UnstructuredCase(boundaries={"top": BoundarySpec("wall", velocity=[1.0, 0.0])}, viscosity=0.01,
                            max_iter=200, tol=0.0, pressure_tol=1e-9)
    s = SimpleSolver(mesh, case, max_coarse=300)
    s.reaggregate = True
    o = OracleSimple(mesh, case)
    for _ in range(45):  # snapshots taken at iterations 20 and 40
        s.step()
        o.step()
    assert s._guard_snap[0]["iteration"] == o._guard_snap[0]["iteration"] == 40
    s._Up[s._cur][1, 7] = float("nan")  # the x-velocity of device cell 7
    o.U[int(s.fv.perm[7]), 0] = np.nan  # the same cell in the reference numbering
    s.step()
    o.step()
    assert len(s.guard_events) == len(o.guard_events) == 1
    _events_equal(s.guard_events, o.guard_events)
    assert s.guard_events[0]["restored_to"] == 40 and not math.isfinite(s.guard_events[0]["continuity"])
    assert s.relax_p == pytest.approx(o.relax_p, rel=1e-15)
    for _ in range(10):
        s.step()
        o.step()
    fs, fo = s.fields(), o.fields()
    for k in ("x-velocity", "y-velocity", "pressure"):
        assert np.isfinite(fs[k]).all()
        assert _rel(fs[k], fo[k]) < 1e-9, k
    assert s.iteration == o.iteration
