"""The oracle's wall reports (``wall_forces``, ``wall_report``, ``wall_profile``; laminar and
with the k-omega SST wall viscosity) against the reference's, through
``tests/golden/report_fixtures.npz`` (made by ``tests/golden/make_report_golden.py``)."""

import json
import os

import numpy as np
import pytest

from gputest_b200.mesh.unstructured import cartesian_mesh_2d, extrude_to_3d
from gputest_b200.unstructured.case import BoundarySpec, UnstructuredCase
from oracle.simplec_oracle import OracleSimple
from tests.golden.report_cases import REPORT_CASES

GOLD = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "report_fixtures.npz"))


def _close(ours, ref, rel):
    """Nested dicts/lists of floats equal to ``rel`` relative to the largest magnitude present."""
    if isinstance(ref, dict):
        assert set(ours) == set(ref)
        for k in ref:
            _close(ours[k], ref[k], rel)
        return
    a, b = np.asarray(ours, dtype=np.float64), np.asarray(ref, dtype=np.float64)
    assert np.abs(a - b).max() <= rel * max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("name", sorted(REPORT_CASES))
def test_oracle_wall_reports_equal_the_reference(name):
    build, kw, n, zone = REPORT_CASES[name]
    bnd = {z: BoundarySpec(**spec) for z, spec in kw["boundaries"].items()}
    o = OracleSimple(build(cartesian_mesh_2d, extrude_to_3d), UnstructuredCase(**{**kw, "boundaries": bnd}))
    for _ in range(n):
        o.step()
    p = f"rep|{name}|"
    for k, v in o.fields().items():
        assert np.array_equal(v, GOLD[p + "field|" + k]), k
    ref = json.loads(bytes(GOLD[p + "json"]).decode())
    _close(o.wall_forces(), ref["wall_forces"], 1e-13)
    _close(o.wall_report(), ref["wall_report"], 1e-13)
    prof = o.wall_profile(zone)
    for k, v in prof.items():
        assert np.allclose(v, GOLD[p + "profile|" + k], rtol=1e-13, atol=0), k


@pytest.mark.parametrize("name", sorted(REPORT_CASES))
def test_product_wall_reports_equal_the_reference(name):
    """``SimpleSolver.wall_forces`` / ``wall_report`` / ``wall_profile`` of the B200 path, run on
    the host arrays of the oracle's state (the same reference numbering the solver's host side
    uses; the boundary pressure and, with the SST model, the wall viscosity taken from the
    oracle), against the reference's reports."""
    from types import SimpleNamespace

    from gputest_b200.unstructured.fvmesh import HostFV
    from gputest_b200.unstructured.simple import SimpleSolver

    build, kw, n, zone = REPORT_CASES[name]
    bnd = {z: BoundarySpec(**spec) for z, spec in kw["boundaries"].items()}
    mesh = build(cartesian_mesh_2d, extrude_to_3d)
    o = OracleSimple(mesh, UnstructuredCase(**{**kw, "boundaries": bnd}))
    for _ in range(n):
        o.step()

    class HostView(SimpleSolver):
        U = property(lambda self: o.U)
        T = property(lambda self: o.T)

        def _pressure_bvals_host(self):
            return o._pressure_bvals(o.p, o._gp)

        def _wall_viscosity_host(self):
            return o._wall_viscosity()

    s = HostView.__new__(HostView)
    s.mesh, s.case, s.energy = mesh, o.case, o.energy
    s.fv = SimpleNamespace(host=HostFV(mesh))
    s.bkind_h, s._ub_fixed_h, s.tkind_h, s._tval_h = o.bkind, o.ub_fixed, o.tkind, o.tval
    ref = json.loads(bytes(GOLD[f"rep|{name}|json"]).decode())
    _close(s.wall_forces(), ref["wall_forces"], 1e-13)
    _close(s.wall_report(), ref["wall_report"], 1e-13)
    for k, v in s.wall_profile(zone).items():
        assert np.allclose(v, GOLD[f"rep|{name}|profile|" + k], rtol=1e-13, atol=0), k
