"""The wall reports of the CUDA path (``SimpleSolver.wall_forces`` / ``wall_report`` /
``wall_profile``, laminar and with the k-omega SST wall viscosity) against the reference's,
after the same outer iterations (``tests/golden/report_fixtures.npz``). The device fields agree
with the reference's to about 1e-9, so the reports are compared at 1e-7."""

import json
import os

import numpy as np
import pytest

from gputest_b200.mesh.unstructured import cartesian_mesh_2d, extrude_to_3d
from gputest_b200.unstructured.case import BoundarySpec, UnstructuredCase
from tests.golden.report_cases import REPORT_CASES
from tests.test_oracle_reports import _close

pytestmark = pytest.mark.gpu
GOLD = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "report_fixtures.npz"))


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


@pytest.mark.parametrize("name", sorted(REPORT_CASES))
def test_cuda_wall_reports_equal_the_reference(name):
    from gputest_b200.unstructured.simple import SimpleSolver

    build, kw, n, zone = REPORT_CASES[name]
    bnd = {z: BoundarySpec(**spec) for z, spec in kw["boundaries"].items()}
    s = SimpleSolver(build(cartesian_mesh_2d, extrude_to_3d), UnstructuredCase(**{**kw, "boundaries": bnd}),
                     max_coarse=300)
    s.reaggregate = True
    for _ in range(n):
        s.step()
    ref = json.loads(bytes(GOLD[f"rep|{name}|json"]).decode())
    _close(s.wall_forces(), ref["wall_forces"], 1e-7)
    _close(s.wall_report(), ref["wall_report"], 1e-7)
    for k, v in s.wall_profile(zone).items():
        g = GOLD[f"rep|{name}|profile|" + k]
        assert np.abs(v - g).max() <= 1e-7 * np.abs(g).max(), k


def test_cuda_sst_diagnostics_report_k_and_omega():
    """As the reference's ``tests/test_diagnostics.py:227-234``: with the SST model the
    diagnostics' field changes include k and omega, and their health counts are reported."""
    from gputest_b200.unstructured.simple import SimpleSolver

    build, kw, _, _ = REPORT_CASES["sst_chan2d"]
    bnd = {z: BoundarySpec(**spec) for z, spec in kw["boundaries"].items()}
    s = SimpleSolver(build(cartesian_mesh_2d, extrude_to_3d), UnstructuredCase(**{**kw, "boundaries": bnd}))
    for _ in range(5):
        s.step()
    d = s.diagnostics()
    ch = d["field_change"]
    assert ch["k"] is not None and ch["omega"] is not None and 0 <= ch["k"] < 1e3
    assert d["health"]["finite"] and {"k", "omega"} <= set(d["health"]["nonfinite_values"])
