"""The k-omega SST model in the mixed-precision solver (float momentum, pressure and energy
systems; the SST stages in double): converged, its fields equal the double solver's converged
fields to 1e-6 relative, as the mixed form promises for the laminar path - without and with the
energy equation (the float energy rows with k/cp + mu_t/Pr_t per face)."""

import numpy as np
import pytest

from gputest_b200.mesh.unstructured import cartesian_mesh_2d
from gputest_b200.unstructured.case import BoundarySpec, UnstructuredCase

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def test_mixed_sst_converges_to_the_double_solution():
    from gputest_b200.unstructured.mixed import MixedSimpleSolver
    from gputest_b200.unstructured.simple import SimpleSolver

    mesh = cartesian_mesh_2d(24, 10, 3.0, 1.0, names=("in", "out", "bottom", "top"))
    kw = dict(boundaries={"in": BoundarySpec("inlet", velocity=[1.0, 0.0]), "out": BoundarySpec("outlet"),
                          "bottom": BoundarySpec("wall"), "top": BoundarySpec("wall")},
              viscosity=1e-3, turbulence="k-omega-sst", max_iter=4000, tol=1e-10)
    d = SimpleSolver(mesh, UnstructuredCase(**kw))
    d.run()
    m = MixedSimpleSolver(mesh, UnstructuredCase(**kw, precision="mixed"))
    m.run()
    assert d.converged and m.converged
    fd, fm = d.fields(), m.fields()
    for k in ("x-velocity", "y-velocity", "pressure", "turb-kinetic-energy", "specific-diss-rate", "viscosity-turb"):
        err = np.abs(fm[k] - fd[k]).max() / np.abs(fd[k]).max()
        assert err <= 1e-6, (k, err)


def test_mixed_sst_with_a_heated_wall_converges_to_the_double_solution():
    from gputest_b200.unstructured.mixed import MixedSimpleSolver
    from gputest_b200.unstructured.simple import SimpleSolver

    mesh = cartesian_mesh_2d(24, 10, 3.0, 1.0, names=("in", "out", "bottom", "top"))
    kw = dict(boundaries={"in": BoundarySpec("inlet", velocity=[1.0, 0.0], value=0.0), "out": BoundarySpec("outlet"),
                          "bottom": BoundarySpec("wall", thermal="flux", value=5.0),
                          "top": BoundarySpec("wall", thermal="temperature", value=1.0)},
              viscosity=1e-3, turbulence="k-omega-sst", energy=True, cp=1.0, conductivity=1e-3 / 0.71,
              max_iter=6000, tol=1e-10)
    d = SimpleSolver(mesh, UnstructuredCase(**kw))
    d.run()
    m = MixedSimpleSolver(mesh, UnstructuredCase(**kw, precision="mixed"))
    m.run()
    assert d.converged and m.converged
    fd, fm = d.fields(), m.fields()
    for k in ("x-velocity", "y-velocity", "pressure", "temperature", "turb-kinetic-energy", "specific-diss-rate"):
        err = np.abs(fm[k] - fd[k]).max() / np.abs(fd[k]).max()
        assert err <= 1e-6, (k, err)
