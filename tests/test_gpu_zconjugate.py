"""Conjugate heat transfer on the CUDA path (``gputest_b200.unstructured.conjugate``) against the
reference's ``ConjugateSolver`` (fixtures of ``tests/golden/conjugate_fixtures.npz``, which the
oracle reproduces): fields, residuals, linear-solver counts and heat flows after a number of
outer iterations on a composite wall, a channel over a heated block (laminar, and turbulent with
the k-omega SST model adding mu_t/Pr_t to the fluid's conductivity) and a lid-driven cavity around
a heated disc; the composite wall's exact solution; ``make_solver``."""

import json
import os

import numpy as np
import pytest

from gputest_b200.unstructured.case import BoundarySpec, UnstructuredCase
from tests.golden.conjugate_cases import CONJUGATE_CASES

pytestmark = pytest.mark.gpu
GOLD = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "conjugate_fixtures.npz"))
# the reference's own temperature on the triangulated cavity moves by ~1e-7, and its energy
# residual by up to 1.5e-4, under 1e-15 relative perturbations of the conductivities
# (test_oracle_conjugate.test_conjugate_temperatures_are_set_to_what_the_gpu_test_asks)
# (on the turbulent heated channel: 1e-7, 3e-5 and 1e-7)
TEMPERATURE_TOL = {"composite": 1e-8, "heated": 1e-8, "heated_sst": 1e-5, "tri_disc": 1e-5}
ENERGY_RESIDUAL_TOL = {"composite": 1e-4, "heated": 1e-4, "heated_sst": 1e-3, "tri_disc": 1e-3}
# and its heat flows there by up to ~6e-6 relative (below 1e-9 on the laminar channel and wall)
HEAT_FLOW_TOL = {"composite": 1e-6, "heated": 1e-6, "heated_sst": 1e-4, "tri_disc": 1e-4}


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _err(a, b):
    """Largest difference relative to the reference field's magnitude (1 where it is zero)."""
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    scale = np.abs(b).max()
    return float(np.abs(a - b).max() / (scale if scale > 0 else 1.0))


def _solver(name):
    from gputest_b200.unstructured.conjugate import ConjugateSolver

    build, kw, n = CONJUGATE_CASES[name]
    bnd = {z: BoundarySpec(**spec) for z, spec in kw["boundaries"].items()}
    s = ConjugateSolver(build(), UnstructuredCase(**{**kw, "boundaries": bnd}), max_coarse=300)
    s.flow.reaggregate = True  # the reference's AMG set-up at every rebuild
    return s, n


@pytest.mark.parametrize("name", sorted(CONJUGATE_CASES))
def test_cuda_conjugate_equals_the_reference(name):
    s, n = _solver(name)
    for _ in range(n):
        s.step()
    p = f"cht|{name}|"
    assert s.iteration == int(GOLD[p + "iterations"][0])
    f = s.fields()
    for k in (k.split("|", 3)[3] for k in GOLD.files if k.startswith(p + "field|")):
        tol = TEMPERATURE_TOL[name] if k == "temperature" else 1e-8
        assert _err(f[k], GOLD[p + "field|" + k]) <= tol, k
    for k, v in s.residuals()["scaled"].items():
        g = float(GOLD[p + "res|" + k][0])
        assert v == pytest.approx(g, rel=ENERGY_RESIDUAL_TOL[name] if k == "energy" else 1e-5, abs=1e-13), k
    lin = list(s.last_linear["momentum_iters"]) + [s.last_linear["pressure_iters"]]
    gold = list(GOLD[p + "linear"])
    assert lin[:-1] == gold[:-1] and abs(lin[-1] - gold[-1]) <= 1
    ref = json.loads(bytes(GOLD[p + "heat_flow"]).decode())
    ours = s.heat_flow()
    assert set(ours) == set(ref)
    for k, v in ref.items():
        assert ours[k] == pytest.approx(v, rel=HEAT_FLOW_TOL[name], abs=1e-9), k
    assert np.all(f["x-velocity"][s.solid] == 0.0)


def test_cuda_composite_wall_is_exact():
    s, _ = _solver("composite")
    s.run(max_steps=60)
    x, T = s.cell_centres()[:, 0], s.fields()["temperature"]
    q = 1 / 3.2
    Te = np.where(x < 1, 1 - q * x / 5, np.where(x < 2, 1 - q / 5 - q * (x - 1), 1 - 1.2 * q - 2 * q * (x - 2)))
    assert np.abs(T - Te).max() < 1e-10


def test_make_solver_picks_the_conjugate_solver_and_the_state_round_trips():
    from gputest_b200.unstructured.conjugate import ConjugateSolver, make_solver

    build, kw, _ = CONJUGATE_CASES["heated"]
    bnd = {z: BoundarySpec(**spec) for z, spec in kw["boundaries"].items()}
    case = UnstructuredCase(**{**kw, "boundaries": bnd})
    a = make_solver(build(), case)
    assert isinstance(a, ConjugateSolver)
    for _ in range(5):
        a.step()
    st = a.state_dict()
    b = make_solver(build(), case)
    b.load_state(st)
    assert np.array_equal(b.fields()["temperature"], a.fields()["temperature"])
    assert np.array_equal(b.state_dict()["U"], st["U"])
