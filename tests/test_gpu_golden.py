"""The CUDA path against fixtures recorded from the reference itself (``tests/golden/``),
through the C ABI: operators, BiCGSTAB, the SA-AMG V-cycle, SIMPLEC iterates and the systems
captured in one iteration (per entry, 1e-12)."""

import os

import numpy as np
import pytest

from gputest_b200.mesh.unstructured import cartesian_mesh_2d, extrude_to_3d
from gputest_b200.unstructured.case import UnstructuredCase
from tests.test_oracle_golden import _runs

pytestmark = pytest.mark.gpu
GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_fixtures.npz"))


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("name", ["tri2d", "hex3d"])
def test_cuda_operators_equal_the_reference(name):
    from gputest_b200.unstructured.fvmesh import FVMesh

    mesh = {"tri2d": cartesian_mesh_2d(20, 16, triangulate=True, warp=0.05),
            "hex3d": extrude_to_3d(cartesian_mesh_2d(6, 5, warp=0.05), 4, 0.5)}[name]
    fv = FVMesh(mesh)
    rng = np.random.default_rng(0)
    phi, phib = rng.standard_normal(fv.nc), rng.standard_normal(fv.n_bf)
    g = rng.standard_normal((fv.nc, fv.dim))
    rng.standard_normal(fv.n_if), rng.standard_normal((fv.n_if, fv.dim))
    d = 4 + rng.random(fv.nc)
    a1, a2 = -rng.random(fv.n_if), -rng.random(fv.n_if)
    p = f"op|{name}|"
    dphi, dphib, dg = fv.cells_to_device(phi), fv.bfaces_to_device(phib), fv.cells_to_device(g)
    assert np.array_equal(fv.faces_to_host(fv.face_interp(dphi)), GOLD[p + "interp"])
    assert _rel(fv.cells_to_host(fv.gradient(dphi, dphib)), GOLD[p + "ls"]) <= 1e-13
    assert _rel(fv.cells_to_host(fv.gradient_gg(dphi, dphib)), GOLD[p + "gg"]) <= 1e-13
    assert _rel(fv.cells_to_host(fv.gradient_gg(dphi, dphib, dg)), GOLD[p + "gg_corr"]) <= 1e-13
    val = fv.matrix_values(fv.cells_to_device(d), fv.faces_to_device(a1), fv.faces_to_device(a2))
    assert np.array_equal(fv.matrix_to_host(val).data, GOLD[p + "matrix_data"])


@pytest.mark.parametrize("tol,maxiter", [(0.1, 30), (1e-10, 500), (1e-10, 3)])
def test_cuda_bicgstab_equals_the_reference(tol, maxiter):
    from gputest_b200.linalg.krylov import bicgstab_jacobi
    from gputest_b200.unstructured.fvmesh import FVMesh

    fv = FVMesh(cartesian_mesh_2d(24, 24, triangulate=True, warp=0.05))
    rng = np.random.default_rng(2)
    d = 4 + rng.random(fv.nc)
    a1, a2 = -rng.random(fv.n_if), -rng.random(fv.n_if)
    b, x0 = rng.standard_normal(fv.nc), rng.standard_normal(fv.nc)
    val = fv.matrix_values(fv.cells_to_device(d), fv.faces_to_device(a1), fv.faces_to_device(a2))
    x, infos = bicgstab_jacobi(fv.rowptr, fv.col, val, fv.cells_to_device(b), fv.cells_to_device(x0),
                               fv.cells_to_device(1.0 / d), tol=tol, maxiter=maxiter)
    it, res, conv = GOLD[f"bicg|{tol}|{maxiter}|info"]
    assert (infos[0].iterations, infos[0].converged) == (int(it), bool(conv))
    assert infos[0].residual == pytest.approx(res, rel=1e-10)
    assert _rel(fv.cells_to_host(x), GOLD[f"bicg|{tol}|{maxiter}|x"]) <= 1e-12


@pytest.mark.parametrize("name", ["tri16", "cavity64", "channel_energy"])
def test_cuda_simplec_equals_the_reference(name):
    from gputest_b200.unstructured.simple import SimpleSolver

    mesh, kw, n = _runs()[name]
    s = SimpleSolver(mesh, UnstructuredCase(**kw), max_coarse=300)
    s.reaggregate = True
    for _ in range(n):
        s.step()
    p = f"simplec|{name}|"
    for k, v in s.fields().items():
        assert _rel(v, GOLD[p + "field|" + k]) <= 1e-9, k
    for k, v in s.residuals()["scaled"].items():
        assert v == pytest.approx(float(GOLD[p + "res|" + k][0]), rel=1e-6), k
    lin = list(s.last_linear["momentum_iters"]) + [s.last_linear["pressure_iters"]]
    gold = list(GOLD[p + "linear"])
    assert lin[:-1] == gold[:-1] and abs(lin[-1] - gold[-1]) <= 1
    if name == "tri16":
        cap = s.captured_systems()
        for key, ours in (("A", cap["A"].data), ("Ar", cap["Ar"].data), ("Ap", cap["Ap"].data),
                          ("b", np.stack(cap["b"], axis=1)), ("br", np.stack(cap["br"], axis=1)),
                          ("mass", cap["mass"]), ("U_old", cap["U_old"]), ("Fst", cap["Fst"])):
            scale = np.abs(GOLD[p + "cap|" + key]).max()
            assert np.abs(ours - GOLD[p + "cap|" + key]).max() <= 1e-9 * scale, key
