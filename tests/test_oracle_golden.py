"""The oracle (and the mesh generators) against fixtures recorded from the reference itself
(``tests/golden/make_golden.py``). CPU only: this pins the checker that the GPU tests use."""

import os

import numpy as np
import pytest

from gputest_b200.mesh.unstructured import cartesian_mesh_2d, extrude_to_3d
from gputest_b200.unstructured.case import BoundarySpec, UnstructuredCase
from oracle.simplec_oracle import OracleFV, OracleSimple, SmoothedAggregationAMG, bicgstab
from tests.golden.make_golden import MESH_CASES, mesh_digest

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_fixtures.npz"))


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("name", list(MESH_CASES))
def test_mesh_generators_reproduce_the_reference_arrays(name):
    assert mesh_digest(cartesian_mesh_2d(**MESH_CASES[name])) == GOLD[f"mesh|{name}"].tobytes().decode()


def test_extrusion_reproduces_the_reference_arrays():
    m = extrude_to_3d(cartesian_mesh_2d(6, 5, warp=0.05), 4, 0.5)
    assert mesh_digest(m) == GOLD["mesh|extrude6x5w"].tobytes().decode()


@pytest.mark.parametrize("name", ["tri2d", "hex3d"])
def test_oracle_operators_equal_the_reference(name):
    mesh = {"tri2d": cartesian_mesh_2d(20, 16, triangulate=True, warp=0.05),
            "hex3d": extrude_to_3d(cartesian_mesh_2d(6, 5, warp=0.05), 4, 0.5)}[name]
    fv = OracleFV(mesh)
    rng = np.random.default_rng(0)
    phi, phib = rng.standard_normal(fv.nc), rng.standard_normal(fv.n_bf)
    g = rng.standard_normal((fv.nc, fv.dim))
    F, G = rng.standard_normal(fv.n_if), rng.standard_normal((fv.n_if, fv.dim))
    d = 4 + rng.random(fv.nc)
    a1, a2 = -rng.random(fv.n_if), -rng.random(fv.n_if)
    p = f"op|{name}|"
    assert np.array_equal(fv.face_interp(phi), GOLD[p + "interp"])
    assert np.array_equal(fv.face_interp_vec(g), GOLD[p + "interp_vec"])
    assert _rel(fv.gradient(phi, phib), GOLD[p + "ls"]) <= 1e-14
    assert _rel(fv.gradient_gg(phi, phib), GOLD[p + "gg"]) <= 1e-14
    assert _rel(fv.gradient_gg(phi, phib, g), GOLD[p + "gg_corr"]) <= 1e-14
    assert np.array_equal(fv.Cdiff @ F, GOLD[p + "cdiff_F"])
    assert np.array_equal(fv.Cown @ G, GOLD[p + "cown_G"])
    A = fv.matrix(d, a1, a2)
    assert np.array_equal(A.indptr, GOLD[p + "matrix_indptr"]) and np.array_equal(A.indices, GOLD[p + "matrix_indices"])
    assert np.array_equal(A.data, GOLD[p + "matrix_data"])


@pytest.mark.parametrize("tol,maxiter", [(0.1, 30), (1e-10, 500), (1e-10, 3)])
def test_oracle_bicgstab_equals_the_reference(tol, maxiter):
    fv = OracleFV(cartesian_mesh_2d(24, 24, triangulate=True, warp=0.05))
    rng = np.random.default_rng(2)
    d = 4 + rng.random(fv.nc)
    A = fv.matrix(d, -rng.random(fv.n_if), -rng.random(fv.n_if))
    b, x0, inv = rng.standard_normal(fv.nc), rng.standard_normal(fv.nc), 1.0 / d
    x, info = bicgstab(lambda v: A @ v, b, M=lambda v: inv * v, x0=x0, tol=tol, maxiter=maxiter, relative_to_initial=True)
    it, res, conv = GOLD[f"bicg|{tol}|{maxiter}|info"]
    assert (info.iterations, info.converged) == (int(it), bool(conv))
    assert info.residual == pytest.approx(res, rel=1e-12)
    assert _rel(x, GOLD[f"bicg|{tol}|{maxiter}|x"]) <= 1e-13


def test_oracle_sa_amg_equals_the_reference():
    import scipy.sparse as sp

    Ap = sp.csr_matrix((GOLD["amg|Ap_data"], GOLD["amg|Ap_indices"], GOLD["amg|Ap_indptr"]))
    amg = SmoothedAggregationAMG(Ap, singular=True)
    assert [lv[0].shape[0] for lv in amg.levels] + [amg.coarse_inv.shape[0]] == list(GOLD["amg|sizes"])
    z = amg(GOLD["amg|b"])
    assert _rel(z - z.mean(), GOLD["amg|vcycle"] - GOLD["amg|vcycle"].mean()) <= 1e-10


def _runs():
    top = {"top": BoundarySpec("wall", velocity=[1.0, 0.0])}
    return {
        "tri16": (cartesian_mesh_2d(16, 16, triangulate=True, warp=0.05),
                  dict(boundaries=top, viscosity=0.01, max_iter=40, tol=0.0, pressure_tol=1e-9), 40),
        "cavity64": (cartesian_mesh_2d(64, 64),
                     dict(boundaries=top, viscosity=0.01, scheme="upwind", pressure_tol=1e-8, max_iter=300, tol=0.0), 30),
        "channel_energy": (cartesian_mesh_2d(24, 8, 3.0, 1.0, names=("in", "out", "bottom", "top"), warp=0.03),
                           dict(boundaries={"in": BoundarySpec("inlet", velocity=[1.0, 0.0], value=1.0),
                                            "out": BoundarySpec("outlet"),
                                            "bottom": BoundarySpec("wall", thermal="temperature", value=0.0),
                                            "top": BoundarySpec("wall", thermal="flux", value=2.0)},
                                energy=True, viscosity=0.01, conductivity=0.02, max_iter=50, tol=0.0), 30),
    }


@pytest.mark.parametrize("name", ["tri16", "cavity64", "channel_energy"])
def test_oracle_simplec_equals_the_reference(name):
    mesh, kw, n = _runs()[name]
    o = OracleSimple(mesh, UnstructuredCase(**kw))
    for _ in range(n):
        o.step()
    p = f"simplec|{name}|"
    for k, v in o.fields().items():
        assert _rel(v, GOLD[p + "field|" + k]) <= 1e-12, k
    for k, v in o.residuals()["scaled"].items():
        assert v == pytest.approx(float(GOLD[p + "res|" + k][0]), rel=1e-9), k
    lin = list(o.last_linear["momentum_iters"]) + [o.last_linear["pressure_iters"]]
    assert lin == list(GOLD[p + "linear"])
    if name == "tri16":
        cap = o._capture
        for key, ours in (("A", cap["A"].data), ("Ar", cap["Ar"].data), ("Ap", cap["Ap"].data),
                          ("b", np.stack(cap["b"], axis=1)), ("br", np.stack(cap["br"], axis=1)),
                          ("mass", cap["mass"]), ("U_old", cap["U_old"]), ("Fst", cap["Fst"])):
            assert _rel(ours, GOLD[p + "cap|" + key]) <= 1e-12, key
