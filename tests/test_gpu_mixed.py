"""The mixed-precision path: float Krylov solvers against their double counterparts through the
C ABI, the double iterative refinement of the pressure-correction solve, and converged
``MixedSimpleSolver`` fields against the double ``SimpleSolver`` (relative error <= 1e-6)."""

import numpy as np
import pytest

from gputest_b200.mesh.unstructured import box_mesh_3d, cartesian_mesh_2d
from gputest_b200.unstructured.case import BoundarySpec, UnstructuredCase

pytestmark = pytest.mark.gpu

FIELD_TOL = 1e-6  # converged mixed-precision fields against the double path, relative to max |field|


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


def _system(n=48, seed=5):
    from gputest_b200.unstructured.fvmesh import FVMesh

    fv = FVMesh(cartesian_mesh_2d(n, n, triangulate=True, warp=0.05))
    rng = np.random.default_rng(seed)
    d = 4 + rng.random(fv.nc)
    a1, a2 = -rng.random(fv.n_if), -rng.random(fv.n_if)
    val = fv.matrix_values(fv.cells_to_device(d), fv.faces_to_device(a1), fv.faces_to_device(a2))
    return fv, val, d, rng


@pytest.mark.parametrize("nrhs", [1, 3])
def test_float_bicgstab_matches_the_double_solver(nrhs):
    import torch

    from gputest_b200 import _lib
    from gputest_b200.linalg.krylov import bicgstab_jacobi, info_buffer, read_info

    fv, val, d, rng = _system()
    n = fv.nc
    b = torch.stack([fv.cells_to_device(rng.standard_normal(n)) for _ in range(nrhs)])
    inv = fv.cells_to_device(1.0 / d)
    x64, infos64 = bicgstab_jacobi(fv.rowptr, fv.col, val, b, torch.zeros_like(b), inv, tol=1e-5, maxiter=200)
    L = _lib.lib()
    val32, b32, inv32 = val.float(), b.float().contiguous(), inv.float()
    x32 = torch.full_like(b32, 123.0)  # not read: zero_x0
    base = torch.randn(b.shape, dtype=torch.float64, device=b.device)
    out = torch.empty_like(base)
    wb = L.b2s_bicgstab_f32_workspace_bytes(n, nrhs)
    work = torch.empty(wb // 8 + 1, dtype=torch.float64, device=b.device)
    info = info_buffer(nrhs, b.device)
    _lib.check(L.b2s_bicgstab_jacobi_f32_d(n, nrhs, fv.rowptr.data_ptr(), fv.col.data_ptr(), val32.data_ptr(),
                                           b32.data_ptr(), inv32.data_ptr(), x32.data_ptr(), 1e-5, 200, 1, 1,
                                           out.data_ptr(), base.data_ptr(), work.data_ptr(), work.numel() * 8,
                                           info.data_ptr(), _lib.stream_ptr()), "b2s_bicgstab_jacobi_f32_d")
    infos32 = read_info(info)
    for k in range(nrhs):
        assert infos32[k].converged and infos64[k].converged
        assert abs(infos32[k].iterations - infos64[k].iterations) <= 2
        assert _rel(x32[k].double().cpu(), x64[k].cpu()) < 1e-4
        assert torch.equal(out[k], base[k] + x32[k].double())


def _cavity_solvers(mesh, **kw):
    from gputest_b200.unstructured.mixed import MixedSimpleSolver
    from gputest_b200.unstructured.simple import SimpleSolver

    top = [1.0, 0.0] if mesh.dim == 2 else [1.0, 0.0, 0.0]
    case = UnstructuredCase(boundaries={"top": BoundarySpec("wall", velocity=top)}, **kw)
    return SimpleSolver(mesh, case), MixedSimpleSolver(mesh, case)


def _face_operator(fv, cf, cb, x):
    """(A x) of the pressure-correction operator from its double face coefficients, on the host
    in reference numbering: sum_f cf_f (x_P - x_N) per cell, plus cb_b x_P on boundary faces."""
    h = fv.host
    cfh, cbh, xh = fv.faces_to_host(cf), fv.bfaces_to_host(cb), fv.cells_to_host(x)
    y = np.zeros(h.nc)
    d = cfh * (xh[h.P] - xh[h.N])
    np.add.at(y, h.P, d)
    np.add.at(y, h.N, -d)
    np.add.at(y, h.Pb, cbh * xh[h.Pb])
    return y


@pytest.mark.parametrize("closed", [True, False])
def test_refined_pressure_solve_reaches_double_accuracy(closed):
    """A pressure-correction tolerance far below float's reach (1e-11): the double refinement
    gets there, checked with the double operator on the host, on a singular (closed cavity) and
    a regular (channel) system."""
    import torch

    from gputest_b200.unstructured.mixed import MixedSimpleSolver

    if closed:
        mesh = cartesian_mesh_2d(40, 40, jitter=0.15)
        case = UnstructuredCase(boundaries={"top": BoundarySpec("wall", velocity=[1.0, 0.0])}, viscosity=0.01,
                                max_iter=50, tol=0.0, pressure_tol=1e-11)
    else:
        mesh = cartesian_mesh_2d(40, 12, 3.0, 1.0, names=("in", "out", "bottom", "top"), jitter=0.15)
        case = UnstructuredCase(boundaries={"in": BoundarySpec("inlet", velocity=[1.0, 0.0]),
                                            "out": BoundarySpec("outlet"), "bottom": BoundarySpec("wall"),
                                            "top": BoundarySpec("wall")}, viscosity=0.01, max_iter=50, tol=0.0,
                                pressure_tol=1e-11)
    smx = MixedSimpleSolver(mesh, case)
    for _ in range(6):
        smx.step()
    assert smx.last_linear["pressure_residual"] < 1e-11
    info = torch.zeros(2, dtype=torch.float64, device=smx.rhs_p.device)
    rhs = smx.rhs_p.clone()
    for tol in (1e-6, 1e-12):
        x = torch.zeros_like(rhs)
        smx._amg.pcg_mixed(smx.fv.cmesh_ref, smx.cf, smx.cb, rhs, x, tol, 400, smx.singular_p, info.data_ptr())
        torch.cuda.synchronize()
        r = smx.fv.cells_to_host(rhs) - _face_operator(smx.fv, smx.cf, smx.cb, x)
        if smx.singular_p:
            r = r - r.mean()
        rel = np.linalg.norm(r) / np.linalg.norm(smx.fv.cells_to_host(rhs))
        assert rel < tol
        assert float(info[1].item()) == pytest.approx(rel, rel=1e-3, abs=1e-3 * tol)


def test_mixed_momentum_matrix_is_the_rounded_double_matrix():
    import torch

    s64, smx = _cavity_solvers(cartesian_mesh_2d(24, 24, triangulate=True, warp=0.05), viscosity=0.01,
                               scheme="second-order", max_iter=20, tol=0.0, pressure_tol=1e-9)
    for _ in range(3):
        s64.step()
        smx.step()
    st = s64.state_dict()
    s64.load_state(st)
    smx.load_state(st)
    s64.step()
    smx.step()
    fv = s64.fv
    # relaxed matrix: float rounding of the double one, entry by entry
    assert torch.equal(smx.val_A32, s64.val_A.float())
    # residual b - A U of the unrelaxed system (double in the kernel, stored in float)
    cap = s64.captured_systems()
    r_ref = np.stack([cap["b"][k] - cap["A"] @ cap["U_old"][:, k] for k in range(2)], axis=1)
    r_mx = fv.cells_to_host(smx.r32.double())
    scale = max(float(np.abs(np.asarray(bk)).max()) for bk in cap["b"])
    assert np.abs(r_mx - r_ref).max() <= 1e-6 * scale


@pytest.mark.parametrize("name", ["cavity_tri", "channel_energy"])
def test_converged_mixed_fields_match_the_double_path(name):
    from gputest_b200.unstructured.mixed import MixedSimpleSolver
    from gputest_b200.unstructured.simple import SimpleSolver

    if name == "cavity_tri":
        mesh = cartesian_mesh_2d(32, 32, triangulate="alternating", jitter=0.2, seed=0)
        case = UnstructuredCase(boundaries={"top": BoundarySpec("wall", velocity=[1.0, 0.0])}, viscosity=0.01,
                                scheme="second-order", max_iter=6000, tol=1e-10)
    else:
        mesh = cartesian_mesh_2d(30, 10, 3.0, 1.0, names=("in", "out", "bottom", "top"), jitter=0.1)
        case = UnstructuredCase(boundaries={"in": BoundarySpec("inlet", velocity=[1.0, 0.0], value=1.0),
                                            "out": BoundarySpec("outlet"),
                                            "bottom": BoundarySpec("wall", thermal="temperature", value=0.0),
                                            "top": BoundarySpec("wall", thermal="flux", value=2.0)},
                                energy=True, viscosity=0.01, conductivity=0.02, max_iter=6000, tol=1e-10)
    s64, smx = SimpleSolver(mesh, case), MixedSimpleSolver(mesh, case)
    s64.run()
    smx.run()
    assert s64.converged and smx.converged
    f64, fmx = s64.fields(), smx.fields()
    for k in f64:
        assert _rel(fmx[k], f64[k]) <= FIELD_TOL, (k, _rel(fmx[k], f64[k]))


def test_mixed_duct_3d_converges_like_the_double_path():
    from gputest_b200.unstructured.mixed import MixedSimpleSolver
    from gputest_b200.unstructured.simple import SimpleSolver

    names = ("inlet", "outlet", "wall", "wall", "wall", "wall")
    mesh = box_mesh_3d(16, 8, 8, 4.0, 1.0, 1.0, jitter=0.1, seed=1, names=names,
                       types=("velocity-inlet", "pressure-outlet", "wall", "wall", "wall", "wall"))
    mu = 1.0 / 50.0
    case = UnstructuredCase(boundaries={"inlet": BoundarySpec("inlet", velocity=[1.0, 0.0, 0.0], value=0.0),
                                        "outlet": BoundarySpec("outlet", pressure=0.0),
                                        "wall": BoundarySpec("wall", thermal="flux", value=5.0)},
                            viscosity=mu, energy=True, cp=1.0, conductivity=mu / 0.71, max_iter=4000, tol=1e-9)
    s64, smx = SimpleSolver(mesh, case, amg_theta=0.0), MixedSimpleSolver(mesh, case, amg_theta=0.0)
    s64.run()
    smx.run()
    assert s64.converged and smx.converged
    f64, fmx = s64.fields(), smx.fields()
    for k in f64:
        assert _rel(fmx[k], f64[k]) <= FIELD_TOL, (k, _rel(fmx[k], f64[k]))
    assert abs(smx.iteration - s64.iteration) <= max(10, s64.iteration // 10)


def test_mixed_solver_refuses_the_double_only_reports():
    from gputest_b200.unstructured.mixed import MixedSimpleSolver

    s = MixedSimpleSolver(cartesian_mesh_2d(8, 8), UnstructuredCase(boundaries={}, max_iter=5, precision="mixed"))
    s.step()
    with pytest.raises(NotImplementedError):
        s.diagnostics()
