"""CUDA finite-volume operators and Krylov solves against the oracle, through the C ABI.

Mirrors the reference's kernel tests (``tests/test_native.py:23-64`` and
``tests/test_gpu_real.py:130-172`` of the reference): the same two meshes, seeded inputs,
bit-equality where the summation order is the reference's, 1e-13 elsewhere, and BiCGSTAB
iteration counts equal to the algorithm's.
"""

import numpy as np
import pytest

from gputest_b200.mesh.unstructured import cartesian_mesh_2d, extrude_to_3d
from oracle.simplec_oracle import OracleFV, OracleSimple, SmoothedAggregationAMG, bicgstab, pcg

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _meshes():
    return {"tri2d": cartesian_mesh_2d(20, 16, triangulate=True, warp=0.05),
            "hex3d": extrude_to_3d(cartesian_mesh_2d(6, 5, warp=0.05), 4, 0.5),
            "alt2d": cartesian_mesh_2d(24, 20, triangulate="alternating", jitter=0.2)}


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.mark.parametrize("name", ["tri2d", "hex3d", "alt2d"])
def test_fv_operators_match_oracle(torch_cuda, name):
    from gputest_b200.unstructured.fvmesh import FVMesh

    mesh = _meshes()[name]
    o = OracleFV(mesh)
    fv = FVMesh(mesh)
    rng = np.random.default_rng(0)
    phi, phib = rng.standard_normal(o.nc), rng.standard_normal(o.n_bf)
    g = rng.standard_normal((o.nc, o.dim))
    d_phi, d_phib, d_g = fv.cells_to_device(phi), fv.bfaces_to_device(phib), fv.cells_to_device(g)
    assert _rel(fv.faces_to_host(fv.face_interp(d_phi)), o.face_interp(phi)) == 0.0
    fi = fv.face_interp(d_g).cpu().numpy()  # [dim][nf] device faces
    ref = o.face_interp_vec(g)[fv.face_ref]
    assert _rel(fi.T, ref) == 0.0
    assert _rel(fv.cells_to_host(fv.gradient(d_phi, d_phib)), o.gradient(phi, phib)) <= 1e-13
    assert _rel(fv.cells_to_host(fv.gradient_gg(d_phi, d_phib)), o.gradient_gg(phi, phib)) <= 1e-13
    assert _rel(fv.cells_to_host(fv.gradient_gg(d_phi, d_phib, d_g)), o.gradient_gg(phi, phib, g)) <= 1e-13
    # several fields in one launch equal one field at a time
    both = fv.gradient(torch_cuda.stack([d_phi, 2.0 * d_phi]), torch_cuda.stack([d_phib, 2.0 * d_phib]))
    assert _rel(fv.cells_to_host(both[1]), 2.0 * fv.cells_to_host(both[0])) == 0.0
    d = 4 + rng.random(o.nc)
    a1, a2 = -rng.random(o.n_if), -rng.random(o.n_if)
    val = fv.matrix_values(fv.cells_to_device(d), fv.faces_to_device(a1), fv.faces_to_device(a2))
    assert _rel(fv.matrix_to_host(val).toarray(), o.matrix(d, a1, a2).toarray()) == 0.0
    x = rng.standard_normal(o.nc)
    Ax = fv.cells_to_host(fv.spmv(val, fv.cells_to_device(x)))
    assert _rel(Ax, o.matrix(d, a1, a2) @ x) == 0.0  # rows keep the reference's summation order


@pytest.mark.parametrize("tol,maxiter", [(0.1, 30), (1e-10, 500), (1e-10, 3)])
def test_bicgstab_follows_the_algorithm(torch_cuda, tol, maxiter):
    """Iteration counts and outcome equal the reference algorithm's (``test_native.py:51-64``)."""
    from gputest_b200.linalg.krylov import bicgstab_jacobi
    from gputest_b200.unstructured.fvmesh import FVMesh

    mesh = cartesian_mesh_2d(24, 24, triangulate=True, warp=0.05)
    o = OracleFV(mesh)
    fv = FVMesh(mesh)
    rng = np.random.default_rng(2)
    d = 4 + rng.random(o.nc)
    a1, a2 = -rng.random(o.n_if), -rng.random(o.n_if)
    A = o.matrix(d, a1, a2)
    b, x0, inv = rng.standard_normal(o.nc), rng.standard_normal(o.nc), 1.0 / d
    xr, ir = bicgstab(lambda v: A @ v, b, M=lambda v: inv * v, x0=x0, tol=tol, maxiter=maxiter, relative_to_initial=True)
    val = fv.matrix_values(fv.cells_to_device(d), fv.faces_to_device(a1), fv.faces_to_device(a2))
    xd, infos = bicgstab_jacobi(fv.rowptr, fv.col, val, fv.cells_to_device(b), fv.cells_to_device(x0),
                                fv.cells_to_device(inv), tol=tol, maxiter=maxiter)
    inn = infos[0]
    assert (inn.iterations, inn.converged) == (ir.iterations, ir.converged)
    assert abs(inn.residual - ir.residual) <= 1e-10 * max(ir.residual, 1e-300)
    assert _rel(fv.cells_to_host(xd), xr) < 1e-12


def test_bicgstab_three_systems_in_one_launch_equal_three_solves(torch_cuda):
    from gputest_b200.linalg.krylov import bicgstab_jacobi
    from gputest_b200.unstructured.fvmesh import FVMesh

    mesh = cartesian_mesh_2d(24, 24, triangulate=True, warp=0.05)
    o = OracleFV(mesh)
    fv = FVMesh(mesh)
    rng = np.random.default_rng(5)
    d = 4 + rng.random(o.nc)
    val = fv.matrix_values(fv.cells_to_device(d), fv.faces_to_device(-rng.random(o.n_if)),
                           fv.faces_to_device(-rng.random(o.n_if)))
    B = torch_cuda.stack([fv.cells_to_device(rng.standard_normal(o.nc)) for _ in range(3)])
    X0 = torch_cuda.stack([fv.cells_to_device(rng.standard_normal(o.nc)) for _ in range(3)])
    inv = fv.cells_to_device(1.0 / d)
    X, infos = bicgstab_jacobi(fv.rowptr, fv.col, val, B, X0, inv, tol=1e-6, maxiter=100)
    for k in range(3):
        xk, ik = bicgstab_jacobi(fv.rowptr, fv.col, val, B[k], X0[k], inv, tol=1e-6, maxiter=100)
        assert (ik[0].iterations, ik[0].converged) == (infos[k].iterations, infos[k].converged)
        assert torch_cuda.equal(xk, X[k])


@pytest.mark.parametrize("name", ["alt2d", "hex3d", "alt2d_large"])
def test_amg_vcycle_and_pcg_match_the_reference_hierarchy(torch_cuda, name):
    """With the reference's max_coarse the device hierarchy is the reference's SA-AMG: one
    V-cycle agrees to round-off and AMG-PCG takes the same number of iterations."""
    from gputest_b200.linalg.amg import AMGHierarchy
    from gputest_b200.linalg.krylov import info_buffer, read_info
    from gputest_b200.unstructured.case import BoundarySpec, UnstructuredCase
    from gputest_b200.unstructured.fvmesh import FVMesh

    # alt2d_large has a finest level above the V-cycle's block-0 tail threshold (grid-wide phases)
    mesh = {"alt2d": lambda: cartesian_mesh_2d(48, 48, triangulate="alternating", jitter=0.2),
            "alt2d_large": lambda: cartesian_mesh_2d(96, 96, triangulate="alternating", jitter=0.2),
            "hex3d": lambda: extrude_to_3d(cartesian_mesh_2d(16, 12, warp=0.05), 8, 0.5)}[name]()
    top = [1.0, 0.0] if mesh.dim == 2 else [1.0, 0.0, 0.0]
    case = UnstructuredCase(boundaries={"top": BoundarySpec("wall", velocity=top)}, viscosity=0.01)
    o = OracleSimple(mesh, case)
    for _ in range(3):
        o.step()
    Ap, mass = o._capture["Ap"], o._capture["mass"]
    ref = SmoothedAggregationAMG(Ap, singular=o.singular_p)
    fv = FVMesh(mesh)
    val = torch_cuda.as_tensor(np.ascontiguousarray(Ap.data[fv.slot_ref]), device=fv.device)
    h = AMGHierarchy(Ap, fv.perm, fv.rowptr, fv.col, fv.t["slot_diag"], val, fv.slot_ref, singular=o.singular_p,
                     max_coarse=300)
    assert h.sizes[:-1] == [lv[0].shape[0] for lv in ref.levels] and h.coarse_n == ref.coarse_inv.shape[0]
    h.rebuild()
    assert not h.strength_changed()  # the device values reproduce the set-up's strength graph
    b = -mass
    z, zr = fv.cells_to_host(h.vcycle(fv.cells_to_device(b))), ref(b)
    tol_v = 1e-9
    if o.singular_p:
        # the reference inverts the singular coarse matrix shifted by 1e-10 mean|diag| (condition
        # ~1e10), so round-off of the two inversions differs along the near-null vector
        z, zr = z - z.mean(), zr - zr.mean()
        tol_v = 1e-7
    assert _rel(z, zr) < tol_v
    proj = (lambda v: v - v.mean()) if o.singular_p else None
    for tol in (0.1, 1e-8):
        xr, ir = pcg(lambda v: Ap @ v, b, M=ref, tol=tol, maxiter=200, project=proj)
        x = torch_cuda.zeros(o.nc, dtype=torch_cuda.float64, device=fv.device)
        info = info_buffer(1, fv.device)
        h.pcg(fv.cells_to_device(b), x, tol, 200, o.singular_p, info.data_ptr())
        i = read_info(info)[0]
        assert i.converged == ir.converged and abs(i.iterations - ir.iterations) <= 1, (i, ir)
        assert np.abs(Ap @ fv.cells_to_host(x) - b).max() <= 10 * tol * np.abs(b).max() + 1e-14
        if i.iterations == ir.iterations:
            assert _rel(fv.cells_to_host(x), xr) < 1e-6


@pytest.mark.parametrize("dim", [2, 3, "batch"])
def test_amg_term_list_rebuild_equals_the_row_owned_rebuild(dim):
    """The rebuild from the set-up's term lists (thread per P row / W entry / A_c entry) gives
    the same hierarchy bit for bit as the row-owned kernels that locate each term's slot by
    binary search (selected by clearing the term-list pointers)."""
    import torch

    from gputest_b200.mesh.unstructured import box_mesh_3d, cartesian_mesh_2d
    from gputest_b200.unstructured.case import BoundarySpec, UnstructuredCase
    from gputest_b200.unstructured.simple import SimpleSolver

    if dim == "batch":  # a block-diagonal batch hierarchy (per-case spectral radii)
        from gputest_b200.unstructured.batch import BatchSimpleSolver

        meshes = [cartesian_mesh_2d(n, n, jitter=0.15, seed=n) for n in (30, 18, 24)]
        cases = [UnstructuredCase(boundaries={"top": BoundarySpec("wall", velocity=[u, 0.0])}, viscosity=0.01,
                                  max_iter=10, tol=0.0) for u in (1.0, 0.5, 2.0)]
        s = BatchSimpleSolver(meshes, cases, max_coarse=40)
    elif dim == 2:
        mesh = cartesian_mesh_2d(48, 48, triangulate=True, jitter=0.2)
        top = [1.0, 0.0]
    else:
        mesh = box_mesh_3d(16, 12, 10, jitter=0.1, seed=1, names=("wall", "wall", "wall", "top", "wall", "wall"))
        top = [1.0, 0.0, 0.0]
    if dim != "batch":
        case = UnstructuredCase(boundaries={"top": BoundarySpec("wall", velocity=top), "wall": BoundarySpec("wall")},
                                viscosity=0.01, max_iter=10, tol=0.0)
        s = SimpleSolver(mesh, case, amg_theta=0.0)
    for _ in range(3):
        s.step()
    amg, h = s._amg, s._amg.c
    assert h.nlevels >= 2 and all(h.levels[l].p_tptr and h.levels[l].w_tptr for l in range(h.nlevels))
    assert h.levels[0].c_tptr
    bufs = [b for b in amg._keep if "p_val" in b]
    nxt = [b["val"] for b in amg._keep if "diag" in b]

    def values():
        torch.cuda.synchronize()
        out = [t.clone() for b in bufs for t in (b["p_val"], b["w_val"], b["rho"])]
        return out + [t.clone() for t in nxt] + [amg.coarse_inv.clone()]

    amg.rebuild()
    a = values()
    names = ("p_tptr", "p_tj", "w_tptr", "w_tj", "w_te", "c_tptr", "c_te", "c_ts")
    saved = [[getattr(h.levels[l], k) for k in names] for l in range(h.nlevels)]
    for l in range(h.nlevels):
        for k in names:
            setattr(h.levels[l], k, None)
    amg.rebuild()
    b = values()
    for l in range(h.nlevels):
        for k, v in zip(names, saved[l]):
            setattr(h.levels[l], k, v)
    for x, y in zip(a, b):
        assert torch.equal(x, y)
