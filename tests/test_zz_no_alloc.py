"""The allocation-free Jacobi-BiCGSTAB entry point against the ordinary one, through the C ABI.

``b2s_bicgstab_jacobi_noalloc_d`` serves callers that cannot allocate device memory (a host
code that reaches the solver only through the C ABI and owns no CUDA allocator, or one whose
device memory is fully handed out before the solve): its work space is a static device array
inside the library. It must give what ``b2s_bicgstab_jacobi_d`` gives with a caller-provided
work array, call after call, although every call reuses the same scratch. This file is named
to be collected last, so a run that stops at the first failure has run every other test first.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _system(seed, nrhs, mesh=None):
    import torch

    from gputest_b200.mesh.unstructured import cartesian_mesh_2d
    from gputest_b200.unstructured.fvmesh import FVMesh

    mesh = mesh if mesh is not None else cartesian_mesh_2d(24, 24, triangulate=True, warp=0.05)
    fv = FVMesh(mesh)
    rng = np.random.default_rng(seed)
    d = 4 + rng.random(fv.nc)
    val = fv.matrix_values(fv.cells_to_device(d), fv.faces_to_device(-rng.random(fv.n_if)),
                           fv.faces_to_device(-rng.random(fv.n_if)))
    B = torch.stack([fv.cells_to_device(rng.standard_normal(fv.nc)) for _ in range(nrhs)]).contiguous()
    X0 = torch.stack([fv.cells_to_device(rng.standard_normal(fv.nc)) for _ in range(nrhs)]).contiguous()
    inv = fv.cells_to_device(1.0 / d)
    return fv, val, B, X0, inv


def _solve(fv, val, B, X0, inv, tol, maxiter, noalloc):
    import torch

    from gputest_b200 import _lib
    from gputest_b200.linalg.krylov import info_buffer, read_info

    L = _lib.lib()
    k, n = B.shape
    x = X0.clone()
    info = info_buffer(k, B.device)
    s = _lib.stream_ptr()
    if noalloc:
        rc = L.b2s_bicgstab_jacobi_noalloc_d(n, k, fv.rowptr.data_ptr(), fv.col.data_ptr(), val.data_ptr(),
                                             B.data_ptr(), inv.data_ptr(), x.data_ptr(), tol, maxiter, 1,
                                             info.data_ptr(), s)
    else:
        work = torch.empty(L.b2s_bicgstab_workspace_bytes(n, k) // 8 + 1, dtype=torch.float64, device=B.device)
        rc = L.b2s_bicgstab_jacobi_d(n, k, fv.rowptr.data_ptr(), fv.col.data_ptr(), val.data_ptr(), B.data_ptr(),
                                     inv.data_ptr(), x.data_ptr(), tol, maxiter, 1, work.data_ptr(), work.numel() * 8,
                                     info.data_ptr(), s)
    assert rc == 0, rc
    torch.cuda.synchronize()
    return x, read_info(info)


def test_noalloc_bicgstab_equals_the_allocating_entry_point_on_consecutive_calls():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    # two calls in a row that share the library's scratch: a 2-system solve, then a 3-system one
    for seed, nrhs, tol, maxiter in ((11, 2, 1e-8, 200), (12, 3, 0.1, 30)):
        fv, val, B, X0, inv = _system(seed, nrhs)
        xa, ia = _solve(fv, val, B, X0, inv, tol, maxiter, noalloc=False)
        xn, inn = _solve(fv, val, B, X0, inv, tol, maxiter, noalloc=True)
        for a, b in zip(ia, inn):
            assert (a.iterations, a.converged) == (b.iterations, b.converged)
            assert abs(a.residual - b.residual) <= 1e-10 * max(a.residual, 1e-300)
        rel = float((xn - xa).abs().max() / xa.abs().max().clamp_min(1e-300))
        assert rel < 1e-12, rel


def test_noalloc_single_system_and_exactly_at_capacity():
    """One right-hand side, then n * nrhs exactly at the capacity (65,536 cells x 2), where the
    static array's vectors and its block partials are packed tightest; both against the
    allocating entry point."""
    import torch

    from gputest_b200.mesh.unstructured import cartesian_mesh_2d

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    cases = ((13, 1, 1e-8, 200, None), (14, 2, 1e-3, 60, cartesian_mesh_2d(256, 256, jitter=0.1, seed=4)))
    for seed, nrhs, tol, maxiter, mesh in cases:
        fv, val, B, X0, inv = _system(seed, nrhs, mesh)
        assert mesh is None or fv.nc * nrhs == 131072
        xa, ia = _solve(fv, val, B, X0, inv, tol, maxiter, noalloc=False)
        xn, inn = _solve(fv, val, B, X0, inv, tol, maxiter, noalloc=True)
        for a, b in zip(ia, inn):
            assert (a.iterations, a.converged) == (b.iterations, b.converged)
            assert abs(a.residual - b.residual) <= 1e-10 * max(a.residual, 1e-300)
        rel = float((xn - xa).abs().max() / xa.abs().max().clamp_min(1e-300))
        assert rel < 1e-12, rel


def test_noalloc_rejects_sizes_beyond_its_capacity():
    import torch

    from gputest_b200 import _lib

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    L = _lib.lib()
    # n * nrhs above the capacity is refused before any pointer is used or any kernel launched
    rc = L.b2s_bicgstab_jacobi_noalloc_d(131072, 2, None, None, None, None, None, None, 0.1, 30, 1, None, None)
    assert rc == -5
    rc = L.b2s_bicgstab_jacobi_noalloc_d(131073, 1, None, None, None, None, None, None, 0.1, 30, 1, None, None)
    assert rc == -5
    rc = L.b2s_bicgstab_jacobi_noalloc_d(43691, 3, None, None, None, None, None, None, 0.1, 30, 1, None, None)
    assert rc == -5  # 131,073 unknowns over three systems
