"""The adjoint's flexible restarted GMRES (``DeviceAdjoint.solve``: classical Gram-Schmidt applied
twice, Givens rotations, right preconditioning by a sweep that may change between calls) on the CPU, with the
operator and the preconditioner given as plain functions in place of the CUDA VJP and the
transposed SIMPLE sweep."""

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla


def _bound_solver(matvec, precondition):
    from gputest_b200.unstructured.adjoint import DeviceAdjoint

    adj = DeviceAdjoint.__new__(DeviceAdjoint)  # no device state: the solve needs only these two
    adj.vjp = matvec
    adj.precondition = precondition
    return adj


def _system(n=600, seed=0):
    """A nonsymmetric convection-diffusion-like sparse matrix, diagonally dominant only in part."""
    rng = np.random.default_rng(seed)
    main = 2.0 + rng.random(n)
    A = sp.diags([main, -1.2 * np.ones(n - 1), -0.6 * np.ones(n - 1), 0.3 * rng.standard_normal(n - 7)],
                 [0, -1, 1, 7], format="csr")
    return A, rng.standard_normal(n)


def test_flexible_gmres_restarts_to_the_tolerance():
    """Restart cycles of 8 with a Jacobi preconditioner reach 1e-10; the returned residual is the
    true one, and the iteration count exceeds one cycle (the restart path ran)."""
    import torch

    A, b = _system()
    At = torch.as_tensor(A.toarray())
    dinv = torch.as_tensor(1.0 / A.diagonal())
    adj = _bound_solver(lambda v: At @ v, lambda r: dinv * r)
    x, its, rel = adj.solve(torch.as_tensor(b), tol=1e-10, restart=8, maxiter=3000)
    true = float(torch.linalg.vector_norm(torch.as_tensor(b) - At @ x) / torch.linalg.vector_norm(torch.as_tensor(b)))
    assert rel < 1e-10 and abs(rel - true) <= 1e-12 and its > 8


def test_flexible_gmres_accepts_a_preconditioner_that_changes_between_calls():
    """An inner Krylov solve as the preconditioner (a different linear map at every call, as the
    device sweep's inner PCG and BiCGSTAB are): the flexible form still converges, to the same
    solution as a direct solve."""
    import torch

    A, b = _system(seed=1)
    At = torch.as_tensor(A.toarray())
    Ap = (A + sp.diags(0.5 * np.ones(A.shape[0]))).tocsr()  # a nearby matrix, solved loosely

    def inner(r):
        y, _ = spla.bicgstab(Ap, r.numpy(), rtol=1e-3, maxiter=30)
        return torch.as_tensor(y)

    adj = _bound_solver(lambda v: At @ v, inner)
    x, its, rel = adj.solve(torch.as_tensor(b), tol=1e-11, restart=20, maxiter=2000)
    assert rel < 1e-11
    np.testing.assert_allclose(x.numpy(), spla.spsolve(A.tocsc(), b), rtol=1e-8, atol=1e-10)


def test_flexible_gmres_returns_zero_for_a_zero_right_hand_side():
    import torch

    A, _ = _system(n=50)
    At = torch.as_tensor(A.toarray())
    adj = _bound_solver(lambda v: At @ v, lambda r: r)
    x, its, rel = adj.solve(torch.zeros(50, dtype=torch.float64))
    assert its == 0 and rel == 0.0 and float(x.abs().max()) == 0.0
