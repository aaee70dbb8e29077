"""The plain-PyTorch transcription of the steady residual (``TorchResidual``), on the CPU with the
oracle: it vanishes at a converged state, and its exact discrete adjoint (a dense solve of the
autograd Jacobian at small size) agrees with central finite differences of re-converged flows."""

import copy

import numpy as np
import pytest

from gputest_b200.mesh.unstructured import cartesian_mesh_2d
from gputest_b200.unstructured.adjoint import TorchResidual, bc_from_oracle, relax_from, state_from_oracle
from gputest_b200.unstructured.case import BoundarySpec, UnstructuredCase
from oracle.simplec_oracle import OracleSimple, load_native


def _channel(nx=24, ny=6):
    m = cartesian_mesh_2d(nx, ny, 4.0, 1.0, names=("in", "out", "bottom", "top"))
    case = UnstructuredCase(boundaries={"in": BoundarySpec("inlet", velocity=[1.0, 0.0]), "out": BoundarySpec("outlet"),
                                        "bottom": BoundarySpec("wall"), "top": BoundarySpec("wall")},
                            viscosity=1 / 200, scheme="upwind", tol=1e-13, max_iter=20000, algorithm="SIMPLE",
                            relax_u=0.3, relax_p=0.3)
    rng = np.random.default_rng(0)
    por = 1e4 / (1 + np.exp(-8 * rng.standard_normal(m.n_cells)))
    return m, case, por


def _solve(m, case, por, u_in=1.0, start=None):
    o = OracleSimple(m, copy.deepcopy(case), native=load_native(), porosity=por)
    if u_in != 1.0:
        ub = o.ub_fixed.copy()
        ub[o.m_inlet > 0, 0] = u_in
        o.ub_fixed = ub
        o.initialize({})
    if start is not None:
        o.load_state(start)
    while not o.finished:
        o.step()
    assert o.converged
    return o


def _x(R, o):
    import torch

    return R.pack(*[torch.as_tensor(a) for a in state_from_oracle(o)])


def test_residual_vanishes_at_a_converged_state():
    import torch

    m, case, por = _channel()
    o = _solve(m, case, por)
    ru, sc = relax_from(o)
    R = TorchResidual(o.fv, bc_from_oracle(o), case, relax_u=ru, simplec=sc)
    x = _x(R, o)
    r = R.residual(x, torch.as_tensor(por), torch.as_tensor(o.ub_fixed))
    for blk, ref in zip(R.split(r), R.split(x)):
        assert float(blk.abs().max()) <= 1e-10 * max(float(ref.abs().max()), 1.0)


def test_exact_discrete_adjoint_matches_central_differences():
    import torch

    m, case, por = _channel()
    o = _solve(m, case, por)
    ru, sc = relax_from(o)
    R = TorchResidual(o.fv, bc_from_oracle(o), case, relax_u=ru, simplec=sc)
    x = _x(R, o).requires_grad_(True)
    al = torch.as_tensor(por).requires_grad_(True)
    ub = torch.as_tensor(o.ub_fixed).requires_grad_(True)
    J = R.objective(x, ub)
    gx, gub_direct = torch.autograd.grad(J, (x, ub))
    Jac = torch.autograd.functional.jacobian(lambda v: R.residual(v, al.detach(), ub.detach()), x.detach())
    lam = torch.linalg.solve(Jac.T, gx)
    ga, gu = torch.autograd.grad(R.residual(x, al, ub), (al, ub), lam)
    d_por = -ga.numpy()
    d_uin = float((gub_direct - gu).numpy()[o.m_inlet > 0, 0].sum())
    st, h = o.state_dict(), 1e-6
    rng = np.random.default_rng(5)
    Jof = lambda oo: float(R.objective(_x(R, oo), torch.as_tensor(oo.ub_fixed)))  # noqa: E731
    for _ in range(2):
        d = rng.standard_normal(m.n_cells) * por
        fd = (Jof(_solve(m, case, por + h * d, start=st)) - Jof(_solve(m, case, por - h * d, start=st))) / (2 * h)
        assert float(d_por @ d) == pytest.approx(fd, rel=1e-5)
    fd = (Jof(_solve(m, case, por, 1 + h, start=st)) - Jof(_solve(m, case, por, 1 - h, start=st))) / (2 * h)
    assert d_uin == pytest.approx(fd, rel=1e-5)


def test_compressed_reverse_products_recover_the_exact_jacobian():
    """``assemble_jacobian`` (one reverse product per residual type and lattice colour) against the
    dense autograd Jacobian of the transcription, in the adjoint's block layout; and
    ``TransposedSolver`` (gradient unknowns eliminated, sparse LU of the rest) against a dense
    solve of the transposed system."""
    import torch

    from gputest_b200.unstructured.adjoint import TransposedSolver, _descriptors, assemble_jacobian, grid_coordinates

    m, case, por = _channel()
    o = _solve(m, case, por)
    ru, sc = relax_from(o)
    R = TorchResidual(o.fv, bc_from_oracle(o), case, relax_u=ru, simplec=sc)
    h = o.fv
    nc, dim = h.nc, h.dim

    def to_ref(v):  # block layout (U [dim][nc], p, g [dim][nc], F, Fb) -> transcription layout
        v = torch.as_tensor(v)
        a = np.cumsum([0, dim * nc, nc, dim * nc])
        return torch.cat([v[a[0]:a[1]].reshape(dim, nc).T.reshape(-1), v[a[1]:a[2]],
                          v[a[2]:a[3]].reshape(dim, nc).T.reshape(-1), v[a[3]:]])

    def to_blk(v):
        U, p, g, F, Fb = R.split(v)
        return torch.cat([U.T.reshape(-1), p, g.T.reshape(-1), F, Fb])

    x = _x(R, o)
    al, ub = torch.as_tensor(por), torch.as_tensor(o.ub_fixed)
    xr = x.clone().requires_grad_(True)
    r = R.residual(xr, al, ub)

    def vjp(lam):
        return to_blk(torch.autograd.grad(r, xr, to_ref(lam), retain_graph=True)[0]).numpy()

    ij = grid_coordinates(h.xc)
    home, typ = _descriptors(dim, nc, ij, h.P, h.N, h.Pb, h.Sb)
    Js = assemble_jacobian(vjp, home, typ, ij, x.numel())
    J = Js.toarray()
    Jd = torch.autograd.functional.jacobian(lambda v: to_blk(R.residual(to_ref(v), al, ub)), to_blk(x)).numpy()
    assert np.abs(J - Jd).max() <= 1e-12 * np.abs(Jd).max()
    # the transposed solve with the gradient unknowns eliminated
    ts = TransposedSolver(Js, dim, nc)
    assert ts.minv is not None
    b = np.random.default_rng(2).standard_normal(J.shape[0])
    y = ts.solve(b)
    assert np.linalg.norm(Jd.T @ y - b) <= 1e-10 * np.linalg.norm(b)
    assert np.allclose(y, np.linalg.solve(Jd.T, b), rtol=1e-8, atol=1e-10 * np.abs(y).max())
