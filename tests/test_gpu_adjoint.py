"""The discrete adjoint on the device: the CUDA vector-Jacobian product of the residual against
autograd through its plain-PyTorch transcription, and the adjoint gradient dJ/d(porosity, inlet
speed) (GMRES on the transposed system, and the sparse LU of the Jacobian assembled from
compressed device products) against central finite differences of re-converged flows, also
through the ``torch.autograd.Function``."""

import numpy as np
import pytest

from gputest_b200.mesh.unstructured import cartesian_mesh_2d
from gputest_b200.unstructured.case import BoundarySpec, UnstructuredCase

pytestmark = pytest.mark.gpu
GRAD_TOL = 1e-5  # relative agreement of the adjoint gradient with central differences


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _problem(nx=48, ny=12, seed=0):
    from gputest_b200.unstructured.adjoint import PorousChannel

    m = cartesian_mesh_2d(nx, ny, 4.0, 1.0, names=("in", "out", "bottom", "top"))
    case = UnstructuredCase(boundaries={"in": BoundarySpec("inlet", velocity=[1.0, 0.0]), "out": BoundarySpec("outlet"),
                                        "bottom": BoundarySpec("wall"), "top": BoundarySpec("wall")},
                            viscosity=1 / 200, scheme="upwind", tol=1e-12, max_iter=50000, algorithm="SIMPLE",
                            relax_u=0.3, relax_p=0.3)
    rng = np.random.default_rng(seed)
    por = 1e4 / (1 + np.exp(-8 * rng.standard_normal(m.n_cells)))
    return PorousChannel(m, case, "in", "out"), por


def test_vjp_kernel_equals_autograd_of_the_transcription():
    import torch

    from gputest_b200.unstructured.adjoint import DeviceAdjoint, objective_gradient

    prob, por = _problem(24, 8)
    s = prob.solve(por, 1.0)
    adj = DeviceAdjoint(s)
    _, _, _, R = objective_gradient(s, "in", "out")
    fv = s.fv
    rng = np.random.default_rng(1)
    lam = torch.as_tensor(rng.standard_normal(adj.n), device=s.torch_device)
    out, opor, oub = adj.vjp(lam, theta=True)
    # the same products by autograd, reference numbering
    lm, lc, lg, lF, lFb = adj.split(lam)
    lam_ref = R.pack(torch.as_tensor(fv.cells_to_host(lm)), torch.as_tensor(fv.cells_to_host(lc)),
                     torch.as_tensor(fv.cells_to_host(lg)), torch.as_tensor(fv.faces_to_host(lF)),
                     torch.as_tensor(fv.bfaces_to_host(lFb)))
    c = s._cur
    x = R.pack(torch.as_tensor(fv.cells_to_host(s._Up[c][1:])), torch.as_tensor(fv.cells_to_host(s._Up[c][0])),
               torch.as_tensor(fv.cells_to_host(s.gpf)), torch.as_tensor(fv.faces_to_host(s._F[c][: fv.n_if])),
               torch.as_tensor(fv.bfaces_to_host(s._Fb[c][: fv.n_bf])))
    x.requires_grad_(True)
    al = torch.as_tensor(por).requires_grad_(True)
    ub = torch.as_tensor(s.ub_fixed).requires_grad_(True)
    gx, ga, gu = torch.autograd.grad(R.residual(x, al, ub), (x, al, ub), lam_ref)
    oU, op, og, oF, oFb = adj.split(out)
    mine = R.pack(torch.as_tensor(fv.cells_to_host(oU)), torch.as_tensor(fv.cells_to_host(op)),
                  torch.as_tensor(fv.cells_to_host(og)), torch.as_tensor(fv.faces_to_host(oF)),
                  torch.as_tensor(fv.bfaces_to_host(oFb)))
    for a, b in zip(R.split(mine), R.split(gx)):
        assert float((a - b).abs().max()) <= 1e-11 * max(float(b.abs().max()), 1.0)
    assert np.allclose(fv.cells_to_host(opor), ga.numpy(), rtol=1e-11, atol=1e-13 * float(ga.abs().max()))
    assert np.allclose(fv.bfaces_to_host(oub[:, : fv.n_bf]), gu.numpy(), rtol=1e-11, atol=1e-13)


@pytest.mark.parametrize("method", ["direct", "gmres"])
def test_adjoint_gradient_matches_central_differences(method):
    prob, por = _problem()
    prob.solve(por, 1.0)
    J0, d_por, d_uin, info = prob.gradient(method=method)
    assert info["method"] == method and info["residual"] < 1e-10
    h = 1e-6
    rng = np.random.default_rng(7)
    for _ in range(3):
        d = rng.standard_normal(por.size) * por
        d /= np.abs(d / por).max()
        prob.solve(por + h * d, 1.0)
        Jp = prob.J()
        prob.solve(por - h * d, 1.0)
        Jm = prob.J()
        fd = (Jp - Jm) / (2 * h)
        assert float(d_por @ d) == pytest.approx(fd, rel=GRAD_TOL)
    prob.solve(por, 1.0 + h)
    Jp = prob.J()
    prob.solve(por, 1.0 - h)
    Jm = prob.J()
    assert d_uin == pytest.approx((Jp - Jm) / (2 * h), rel=GRAD_TOL)


def test_autograd_function_returns_the_adjoint_gradient():
    import torch

    from gputest_b200.unstructured.adjoint import porous_objective

    prob, por = _problem(32, 8)
    f = porous_objective(prob)
    a = torch.as_tensor(por).requires_grad_(True)
    u = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    J = f(a, u)
    J.backward()
    J2, d_por, d_uin, _ = prob.gradient()
    assert float(J) == pytest.approx(J2, rel=1e-12)
    assert np.allclose(a.grad.numpy(), d_por, rtol=1e-6, atol=1e-9 * np.abs(d_por).max())
    assert float(u.grad) == pytest.approx(d_uin, rel=1e-6)


def test_device_jacobian_reproduces_the_vjp_kernel():
    """The Jacobian assembled from compressed device products, transposed and applied to random
    vectors, equals the CUDA VJP itself (no two rows of one seed share an unknown)."""
    import torch

    from gputest_b200.unstructured.adjoint import DeviceAdjoint, device_jacobian

    prob, por = _problem(24, 8)
    adj = DeviceAdjoint(prob.solve(por, 1.0))
    J = device_jacobian(adj)
    rng = np.random.default_rng(3)
    for _ in range(3):
        lam = rng.standard_normal(adj.n)
        ref = adj.vjp(torch.as_tensor(lam, device=adj.U.device)).cpu().numpy()
        assert np.abs(J.T @ lam - ref).max() <= 1e-11 * np.abs(ref).max()
