"""The device set-up of the finite-volume data (``FVMesh`` from the raw mesh on the GPU,
``b2s_setup.cu``) against the host set-up (``HostFV``: the reference's
``flowtrace/mesh/unstructured.py:171-261`` and ``flowtrace/unstructured/fvmesh.py:61-230``):
every device array equal bit for bit, the least-squares inverses to rounding (LU here,
LAPACK on the host), on 2-D quads, warped and alternating triangles, jittered hexahedra and an
extruded prism mesh."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _meshes():
    from gputest_b200.mesh.unstructured import box_mesh_3d, cartesian_mesh_2d, extrude_to_3d

    return {
        "quads": lambda: cartesian_mesh_2d(33, 17),
        "warped-triangles": lambda: cartesian_mesh_2d(40, 30, triangulate=True, warp=0.1),
        "alternating": lambda: cartesian_mesh_2d(64, 64, triangulate="alternating", jitter=0.2, seed=0),
        "hexahedra": lambda: box_mesh_3d(12, 8, 6, 2.0, 1.0, 1.0, jitter=0.1, seed=1),
        "prisms": lambda: extrude_to_3d(cartesian_mesh_2d(10, 8, triangulate=True, warp=0.05), 3, 0.5),
    }


@pytest.mark.parametrize("name", list(_meshes()))
def test_device_fv_set_up_equals_the_host_set_up(name):
    import torch

    from gputest_b200.unstructured.fvmesh import FVMesh

    mesh = _meshes()[name]()
    fd = FVMesh(mesh, torch.device("cuda"))
    fh = FVMesh(mesh, torch.device("cuda"), device_setup=False)
    assert fd.nnz == fh.nnz and fd.n_if == fh.n_if and fd.n_bf == fh.n_bf
    assert fd.row_terms_max == fh.row_terms_max and fd.cell_faces_max == fh.cell_faces_max
    assert fd.non_orthogonality_deg == fh.non_orthogonality_deg
    for a in ("perm", "face_ref", "bface_ref", "slot_ref"):
        np.testing.assert_array_equal(getattr(fd, a), getattr(fh, a), err_msg=a)
    np.testing.assert_array_equal(fd.bzone, fh.host.bzone)
    assert fd.flipped_faces == fh.host.geometry.flipped_faces
    assert set(fd.t) == set(fh.t)
    for k in fd.t:
        if k == "Ginv":
            continue
        assert torch.equal(fd.t[k], fh.t[k]), k
    gi_d, gi_h = fd.t["Ginv"], fh.t["Ginv"]
    scale = gi_h.abs().amax(dim=0, keepdim=True)
    assert float(((gi_d - gi_h).abs() / scale).max()) < 1e-13
    h = fh.host
    np.testing.assert_array_equal(fd._ref["xc"].cpu().numpy(), h.xc)
    np.testing.assert_array_equal(fd._ref["yb"].cpu().numpy(), h.yb)
    np.testing.assert_array_equal(fd.boundary_normals_host(), h.nb)
    vals = torch.arange(1, fd.nnz + 1, dtype=torch.float64, device="cuda")
    A, B = fd.matrix_to_host(vals), fh.matrix_to_host(vals)
    assert (A != B).nnz == 0 and np.array_equal(A.indptr, B.indptr) and np.array_equal(A.indices, B.indices)


def test_solver_with_the_device_set_up_equals_the_host_set_up():
    """The same 30 iterations from either set-up: fields equal to rounding of the inverses."""
    from gputest_b200.mesh.unstructured import cartesian_mesh_2d
    from gputest_b200.unstructured import fvmesh
    from gputest_b200.unstructured.case import BoundarySpec, UnstructuredCase
    from gputest_b200.unstructured.simple import SimpleSolver

    mesh = cartesian_mesh_2d(48, 48, triangulate=True, warp=0.08)
    case = UnstructuredCase(boundaries={"top": BoundarySpec("wall", velocity=[1.0, 0.0])}, viscosity=0.01,
                            max_iter=1000, tol=0.0, init_velocity=[0.3, -0.1])
    out = []
    orig = fvmesh.FVMesh.__init__
    for dev_setup in (True, False):
        def init(self, *a, _d=dev_setup, **k):
            k["device_setup"] = _d
            orig(self, *a, **k)

        fvmesh.FVMesh.__init__ = init
        try:
            s = SimpleSolver(mesh, case, max_coarse=300)
        finally:
            fvmesh.FVMesh.__init__ = orig
        F0 = s._F[s._cur].cpu().numpy().copy()
        for _ in range(30):
            s.step()
        out.append((F0, s.fields()))
    np.testing.assert_array_equal(out[0][0], out[1][0])
    for k in ("x-velocity", "y-velocity", "pressure"):
        a, b = out[0][1][k], out[1][1][k]
        assert np.abs(a - b).max() <= 1e-12 * max(np.abs(b).max(), 1e-300), k
