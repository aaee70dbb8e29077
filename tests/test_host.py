"""Host-side logic on CPU: the C ABI library loads and exports what the header declares, the
device layout maps back to the reference's numbering, the AMG host set-up reproduces the
reference's hierarchy, and the case objects validate like the reference's."""

import os
import re

import numpy as np
import pytest

from gputest_b200.mesh.unstructured import box_mesh_3d, cartesian_mesh_2d, compute_geometry, extrude_to_3d
from gputest_b200.unstructured.case import BoundarySpec, UnstructuredCase, default_boundaries

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_loads_and_exports_every_declared_symbol():
    from gputest_b200 import _lib

    L = _lib.lib()
    assert L.b2s_abi_version() == _lib.ABI_VERSION
    header = open(os.path.join(ROOT, "include", "b2simplec.h")).read()
    declared = re.findall(r"^B2S_API\s+\w+\s+(b2s_\w+)\s*\(", header, flags=re.M)
    assert len(declared) >= 20
    for name in declared:
        assert hasattr(L, name), name
        assert name in _lib._SIGS, f"{name} is declared in the header but not bound"


def test_host_aggregation_is_the_reference_greedy_algorithm():
    import scipy.sparse as sp

    from gputest_b200.linalg.amg import aggregate, strength
    from oracle.simplec_oracle import _aggregate_py

    rng = np.random.default_rng(4)
    A = sp.random(300, 300, density=0.02, random_state=5, format="csr")
    A = A + A.T + sp.eye(300) * 5
    S = strength(A.tocsr(), 0.08)
    a1, n1 = aggregate(S)
    a2, n2 = _aggregate_py(S.indptr, S.indices, 300)
    assert n1 == n2 and np.array_equal(a1, a2)
    assert rng is not None


@pytest.mark.parametrize("mesh", [cartesian_mesh_2d(20, 16, triangulate=True, warp=0.05),
                                  cartesian_mesh_2d(30, 20, triangulate="alternating", jitter=0.2),
                                  box_mesh_3d(6, 5, 4, 4, 1, 1, jitter=0.1, seed=1),
                                  extrude_to_3d(cartesian_mesh_2d(6, 5, warp=0.05), 4, 0.5)],
                         ids=["tri", "alt", "box", "extruded"])
def test_device_layout_maps_back_to_the_reference_numbering(mesh):
    from gputest_b200.unstructured.fvmesh import FVMesh
    from oracle.simplec_oracle import OracleFV

    fv = FVMesh(mesh, device="cpu")
    o = OracleFV(mesh)
    t = {k: v.numpy() for k, v in fv.t.items()}
    perm, nc = fv.perm, fv.nc
    assert np.array_equal(perm[t["fP"]], o.P[fv.face_ref]) and np.array_equal(perm[t["fN"]], o.N[fv.face_ref])
    assert np.array_equal(perm[t["bP"]], o.Pb[fv.bface_ref])
    assert np.array_equal(np.diff(t["own_ptr"]), np.bincount(t["fP"], minlength=nc))
    assert np.all(t["fP"][np.repeat(np.arange(fv.n_if), 1)] == np.repeat(np.arange(nc), np.diff(t["own_ptr"])))
    assert np.array_equal(t["fN"][t["nei_face"]], np.repeat(np.arange(nc), np.diff(t["nei_ptr"])))
    rows = np.repeat(np.arange(nc), np.diff(t["rowptr"]))
    assert np.array_equal(rows[t["slot_PN"]], t["fP"]) and np.array_equal(t["col"][t["slot_PN"]], t["fN"])
    assert np.array_equal(rows[t["slot_NP"]], t["fN"]) and np.array_equal(t["col"][t["slot_NP"]], t["fP"])
    assert np.array_equal(t["col"][t["slot_diag"]], np.arange(nc))
    # every device CSR row holds its reference row's columns in the reference's order
    ref_cols = [o.indices[o.indptr[perm[c]]:o.indptr[perm[c] + 1]] for c in range(nc)]
    dev_cols = [perm[t["col"][t["rowptr"][c]:t["rowptr"][c + 1]]] for c in range(nc)]
    assert all(np.array_equal(a, b) for a, b in zip(ref_cols, dev_cols))
    assert np.array_equal(t["S"].T, o.S[fv.face_ref])
    assert np.array_equal(t["Ginv"].T.reshape(nc, fv.dim, fv.dim), o.Ginv[perm])
    # matrix_to_host inverts the slot permutation exactly
    vals = np.arange(fv.nnz, dtype=np.float64)
    import torch

    A = fv.matrix_to_host(torch.as_tensor(vals))
    assert np.array_equal(A.indptr, o.indptr) and np.array_equal(A.indices, o.indices)
    assert np.array_equal(A.data[fv.slot_ref], vals)
    # reverse Cuthill-McKee does not widen the cell bandwidth
    assert np.abs(t["fP"] - t["fN"]).max() <= np.abs(o.P - o.N).max()


def test_amg_host_setup_reproduces_the_reference_hierarchy():
    import torch

    from gputest_b200.linalg.amg import AMGHierarchy
    from gputest_b200.unstructured.fvmesh import FVMesh
    from oracle.simplec_oracle import OracleSimple, SmoothedAggregationAMG

    mesh = cartesian_mesh_2d(48, 48, triangulate="alternating", jitter=0.2)
    case = UnstructuredCase(boundaries={"top": BoundarySpec("wall", velocity=[1.0, 0.0])}, viscosity=0.01)
    o = OracleSimple(mesh, case)
    for _ in range(3):
        o.step()
    Ap = o._capture["Ap"]
    fv = FVMesh(mesh, device="cpu")
    h = AMGHierarchy(Ap, fv.perm, fv.rowptr, fv.col, fv.t["slot_diag"], torch.as_tensor(Ap.data[fv.slot_ref]),
                     fv.slot_ref, singular=True, max_coarse=300)
    ref = SmoothedAggregationAMG(Ap, singular=True)
    assert h.sizes == [lv[0].shape[0] for lv in ref.levels] + [ref.coarse_inv.shape[0]]
    agg0 = h._keep[0]["agg"].numpy()
    assert np.array_equal(agg0, ref.aggregates[0][fv.perm])  # device rows carry the reference aggregates


def test_generated_meshes_are_valid():
    for m, vol in ((cartesian_mesh_2d(16, 12, triangulate="alternating", jitter=0.2), 1.0),
                   (box_mesh_3d(8, 4, 4, 4.0, 1.0, 1.0, jitter=0.1, seed=1), 4.0)):
        g = compute_geometry(m)
        assert g.flipped_faces == 0 and np.all(g.cell_volume > 0)
        assert g.total_volume == pytest.approx(vol, rel=1e-12)
    alt = cartesian_mesh_2d(4, 4, triangulate="alternating")
    assert alt.n_cells == 32 and int((alt.neighbour >= 0).sum()) == 16 + 12 + 12


def test_case_validation_matches_the_reference():
    with pytest.raises(ValueError):
        BoundarySpec(kind="nonsense")
    with pytest.raises(ValueError):
        UnstructuredCase(algorithm="PISO")
    assert UnstructuredCase(algorithm="simple").relax_p == 0.3
    with pytest.raises(ValueError):
        UnstructuredCase(radiation="p1")
    m = cartesian_mesh_2d(7, 3, 4.0, 1.0, names=("inlet", "outlet", "bottom", "top"),
                          types=("velocity-inlet", "pressure-outlet", "wall", "wall"))
    b = default_boundaries(m)
    assert b["inlet"].kind == "inlet" and b["inlet"].normal_speed == 1.0 and b["outlet"].kind == "outlet"


def test_solver_refuses_unsupported_models_without_a_device():
    from gputest_b200.unstructured.simple import _check_scope

    with pytest.raises(NotImplementedError):
        _check_scope(UnstructuredCase(turbulence="k-omega-sst"))
    with pytest.raises(NotImplementedError):
        _check_scope(UnstructuredCase(unsteady=True))
    _check_scope(UnstructuredCase())


def test_product_path_raises_without_a_cuda_device():
    import torch

    from gputest_b200 import _lib

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    with pytest.raises(RuntimeError, match="CUDA device"):
        _lib.require_device()


def test_union_mesh_keeps_every_case_and_its_geometry():
    """The disjoint union of a batch: each case's cells contiguous (reference and device order),
    zones renamed per case, geometry identical to the case's own."""
    from gputest_b200.mesh.unstructured import cartesian_mesh_2d, compute_geometry, union_groups, union_mesh
    from gputest_b200.unstructured.fvmesh import FVMesh

    meshes = [cartesian_mesh_2d(5, 4, jitter=0.1, seed=1),
              cartesian_mesh_2d(8, 3, 4.0, 1.0, names=("in", "out", "bottom", "top"), jitter=0.1, seed=2),
              cartesian_mesh_2d(3, 3, triangulate=True)]
    u = union_mesh(meshes)
    g = union_groups(meshes)
    assert u.n_cells == sum(m.n_cells for m in meshes)
    gu = compute_geometry(u)
    off = 0
    for i, m in enumerate(meshes):
        gm = compute_geometry(m)
        assert np.allclose(gu.cell_volume[off:off + m.n_cells], gm.cell_volume, rtol=0, atol=1e-15)
        assert np.allclose(gu.cell_centre[off:off + m.n_cells], gm.cell_centre, rtol=0, atol=1e-15)
        for z in m.boundary_zones():
            zu = u.zone_by_name(f"c{i}/{z.name}")
            assert zu is not None and zu.count == z.count and zu.type == z.type
        off += m.n_cells
    fv = FVMesh(u, device="cpu", groups=g)
    gd = g[fv.perm]
    assert np.all(np.diff(gd) >= 0)
    # no interior face joins two cases
    assert np.all(g[fv.host.P] == g[fv.host.N])


def test_amg_term_lists_reproduce_the_row_owned_products_bit_for_bit():
    """The term lists of P, W = A P and A_c = R W (``linalg.amg.term_lists``), summed slot by
    slot in list order, equal the row-owned products of the rebuild kernels (pvals_k, wvals_k,
    acvals_k, restated here as loops) exactly, on a random pattern with unsorted stored rows."""
    import scipy.sparse as sp

    from gputest_b200.linalg.amg import _pattern, term_lists

    rng = np.random.default_rng(4)
    n, na = 80, 17
    M = sp.random(n, n, density=0.06, random_state=5) + sp.eye(n)
    M = sp.csr_matrix(M + M.T)
    rp, cl = M.indptr.astype(np.int64), M.indices.astype(np.int64).copy()
    for i in range(n):  # stored order within rows need not be sorted
        seg = cl[rp[i]:rp[i + 1]]
        cl[rp[i]:rp[i + 1]] = seg[rng.permutation(seg.size)]
    agg = rng.integers(0, na, n)
    agg[:na] = np.arange(na)
    Apat = sp.csr_matrix((np.ones(cl.size), cl, rp), shape=(n, n))
    T = sp.csr_matrix((np.ones(n), (np.arange(n), agg)), shape=(n, na))
    Pp = _pattern(_pattern(Apat) @ T)
    Wp = _pattern(_pattern(Apat) @ Pp)
    Cp = _pattern(Pp.T.tocsr() @ Wp)
    prow = np.repeat(np.arange(n), np.diff(Pp.indptr))
    order = np.lexsort((prow, Pp.indices))
    r_col = prow[order]
    r_rowptr = np.concatenate([[0], np.cumsum(np.bincount(Pp.indices, minlength=na))])
    a, dinv, tval = rng.standard_normal(cl.size), 1 / (1 + rng.random(n)), 1 / np.sqrt(1 + rng.random(na))
    c = 4.0 / 3.0 / 1.7
    # row-owned products in the kernels' order
    p = np.zeros(Pp.nnz)
    for i in range(n):
        p0, p1 = Pp.indptr[i], Pp.indptr[i + 1]
        for j in range(rp[i], rp[i + 1]):
            J = agg[cl[j]]
            s = p0 + int(np.searchsorted(Pp.indices[p0:p1], J))
            p[s] += (dinv[i] * a[j]) * tval[J]
        for s in range(p0, p1):
            J = Pp.indices[s]
            p[s] = (tval[J] if J == agg[i] else 0.0) - c * p[s]
    w = np.zeros(Wp.nnz)
    for i in range(n):
        w0, w1 = Wp.indptr[i], Wp.indptr[i + 1]
        for j in range(rp[i], rp[i + 1]):
            k = cl[j]
            for e in range(Pp.indptr[k], Pp.indptr[k + 1]):
                s = w0 + int(np.searchsorted(Wp.indices[w0:w1], Pp.indices[e]))
                w[s] += a[j] * p[e]
    r = p[order]
    ac = np.zeros(Cp.nnz)
    for I in range(na):
        c0, c1 = Cp.indptr[I], Cp.indptr[I + 1]
        for q in range(r_rowptr[I], r_rowptr[I + 1]):
            i = r_col[q]
            for s in range(Wp.indptr[i], Wp.indptr[i + 1]):
                t = c0 + int(np.searchsorted(Cp.indices[c0:c1], Wp.indices[s]))
                ac[t] += r[q] * w[s]
    # the same from the term lists
    tl = {k: v.numpy() for k, v in term_lists(rp, cl, agg, na, Pp, Wp, Cp, r_col, r_rowptr).items()}
    p2 = np.empty(Pp.nnz)
    for i in range(n):
        for s in range(Pp.indptr[i], Pp.indptr[i + 1]):
            J = Pp.indices[s]
            acc = 0.0
            for t in range(tl["p_tptr"][s], tl["p_tptr"][s + 1]):
                acc += (dinv[i] * a[tl["p_tj"][t]]) * tval[J]
            p2[s] = (tval[J] if J == agg[i] else 0.0) - c * acc
    w2 = np.array([sum((a[tl["w_tj"][t]] * p2[tl["w_te"][t]] for t in range(tl["w_tptr"][s], tl["w_tptr"][s + 1])),
                       0.0) for s in range(Wp.nnz)])
    ac2 = np.array([sum((r[tl["c_te"][t]] * w2[tl["c_ts"][t]] for t in range(tl["c_tptr"][s], tl["c_tptr"][s + 1])),
                        0.0) for s in range(Cp.nnz)])
    assert np.array_equal(p, p2) and np.array_equal(w, w2) and np.array_equal(ac, ac2)
    assert tl["c_tptr"][-1] == sum(np.diff(Wp.indptr)[r_col])


def test_ctypes_structs_match_the_c_header_layout(tmp_path):
    """Every struct of ``include/b2simplec.h`` and its ctypes mirror in ``gputest_b200/_lib.py``
    have the same size and the same offset for every field (compiled with gcc against the header)."""
    import ctypes
    import shutil
    import subprocess

    from gputest_b200 import _lib

    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("gcc not available")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    pairs = {"b2s_mesh": _lib.Mesh, "b2s_bc": _lib.BC, "b2s_flow_params": _lib.FlowParams,
             "b2s_solve_info": _lib.SolveInfo, "b2s_amg_level": _lib.AmgLevel, "b2s_amg": _lib.Amg,
             "b2s_amg_f32": _lib.Amg32, "b2s_team_config": _lib.TeamConfig, "b2s_sst": _lib.SST}
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "b2simplec.h"', "int main(void) {"]
    for cname, py in pairs.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("  return 0;\n}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([gcc, "-std=c11", "-I", os.path.join(root, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l}
    for cname, py in pairs.items():
        assert got[(cname, "size")] == ctypes.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)


def test_extract_cells_equals_the_reference_and_orients_the_interfaces():
    """``extract_cells`` (the fluid part of a conjugate mesh) against digests of the reference's
    own ``extract_cells`` (``tests/golden/extract_digests.json``): sub-mesh arrays, zones, face
    and cell maps; the interface faces point out of the kept cells and the kept volume is the
    fluid volume."""
    import json

    from gputest_b200.mesh.unstructured import compute_geometry, extract_cells
    from tests.golden.mesh_cases import extract_digest, zoned_meshes

    ref = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "extract_digests.json")))
    for key, (m, keep) in zoned_meshes().items():
        sub, fmap, cmap = extract_cells(m, keep)
        assert extract_digest(sub, fmap, cmap) == ref[key], key
        g, g0 = compute_geometry(sub), compute_geometry(m)
        assert g.flipped_faces == 0
        assert np.isclose(g.cell_volume.sum(), g0.cell_volume[keep].sum(), rtol=1e-13)
        iface = [z for z in sub.boundary_zones() if z.name.startswith("interface-")]
        assert len(iface) == 1 and iface[0].count > 0


def test_host_geometry_errors_and_orientation_repair():
    """The library's host geometry (``b2s_host_geometry``): a turned face is turned back and
    counted, a face with a node count the dimension does not allow and a cell of non-positive
    volume raise, as the reference's ``compute_geometry`` does."""
    import copy

    import pytest as _pytest

    from gputest_b200.mesh.unstructured import face_centres_and_areas

    m = cartesian_mesh_2d(6, 5, triangulate=True, warp=0.05)
    g0 = compute_geometry(m)
    # reverse the node order of three faces: their area vectors flip and the repair restores them
    m2 = copy.deepcopy(m)
    for f in (0, 7, 20):
        a, b = m2.face_ptr[f], m2.face_ptr[f + 1]
        m2.face_nodes[a:b] = m2.face_nodes[a:b][::-1].copy()
    g2 = compute_geometry(m2)
    assert g2.flipped_faces == g0.flipped_faces + 3
    np.testing.assert_array_equal(g2.face_area_vec, g0.face_area_vec)
    np.testing.assert_array_equal(g2.cell_volume, g0.cell_volume)
    fc, S = face_centres_and_areas(m)
    np.testing.assert_array_equal(fc, g0.face_centre)
    # a 2-D mesh whose first face lists three nodes
    m3 = copy.deepcopy(m)
    m3.face_ptr = m3.face_ptr.copy()
    m3.face_nodes = np.insert(m3.face_nodes, 2, m3.face_nodes[0])
    m3.face_ptr[1:] += 1
    with _pytest.raises(ValueError, match="2-node faces"):
        compute_geometry(m3)
    # without the repair, a turned boundary face gives a cell of non-positive volume
    m4 = cartesian_mesh_2d(1, 1)
    for f in range(m4.n_faces):
        a, b = m4.face_ptr[f], m4.face_ptr[f + 1]
        m4.face_nodes[a:b] = m4.face_nodes[a:b][::-1].copy()
    with _pytest.raises(ValueError, match="non-positive volume"):
        compute_geometry(m4, repair=False)
