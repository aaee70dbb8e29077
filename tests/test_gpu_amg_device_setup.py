"""The device AMG set-up on a B200 against the host set-up (the reference's algorithm,
``flowtrace/linalg/amg.py:25-117``): strength flags, the greedy aggregation in the reference's
visiting order (``b2s_amg_aggregate_d``), whole hierarchies (aggregates, patterns, V-cycle bit
for bit) and the solver re-aggregating on the device against the host set-up."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


@pytest.fixture(params=[2048, 0], ids=["warp-rows", "thread-rows"])
def warp_cols(request):
    """The pattern builders' warp-per-row threshold for one test (2048: the default, coarse levels
    one warp per row; 0: one thread per row on every level), restored afterwards."""
    from gputest_b200 import _lib

    L = _lib.lib()
    prev = L.b2s_amg_pattern_warp_cols(request.param)
    yield request.param
    L.b2s_amg_pattern_warp_cols(prev)


def _device_csr(A, rng):
    """A's rows on the device with each row's entries shuffled (the device code may not rely on
    sorted columns), plus the diagonal slots."""
    import torch

    n = A.shape[0]
    rp = A.indptr.astype(np.int64)
    src = np.concatenate([rp[i] + rng.permutation(rp[i + 1] - rp[i]) for i in range(n)])
    cl = A.indices[src].astype(np.int64)
    rows = np.repeat(np.arange(n), np.diff(rp))
    diag = np.flatnonzero(cl == rows)
    assert diag.size == n
    t = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device="cuda")  # noqa: E731
    return (t(rp, torch.int32), t(cl, torch.int32), t(A.data[src], torch.float64), t(diag, torch.int32), src)


@pytest.mark.parametrize("kind,seed,theta,order,n", [
    ("grid", 1, 0.08, "identity", 400), ("grid", 2, 0.25, "random", 2500), ("random", 4, 0.08, "random", 3000),
    ("random", 6, 0.0, "random", 3000), ("grid", 9, 0.08, "random", 131044), ("grid", 10, 0.08, "identity", 262144),
])
def test_device_aggregation_equals_the_host_greedy(kind, seed, theta, order, n):
    import torch

    from gputest_b200.linalg import amg
    from tests.test_amg_device_setup import _graph, _greedy_in_priority_order

    A = _graph(seed, n, kind)
    n = A.shape[0]
    rng = np.random.default_rng(seed)
    rp, cl, val, diag, src = _device_csr(A, rng)
    strong = amg.device_strength(rp, cl, val, diag, theta)
    want_strong = amg.strong_mask(A, theta)[src]
    np.testing.assert_array_equal(strong.cpu().numpy().astype(bool), want_strong)
    tslot, missing = amg.device_transpose_slots(rp, cl, False)
    assert int(missing.item()) == 0
    prio = np.arange(n) if order == "identity" else rng.permutation(n)
    rank = np.argsort(prio)
    pr = torch.as_tensor(prio, dtype=torch.int32, device="cuda")
    rk = torch.as_tensor(rank, dtype=torch.int32, device="cuda")
    agg, counts, info = amg.device_aggregate(rp, cl, strong, tslot, pr, rk)
    info = info.cpu().numpy()
    assert info[1] == 0
    want, na = _greedy_in_priority_order(A.indptr.astype(np.int64), A.indices.astype(np.int64),
                                         amg.strong_mask(A, theta).astype(np.uint8), prio)
    assert info[0] == na
    np.testing.assert_array_equal(agg.cpu().numpy(), want)
    np.testing.assert_array_equal(counts.cpu().numpy()[:na], np.bincount(want, minlength=na))


def _pressure_system(mesh_fn, iterations=3):
    from gputest_b200.unstructured.case import BoundarySpec, UnstructuredCase
    from gputest_b200.unstructured.simple import SimpleSolver

    mesh = mesh_fn()
    case = UnstructuredCase(boundaries={"top": BoundarySpec("wall", velocity=[1.0, 0.0])}, viscosity=0.01,
                            max_iter=1000, tol=0.0)
    s = SimpleSolver(mesh, case, max_coarse=300)
    for _ in range(iterations):
        s.step()
    return s


def _meshes():
    from gputest_b200.mesh.unstructured import cartesian_mesh_2d

    return [lambda: cartesian_mesh_2d(48, 40, triangulate=True, warp=0.08),
            lambda: cartesian_mesh_2d(96, 96)]


@pytest.mark.parametrize("which", [0, 1])
@pytest.mark.parametrize("theta", [0.08, 0.0])
def test_device_hierarchy_equals_the_host_hierarchy(which, theta, warp_cols):
    """Both set-ups from the same pressure-correction matrix: the same levels, aggregates,
    patterns and strong flags, and the same V-cycle bit for bit; with the products' patterns
    built one warp per row on the levels of at most 2048 aggregates, or one thread per row on
    every level."""
    import torch

    from gputest_b200.linalg.amg import AMGHierarchy

    s = _pressure_system(_meshes()[which])
    fv = s.fv
    A_host = fv.matrix_to_host(s.val_P)
    host = AMGHierarchy(A_host, fv.perm, fv.rowptr, fv.col, fv.t["slot_diag"], s.val_P, fv.slot_ref,
                        singular=s.singular_p, max_coarse=300, theta=theta)
    host.rebuild()
    dev = AMGHierarchy.on_device(torch.as_tensor(fv.perm, device="cuda"), fv.rowptr, fv.col, fv.t["slot_diag"],
                                 s.val_P, singular=s.singular_p, max_coarse=300, theta=theta)
    assert dev.n_levels == host.n_levels >= 3 and dev.sizes == host.sizes
    for l in range(host.n_levels - 1):
        kh, kd = host._keep[2 * l], dev._keep[2 * l]
        for k in ("agg", "tval", "x0", "p_rowptr", "p_col", "r_rowptr", "r_col", "r_from_p", "w_rowptr", "w_col",
                  "strong", "p_tptr", "p_tj", "w_tptr", "w_tj", "w_te", "c_tptr", "c_te", "c_ts"):
            assert torch.equal(kh[k], kd[k].to(kh[k].dtype)), (l, k)
        for k in ("p_val", "w_val", "dinv", "rho"):
            assert torch.equal(kh[k], kd[k]), (l, k)
    assert torch.equal(host.coarse_val, dev.coarse_val) and torch.equal(host.coarse_inv, dev.coarse_inv)
    b = torch.randn(fv.rowptr.numel() - 1, dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(5))
    assert torch.equal(host.vcycle(b), dev.vcycle(b))


def test_solver_reaggregating_on_the_device_equals_the_host_set_up():
    """reaggregate=True with the device set-up against the same solver with the host set-up:
    the same set-up count and the same fields bit for bit after 60 iterations."""
    from gputest_b200.mesh.unstructured import cartesian_mesh_2d
    from gputest_b200.unstructured.case import BoundarySpec, UnstructuredCase
    from gputest_b200.unstructured.simple import SimpleSolver

    mesh = cartesian_mesh_2d(40, 40, triangulate=True, warp=0.1)
    case = UnstructuredCase(boundaries={"top": BoundarySpec("wall", velocity=[1.0, 0.0])}, viscosity=0.005,
                            max_iter=1000, tol=0.0)
    out = []
    for host in (True, False):
        s = SimpleSolver(mesh, case, max_coarse=300)
        s.reaggregate = True
        s.host_amg_setup = host
        for _ in range(60):
            s.step()
        out.append((s.amg_setups, s.fields()))
    assert out[0][0] == out[1][0] >= 2
    for k in ("x-velocity", "y-velocity", "pressure"):
        np.testing.assert_array_equal(out[0][1][k], out[1][1][k])


def test_partial_reaggregation_equals_a_full_device_set_up():
    """With reaggregate on, a re-aggregation resumes at the first level whose strength graph
    changed and shares the levels above it: at every re-aggregation the solver's hierarchy equals
    a full device set-up from the same matrix (levels, aggregates, patterns, V-cycle bit for bit),
    and some of them did start below level 0."""
    import torch

    from gputest_b200.linalg.amg import AMGHierarchy
    from gputest_b200.mesh.unstructured import cartesian_mesh_2d
    from gputest_b200.unstructured.case import BoundarySpec, UnstructuredCase
    from gputest_b200.unstructured.simple import SimpleSolver

    mesh = cartesian_mesh_2d(64, 64, triangulate=True, warp=0.1)
    case = UnstructuredCase(boundaries={"top": BoundarySpec("wall", velocity=[1.0, 0.0])}, viscosity=0.002,
                            max_iter=1000, tol=0.0)
    s = SimpleSolver(mesh, case, max_coarse=150)
    s.reaggregate = True
    starts = []
    orig = s._setup_amg

    def spy(start=0):
        starts.append(start)
        orig(start)

    s._setup_amg = spy
    b = torch.randn(mesh.n_cells, dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(3))
    checked = 0
    for _ in range(120):
        n0 = len(starts)
        s.step()
        if len(starts) == n0 or starts[-1] == 0:
            continue
        got = s._amg
        full = AMGHierarchy.on_device(torch.as_tensor(s.fv.perm, device="cuda"), s.fv.rowptr, s.fv.col,
                                      s.fv.t["slot_diag"], s.val_P, singular=s.singular_p, max_coarse=150,
                                      theta=s.amg_theta)
        assert got.sizes == full.sizes
        for l in range(full.n_levels - 1):
            for k in ("agg", "p_col", "w_col", "c_ts", "strong", "p_val", "w_val"):
                assert torch.equal(got._keep[2 * l][k], full._keep[2 * l][k]), (l, k)
        assert torch.equal(got.coarse_inv, full.coarse_inv)
        assert torch.equal(got.vcycle(b), full.vcycle(b))
        checked += 1
    assert checked >= 2


@pytest.mark.parametrize("kind,n,seed", [("grid", 2500, 11), ("grid", 10000, 14), ("random", 3000, 12)])
def test_row_product_kernels_equal_the_key_based_patterns(kind, n, seed, warp_cols):
    """``row_products`` (P, W, R = P^T and A_c by the per-row kernels) against the sorted-key
    construction of ``product_patterns`` on the same level and aggregates, one warp per row and
    one thread per row: every pattern and term list equal, the diagonal slots and the next
    level's conflict bound from the same pattern. One thread per row handles at most 64 distinct
    P columns, 128 distinct W columns and 128 distinct A_c columns a row (a warp has no such
    limit); where an A_c row does not fit (the random graph: up to 550 columns) P and W come back
    alone and the sorted keys complete them; where a P row does not fit the level is handed back
    (None)."""
    import scipy.sparse as sp
    import torch

    from gputest_b200.linalg import amg
    from tests.test_amg_device_setup import _graph

    A = _graph(seed, n, kind)
    n = A.shape[0]
    rng = np.random.default_rng(seed)
    rp, cl, val, diag, _ = _device_csr(A, rng)
    S = amg.strength(A, 0.08)
    agg_h, na = amg.aggregate(S)
    T = sp.csr_matrix((np.ones(n), (np.arange(n), agg_h)), shape=(n, na))
    Pp = amg._pattern(amg._pattern(A) @ T)
    Wp = amg._pattern(amg._pattern(A) @ Pp)
    Cp = amg._pattern(Pp.T @ Wp)
    by_warp = na <= warp_cols
    assert na <= 2048
    pw_fits = by_warp or (int(np.diff(Pp.indptr).max()) <= 64 and int(np.diff(Wp.indptr).max()) <= 128)
    rc_fits = int(np.bincount(Pp.indices, minlength=na).max()) <= 256 and (
        by_warp or int(np.diff(Cp.indptr).max()) <= 128)
    assert pw_fits and rc_fits == (by_warp or kind == "grid")
    agg = torch.as_tensor(agg_h, dtype=torch.int32, device="cuda")
    pw = amg.row_products(rp, cl, agg, na)
    assert pw is not None and pw["complete"] == rc_fits
    ref = amg.product_patterns(rp.long(), cl.long(), agg.long(), na)
    got = pw if rc_fits else amg.product_patterns(rp.long(), cl.long(), agg.long(), na, pw=pw)
    for k in ("p_ptr", "p_idx", "w_ptr", "w_idx", "r_rowptr", "r_col", "r_from_p", "c_ptr", "c_idx"):
        assert torch.equal(got[k].long(), ref[k]), k
    for k in ("p_tptr", "p_tj", "w_tptr", "w_tj", "w_te", "c_tptr", "c_te", "c_ts"):
        assert torch.equal(got[k], ref[k]), k
    if rc_fits:
        assert int(pw["check"].item()) == 0
        ar = torch.arange(na, device="cuda")
        assert torch.equal(pw["c_diag"].long(), torch.searchsorted(ref["c_keys"], ar * na + ar))
        cl_len = ref["c_ptr"][1:] - ref["c_ptr"][:-1]
        assert pw["conflicts"] == ref["c_idx"].numel() + int((cl_len * cl_len).sum())
    # a star of 70 nodes, each its own aggregate: the centre's P row has 70 distinct columns,
    # over one thread's 64 (the level is handed back), within a warp's reach
    star = sp.csr_matrix((np.ones(138), (np.r_[np.zeros(69, int), np.arange(1, 70)],
                                         np.r_[np.arange(1, 70), np.zeros(69, int)])), shape=(70, 70)) + sp.eye(70)
    star = sp.csr_matrix(star)
    star.sort_indices()
    rp2, cl2, _, _, _ = _device_csr(star, rng)
    agg2 = torch.arange(70, dtype=torch.int32, device="cuda")
    got = amg.row_products(rp2, cl2, agg2, 70)
    if by_warp:
        ref = amg.product_patterns(rp2.long(), cl2.long(), agg2.long(), 70)
        assert got["complete"] and all(torch.equal(got[k].long(), ref[k].long()) for k in ("p_idx", "w_idx", "c_idx", "c_ts"))
    else:
        assert got is None


@pytest.mark.parametrize("m", [300, 256])
def test_row_products_hand_r_and_a_c_back_where_a_row_does_not_fit(m, warp_cols):
    """A path of m nodes whose even nodes form aggregate 0 and whose odd nodes are singletons:
    P and W fit every kernel, but R's row 0 holds every node (over 256 entries for m = 300), or
    A_c's row 0 every aggregate of the path (129 distinct columns for m = 256: over one thread's
    128, within a warp's reach). Where a row does not fit, P and W come back with ``complete``
    False and ``product_patterns`` completes them; either way the level equals the key-based
    one."""
    import scipy.sparse as sp
    import torch

    from gputest_b200.linalg import amg

    i = np.arange(m - 1)
    A = sp.csr_matrix((np.ones(2 * (m - 1)), (np.r_[i, i + 1], np.r_[i + 1, i])), shape=(m, m)) + sp.eye(m)
    A = sp.csr_matrix(A)
    A.sort_indices()
    agg_h = np.where(np.arange(m) % 2 == 0, 0, (np.arange(m) + 1) // 2)
    na = int(agg_h.max()) + 1
    rp, cl, _, _, _ = _device_csr(A, np.random.default_rng(m))
    agg = torch.as_tensor(agg_h, dtype=torch.int32, device="cuda")
    pw = amg.row_products(rp, cl, agg, na)
    assert pw is not None and pw["complete"] == (m == 256 and warp_cols > 0)
    got = pw if pw["complete"] else amg.product_patterns(rp.long(), cl.long(), agg.long(), na, pw=pw)
    ref = amg.product_patterns(rp.long(), cl.long(), agg.long(), na)
    for k in ("p_ptr", "p_idx", "w_ptr", "w_idx", "r_rowptr", "r_col", "r_from_p", "c_ptr", "c_idx"):
        assert torch.equal(got[k].long(), ref[k]), k
    for k in ("p_tptr", "p_tj", "w_tptr", "w_tj", "w_te", "c_tptr", "c_te", "c_ts"):
        assert torch.equal(got[k], ref[k]), k
