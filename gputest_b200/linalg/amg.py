"""Smoothed-aggregation AMG hierarchy for the pressure-correction solve on B200.

The set-up is the reference's (``flowtrace/linalg/amg.py:80-117``): strength of connection,
the greedy three-pass aggregation, P = (I - 4/(3 rho) D^-1 A) T, W = A P and A_c = P^T W,
level by level. ``AMGHierarchy.on_device`` does it on the device: strength flags and the
aggregation in CUDA (``b2s_amg_strength_d``, ``b2s_amg_aggregate_d``, which reproduces the
sequential greedy exactly), the patterns and term lists of the products (P, W, R and A_c one
row per thread, ``row_products``; rows too long for those kernels from sorted distinct keys,
``product_patterns``), and each level's numeric rebuild, whose Galerkin product gives the
next level's values. ``AMGHierarchy(...)`` is the same set-up on the host (SciPy, the C++ helper
``b2s_host_aggregate``); batches of independent cases use it. Afterwards every numeric quantity
is rebuilt on the device by ``rebuild()`` (``b2s_amg_rebuild_d``): D^-1, the spectral radius by
15 power iterations from the reference's start vector (``default_rng(0)``, ``amg.py:69-77``),
P, R = P^T, the Galerkin products and the inverse of the coarsest matrix. The V-cycle (2+2
damped-Jacobi sweeps, w = 0.8) runs inside the PCG kernel.

The reference re-aggregates at every rebuild. Callers choose: keep the first set-up's
aggregates (the solvers' default), or re-aggregate when ``first_strength_change()`` reports a
level whose strength graph changed, resuming the device set-up at that level
(``on_device(prev=..., start=...)``) - the reference's hierarchy at every rebuild.
``max_coarse`` defaults to 150 (the reference's 300) so that the coarsest matrix is inverted in
one block's shared memory; 300 reproduces the reference's hierarchy exactly.
"""

from __future__ import annotations

import ctypes

import numpy as np
import scipy.sparse as sp

from .. import _lib


def strength(A: sp.csr_matrix, theta: float) -> sp.csr_matrix:
    """|a_ij| >= theta sqrt(|a_ii a_jj|), i != j (``flowtrace/linalg/amg.py:60-66``)."""
    A = A.tocoo()
    d = np.abs(A.diagonal())
    mask = (A.row != A.col) & (np.abs(A.data) >= theta * np.sqrt(d[A.row] * d[A.col]))
    S = sp.csr_matrix((np.ones(int(mask.sum())), (A.row[mask], A.col[mask])), shape=A.shape)
    S.sort_indices()
    return S


def aggregate(S: sp.csr_matrix):
    """Greedy aggregation of the strength graph (``flowtrace/linalg/amg.py:25-57``), in C++."""
    n = S.shape[0]
    indptr = np.ascontiguousarray(S.indptr, dtype=np.int64)
    indices = np.ascontiguousarray(S.indices, dtype=np.int64)
    agg = np.empty(n, dtype=np.int64)
    na = _lib.lib().b2s_host_aggregate(n, indptr.ctypes.data, indices.ctypes.data, agg.ctypes.data)
    if na < 0:
        raise RuntimeError("b2s_host_aggregate failed")
    return agg, int(na)


def spectral_radius(M, iters=15, seed=0) -> float:
    """Power iteration of ``flowtrace/linalg/amg.py:69-77`` (host, set-up only)."""
    x = np.random.default_rng(seed).standard_normal(M.shape[0])
    lam = 1.0
    for _ in range(iters):
        y = M @ x
        lam = np.linalg.norm(y) / max(np.linalg.norm(x), 1e-300)
        x = y / max(np.linalg.norm(y), 1e-300)
    return lam


def strong_mask(A: sp.csr_matrix, theta: float) -> np.ndarray:
    """Per stored entry of A (CSR order): True where the connection is strong (amg.py:60-66)."""
    A = sp.csr_matrix(A)
    rows = np.repeat(np.arange(A.shape[0]), np.diff(A.indptr))
    d = np.abs(A.diagonal())
    return (rows != A.indices) & (np.abs(A.data) >= theta * np.sqrt(d[rows] * d[A.indices]))


def _pattern(M) -> sp.csr_matrix:
    M = sp.csr_matrix(M)
    M = sp.csr_matrix((np.ones(M.nnz, dtype=np.float64), M.indices, M.indptr), shape=M.shape)
    M.sum_duplicates()
    M.sort_indices()
    return M


TERM_CAP = 1 << 26  # largest term list built per product (larger products keep the row-owned kernel)


def _expand(ptr, idx):
    """For each i in idx, the positions ptr[i] .. ptr[i+1]-1, concatenated; with the index of
    the idx entry each position came from (int64 torch tensors on one device)."""
    import torch

    lens = ptr[idx + 1] - ptr[idx]
    src = torch.repeat_interleave(torch.arange(idx.numel(), device=idx.device), lens)
    start = torch.repeat_interleave(ptr[idx] - (torch.cumsum(lens, 0) - lens), lens)
    return src, start + torch.arange(src.numel(), device=idx.device)


def _slot_lists(slot, nslot):
    """Stable grouping of terms (in generation order) by output slot: (ptr, term order)."""
    import torch

    order = torch.sort(slot, stable=True).indices
    ptr = torch.zeros(nslot + 1, dtype=torch.int64, device=slot.device)
    ptr[1:] = torch.cumsum(torch.bincount(slot, minlength=nslot), 0)
    return ptr, order


def _row_keys(indptr, indices, ncols):
    """row * ncols + column of every stored entry of a CSR pattern (sorted when the pattern is)."""
    import torch

    rows = torch.repeat_interleave(torch.arange(indptr.numel() - 1, device=indptr.device), indptr[1:] - indptr[:-1])
    return rows * ncols + indices


def term_lists(rp, cl, agg, na, Pp, Wp, Cp, r_col, r_rowptr, cap=TERM_CAP, device="cpu"):
    """Term lists of P, W = A P and A_c = R W on fixed patterns (see ``b2s_amg_level``): for
    every output slot, the terms in the order the row-owned kernels add them (A entries in
    stored order; then P entries in sorted order; R entries in R order, each W row once).
    (rp, cl): the level's CSR in stored order; agg: aggregate of each row; Pp, Wp, Cp: sorted
    scipy patterns; r_col, r_rowptr: R = P^T. Computed with torch on ``device`` (sorts and
    searches on the GPU at set-up); returns a dict of int32 tensors there, or None when the W
    lists would exceed ``cap`` terms; the A_c lists are None when they would."""
    import torch

    T = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.int64), device=device)  # noqa: E731
    rp_t, cl_t, agg_t = T(rp), T(cl), T(agg)
    p_ptr, p_idx, w_ptr, w_idx = T(Pp.indptr), T(Pp.indices), T(Wp.indptr), T(Wp.indices)
    n = rp_t.numel() - 1
    rows = torch.repeat_interleave(torch.arange(n, device=device), rp_t[1:] - rp_t[:-1])
    i32 = lambda t: t.to(torch.int32).contiguous()  # noqa: E731
    out = {}
    # P: A entry j of row i -> slot (i, agg[col j])
    sp_ = torch.searchsorted(_row_keys(p_ptr, p_idx, na), rows * na + agg_t[cl_t])
    ptr, order = _slot_lists(sp_, Pp.nnz)
    out["p_tptr"], out["p_tj"] = i32(ptr), i32(order)
    # W: (A entry j, P entry e of row col j) -> slot (row j, col e)
    lens = p_ptr[cl_t + 1] - p_ptr[cl_t]
    if int(lens.sum()) > cap:
        return None
    jj, e = _expand(p_ptr, cl_t)
    sw = torch.searchsorted(_row_keys(w_ptr, w_idx, na), rows[jj] * na + p_idx[e])
    ptr, order = _slot_lists(sw, Wp.nnz)
    out["w_tptr"], out["w_tj"], out["w_te"] = i32(ptr), i32(jj[order]), i32(e[order])
    # A_c: (R entry q of coarse row I, W entry s of row r_col[q]) -> slot (I, col s)
    rc, rr = T(r_col), T(r_rowptr)
    if int((w_ptr[rc + 1] - w_ptr[rc]).sum()) > cap:
        out["c_tptr"] = out["c_te"] = out["c_ts"] = None
        return out
    qrow = torch.repeat_interleave(torch.arange(rr.numel() - 1, device=device), rr[1:] - rr[:-1])
    q, s_ = _expand(w_ptr, rc)
    sc = torch.searchsorted(_row_keys(T(Cp.indptr), T(Cp.indices), na), qrow[q] * na + w_idx[s_])
    ptr, order = _slot_lists(sc, Cp.nnz)
    out["c_tptr"], out["c_te"], out["c_ts"] = i32(ptr), i32(q[order]), i32(s_[order])
    return out


def _sorted_ptr(sorted_rows, nrows):
    """CSR offsets of nrows rows from the (ascending) row of every entry, without a host sync."""
    import torch

    return torch.searchsorted(sorted_rows, torch.arange(nrows + 1, device=sorted_rows.device))


def _unique_pattern(keys, nrows, ncols):
    """CSR pattern of the distinct row * ncols + col keys: (indptr, indices, sorted keys), int64."""
    import torch

    u = torch.unique(keys, sorted=True)
    return _sorted_ptr(u // ncols, nrows), u % ncols, u


def _grouped(slot, nslot):
    """``_slot_lists`` without a host sync: stable grouping of terms by output slot."""
    import torch

    srt = torch.sort(slot, stable=True)
    return _sorted_ptr(srt.values, nslot), srt.indices


def _expand_sized(ptr, idx, total):
    """``_expand`` with its output size known (no host sync)."""
    import torch

    lens = ptr[idx + 1] - ptr[idx]
    src = torch.repeat_interleave(torch.arange(idx.numel(), device=idx.device), lens, output_size=total)
    start = torch.repeat_interleave(ptr[idx] - (torch.cumsum(lens, 0) - lens), lens, output_size=total)
    return src, start + torch.arange(total, device=idx.device)


def _rows_of(ptr, nnz):
    import torch

    n = ptr.numel() - 1
    return torch.repeat_interleave(torch.arange(n, device=ptr.device), ptr[1:] - ptr[:-1], output_size=nnz)


def row_products(rp, cl, agg, na, stream=None):
    """Every pattern and term list of a level's products by the per-row kernels: P and W
    (``b2s_amg_p_pattern_d``, ``b2s_amg_w_pattern_d``), R = P^T (``b2s_amg_r_pattern_d``) and
    A_c = R W (``b2s_amg_c_pattern_d``); rp, cl, agg int32 device tensors, na aggregates. The
    keys of ``product_patterns`` as int32 tensors, with ``c_diag`` (the slot of each coarse
    row's diagonal) in place of ``c_keys``, ``conflicts`` (the next level's aggregation work-space
    bound: A_c's entries plus its squared row lengths) and ``check``, a device int that is
    nonzero if A_c's fill pass found its offsets inconsistent (read at the caller's next
    synchronisation). Two host synchronisations. Levels of at most ``b2s_amg_pattern_warp_cols``
    (2048) aggregates are built one warp per row, larger ones one thread per row. Where a row
    exceeds a thread's capacity (64 distinct P columns, 128 distinct W columns) the result is
    None; where an R row has over 256 entries, an A_c row built by one thread over 128 distinct
    columns, or a term list over ``TERM_CAP`` terms, it holds P and W only, with ``complete``
    False (``product_patterns`` adds R and A_c from sorted keys)."""
    import torch

    L = _lib.lib()
    sp_ = _lib.stream_ptr(stream)
    dev = cl.device
    n, nnz = rp.numel() - 1, cl.numel()
    e32 = lambda k: torch.empty(max(int(k), 1), dtype=torch.int32, device=dev)  # noqa: E731
    ov = torch.zeros(1, dtype=torch.int32, device=dev)  # P and W kernels
    ovc = torch.zeros(1, dtype=torch.int32, device=dev)  # R and A_c kernels
    ws = e32(L.b2s_scan_workspace_bytes(max(n, na)) // 4 + 1)

    def scan(counts, m):
        out = e32(m + 1)
        _lib.check(L.b2s_scan_counts_d(m, counts.data_ptr(), out.data_ptr(), ws.data_ptr(), ws.numel() * 4, sp_),
                   "b2s_scan_counts_d")
        return out

    # P: counts, offsets, then the fill into room for nnz entries (a P row has at most as many
    # entries as the A row), so the sizes are read once, together with W's
    pcnt = e32(n)
    _lib.check(L.b2s_amg_p_pattern_d(n, na, rp.data_ptr(), cl.data_ptr(), agg.data_ptr(), 0, pcnt.data_ptr(), None,
                                     0, None, None, None, nnz, ov.data_ptr(), sp_), "b2s_amg_p_pattern_d")
    p_ptr = scan(pcnt, n)
    p_idx, p_tptr, p_tj = e32(nnz), e32(nnz + 1), e32(nnz)
    _lib.check(L.b2s_amg_p_pattern_d(n, na, rp.data_ptr(), cl.data_ptr(), agg.data_ptr(), 1, None, p_ptr.data_ptr(),
                                     nnz, p_idx.data_ptr(), p_tptr.data_ptr(), p_tj.data_ptr(), nnz, ov.data_ptr(),
                                     sp_), "b2s_amg_p_pattern_d")
    wcnt, tcnt = e32(n), e32(n)
    _lib.check(L.b2s_amg_w_pattern_d(n, na, rp.data_ptr(), cl.data_ptr(), p_ptr.data_ptr(), p_idx.data_ptr(), 0,
                                     wcnt.data_ptr(), tcnt.data_ptr(), None, None, 0, 0, None, None, None, None,
                                     ov.data_ptr(), sp_), "b2s_amg_w_pattern_d")
    w_ptr, t_ptr = scan(wcnt, n), scan(tcnt, n)
    h = torch.cat([ov, p_ptr[n:], w_ptr[n:], t_ptr[n:]]).cpu()
    if int(h[0]) or int(h[3]) > TERM_CAP:
        return None
    p_nnz, w_nnz, w_terms = int(h[1]), int(h[2]), int(h[3])
    w_idx, w_tptr, w_tj, w_te = e32(w_nnz), e32(w_nnz + 1), e32(w_terms), e32(w_terms)
    _lib.check(L.b2s_amg_w_pattern_d(n, na, rp.data_ptr(), cl.data_ptr(), p_ptr.data_ptr(), p_idx.data_ptr(), 1,
                                     None, None, w_ptr.data_ptr(), t_ptr.data_ptr(), w_nnz, w_terms, w_idx.data_ptr(),
                                     w_tptr.data_ptr(), w_tj.data_ptr(), w_te.data_ptr(), ov.data_ptr(), sp_),
               "b2s_amg_w_pattern_d")
    out = {"p_ptr": p_ptr, "p_idx": p_idx[:p_nnz], "p_tptr": p_tptr[:p_nnz + 1], "p_tj": p_tj[:nnz],
           "w_ptr": w_ptr, "w_idx": w_idx[:w_nnz], "w_tptr": w_tptr[:w_nnz + 1], "w_tj": w_tj[:w_terms],
           "w_te": w_te[:w_terms], "complete": False}
    # R = P^T (no sizes to read), then A_c's counts
    r_rowptr, r_col, r_from_p = e32(na + 1), e32(p_nnz), e32(p_nnz)
    rw = e32(L.b2s_amg_r_workspace_bytes(na) // 4 + 1)
    _lib.check(L.b2s_amg_r_pattern_d(n, na, p_ptr.data_ptr(), p_idx.data_ptr(), p_nnz, r_rowptr.data_ptr(),
                                     r_col.data_ptr(), r_from_p.data_ptr(), rw.data_ptr(), rw.numel() * 4,
                                     ovc.data_ptr(), sp_), "b2s_amg_r_pattern_d")
    ccnt, ctc = e32(na), e32(na)
    _lib.check(L.b2s_amg_c_pattern_d(na, r_rowptr.data_ptr(), r_col.data_ptr(), w_ptr.data_ptr(), w_idx.data_ptr(), 0,
                                     ccnt.data_ptr(), ctc.data_ptr(), None, None, 0, 0, None, None, None, None, None,
                                     ovc.data_ptr(), sp_), "b2s_amg_c_pattern_d")
    c_ptr, ct_ptr = scan(ccnt, na), scan(ctc, na)
    sq = ccnt[:na].to(torch.int64)
    h = torch.cat([ov.to(torch.int64), ovc.to(torch.int64), c_ptr[na:].to(torch.int64),
                   ct_ptr[na:].to(torch.int64), (sq * sq).sum().view(1)]).cpu()
    if int(h[0]):
        raise RuntimeError("AMG set-up: the W pattern kernel's offsets disagree with its counts")
    if int(h[1]) or int(h[3]) > TERM_CAP:
        return out  # a row too long for the R or A_c kernel
    c_nnz, c_terms = int(h[2]), int(h[3])
    c_idx, c_diag, c_tptr, c_te, c_ts = e32(c_nnz), e32(na), e32(c_nnz + 1), e32(c_terms), e32(c_terms)
    _lib.check(L.b2s_amg_c_pattern_d(na, r_rowptr.data_ptr(), r_col.data_ptr(), w_ptr.data_ptr(), w_idx.data_ptr(), 1,
                                     None, None, c_ptr.data_ptr(), ct_ptr.data_ptr(), c_nnz, c_terms, c_idx.data_ptr(),
                                     c_diag.data_ptr(), c_tptr.data_ptr(), c_te.data_ptr(), c_ts.data_ptr(),
                                     ovc.data_ptr(), sp_), "b2s_amg_c_pattern_d")
    out.update(r_rowptr=r_rowptr, r_col=r_col[:p_nnz], r_from_p=r_from_p[:p_nnz], c_ptr=c_ptr, c_idx=c_idx[:c_nnz],
               c_diag=c_diag[:na], c_tptr=c_tptr[:c_nnz + 1], c_te=c_te[:c_terms], c_ts=c_ts[:c_terms],
               conflicts=c_nnz + int(h[4]), check=ovc, complete=True)
    return out


def product_patterns(rp, cl, agg, na, cap=TERM_CAP, pw=None):
    """Patterns of P = A T, W = A P, A_c = P^T W and R = P^T for the aggregates ``agg`` (``na`` of
    them) of the level whose CSR in stored order is (rp, cl) (int64 torch tensors on one device),
    with the term lists of ``term_lists``, computed from sorted distinct keys instead of SciPy
    products: every structure the device set-up needs, on the tensors' device (four host
    synchronisations: the sizes of the products). ``pw``: the P and W parts already built by
    ``row_products`` (which hands a level back with P and W alone where an R or A_c row does
    not fit its kernels). Returns a dict of int64 tensors (patterns: p_ptr/p_idx, w_ptr/w_idx,
    c_ptr/c_idx, r_rowptr/r_col/r_from_p) and int32 term lists (None where a list would exceed
    ``cap`` terms)."""
    import torch

    dev = rp.device
    n, nnz = rp.numel() - 1, cl.numel()
    i32 = lambda t: t.to(torch.int32).contiguous()  # noqa: E731
    out = {}
    if pw is not None:
        i64 = lambda t: t.to(torch.int64)  # noqa: E731
        p_ptr, p_idx, w_ptr, w_idx = i64(pw["p_ptr"]), i64(pw["p_idx"]), i64(pw["w_ptr"]), i64(pw["w_idx"])
        p_nnz = p_idx.numel()
        out.update(p_ptr=p_ptr, p_idx=p_idx, w_ptr=w_ptr, w_idx=w_idx)
        for k in ("p_tptr", "p_tj", "w_tptr", "w_tj", "w_te"):
            out[k] = pw[k].contiguous()
    else:
        rows = _rows_of(rp, nnz)
        # P: A entry j of row i -> (i, agg[col j])
        kp = rows * na + agg[cl]
        p_ptr, p_idx, p_keys = _unique_pattern(kp, n, na)
        p_nnz = p_idx.numel()
        out.update(p_ptr=p_ptr, p_idx=p_idx)
        ptr, order = _grouped(torch.searchsorted(p_keys, kp), p_nnz)
        out["p_tptr"], out["p_tj"] = i32(ptr), i32(order)
        # W: (A entry j of row i, P entry e of row col j) -> (i, col e), generated j-major
        lens = p_ptr[cl + 1] - p_ptr[cl]
        w_terms = int(lens.sum())
        jj, e = _expand_sized(p_ptr, cl, w_terms)
        kw = rows[jj] * na + p_idx[e]
        w_ptr, w_idx, w_keys = _unique_pattern(kw, n, na)
        out.update(w_ptr=w_ptr, w_idx=w_idx)
        if w_terms <= cap:
            ptr, order = _grouped(torch.searchsorted(w_keys, kw), w_idx.numel())
            out["w_tptr"], out["w_tj"], out["w_te"] = i32(ptr), i32(jj[order]), i32(e[order])
        else:
            out["w_tptr"] = out["w_tj"] = out["w_te"] = None
        del jj, e, kw
    # R = P^T: P entries by (column, row)
    prow = _rows_of(p_ptr, p_nnz)
    r_from_p = torch.argsort(p_idx * n + prow)
    out.update(r_rowptr=_sorted_ptr(p_idx[r_from_p], na), r_col=prow[r_from_p], r_from_p=r_from_p)
    # A_c: (R entry q of coarse row I, W entry s of row r_col[q]) -> (I, col s), generated q-major
    qrow = _rows_of(out["r_rowptr"], p_nnz)
    rc = out["r_col"]
    c_terms = int((w_ptr[rc + 1] - w_ptr[rc]).sum())
    q, s_ = _expand_sized(w_ptr, rc, c_terms)
    kc = qrow[q] * na + w_idx[s_]
    c_ptr, c_idx, c_keys = _unique_pattern(kc, na, na)
    out.update(c_ptr=c_ptr, c_idx=c_idx, c_keys=c_keys)
    if c_terms <= cap and out["w_tptr"] is not None:
        ptr, order = _grouped(torch.searchsorted(c_keys, kc), c_idx.numel())
        out["c_tptr"], out["c_te"], out["c_ts"] = i32(ptr), i32(q[order]), i32(s_[order])
    else:
        out["c_tptr"] = out["c_te"] = out["c_ts"] = None
    return out


def device_strength(rowptr, col, val, diag_slot, theta, stream=None):
    """Strong flags of every stored entry (``b2s_amg_strength_d``): uint8 tensor [nnz]."""
    import torch

    n = rowptr.numel() - 1
    strong = torch.empty(col.numel(), dtype=torch.uint8, device=col.device)
    _lib.check(_lib.lib().b2s_amg_strength_d(n, rowptr.data_ptr(), col.data_ptr(), val.data_ptr(),
                                             diag_slot.data_ptr(), float(theta), strong.data_ptr(),
                                             _lib.stream_ptr(stream)), "b2s_amg_strength_d")
    return strong


def device_transpose_slots(rowptr, col, sorted_cols, stream=None):
    """Slot of every entry's transpose (``b2s_csr_transpose_slots_d``) and the device count of
    entries without one (int32 tensors)."""
    import torch

    n = rowptr.numel() - 1
    tslot = torch.empty(col.numel(), dtype=torch.int32, device=col.device)
    missing = torch.zeros(1, dtype=torch.int32, device=col.device)
    _lib.check(_lib.lib().b2s_csr_transpose_slots_d(n, rowptr.data_ptr(), col.data_ptr(), int(bool(sorted_cols)),
                                                    tslot.data_ptr(), missing.data_ptr(), _lib.stream_ptr(stream)),
               "b2s_csr_transpose_slots_d")
    return tslot, missing


def device_aggregate(rowptr, col, strong, tslot, prio, rank_node, stream=None, capacity=None):
    """The reference's greedy aggregation on the device (``b2s_amg_aggregate_d``), nodes visited
    in the order ``prio``: (agg int32 [n], counts int32 [n], info int32 [4]) on the device;
    info[0] is the number of aggregates, info[1] an error code. ``capacity``: the conflict lists'
    room, nnz plus the sum of squared row lengths (computed here, with a host synchronisation,
    when not given)."""
    import torch

    n = rowptr.numel() - 1
    dev = col.device
    L = _lib.lib()
    if capacity is None:
        rl = (rowptr[1:] - rowptr[:-1]).to(torch.int64)
        capacity = int(col.numel() + int((rl * rl).sum()))  # bounds every node's conflict list
    wb = L.b2s_amg_aggregate_workspace_bytes(n, capacity)
    if wb < 0:
        raise RuntimeError("invalid aggregation size")
    work = torch.empty(wb // 4 + 1, dtype=torch.int32, device=dev)
    agg = torch.empty(n, dtype=torch.int32, device=dev)
    counts = torch.empty(n, dtype=torch.int32, device=dev)
    info = torch.zeros(4, dtype=torch.int32, device=dev)
    _lib.check(L.b2s_amg_aggregate_d(n, rowptr.data_ptr(), col.data_ptr(), strong.data_ptr(), tslot.data_ptr(),
                                     prio.data_ptr(), rank_node.data_ptr(), agg.data_ptr(), counts.data_ptr(),
                                     info.data_ptr(), work.data_ptr(), work.numel() * 4, _lib.stream_ptr(stream)),
               "b2s_amg_aggregate_d")
    return agg, counts, info


def _pattern_checks(flags):
    """Raise where an A_c fill pass (``row_products``) found its offsets inconsistent."""
    if flags.numel() and bool((flags != 0).any()):
        raise RuntimeError("AMG set-up: the A_c pattern kernel's offsets disagree with its counts")


_START_VECTORS = {}


def _start_vector(n, dev):
    """The reference's power-iteration start vector (``default_rng(0)``, ``amg.py:69-77``) of
    length n, on the device. A draw of n normals is the first n values of a longer draw from the
    same seed, so one vector per device, as long as the longest level yet, serves every level
    (re-aggregated hierarchies change their coarse sizes; the cache does not grow with them)."""
    import torch

    key = str(dev)
    v = _START_VECTORS.get(key)
    if v is None or v.numel() < n:
        v = torch.as_tensor(np.random.default_rng(0).standard_normal(max(int(n), 1)), device=dev)
        _START_VECTORS[key] = v
    return v[: int(n)]


class AMGHierarchy:
    """Fixed-pattern SA-AMG hierarchy whose numeric part lives on the device.

    ``A_host`` is the first matrix in the reference's numbering (SciPy CSR); ``perm`` maps
    device rows to reference rows for level 0, whose device pattern is ``(rowptr, col)`` with
    ``diag_slot``; ``val`` is the device tensor of level-0 values that the solver rewrites
    before every rebuild.
    """

    ROW_PATTERNS = True  # device set-up: the products' patterns by the per-row kernels where rows fit them

    def __init__(self, A_host, perm, rowptr, col, diag_slot, val, slot_ref, singular=False, theta=0.08,
                 max_coarse=150, max_levels=20, sweeps=2, omega=0.8, groups=None, group_singular=None):
        """``groups`` (batches of independent cases, optional): the case of every row of A_host
        (reference numbering; A_host block diagonal by case, each case's rows contiguous in the
        device order). Aggregates are then numbered case by case, coarsening goes on until every
        case has at most ``max_coarse`` rows, and the coarsest level keeps one dense inverse per
        case (shifted where ``group_singular``)."""
        import torch

        dev = val.device
        self.singular, self.sweeps, self.omega, self.theta = bool(singular), int(sweeps), float(omega), theta
        A = sp.csr_matrix(A_host, dtype=np.float64)
        perm = np.asarray(perm, dtype=np.int64)
        n0 = A.shape[0]
        batched = groups is not None
        if batched:
            gl = np.asarray(groups, dtype=np.int64)
            ngroups = int(gl.max()) + 1
            level_groups = [gl]

        def too_big(A):
            if not batched:
                return A.shape[0] > max_coarse
            return np.bincount(level_groups[-1], minlength=ngroups).max() > max_coarse

        # ---- host set-up on the reference numbering (values drive the coarse strength graphs)
        aggs, counts, mats = [], [], []
        while too_big(A) and len(aggs) < max_levels - 1:
            S = strength(A, theta)
            if batched:
                # cases already at most max_coarse rows keep their size: no strong connections, so
                # every row of theirs is an aggregate of its own (a case coarsened to a handful of
                # rows would make a singular case's coarse block numerically zero)
                gsz = np.bincount(level_groups[-1], minlength=ngroups)
                big_row = gsz[level_groups[-1]] > max_coarse
                S = S.tocoo()
                keep = big_row[S.row]
                S = sp.csr_matrix((S.data[keep], (S.row[keep], S.col[keep])), shape=S.shape)
            agg, na = aggregate(S)
            if batched:
                n_big = int(big_row.sum())
                na_big = na - int((~big_row).sum())
                if na_big >= n_big * 0.9:
                    break
            elif na >= A.shape[0] * 0.9:
                break
            if batched:  # number the aggregates case by case (aggregates never cross cases)
                g_of = np.empty(na, dtype=np.int64)
                g_of[agg] = level_groups[-1]
                order = np.argsort(g_of, kind="stable")
                new_id = np.empty(na, dtype=np.int64)
                new_id[order] = np.arange(na)
                agg = new_id[agg]
                level_groups.append(g_of[order])
            T = sp.csr_matrix((np.ones(A.shape[0]), (np.arange(A.shape[0]), agg)), shape=(A.shape[0], na))
            cnt = np.asarray(T.sum(axis=0)).ravel()
            T = T @ sp.diags(1.0 / np.sqrt(cnt))
            Dinv = 1.0 / A.diagonal()
            DA = sp.diags(Dinv) @ A
            rho = spectral_radius(DA)
            P = (T - (4.0 / 3.0 / rho) * (DA @ T)).tocsr()
            aggs.append(agg)
            counts.append(cnt)
            mats.append(A)
            A = (P.T @ A @ P).tocsr()
        # no aggregation (at most max_coarse rows, or too weakly connected): the preconditioner is
        # the coarse solve of the matrix itself, as in the reference
        self.n_levels = len(aggs) + 1
        # ---- structural patterns and device buffers, level 0 in device numbering
        i32 = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.int32), device=dev)  # noqa: E731
        f64 = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=dev)  # noqa: E731
        self._keep = []
        self.sizes = []
        h = self.c = _lib.Amg()
        h.nlevels = len(aggs)
        h.singular = int(self.singular)
        h.sweeps = self.sweeps
        h.omega = self.omega
        rp = np.asarray(rowptr.cpu().numpy(), dtype=np.int64)
        cl = np.asarray(col.cpu().numpy(), dtype=np.int64)
        Apat = sp.csr_matrix((np.ones(cl.size), cl, rp), shape=(n0, n0))
        lv_rp, lv_cl = rp, cl  # the current level's CSR in stored order
        # the hierarchy's own copy of the level-0 values: like the reference's preconditioner
        # object, the V-cycle keeps the matrix of the last rebuild until the next one
        self.src_val = val
        self.src_val32 = None
        self.val0 = torch.empty_like(val)
        self.val0.copy_(val)
        level_val = self.val0
        level_rowptr, level_col, level_diag = rowptr, col, diag_slot
        self.rowptr0, self.col0, self.n0 = rowptr, col, n0
        for l, (agg, cnt) in enumerate(zip(aggs, counts)):
            n = Apat.shape[0]
            na = cnt.size
            if l == 0:
                agg_l = agg[perm]
                x0 = np.random.default_rng(0).standard_normal(n)[perm]
            else:
                agg_l = agg
                x0 = np.random.default_rng(0).standard_normal(n)
            T = sp.csr_matrix((np.ones(n), (np.arange(n), agg_l)), shape=(n, na))
            Pp = _pattern(_pattern(Apat) @ T)
            Wp = _pattern(_pattern(Apat) @ Pp)
            Cp = _pattern(Pp.T.tocsr() @ Wp)
            # R = P^T with the map from R entries to P entries
            prow = np.repeat(np.arange(n), np.diff(Pp.indptr))
            order = np.lexsort((prow, Pp.indices))
            r_col = prow[order]
            r_rowptr = np.concatenate([[0], np.cumsum(np.bincount(Pp.indices, minlength=na))])
            # strength flags of the set-up on this level's device pattern
            if l == 0:
                flags = strong_mask(mats[0], theta)[slot_ref]
            else:
                Sh = mats[l]
                rows_h = np.repeat(np.arange(n), np.diff(Sh.indptr))
                keys_s = (rows_h * n + Sh.indices)[strong_mask(Sh, theta)]
                rows_p = np.repeat(np.arange(n), np.diff(Apat.indptr))
                flags = np.isin(rows_p.astype(np.int64) * n + Apat.indices, keys_s)
            L = h.levels[l]
            L.n, L.nnz, L.nc, L.p_nnz, L.w_nnz = n, Apat.nnz, na, Pp.nnz, Wp.nnz
            bufs = {
                "rowptr": level_rowptr, "col": level_col, "val": level_val, "diag_slot": level_diag,
                "dinv": torch.empty(n, dtype=torch.float64, device=dev), "agg": i32(agg_l),
                "tval": f64(1.0 / np.sqrt(cnt)), "x0": f64(x0), "p_rowptr": i32(Pp.indptr), "p_col": i32(Pp.indices),
                "p_val": torch.empty(Pp.nnz, dtype=torch.float64, device=dev), "r_rowptr": i32(r_rowptr),
                "r_col": i32(r_col), "r_from_p": i32(order), "r_val": torch.empty(Pp.nnz, dtype=torch.float64, device=dev),
                "w_rowptr": i32(Wp.indptr), "w_col": i32(Wp.indices),
                "w_val": torch.empty(Wp.nnz, dtype=torch.float64, device=dev),
                "rho": torch.zeros(ngroups if batched else 1, dtype=torch.float64, device=dev),
                "strong": torch.as_tensor(np.ascontiguousarray(flags, dtype=np.uint8), device=dev),
            }
            if batched:
                bufs["group_ptr"] = i32(np.concatenate([[0], np.cumsum(np.bincount(level_groups[l],
                                                                                    minlength=ngroups))]))
            tl = term_lists(lv_rp, lv_cl, agg_l, na, Pp, Wp, Cp, r_col, r_rowptr, device=dev)
            if tl is not None:
                for k, v in tl.items():
                    if v is not None:
                        bufs[k] = v
                L.c_nnz = Cp.nnz
            for k, v in bufs.items():
                setattr(L, k, v.data_ptr())
            self._keep.append(bufs)
            self.sizes.append(n)
            # next level: pattern Cp in aggregate numbering
            Apat = Cp
            lv_rp, lv_cl = Cp.indptr.astype(np.int64), Cp.indices.astype(np.int64)
            level_rowptr, level_col = i32(Cp.indptr), i32(Cp.indices)
            level_val = torch.empty(Cp.nnz, dtype=torch.float64, device=dev)
            rows = np.repeat(np.arange(Cp.shape[0]), np.diff(Cp.indptr))
            dpos = np.flatnonzero(Cp.indices == rows)
            if dpos.size != Cp.shape[0]:
                raise RuntimeError("a coarse matrix lacks a diagonal entry")
            level_diag = i32(dpos)
            self._keep.append({"rowptr": level_rowptr, "col": level_col, "val": level_val, "diag": level_diag})
        nc = Apat.shape[0]
        self.coarse_n = nc
        self.sizes.append(nc)
        self.coarse_val = level_val
        if batched:
            sizes_g = np.bincount(level_groups[-1], minlength=ngroups)
            if sizes_g.max() > 160:
                raise RuntimeError("a case's coarsest AMG level has more than 160 rows")
            off = np.concatenate([[0], np.cumsum(sizes_g.astype(np.int64) ** 2)])
            self.coarse_inv = torch.empty(int(off[-1]), dtype=torch.float64, device=dev)
            gs = np.zeros(ngroups, dtype=np.int32) if group_singular is None else np.asarray(group_singular)
            self._keep.append({"cgp": i32(np.concatenate([[0], np.cumsum(sizes_g)])),
                               "off": torch.as_tensor(off[:-1].astype(np.int64), device=dev), "gs": i32(gs)})
            h.ngroups = ngroups
            h.coarse_group_ptr = self._keep[-1]["cgp"].data_ptr()
            h.coarse_inv_off = self._keep[-1]["off"].data_ptr()
            h.group_singular = self._keep[-1]["gs"].data_ptr()
            self.ngroups = ngroups
        else:
            self.coarse_inv = torch.empty((nc, nc), dtype=torch.float64, device=dev)
            self.ngroups = 0
        h.coarse_n = nc
        h.coarse_rowptr, h.coarse_col = level_rowptr.data_ptr(), level_col.data_ptr()
        h.coarse_val, h.coarse_inv = level_val.data_ptr(), self.coarse_inv.data_ptr()
        self._finish(dev)

    @classmethod
    def on_device(cls, perm, rowptr, col, diag_slot, val, singular=False, theta=0.08, max_coarse=150, max_levels=20,
                  sweeps=2, omega=0.8, stream=None, prev=None, start=0):
        """The set-up of ``flowtrace/linalg/amg.py:88-117`` done on the device, level by level:
        strength (``b2s_amg_strength_d``), the greedy aggregation in the reference's visiting
        order (``b2s_amg_aggregate_d``: the reference numbering ``perm`` on level 0, the aggregate
        numbering below), the patterns and term lists of P, W, R and A_c from sorted distinct keys
        (``product_patterns``), and the level's numeric rebuild (``b2s_amg_level_rebuild_d``),
        whose Galerkin product gives the next level's values and so its strength graph. Same
        aggregates, patterns and term lists as the host set-up; no host copy of the matrix. A
        single case only (no ``groups``). ``perm`` maps device rows to reference rows (numpy or
        a device tensor).

        Re-aggregation (``prev``, ``start``): ``prev`` is a hierarchy of the same level-0 pattern
        just rebuilt from the current matrix, whose levels below ``start`` kept their strength
        graphs - so the reference would build the same aggregates there. Those levels are shared
        with it and the set-up resumes at level ``start`` from its current values."""
        import torch

        self = cls.__new__(cls)
        dev = val.device
        L = _lib.lib()
        sp_ = _lib.stream_ptr(stream)
        self._row_patterns = cls.ROW_PATTERNS
        self.singular, self.sweeps, self.omega, self.theta = bool(singular), int(sweeps), float(omega), theta
        self._keep, self.sizes = [], []
        h = self.c = _lib.Amg()
        h.singular, h.sweeps, h.omega = int(self.singular), self.sweeps, self.omega
        self.src_val, self.src_val32 = val, None
        n0 = rowptr.numel() - 1
        self.rowptr0, self.col0, self.n0 = rowptr, col, n0
        i32 = lambda t: t.to(torch.int32).contiguous()  # noqa: E731
        start = int(start) if prev is not None else 0
        if start > 0:
            if start >= prev.n_levels:
                raise ValueError("start beyond the previous hierarchy's levels")
            self.val0 = prev.val0  # the shared level 0 keeps the previous rebuild's values
            for l in range(start):
                h.levels[l] = prev.c.levels[l]
                self._keep += prev._keep[2 * l:2 * l + 2]
                self.sizes.append(prev.sizes[l])
            nxt = prev._keep[2 * start - 1]
            lv_rp, lv_cl, lv_val, lv_diag = nxt["rowptr"], nxt["col"], nxt["val"], nxt["diag"]
            lv_rp64, lv_cl64 = nxt.get("rowptr64", lv_rp), nxt.get("col64", lv_cl)
            n = prev.sizes[start]
            prio = rank_node = torch.arange(n, dtype=torch.int32, device=dev)
            x0_src = _start_vector(n, dev)
            sorted_cols = True
        else:
            self.val0 = torch.empty_like(val)
            self.val0.copy_(val)
            perm_t = torch.as_tensor(np.asarray(perm, dtype=np.int64) if not torch.is_tensor(perm) else perm,
                                     device=dev).to(torch.int64)
            prio = i32(perm_t)
            rank_node = torch.empty(n0, dtype=torch.int32, device=dev)
            rank_node[perm_t] = torch.arange(n0, dtype=torch.int32, device=dev)
            lv_rp, lv_cl, lv_val, lv_diag = rowptr, col, self.val0, diag_slot
            lv_rp64, lv_cl64 = rowptr, col  # widened where the sorted-key construction needs them
            x0_src = _start_vector(n0, dev)[perm_t]
            sorted_cols = False  # level 0's columns are in the reference's order, not the device's
            n = n0
        nlev = start
        conflicts, checks = None, []
        while n > max_coarse and nlev < max_levels - 1:
            strong = device_strength(lv_rp, lv_cl, lv_val, lv_diag, theta, stream)
            tslot, missing = device_transpose_slots(lv_rp, lv_cl, sorted_cols, stream)
            agg, counts, info = device_aggregate(lv_rp, lv_cl, strong, tslot, prio, rank_node, stream, conflicts)
            # the level's read-back: aggregates and errors, and the previous level's A_c check
            ih = torch.cat([info, missing] + checks).cpu()
            _pattern_checks(ih[5:])
            checks = []
            if int(ih[4]) != 0:
                raise RuntimeError("AMG set-up: the level's pattern is not structurally symmetric")
            if int(ih[1]) != 0:
                raise RuntimeError(f"device aggregation failed (code {int(ih[1])})")
            na = int(ih[0])
            if na >= n * 0.9:
                break
            pat = row_products(lv_rp, lv_cl, agg, na, stream) if self._row_patterns else None
            if pat is None or not pat["complete"]:
                pat = product_patterns(lv_rp64.to(torch.int64), lv_cl64.to(torch.int64), agg.to(torch.int64), na,
                                       pw=pat)
            else:
                checks.append(pat["check"])
            conflicts = pat.get("conflicts")
            Lv = h.levels[nlev]
            Lv.n, Lv.nnz, Lv.nc = n, lv_cl.numel(), na
            Lv.p_nnz, Lv.w_nnz = pat["p_idx"].numel(), pat["w_idx"].numel()
            c_nnz = pat["c_idx"].numel()
            Lv.c_nnz = c_nnz if pat["c_tptr"] is not None else 0
            bufs = {
                "rowptr": lv_rp, "col": lv_cl, "val": lv_val, "diag_slot": lv_diag,
                "dinv": torch.empty(n, dtype=torch.float64, device=dev), "agg": agg,
                "tval": 1.0 / torch.sqrt(counts[:na].to(torch.float64)), "x0": x0_src.contiguous(),
                "p_rowptr": i32(pat["p_ptr"]), "p_col": i32(pat["p_idx"]),
                "p_val": torch.empty(Lv.p_nnz, dtype=torch.float64, device=dev),
                "r_rowptr": i32(pat["r_rowptr"]), "r_col": i32(pat["r_col"]), "r_from_p": i32(pat["r_from_p"]),
                "r_val": torch.empty(Lv.p_nnz, dtype=torch.float64, device=dev),
                "w_rowptr": i32(pat["w_ptr"]), "w_col": i32(pat["w_idx"]),
                "w_val": torch.empty(Lv.w_nnz, dtype=torch.float64, device=dev),
                "rho": torch.zeros(1, dtype=torch.float64, device=dev), "strong": strong,
            }
            for k in ("p_tptr", "p_tj", "w_tptr", "w_tj", "w_te", "c_tptr", "c_te", "c_ts"):
                if pat[k] is not None:
                    bufs[k] = pat[k]
            for k, v in bufs.items():
                setattr(Lv, k, v.data_ptr())
            self._keep.append(bufs)
            self.sizes.append(n)
            # the next level: A_c on its pattern, from this level's numeric rebuild; its diagonal
            # is in the pattern (a_ii p_iI^2 contributes to entry (I, I) of P^T A P)
            c_rp, c_cl = i32(pat["c_ptr"]), i32(pat["c_idx"])
            c_val = torch.empty(c_nnz, dtype=torch.float64, device=dev)
            wl = L.b2s_amg_level_workspace_bytes(ctypes.byref(Lv))
            work = torch.empty(max(wl, 8) // 8 + 1, dtype=torch.float64, device=dev)
            _lib.check(L.b2s_amg_level_rebuild_d(ctypes.byref(Lv), c_rp.data_ptr(), c_cl.data_ptr(), c_val.data_ptr(),
                                                 work.data_ptr(), work.numel() * 8, sp_), "b2s_amg_level_rebuild_d")
            ar = torch.arange(na, device=dev)
            lv_diag = pat["c_diag"] if "c_diag" in pat else i32(torch.searchsorted(pat["c_keys"], ar * na + ar))
            lv_rp, lv_cl, lv_val = c_rp, c_cl, c_val
            lv_rp64, lv_cl64 = pat["c_ptr"], pat["c_idx"]
            self._keep.append({"rowptr": lv_rp, "col": lv_cl, "val": lv_val, "diag": lv_diag, "work": work,
                               "rowptr64": lv_rp64, "col64": lv_cl64})
            prio = rank_node = ar.to(torch.int32)
            x0_src = _start_vector(na, dev)
            sorted_cols = True
            n = na
            nlev += 1
        if checks:
            _pattern_checks(torch.cat(checks).cpu())
        h.nlevels = nlev
        self.n_levels = nlev + 1
        self.coarse_n = n
        self.sizes.append(n)
        self.coarse_val = lv_val
        self.coarse_inv = torch.empty((n, n), dtype=torch.float64, device=dev)
        self.ngroups = 0
        h.coarse_n = n
        h.coarse_rowptr, h.coarse_col = lv_rp.data_ptr(), lv_cl.data_ptr()
        h.coarse_val, h.coarse_inv = lv_val.data_ptr(), self.coarse_inv.data_ptr()
        self._keep.append({"coarse_rowptr": lv_rp, "coarse_col": lv_cl})
        self._finish(dev)
        _lib.check(L.b2s_amg_coarse_inverse_d(self.cref, self.work_rebuild.data_ptr(), self.work_rebuild.numel() * 8,
                                              sp_), "b2s_amg_coarse_inverse_d")
        return self

    def first_strength_change(self, stream=None) -> int:
        """The first level whose strength graph, with the current level matrices, differs from the
        set-up's (the reference would aggregate it differently), or -1. Synchronises the stream."""
        import torch

        nl = max(self.c.nlevels, 1)
        if self._level_counts is None or self._level_counts.numel() < nl:
            self._level_counts = torch.zeros(nl, dtype=torch.int32, device=self._count.device)
            self._level_counts_host = torch.zeros(nl, dtype=torch.int32)
            if self._count.device.type == "cuda":
                self._level_counts_host = self._level_counts_host.pin_memory()
        if self.c.nlevels == 0:
            return -1
        _lib.check(_lib.lib().b2s_amg_level_strength_changes_d(self.cref, self.theta, self._level_counts.data_ptr(),
                                                               _lib.stream_ptr(stream)),
                   "b2s_amg_level_strength_changes_d")
        self._level_counts_host.copy_(self._level_counts, non_blocking=True)
        (stream or torch.cuda.current_stream()).synchronize()
        changed = np.flatnonzero(self._level_counts_host.numpy()[: self.c.nlevels])
        return int(changed[0]) if changed.size else -1

    def to_f32(self, stream=None):
        """Refresh the float copies of the level values (mixed precision) without a rebuild."""
        if self.src_val32 is not None:
            _lib.check(_lib.lib().b2s_amg_to_f32_d(self.cref, self.c32ref, _lib.stream_ptr(stream)), "b2s_amg_to_f32_d")

    def _finish(self, dev):
        """Workspaces and the strength-change counter of a complete hierarchy."""
        import torch

        self.cref = ctypes.byref(self.c)
        L = _lib.lib()
        wb = L.b2s_amg_workspace_bytes(self.cref)
        pb = L.b2s_pcg_workspace_bytes(self.cref)
        if wb < 0 or pb < 0:
            raise RuntimeError("invalid AMG hierarchy")
        self.work_rebuild = torch.empty(max(wb, 8) // 8 + 1, dtype=torch.float64, device=dev)
        self.work_pcg = torch.empty(max(pb, 8) // 8 + 1, dtype=torch.float64, device=dev)
        self._count = torch.zeros(1, dtype=torch.int32, device=dev)
        self._level_counts = None
        self._count_host = torch.zeros(1, dtype=torch.int32)
        if dev.type == "cuda":
            self._count_host = self._count_host.pin_memory()

    def strength_changed(self, stream=None) -> bool:
        """True when, with the current level matrices, some level's strength graph differs from the
        set-up's: the reference would then build different aggregates (it re-aggregates at every
        rebuild). Synchronises the stream."""
        import torch

        _lib.check(_lib.lib().b2s_amg_strength_changes_d(self.cref, self.theta, self._count.data_ptr(),
                                                         _lib.stream_ptr(stream)), "b2s_amg_strength_changes_d")
        self._count_host.copy_(self._count, non_blocking=True)
        (stream or torch.cuda.current_stream()).synchronize()
        return int(self._count_host[0]) != 0

    def rebuild(self, stream=None):
        """Copy the current level-0 values and recompute every numeric quantity (device). With a
        float source (``enable_mixed``) the values are widened first and the float copies of the
        level values are refreshed after the rebuild."""
        if self.src_val32 is not None:
            self.src_val.copy_(self.src_val32)
        self.val0.copy_(self.src_val)
        _lib.check(_lib.lib().b2s_amg_rebuild_d(self.cref, self.work_rebuild.data_ptr(),
                                                self.work_rebuild.numel() * 8, _lib.stream_ptr(stream)),
                   "b2s_amg_rebuild_d")
        if self.src_val32 is not None:
            _lib.check(_lib.lib().b2s_amg_to_f32_d(self.cref, self.c32ref, _lib.stream_ptr(stream)), "b2s_amg_to_f32_d")

    def enable_mixed(self, val32):
        """Prepare the float solve: float copies of every level's values (refreshed by ``rebuild``)
        and the workspace of ``pcg_mixed``; val32 is the float level-0 operator, whose values
        ``rebuild`` widens into ``src_val`` before rebuilding."""
        import torch

        dev = val32.device
        self.src_val32 = val32
        h = self.c
        h32 = self.c32 = _lib.Amg32()
        self._keep32 = []
        for l in range(h.nlevels):
            L = h.levels[l]
            bufs = {"val": torch.empty(L.nnz, dtype=torch.float32, device=dev),
                    "dinv": torch.empty(L.n, dtype=torch.float32, device=dev),
                    "p_val": torch.empty(L.p_nnz, dtype=torch.float32, device=dev),
                    "r_val": torch.empty(L.p_nnz, dtype=torch.float32, device=dev)}
            for k, v in bufs.items():
                getattr(h32, k)[l] = v.data_ptr()
            self._keep32.append(bufs)
        self.c32ref = ctypes.byref(h32)
        mb = (_lib.lib().b2s_pcg_groups_workspace_bytes(self.cref) if self.ngroups
              else _lib.lib().b2s_pcg_mixed_workspace_bytes(self.cref))
        if mb < 0:
            raise RuntimeError("invalid AMG hierarchy")
        self.work_mixed = torch.empty(mb // 8 + 1, dtype=torch.float64, device=dev)

    def pcg_mixed(self, mesh_ref, cf, cb, b, x, tol, maxiter, project, info, maxpass=8, min_inner_tol=1e-5,
                  stream=None):
        """Solve A x = b (double b, x) by float AMG-PCG passes with double iterative refinement,
        A applied in double from the face coefficients cf, cb of the mesh (``b2s_pcg_amg_mixed_d``)."""
        _lib.check(_lib.lib().b2s_pcg_amg_mixed_d(self.cref, self.c32ref, mesh_ref, cf.data_ptr(), cb.data_ptr(),
                                                  self.n0, self.rowptr0.data_ptr(), self.col0.data_ptr(),
                                                  self.src_val32.data_ptr(), b.data_ptr(), x.data_ptr(), float(tol),
                                                  int(maxiter), int(bool(project)), int(maxpass), float(min_inner_tol),
                                                  self.work_mixed.data_ptr(), self.work_mixed.numel() * 8, info,
                                                  _lib.stream_ptr(stream)), "b2s_pcg_amg_mixed_d")

    def vcycle(self, b, stream=None):
        import torch

        x = torch.empty_like(b)
        _lib.check(_lib.lib().b2s_amg_vcycle_d(self.cref, b.contiguous().data_ptr(), x.data_ptr(),
                                               self.work_pcg.data_ptr(), self.work_pcg.numel() * 8,
                                               _lib.stream_ptr(stream)), "b2s_amg_vcycle_d")
        return x

    def pcg(self, b, x, tol, maxiter, project, info, stream=None):
        """Solve A x = b by AMG-PCG, A the current level-0 matrix (``src_val``); info is the device
        address of a b2s_solve_info record."""
        _lib.check(_lib.lib().b2s_pcg_amg_d(self.cref, self.n0, self.rowptr0.data_ptr(), self.col0.data_ptr(),
                                            self.src_val.data_ptr(), b.data_ptr(), x.data_ptr(), float(tol), int(maxiter),
                                            int(bool(project)), self.work_pcg.data_ptr(), self.work_pcg.numel() * 8,
                                            info, _lib.stream_ptr(stream)), "b2s_pcg_amg_d")

    def pcg_groups_mixed(self, mesh_ref, order, project, cf, cb, b, x, tol, maxiter, info, maxpass=8,
                         min_inner_tol=1e-5, stream=None, team=None):
        """Per-case refined solves of a batch hierarchy (``b2s_pcg_groups_mixed_d``): order and
        project are device int32 tensors [ngroups]; info the device address of ngroups records;
        team a ``_lib.TeamConfig`` (None: the library's default team shape)."""
        _lib.check(_lib.lib().b2s_pcg_groups_mixed_d(self.cref, self.c32ref, order.data_ptr(), project.data_ptr(),
                                                     mesh_ref, cf.data_ptr(), cb.data_ptr(), self.n0,
                                                     self.rowptr0.data_ptr(), self.col0.data_ptr(),
                                                     self.src_val32.data_ptr(), b.data_ptr(), x.data_ptr(), float(tol),
                                                     int(maxiter), int(maxpass), float(min_inner_tol),
                                                     self.work_mixed.data_ptr(), self.work_mixed.numel() * 8, info,
                                                     None if team is None else ctypes.byref(team),
                                                     _lib.stream_ptr(stream)), "b2s_pcg_groups_mixed_d")
