"""The device AMG set-up's rules on the CPU: the parallel formulation of the reference's greedy
aggregation (``flowtrace/linalg/amg.py:25-57``) that ``b2s_amg_aggregate_d`` implements -
pass 1 as a lexicographically-first independent set over conflicting nodes, roots numbered in
priority order, pass 2 by links down in priority - restated here step by step and compared
with the sequential greedy (``b2s_host_aggregate``) on structurally symmetric graphs with
symmetric and non-symmetric strengths and arbitrary visiting orders; and the key-based product
patterns and term lists of the device set-up (``product_patterns``) against the SciPy patterns
and ``term_lists`` of the host set-up."""

import numpy as np
import pytest
import scipy.sparse as sp

from gputest_b200.linalg import amg

UND, ROOT, NOT = 0, 1, 2


def _transpose_slots(rp, cl):
    pos = {(i, int(cl[e])): e for i in range(len(rp) - 1) for e in range(rp[i], rp[i + 1])}
    return np.array([pos[(int(cl[e]), i)] for i in range(len(rp) - 1) for e in range(rp[i], rp[i + 1])])


def _parallel_rules(rp, cl, strong, prio):
    """The kernel's rules, evaluated in priority order (the dataflow kernel's unique fixed point:
    every dependency of a node has a lower priority)."""
    n = len(rp) - 1
    ts = _transpose_slots(rp, cl)
    rank_node = np.argsort(prio)
    deps = []
    for i in range(n):
        d = set()
        for e in range(rp[i], rp[i + 1]):
            j = int(cl[e])
            if j == i:
                continue
            if (strong[e] or strong[ts[e]]) and prio[j] < prio[i]:
                d.add(j)
            if strong[e]:
                for e2 in range(rp[j], rp[j + 1]):
                    r = int(cl[e2])
                    if r in (i, j) or not strong[ts[e2]] or prio[r] >= prio[i]:
                        continue
                    d.add(r)
        deps.append(d)
    st = np.zeros(n, dtype=int)
    for p in range(n):
        i = rank_node[p]
        st[i] = NOT if any(st[r] == ROOT for r in deps[i]) else ROOT
    rid = np.cumsum([st[rank_node[p]] == ROOT for p in range(n)]) - 1
    na1 = int((st == ROOT).sum())
    agg1 = -np.ones(n, dtype=int)
    for i in range(n):
        if st[i] == ROOT:
            agg1[i] = rid[prio[i]]
            continue
        for e in range(rp[i], rp[i + 1]):
            r = int(cl[e])
            if r != i and strong[ts[e]] and st[r] == ROOT:
                agg1[i] = rid[prio[r]]
                break
    link = np.empty(n, dtype=int)
    for i in range(n):
        if agg1[i] >= 0:
            link[i] = i
            continue
        best, bp = -1, n + 1
        for e in range(rp[i], rp[i + 1]):
            j = int(cl[e])
            if j != i and strong[e] and (agg1[j] >= 0 or prio[j] < prio[i]) and prio[j] < bp:
                best, bp = j, prio[j]
        link[i] = best
    agg = agg1.copy()
    for i in range(n):
        x = i
        while agg[i] < 0 and link[x] >= 0:
            x = link[x]
            agg[i] = agg1[x]
    late = [i for i in rank_node if agg[i] < 0]
    for k, i in enumerate(late):
        agg[i] = na1 + k
    return agg, na1 + len(late)


def _greedy_in_priority_order(rp, cl, strong, prio):
    """The reference's sequential greedy on the strength graph renumbered by priority."""
    n = len(rp) - 1
    rows = np.repeat(np.arange(n), np.diff(rp))
    m = strong.astype(bool)
    S = sp.csr_matrix((np.ones(int(m.sum())), (prio[rows[m]], prio[cl[m]])), shape=(n, n))
    S.sort_indices()
    agg_p, na = amg.aggregate(S)
    return agg_p[prio], na


def _graph(seed, n, kind):
    rng = np.random.default_rng(seed)
    if kind == "grid":  # 2-D 5-point pattern with anisotropy and random jitter
        nx = int(np.sqrt(n))
        A = sp.diags([1.0], [0], shape=(nx * nx, nx * nx)).tolil()
        for y in range(nx):
            for x in range(nx):
                i = y * nx + x
                for dx, dy, w in ((1, 0, 1.0), (0, 1, 0.05 + rng.random())):
                    if x + dx < nx and y + dy < nx:
                        j = (y + dy) * nx + x + dx
                        a = -w * (0.5 + rng.random())
                        A[i, j] = a
                        A[j, i] = a
        A = A.tocsr()
        A.setdiag(-np.asarray(A.sum(axis=1)).ravel() + 1e-3 + A.diagonal())
    else:  # random structurally symmetric pattern, values not symmetric
        B = sp.random(n, n, density=4.0 / n, random_state=seed, format="coo")
        pat = sp.csr_matrix((np.ones(B.nnz), (B.row, B.col)), shape=(n, n))
        pat = ((pat + pat.T) > 0).astype(float).tocoo()
        vals = -rng.random(pat.nnz) ** 3
        A = sp.csr_matrix((vals, (pat.row, pat.col)), shape=(n, n))
        A.setdiag(0.0)
        A.eliminate_zeros()
        A = A + sp.diags(np.abs(np.asarray(A.sum(axis=1)).ravel()) + 0.5)
    A = sp.csr_matrix(A)
    A.sort_indices()
    return A


@pytest.mark.parametrize("kind,seed,theta,order", [
    ("grid", 1, 0.08, "identity"), ("grid", 2, 0.25, "random"), ("grid", 3, 0.5, "random"),
    ("random", 4, 0.08, "random"), ("random", 5, 0.25, "identity"), ("random", 6, 0.0, "random"),
])
def test_parallel_aggregation_rules_equal_the_sequential_greedy(kind, seed, theta, order):
    A = _graph(seed, 400, kind)
    n = A.shape[0]
    rp, cl = A.indptr.astype(np.int64), A.indices.astype(np.int64)
    strong = amg.strong_mask(A, theta).astype(np.uint8)
    rng = np.random.default_rng(seed + 100)
    prio = np.arange(n) if order == "identity" else rng.permutation(n)
    # the device visits rows in priority order whatever their storage order: shuffle the rows'
    # entries so that nothing relies on sorted columns
    perm_e = np.concatenate([rp[i] + rng.permutation(rp[i + 1] - rp[i]) for i in range(n)])
    cl_s, strong_s = cl[perm_e], strong[perm_e]
    got, na = _parallel_rules(rp, cl_s, strong_s, prio)
    want, na_ref = _greedy_in_priority_order(rp, cl, strong, prio)
    assert na == na_ref
    np.testing.assert_array_equal(got, want)


def test_product_patterns_equal_the_scipy_patterns_and_term_lists():
    import torch

    A = _graph(7, 900, "grid")
    n = A.shape[0]
    S = amg.strength(A, 0.08)
    agg, na = amg.aggregate(S)
    # a level in "device" order: rows renumbered and each row's entries shuffled
    rng = np.random.default_rng(8)
    perm = rng.permutation(n)
    iperm = np.empty(n, dtype=np.int64)
    iperm[perm] = np.arange(n)
    rl = np.diff(A.indptr)
    rp = np.concatenate([[0], np.cumsum(rl[perm])])
    src = np.concatenate([A.indptr[perm[i]] + rng.permutation(rl[perm[i]]) for i in range(n)])
    cl = iperm[A.indices[src]]
    agg_l = agg[perm]
    Apat = sp.csr_matrix((np.ones(cl.size), cl, rp), shape=(n, n))
    T = sp.csr_matrix((np.ones(n), (np.arange(n), agg_l)), shape=(n, na))
    Pp = amg._pattern(amg._pattern(Apat) @ T)
    Wp = amg._pattern(amg._pattern(Apat) @ Pp)
    Cp = amg._pattern(Pp.T.tocsr() @ Wp)
    prow = np.repeat(np.arange(n), np.diff(Pp.indptr))
    order = np.lexsort((prow, Pp.indices))
    r_col = prow[order]
    r_rowptr = np.concatenate([[0], np.cumsum(np.bincount(Pp.indices, minlength=na))])
    ref = amg.term_lists(rp, cl, agg_l, na, Pp, Wp, Cp, r_col, r_rowptr)
    t = lambda a: torch.as_tensor(np.asarray(a, dtype=np.int64))  # noqa: E731
    got = amg.product_patterns(t(rp), t(cl), t(agg_l), na)
    for key, M in (("p", Pp), ("w", Wp), ("c", Cp)):
        np.testing.assert_array_equal(got[key + "_ptr"].numpy(), M.indptr)
        np.testing.assert_array_equal(got[key + "_idx"].numpy(), M.indices)
    np.testing.assert_array_equal(got["r_rowptr"].numpy(), r_rowptr)
    np.testing.assert_array_equal(got["r_col"].numpy(), r_col)
    np.testing.assert_array_equal(got["r_from_p"].numpy(), order)
    for k, v in ref.items():
        np.testing.assert_array_equal(got[k].numpy(), v.numpy(), err_msg=k)


def _shuffled_level(seed, n):
    """A grid level in "device" order (rows renumbered, each row's entries shuffled) with its
    greedy aggregates: (rp, cl, agg, na) as int64 torch tensors on the CPU and na."""
    import torch

    A = _graph(seed, n, "grid")
    n = A.shape[0]
    agg, na = amg.aggregate(amg.strength(A, 0.08))
    rng = np.random.default_rng(seed + 1)
    perm = rng.permutation(n)
    iperm = np.empty(n, dtype=np.int64)
    iperm[perm] = np.arange(n)
    rl = np.diff(A.indptr)
    rp = np.concatenate([[0], np.cumsum(rl[perm])])
    src = np.concatenate([A.indptr[perm[i]] + rng.permutation(rl[perm[i]]) for i in range(n)])
    t = lambda a: torch.as_tensor(np.asarray(a, dtype=np.int64))  # noqa: E731
    return t(rp), t(iperm[A.indices[src]]), t(agg[perm]), na


def test_product_patterns_complete_a_level_handed_back_with_p_and_w_only():
    """Where an R or A_c row does not fit the per-row kernels, ``row_products`` hands the level
    back with P and W alone (int32 patterns, ``complete`` False); ``product_patterns`` adds R and
    A_c from sorted keys, and the level equals the key-based construction of all four."""
    import torch

    rp, cl, agg, na = _shuffled_level(11, 1600)
    full = amg.product_patterns(rp, cl, agg, na)
    pw = {k: full[k].to(torch.int32) for k in ("p_ptr", "p_idx", "w_ptr", "w_idx")}
    pw.update({k: full[k] for k in ("p_tptr", "p_tj", "w_tptr", "w_tj", "w_te")}, complete=False)
    got = amg.product_patterns(rp, cl, agg, na, pw=pw)
    assert set(got) == set(full)
    for k, v in full.items():
        assert (got[k] is None) == (v is None), k
        if v is not None:
            assert torch.equal(got[k].long(), v.long()), k


def test_pattern_checks_raise_on_an_inconsistent_fill():
    """The A_c fill passes' consistency flags, read at the set-up's next synchronisation: zero
    flags (or none) pass, any nonzero flag raises."""
    import torch

    amg._pattern_checks(torch.zeros(0, dtype=torch.int32))
    amg._pattern_checks(torch.zeros(3, dtype=torch.int32))
    with pytest.raises(RuntimeError, match="A_c pattern kernel"):
        amg._pattern_checks(torch.tensor([0, 2, 0], dtype=torch.int32))
