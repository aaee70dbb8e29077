"""Device-resident finite-volume data of an unstructured mesh, laid out for B200.

Host set-up (once, FP64, NumPy) computes the quantities of
``flowtrace/unstructured/fvmesh.py:61-230`` in the reference's numbering: interior/boundary
split, d, w, alpha = S.S/S.d, T = S - alpha d, non-orthogonality, least-squares matrices and
their inverses, the CSR pattern and its slot maps. It then lays them out for the device:

* cells in reverse Cuthill-McKee order (``perm``: device -> reference cell), so that a cell's
  neighbours, and the faces it shares with them, sit close in memory;
* interior faces sorted by (device owner, reference face index): a cell's owned faces are a
  contiguous range; faces it neighbours are listed per cell, by reference face index;
* boundary faces sorted by (device owner, reference boundary-face index);
* geometry in SoA form (component-major), so each component streams contiguously;
* the CSR pattern in device rows, each row keeping the reference's column order, so a row
  product sums its terms in the reference's order.

Everything maps back to the reference's numbering through ``perm``, ``face_ref`` and
``bface_ref``; connectivity and slot maps are checked against the reference bit for bit in
the tests.
"""

from __future__ import annotations

import ctypes

import numpy as np
import scipy.sparse as sp
from scipy.sparse.csgraph import reverse_cuthill_mckee

from .. import _lib
from ..mesh.unstructured import UnstructuredMesh, compute_geometry


def _batched_inverse(G: np.ndarray) -> np.ndarray:
    """Inverse of every (dim x dim) least-squares matrix; the pseudo-inverse where singular
    (``flowtrace/unstructured/fvmesh.py:25-39``)."""
    out = np.empty_like(G)
    ok = np.abs(np.linalg.det(G)) > 1e-300
    if ok.any():
        out[ok] = np.linalg.inv(G[ok])
        bad = ~ok | ~np.isfinite(out).all(axis=(1, 2))
    else:
        bad = ok == ok
    if bad.any():
        out[bad] = np.linalg.pinv(G[bad])
    return out


class HostFV:
    """The reference's FV quantities, in the reference's numbering (host, FP64)."""

    def __init__(self, mesh: UnstructuredMesh):
        if mesh.periodic:
            raise NotImplementedError("periodic meshes are not supported by the B200 SIMPLEC path")
        self.mesh = mesh
        self.dim = dim = mesh.dim
        geo = self.geometry = compute_geometry(mesh)
        self.nc = nc = mesh.n_cells
        interior = mesh.neighbour >= 0
        boundary = ~interior
        self.if_idx = np.flatnonzero(interior)
        self.bf_idx = np.flatnonzero(boundary)
        P = mesh.owner[interior].astype(np.int64)
        N = mesh.neighbour[interior].astype(np.int64)
        Pb = mesh.owner[boundary].astype(np.int64)
        if np.any(P == N):
            raise ValueError("a face connects a cell to itself")
        self.n_if, self.n_bf = P.size, Pb.size
        xc = geo.cell_centre
        S, Sb = geo.face_area_vec[interior], geo.face_area_vec[boundary]
        xf, xfb = geo.face_centre[interior], geo.face_centre[boundary]
        xN = xc[N]
        d = xN - xc[P]
        db = xfb - xc[Pb]
        dd = np.einsum("fd,fd->f", d, d)
        w = np.clip(np.einsum("fd,fd->f", xN - xf, d) / dd, 0.0, 1.0)
        Sd = np.einsum("fd,fd->f", S, d)
        Sdb = np.einsum("fd,fd->f", Sb, db)
        SS = np.einsum("fd,fd->f", S, S)
        SSb = np.einsum("fd,fd->f", Sb, Sb)
        alpha, alpha_b = SS / Sd, SSb / Sdb
        self.non_orthogonality_deg = float(np.degrees(np.arccos(np.clip(Sd / np.sqrt(SS * dd), -1, 1))).max()) \
            if P.size else 0.0
        wl = 1.0 / dd
        wlb = 1.0 / np.einsum("fd,fd->f", db, db)
        Gm = np.zeros((nc, dim, dim))
        for a in range(dim):
            for b in range(a, dim):
                o = wl * d[:, a] * d[:, b]
                Gm[:, a, b] = (np.bincount(P, o, minlength=nc) + np.bincount(N, o, minlength=nc)
                               + np.bincount(Pb, wlb * db[:, a] * db[:, b], minlength=nc))
                Gm[:, b, a] = Gm[:, a, b]
        self.Ginv = _batched_inverse(Gm)
        rows = np.concatenate([np.arange(nc), P, N])
        cols = np.concatenate([np.arange(nc), N, P])
        pat = sp.csr_matrix((np.ones(rows.size, dtype=np.int8), (rows, cols)), shape=(nc, nc))
        pat.sum_duplicates()
        pat.sort_indices()
        row_of = np.repeat(np.arange(nc), np.diff(pat.indptr))
        keys = row_of.astype(np.int64) * nc + pat.indices
        self.nnz = int(pat.nnz)
        self.slot_diag = np.searchsorted(keys, np.arange(nc, dtype=np.int64) * nc + np.arange(nc))
        self.slot_PN = np.searchsorted(keys, P * nc + N)
        self.slot_NP = np.searchsorted(keys, N * nc + P)
        self.indptr, self.indices = pat.indptr.astype(np.int64), pat.indices.astype(np.int64)
        self.duplicate_pairs = bool(np.unique(self.slot_PN).size != self.slot_PN.size)
        self.bzone = mesh.face_zone[boundary]
        self.P, self.N, self.Pb = P, N, Pb
        self.S, self.Sb, self.d, self.db, self.w = S, Sb, d, db, w
        self.alpha, self.alpha_b = alpha, alpha_b
        self.Tvec = S - alpha[:, None] * d
        self.Sb_mag = np.sqrt(SSb)
        self.nb = Sb / np.sqrt(SSb)[:, None]
        self.db_t = db - np.einsum("fd,fd->f", db, self.nb)[:, None] * self.nb
        self.vol, self.xc, self.xfb = geo.cell_volume, xc, xfb
        self.yb = np.abs(np.einsum("fd,fd->f", db, Sb)) / np.sqrt(SSb)
        self.wl, self.wlb = wl, wlb
        self.dP_f = xf - xc[P]
        self.dN_f = xf - xN
        self.dxm = xf - (w[:, None] * xc[P] + (1.0 - w)[:, None] * xN)


class FVMesh:
    """Device layout of a mesh (see the module docstring). ``device`` defaults to the current
    CUDA device; there is no CPU variant."""

    def __init__(self, mesh: UnstructuredMesh, device=None, reorder: bool = True, groups=None,
                 device_setup: bool = True):
        """``groups`` (one label per cell, optional): cells of one group are kept contiguous in the
        device order, groups in increasing label order (the reverse Cuthill-McKee order within
        each) - the layout of a block-diagonal batch of independent cases. ``device_setup``: the
        geometry, face quantities, least-squares matrices, CSR pattern and layout are computed on
        the device (``b2s_setup.cu``) from the raw mesh; False computes them on the host
        (``HostFV``) and uploads them. Both give the same arrays (the least-squares inverses to
        rounding); ``host`` is available either way (built on first use in the device set-up)."""
        self.device = device if device is not None else _lib.require_device()
        if mesh.periodic:
            raise NotImplementedError("periodic meshes are not supported by the B200 SIMPLEC path")
        self.mesh = mesh
        self._host = None
        self._geometry = None
        dev = self.device
        if device_setup and getattr(dev, "type", str(dev)) == "cuda":
            ref = self._reference_arrays_on_device(mesh)
        else:
            ref = self._reference_arrays_from_host(mesh)
        self._layout(ref, reorder, groups)

    @property
    def host(self) -> HostFV:
        """The reference's FV quantities on the host (``HostFV``), built on first use."""
        if self._host is None:
            self._host = HostFV(self.mesh)
        return self._host

    @property
    def geometry(self):
        return self.host.geometry

    def _reference_arrays_from_host(self, mesh):
        """The FV quantities in the reference's numbering, from ``HostFV`` (host, then uploaded)."""
        import torch

        h = self._host = HostFV(mesh)
        dev = self.device
        T = lambda a, dt=torch.float64: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=dev)  # noqa: E731
        self.h2d_bytes = 8 * sum(np.asarray(a).size for a in (h.w, h.alpha, h.wl, h.S, h.d, h.Tvec, h.dxm, h.dP_f,
                                                              h.dN_f, h.alpha_b, h.wlb, h.Sb_mag, h.Sb, h.db, h.nb,
                                                              h.db_t, h.vol, h.Ginv))
        return {"dim": h.dim, "nc": h.nc, "P": h.P, "N": h.N, "Pb": h.Pb, "bzone": h.bzone, "xfb": h.xfb,
                "non_orthogonality_deg": h.non_orthogonality_deg,
                "w": T(h.w), "alpha": T(h.alpha), "wl": T(h.wl), "S": T(h.S), "d": T(h.d), "Tv": T(h.Tvec),
                "dxm": T(h.dxm), "dPf": T(h.dP_f), "dNf": T(h.dN_f), "alpha_b": T(h.alpha_b), "wlb": T(h.wlb),
                "Sb_mag": T(h.Sb_mag), "Sb": T(h.Sb), "db": T(h.db), "nbv": T(h.nb), "dbt": T(h.db_t),
                "vol": T(h.vol), "Ginv": T(h.Ginv)}

    def _reference_arrays_on_device(self, mesh):
        """The FV quantities in the reference's numbering, computed on the device from the raw
        mesh (nodes, face-node lists, owner, neighbour): ``b2s_face_geometry_d``,
        ``b2s_cell_geometry_d``, ``b2s_fv_faces_d`` and ``b2s_ls_matrices_d``, with the per-cell
        face lists in the reference's face order (stable sorts)."""
        import torch

        dev = self.device
        L = _lib.lib()
        sp_ = _lib.stream_ptr()
        dim, nc = mesh.dim, mesh.n_cells
        owner = np.asarray(mesh.owner, dtype=np.int64)
        neighbour = np.asarray(mesh.neighbour, dtype=np.int64)
        nf_all = owner.size
        interior = neighbour >= 0
        if_idx = np.flatnonzero(interior)
        bf_idx = np.flatnonzero(~interior)
        P, N, Pb = owner[if_idx], neighbour[if_idx], owner[bf_idx]
        if np.any(P == N):
            raise ValueError("a face connects a cell to itself")
        n_if, n_bf = if_idx.size, bf_idx.size
        i32 = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.int32), device=dev)  # noqa: E731
        f64 = lambda *sh: torch.empty(*sh, dtype=torch.float64, device=dev)  # noqa: E731
        X = torch.as_tensor(np.ascontiguousarray(mesh.nodes, dtype=np.float64), device=dev)
        fptr, fnodes = i32(mesh.face_ptr), i32(mesh.face_nodes)
        own_t, nei_t = i32(owner), i32(neighbour)
        if_t, bf_t, P_t, N_t, Pb_t = i32(if_idx), i32(bf_idx), i32(P), i32(N), i32(Pb)
        self.h2d_bytes = sum(a.numel() * a.element_size() for a in (X, fptr, fnodes, own_t, nei_t, if_t, bf_t, P_t,
                                                                     N_t, Pb_t))
        ar = torch.arange(nc + 1, device=dev)

        def lists(keys):
            """Entries grouped by key (stable: increasing position within a key) and offsets."""
            srt = torch.sort(keys, stable=True)
            return torch.searchsorted(srt.values, ar).to(torch.int32), srt.indices.to(torch.int32)

        own_ptr, own = lists(own_t)  # every face a cell owns, increasing face index
        nei_ptr, nei_i = lists(N_t)  # interior faces by neighbour, increasing index
        nei = if_t[nei_i.long()].contiguous()
        pi_ptr, pi = lists(P_t)  # interior faces (interior index) by owner
        pb_ptr, pb = lists(Pb_t)  # boundary faces (boundary index) by owner
        fc, S = f64(nf_all, dim), f64(nf_all, dim)
        cnt = torch.zeros(8, dtype=torch.int32, device=dev)
        _lib.check(L.b2s_face_geometry_d(dim, nf_all, X.data_ptr(), fptr.data_ptr(), fnodes.data_ptr(), fc.data_ptr(),
                                         S.data_ptr(), cnt.data_ptr(), sp_), "b2s_face_geometry_d")
        ca, vol, xc = f64(nc, dim), f64(nc), f64(nc, dim)
        _lib.check(L.b2s_cell_geometry_d(dim, nc, nf_all, own_t.data_ptr(), nei_t.data_ptr(), own_ptr.data_ptr(),
                                         own.data_ptr(), nei_ptr.data_ptr(), nei.data_ptr(), fc.data_ptr(), S.data_ptr(),
                                         ca.data_ptr(), vol.data_ptr(), xc.data_ptr(), cnt[1:].data_ptr(), sp_),
                   "b2s_cell_geometry_d")
        o = {k: f64(n_if, dim) for k in ("d", "Tv", "dPf", "dNf", "dxm")}
        o.update({k: f64(max(n_if, 1)) for k in ("w", "alpha", "wl")})
        o.update({k: f64(n_bf, dim) for k in ("db", "nbv", "dbt")})
        o.update({k: f64(max(n_bf, 1)) for k in ("alpha_b", "wlb", "Sb_mag", "yb")})
        cmin = f64(1)
        _lib.check(L.b2s_fv_faces_d(dim, n_if, if_t.data_ptr(), P_t.data_ptr(), N_t.data_ptr(), n_bf, bf_t.data_ptr(),
                                    Pb_t.data_ptr(), xc.data_ptr(), fc.data_ptr(), S.data_ptr(),
                                    *[o[k].data_ptr() for k in ("d", "w", "alpha", "wl", "Tv", "dPf", "dNf", "dxm",
                                                                "db", "alpha_b", "wlb", "Sb_mag", "nbv", "dbt", "yb")],
                                    cmin.data_ptr(), sp_), "b2s_fv_faces_d")
        G, Ginv = f64(nc, dim, dim), f64(nc, dim, dim)
        flag = torch.empty(nc, dtype=torch.int32, device=dev)
        _lib.check(L.b2s_ls_matrices_d(dim, nc, pi_ptr.data_ptr(), pi.data_ptr(), nei_ptr.data_ptr(), nei_i.data_ptr(),
                                       pb_ptr.data_ptr(), pb.data_ptr(), o["d"].data_ptr(), o["wl"].data_ptr(),
                                       o["db"].data_ptr(), o["wlb"].data_ptr(), G.data_ptr(), Ginv.data_ptr(),
                                       flag.data_ptr(), sp_), "b2s_ls_matrices_d")
        nflag = flag.sum(dtype=torch.int32).reshape(1)
        chk = torch.cat([cnt[:3], nflag]).cpu().numpy()  # bad faces, flipped, non-positive volumes, singular G
        if chk[0]:
            raise ValueError("2-D meshes must have 2-node faces" if dim == 2 else "a face has fewer than 3 or more "
                             "than 32 nodes")
        if chk[2]:
            raise ValueError(f"{int(chk[2])} cells have non-positive volume")
        if chk[3]:  # singular least-squares matrices: the pseudo-inverse, as the reference
            bad = torch.nonzero(flag).flatten()
            Ginv[bad] = torch.as_tensor(np.linalg.pinv(G[bad].cpu().numpy()), device=dev)
        cm = float(cmin.item()) if n_if else 1.0
        self.flipped_faces = int(chk[1])
        Sif, Sbf = S[if_t.long()], S[bf_t.long()]
        return {"dim": dim, "nc": nc, "P": P, "N": N, "Pb": Pb, "bzone": np.asarray(mesh.face_zone)[bf_idx],
                "non_orthogonality_deg": float(np.degrees(np.arccos(cm))) if n_if else 0.0,
                "w": o["w"][:n_if], "alpha": o["alpha"][:n_if], "wl": o["wl"][:n_if], "S": Sif, "d": o["d"],
                "Tv": o["Tv"], "dxm": o["dxm"], "dPf": o["dPf"], "dNf": o["dNf"], "alpha_b": o["alpha_b"][:n_bf],
                "wlb": o["wlb"][:n_bf], "Sb_mag": o["Sb_mag"][:n_bf], "Sb": Sbf, "db": o["db"], "nbv": o["nbv"],
                "dbt": o["dbt"], "vol": vol, "Ginv": Ginv, "xc": xc, "yb": o["yb"][:n_bf], "xfb": fc[bf_t.long()]}

    def _layout(self, r, reorder, groups):
        """The device layout (module docstring) of reference-numbered quantities ``r``: the cell
        order, the face orders, the CSR pattern and its slot maps, SoA device tensors."""
        import torch

        dev = self.device
        dim, nc = r["dim"], r["nc"]
        P, N, Pb = r["P"], r["N"], r["Pb"]
        nf, nb = P.size, Pb.size
        self.dim, self.nc, self.n_if, self.n_bf = dim, nc, nf, nb
        self.non_orthogonality_deg = r["non_orthogonality_deg"]
        self.bzone = r["bzone"]
        self._ref = r
        L64 = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.int64), device=dev)  # noqa: E731
        P_t, N_t, Pb_t = L64(P), L64(N), L64(Pb)
        ar = torch.arange(nc + 1, device=dev)
        # ---- cell order: reverse Cuthill-McKee (SciPy, host) of the cell adjacency, whose sorted
        # CSR is built from distinct keys on the device
        if reorder and nf:
            akeys = torch.unique(torch.cat([P_t * nc + N_t, N_t * nc + P_t]), sorted=True)
            adj = sp.csr_matrix((np.ones(akeys.numel(), dtype=np.int8), (akeys % nc).cpu().numpy(),
                                 torch.searchsorted(akeys // nc, ar).cpu().numpy()), shape=(nc, nc))
            perm = np.asarray(reverse_cuthill_mckee(adj, symmetric_mode=True), dtype=np.int64)
        else:
            perm = np.arange(nc, dtype=np.int64)
        if groups is not None:
            groups = np.asarray(groups)
            perm = perm[np.argsort(groups[perm], kind="stable")]
        iperm = np.empty(nc, dtype=np.int64)
        iperm[perm] = np.arange(nc)
        self.perm, self.iperm = perm, iperm  # device -> reference, reference -> device
        perm_t, iperm_t = L64(perm), L64(iperm)
        self.h2d_bytes += 8 * (2 * nc + 2 * nf + nb)
        # ---- interior faces by (device owner, reference index); faces by neighbour
        Pn, Nn = iperm_t[P_t], iperm_t[N_t]
        forder = torch.sort(Pn, stable=True).indices
        fP, fN = Pn[forder], Nn[forder]
        own_ptr = torch.searchsorted(fP, ar)
        norder = torch.argsort(fN * max(nf, 1) + forder)
        nei_ptr = torch.searchsorted(fN[norder], ar)
        # ---- boundary faces by (device owner, reference index)
        bPn = iperm_t[Pb_t]
        border = torch.sort(bPn, stable=True).indices
        bP = bPn[border]
        bptr = torch.searchsorted(bP, ar)
        # ---- the CSR pattern in the reference's numbering, then its rows in device order
        dg = torch.arange(nc, device=dev)
        keys = torch.unique(torch.cat([dg * nc + dg, P_t * nc + N_t, N_t * nc + P_t]), sorted=True)
        nnz = keys.numel()
        r_indptr = torch.searchsorted(keys // nc, ar)
        r_indices = keys % nc
        slot_diag = torch.searchsorted(keys, dg * nc + dg)
        slot_PN = torch.searchsorted(keys, P_t * nc + N_t)
        slot_NP = torch.searchsorted(keys, N_t * nc + P_t)
        rl = r_indptr[1:] - r_indptr[:-1]
        rlp = rl[perm_t]
        rowptr = torch.zeros(nc + 1, dtype=torch.int64, device=dev)
        rowptr[1:] = torch.cumsum(rlp, 0)
        src = torch.repeat_interleave(r_indptr[:-1][perm_t] - rowptr[:-1], rlp, output_size=nnz) + torch.arange(
            nnz, device=dev)  # device slot -> reference slot
        col = iperm_t[r_indices[src]]
        slot_new = torch.empty(nnz, dtype=torch.int64, device=dev)
        slot_new[src] = torch.arange(nnz, device=dev)  # reference slot -> device slot
        per_cell = (torch.bincount(P_t, minlength=nc) + torch.bincount(N_t, minlength=nc)
                    + torch.bincount(Pb_t, minlength=nc))
        spn = torch.sort(slot_PN).values
        dup = (spn[1:] == spn[:-1]).any() if nf > 1 else torch.zeros((), dtype=torch.bool, device=dev)
        stats = torch.stack([rl.max() if nc else torch.zeros((), dtype=torch.int64, device=dev),
                             per_cell.max() if nc else torch.zeros((), dtype=torch.int64, device=dev),
                             dup.to(torch.int64)]).cpu().numpy()
        self.nnz = int(nnz)
        if max(nc, nf, nb, self.nnz) >= 2 ** 31 - 1:
            raise ValueError("mesh too large for 32-bit indices")
        self.duplicate_pairs = bool(stats[2])
        if self.duplicate_pairs:
            raise NotImplementedError("meshes with two faces joining the same pair of cells are not supported")
        self._ref_csr = (r_indptr, r_indices)
        self.bface_ref = border.cpu().numpy()  # device boundary face -> reference boundary face
        self._maps = {"face_ref": forder, "slot_ref": src}  # host copies made on first use
        # ---- device tensors
        i32 = lambda t: t.to(torch.int32).contiguous()  # noqa: E731
        soa = lambda t: t.t().contiguous()  # (n, k) -> [k][n]  # noqa: E731
        t = self.t = {}
        t["fP"], t["fN"], t["forig"] = i32(fP), i32(fN), i32(forder)
        t["own_ptr"], t["nei_ptr"], t["nei_face"] = i32(own_ptr), i32(nei_ptr), i32(norder)
        t["bP"], t["bptr"] = i32(bP), i32(bptr)
        t["w"], t["alpha"], t["wl"] = r["w"][forder].contiguous(), r["alpha"][forder].contiguous(), r["wl"][forder].contiguous()
        for name in ("S", "d", "Tv", "dxm", "dPf", "dNf"):
            t[name] = soa(r[name][forder])
        for name in ("alpha_b", "wlb", "Sb_mag"):
            t[name] = r[name][border].contiguous()
        for name in ("Sb", "db", "nbv", "dbt"):
            t[name] = soa(r[name][border])
        t["vol"] = r["vol"][perm_t].contiguous()
        t["Ginv"] = r["Ginv"][perm_t].reshape(nc, dim * dim).t().contiguous()
        t["rowptr"], t["col"] = i32(rowptr), i32(col)
        t["slot_diag"] = i32(slot_new[slot_diag[perm_t]])
        t["slot_PN"] = i32(slot_new[slot_PN[forder]])
        t["slot_NP"] = i32(slot_new[slot_NP[forder]])
        for k, v in list(t.items()):
            if v.numel() == 0:  # a mesh without interior or boundary faces: keep valid pointers
                t[k] = torch.zeros(1, dtype=v.dtype, device=dev)
        self.vol = t["vol"]
        self.rowptr, self.col = t["rowptr"], t["col"]
        self.cmesh = _lib.Mesh(nc=nc, nf=nf, nb=nb, dim=dim, nnz=self.nnz,
                               **{k: v.data_ptr() for k, v in t.items()})
        self.cmesh_ref = ctypes.byref(self.cmesh)
        self.row_terms_max = int(stats[0]) + 1 if nc else 1
        self.cell_faces_max = int(stats[1]) if nc else 1

    @property
    def face_ref(self):
        """Device interior face -> reference interior face (host array)."""
        m = self._maps["face_ref"]
        if not isinstance(m, np.ndarray):
            m = self._maps["face_ref"] = m.cpu().numpy()
        return m

    @property
    def slot_ref(self):
        """Device CSR slot -> reference CSR slot (host array)."""
        m = self._maps["slot_ref"]
        if not isinstance(m, np.ndarray):
            m = self._maps["slot_ref"] = m.cpu().numpy()
        return m

    def boundary_centres_host(self):
        """Boundary-face centres, (nb, dim), reference order."""
        x = self._ref["xfb"]
        return x.detach().cpu().numpy() if hasattr(x, "detach") else np.asarray(x)

    def boundary_normals_host(self):
        """Unit outward normals of the boundary faces, (nb, dim), reference order."""
        nbv = self._ref["nbv"]
        return nbv.detach().cpu().numpy() if hasattr(nbv, "detach") else np.asarray(nbv)

    # ---- conversions between the reference's and the device's numbering ------------------------------
    def cells_to_device(self, a):
        """(nc, ...) host array in reference order -> device SoA tensor [...][nc]."""
        import torch

        a = np.asarray(a, dtype=np.float64)[self.perm]
        return torch.as_tensor(np.ascontiguousarray(a.T if a.ndim > 1 else a), device=self.device)

    def set_tiling(self, tiles) -> None:
        """Tile the cells (``b2s_mesh.tiles``): tiles[t] .. tiles[t+1]-1 are the cells of tile t,
        at most 256 each, in device numbering; the partial-sum stages then give one partial per
        tile."""
        import torch

        tiles = np.asarray(tiles, dtype=np.int64)
        if tiles[0] != 0 or tiles[-1] != self.nc or np.any(np.diff(tiles) <= 0) or np.any(np.diff(tiles) > 256):
            raise ValueError("invalid tiling")
        self.t["tiles"] = torch.as_tensor(tiles.astype(np.int32), device=self.device)
        self.cmesh.tiles = self.t["tiles"].data_ptr()
        self.cmesh.ntiles = int(tiles.size - 1)

    def cells_to_host(self, t):
        """Device SoA tensor [...][nc] -> (nc, ...) host array in reference order."""
        a = t.detach().double().cpu().numpy()
        a = a.reshape(-1, self.nc).T if a.ndim > 1 else a
        out = np.empty_like(a)
        out[self.perm] = a
        return out

    def faces_to_host(self, t):
        a = t.detach().double().cpu().numpy()
        out = np.empty_like(a)
        out[self.face_ref] = a
        return out

    def faces_to_device(self, a):
        import torch

        return torch.as_tensor(np.ascontiguousarray(np.asarray(a, dtype=np.float64)[self.face_ref]), device=self.device)

    def bfaces_to_host(self, t):
        """Device SoA tensor [...][nb] -> (nb, ...) host array in reference order."""
        a = t.detach().double().cpu().numpy()
        a = a.reshape(-1, self.n_bf).T if a.ndim > 1 else a
        out = np.empty_like(a)
        out[self.bface_ref] = a
        return out

    def bfaces_to_device(self, a):
        import torch

        a = np.asarray(a, dtype=np.float64)[self.bface_ref]
        return torch.as_tensor(np.ascontiguousarray(a.T if a.ndim > 1 else a), device=self.device)

    def matrix_to_host(self, val):
        """CSR values of a device matrix -> SciPy CSR in the reference's numbering."""
        if not hasattr(self, "_ref_csr_host"):
            ip, ix = self._ref_csr
            self._ref_csr_host = (ip.cpu().numpy(), ix.cpu().numpy())
        indptr, indices = self._ref_csr_host
        v = val.detach().double().cpu().numpy()
        data = np.empty(self.nnz)
        data[self.slot_ref] = v
        return sp.csr_matrix((data, indices, indptr), shape=(self.nc, self.nc))

    # ---- operators (device in, device out), mirroring flowtrace.unstructured.fvmesh.FVMesh ------------
    def _stream(self):
        return _lib.stream_ptr()

    def face_interp(self, phi):
        """w phi_P + (1 - w) phi_N; phi [k][nc] or [nc] (``fvmesh.py:318-330``)."""
        import torch

        k = 1 if phi.dim() == 1 else phi.shape[0]
        out = torch.empty((self.n_if,) if phi.dim() == 1 else (k, self.n_if), dtype=torch.float64, device=self.device)
        _lib.check(_lib.lib().b2s_face_interp_d(self.cmesh_ref, k, phi.contiguous().data_ptr(), out.data_ptr(),
                                                self._stream()), "b2s_face_interp_d")
        return out

    def gradient(self, phi, phi_b):
        """Least-squares gradients; phi [k][nc] or [nc], phi_b [k][nb] or [nb]; out [k][dim][nc]
        or [dim][nc] (``fvmesh.py:268-286``)."""
        import torch

        k = 1 if phi.dim() == 1 else phi.shape[0]
        out = torch.empty((k, self.dim, self.nc), dtype=torch.float64, device=self.device)
        _lib.check(_lib.lib().b2s_ls_gradient_d(self.cmesh_ref, k, phi.contiguous().data_ptr(),
                                                phi_b.contiguous().data_ptr(), out.data_ptr(), self._stream()),
                   "b2s_ls_gradient_d")
        return out[0] if phi.dim() == 1 else out

    def gradient_gg(self, phi, phi_b, grad=None):
        """Green-Gauss gradient with skewness correction (``fvmesh.py:288-309``); out [dim][nc]."""
        import torch

        out = torch.empty((self.dim, self.nc), dtype=torch.float64, device=self.device)
        _lib.check(_lib.lib().b2s_gg_gradient_d(self.cmesh_ref, phi.contiguous().data_ptr(),
                                                phi_b.contiguous().data_ptr(),
                                                None if grad is None else grad.contiguous().data_ptr(),
                                                out.data_ptr(), self._stream()), "b2s_gg_gradient_d")
        return out

    def matrix_values(self, diag, a_PN, a_NP):
        """CSR values from the diagonal and face coefficients (``fvmesh.py:332-348``)."""
        import torch

        val = torch.empty(self.nnz, dtype=torch.float64, device=self.device)
        _lib.check(_lib.lib().b2s_assemble_d(self.cmesh_ref, diag.contiguous().data_ptr(),
                                             a_PN.contiguous().data_ptr(), a_NP.contiguous().data_ptr(),
                                             val.data_ptr(), self._stream()), "b2s_assemble_d")
        return val

    def spmv(self, val, x):
        """A x for x [k][nc] or [nc] with the mesh's CSR pattern."""
        import torch

        k = 1 if x.dim() == 1 else x.shape[0]
        y = torch.empty_like(x, dtype=torch.float64)
        _lib.check(_lib.lib().b2s_spmv_d(self.nc, k, self.rowptr.data_ptr(), self.col.data_ptr(), val.data_ptr(),
                                         x.contiguous().data_ptr(), y.data_ptr(), self._stream()), "b2s_spmv_d")
        return y
