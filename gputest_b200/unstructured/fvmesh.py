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

    def __init__(self, mesh: UnstructuredMesh, device=None, reorder: bool = True, groups=None):
        """``groups`` (one label per cell, optional): cells of one group are kept contiguous in the
        device order, groups in increasing label order (the reverse Cuthill-McKee order within
        each) - the layout of a block-diagonal batch of independent cases."""
        import torch

        self.device = device if device is not None else _lib.require_device()
        h = self.host = HostFV(mesh)
        self.mesh = mesh
        self.dim, self.nc, self.n_if, self.n_bf, self.nnz = h.dim, h.nc, h.n_if, h.n_bf, h.nnz
        self.non_orthogonality_deg = h.non_orthogonality_deg
        self.geometry = h.geometry
        nc, nf, nb, dim = h.nc, h.n_if, h.n_bf, h.dim
        if max(nc, nf, nb, h.nnz) >= 2 ** 31 - 1:
            raise ValueError("mesh too large for 32-bit indices")
        # ---- cell order: reverse Cuthill-McKee of the cell adjacency
        if reorder and nf:
            adj = sp.csr_matrix((np.ones(2 * nf, dtype=np.int8), (np.concatenate([h.P, h.N]),
                                                                   np.concatenate([h.N, h.P]))), shape=(nc, nc))
            perm = np.asarray(reverse_cuthill_mckee(adj, symmetric_mode=True), dtype=np.int64)
        else:
            perm = np.arange(nc, dtype=np.int64)
        if groups is not None:
            groups = np.asarray(groups)
            perm = perm[np.argsort(groups[perm], kind="stable")]
        iperm = np.empty(nc, dtype=np.int64)
        iperm[perm] = np.arange(nc)
        self.perm, self.iperm = perm, iperm  # device -> reference, reference -> device
        # ---- interior faces by (device owner, reference index)
        Pn, Nn = iperm[h.P], iperm[h.N]
        forder = np.lexsort((np.arange(nf), Pn))
        self.face_ref = forder  # device face -> reference interior face
        fP, fN = Pn[forder], Nn[forder]
        own_ptr = np.concatenate([[0], np.cumsum(np.bincount(fP, minlength=nc))])
        norder = np.lexsort((forder, fN))  # device faces grouped by neighbour, by reference index
        nei_ptr = np.concatenate([[0], np.cumsum(np.bincount(fN, minlength=nc))])
        # ---- boundary faces by (device owner, reference index)
        bPn = iperm[h.Pb]
        border = np.lexsort((np.arange(nb), bPn))
        self.bface_ref = border  # device boundary face -> reference boundary face
        bP = bPn[border]
        bptr = np.concatenate([[0], np.cumsum(np.bincount(bP, minlength=nc))])
        # ---- CSR rows in device order, each keeping the reference's column order
        rl = np.diff(h.indptr)
        rowptr = np.concatenate([[0], np.cumsum(rl[perm])])
        src = np.repeat(h.indptr[:-1][perm] - rowptr[:-1], rl[perm]) + np.arange(h.nnz)  # device slot -> ref slot
        col = iperm[h.indices[src]]
        slot_new = np.empty(h.nnz, dtype=np.int64)
        slot_new[src] = np.arange(h.nnz)  # reference slot -> device slot
        self.slot_ref = src
        self.duplicate_pairs = h.duplicate_pairs
        if h.duplicate_pairs:
            raise NotImplementedError("meshes with two faces joining the same pair of cells are not supported")
        # ---- device tensors
        dev = self.device
        i32 = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.int32), device=dev)  # noqa: E731
        f64 = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=dev)  # noqa: E731
        soa = lambda a: f64(np.ascontiguousarray(np.asarray(a).T))  # (n, k) -> [k][n]  # noqa: E731
        t = self.t = {}
        t["fP"], t["fN"], t["forig"] = i32(fP), i32(fN), i32(forder)
        t["own_ptr"], t["nei_ptr"], t["nei_face"] = i32(own_ptr), i32(nei_ptr), i32(norder)
        t["bP"], t["bptr"] = i32(bP), i32(bptr)
        t["w"], t["alpha"], t["wl"] = f64(h.w[forder]), f64(h.alpha[forder]), f64(h.wl[forder])
        for name, arr in (("S", h.S), ("d", h.d), ("Tv", h.Tvec), ("dxm", h.dxm), ("dPf", h.dP_f), ("dNf", h.dN_f)):
            t[name] = soa(arr[forder])
        t["alpha_b"], t["wlb"], t["Sb_mag"] = f64(h.alpha_b[border]), f64(h.wlb[border]), f64(h.Sb_mag[border])
        for name, arr in (("Sb", h.Sb), ("db", h.db), ("nbv", h.nb), ("dbt", h.db_t)):
            t[name] = soa(arr[border])
        t["vol"] = f64(h.vol[perm])
        t["Ginv"] = f64(np.ascontiguousarray(h.Ginv[perm].reshape(nc, dim * dim).T))
        t["rowptr"], t["col"] = i32(rowptr), i32(col)
        t["slot_diag"] = i32(slot_new[h.slot_diag[perm]])
        t["slot_PN"] = i32(slot_new[h.slot_PN[forder]])
        t["slot_NP"] = i32(slot_new[h.slot_NP[forder]])
        self.vol = t["vol"]
        self.rowptr, self.col = t["rowptr"], t["col"]
        self.cmesh = _lib.Mesh(nc=nc, nf=nf, nb=nb, dim=dim, nnz=h.nnz,
                               **{k: v.data_ptr() for k, v in t.items()})
        self.cmesh_ref = ctypes.byref(self.cmesh)
        self.row_terms_max = int(rl.max()) + 1 if nc else 1
        per_cell = np.bincount(h.P, minlength=nc) + np.bincount(h.N, minlength=nc) + np.bincount(h.Pb, minlength=nc)
        self.cell_faces_max = int(per_cell.max()) if nc else 1

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
        h = self.host
        v = val.detach().double().cpu().numpy()
        data = np.empty(h.nnz)
        data[self.slot_ref] = v
        return sp.csr_matrix((data, h.indices, h.indptr), shape=(h.nc, h.nc))

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
