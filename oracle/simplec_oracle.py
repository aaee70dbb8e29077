"""ORACLE — test infrastructure only. Never imported by the product (``gputest_b200``).

A CPU restatement, in NumPy/SciPy, of FlowTrace's unstructured SIMPLEC outer iteration:
finite-volume operators, the Jacobi-BiCGSTAB and AMG-PCG linear solves, the smoothed-
aggregation AMG and ``SimpleSolver.step``. It is the checker of the CUDA path in
``tests/``, the CPU baseline of ``bench.py`` and the reference of ``__graft_entry__.smoke``.

Every function cites the reference file:line it follows; the operations are written in the
same order as the reference's NumPy path so that results agree with it to round-off.
Pinned against the reference itself: ``tests/golden/make_golden.py`` runs the reference
(when it is importable) and this oracle side by side and stores the reference's outputs
as fixtures; ``tests/test_oracle_golden.py`` re-checks the oracle against them.

Scope: steady laminar flow (SIMPLE/SIMPLEC), energy with adiabatic/temperature/flux walls,
upwind and bounded second-order convection, Green-Gauss or least-squares pressure force,
uniform body force and per-cell momentum/energy sources, the divergence guard, and the
k-omega SST model (``oracle/sst_oracle.py``: face viscosities with Spalding's wall law,
transpose stress, turbulent energy diffusivity, the k and omega transport solves). Two
features the reference lacks are added the way its test harness would add them:
a per-cell Brinkman drag ``alpha V`` on the momentum diagonal, and a per-face boundary
velocity profile written into ``ub_fixed`` (followed by ``initialize({})``).

Optionally (``native=``) the operators call the reference's own C++ kernels compiled from
its sources into ``oracle/_ref`` (see ``oracle/Makefile``), exactly as the reference's
native CPU path does (``flowtrace/unstructured/fvmesh.py:232-346``).
"""

from __future__ import annotations

import ctypes
import math
import os
from collections import defaultdict
from dataclasses import dataclass
from typing import Callable, Dict, Optional

import numpy as np
import scipy.sparse as sp

HERE = os.path.dirname(os.path.abspath(__file__))
WALL, INLET, OUTLET, PRESSURE, SYMMETRY = range(5)
T_ADIABATIC, T_FIXED, T_FLUX = range(3)
_KIND_CODE = {"wall": WALL, "inlet": INLET, "outlet": OUTLET, "pressure": PRESSURE, "symmetry": SYMMETRY}
FLUENT_TO_KIND = {"wall": "wall", "velocity-inlet": "inlet", "mass-flow-inlet": "inlet", "pressure-inlet": "pressure",
                  "pressure-outlet": "outlet", "outflow": "outlet", "pressure-far-field": "outlet",
                  "outlet-vent": "outlet", "exhaust-fan": "outlet", "inlet-vent": "pressure", "intake-fan": "pressure",
                  "symmetry": "symmetry", "axis": "symmetry"}


# ------------------------------------------------------------------------------------------- geometry
def _face_geometry(mesh):
    """``flowtrace/mesh/unstructured.py:171-212``."""
    X, ptr, fn, dim = mesh.nodes, mesh.face_ptr, mesh.face_nodes, mesh.dim
    nf = mesh.owner.shape[0]
    if dim == 2:
        a = X[fn[ptr[:-1]]]
        b = X[fn[ptr[:-1] + 1]]
        d = b - a
        return 0.5 * (a + b), np.stack([d[:, 1], -d[:, 0]], axis=1)
    fc, S = np.zeros((nf, dim)), np.zeros((nf, dim))
    counts = np.diff(ptr)
    for k in np.unique(counts):
        idx = np.nonzero(counts == k)[0]
        nodes = fn[ptr[idx][:, None] + np.arange(k)[None, :]]
        P = X[nodes]
        xc = P.mean(axis=1)
        Pn = np.roll(P, -1, axis=1)
        tri = 0.5 * np.cross(P - xc[:, None, :], Pn - xc[:, None, :])
        Sk = tri.sum(axis=1)
        nhat = Sk / np.maximum(np.linalg.norm(Sk, axis=1, keepdims=True), 1e-300)
        w = np.einsum("mkd,md->mk", tri, nhat)
        cent = (xc[:, None, :] + P + Pn) / 3.0
        wsum = w.sum(axis=1, keepdims=True)
        fc[idx] = (w[:, :, None] * cent).sum(axis=1) / np.where(np.abs(wsum) > 0, wsum, 1.0)
        S[idx] = Sk
    return fc, S


def compute_geometry(mesh):
    """Face centres/areas, repaired orientation, cell volumes and centroids
    (``flowtrace/mesh/unstructured.py:215-261``). Returns (fc, S, cc, vol)."""
    dim, nc = mesh.dim, mesh.n_cells
    own, nei = mesh.owner, mesh.neighbour
    interior = nei >= 0
    fc, S = _face_geometry(mesh)
    cnt = np.bincount(own, minlength=nc) + np.bincount(nei[interior], minlength=nc)
    ca = np.zeros((nc, dim))
    for d in range(dim):
        ca[:, d] = np.bincount(own, fc[:, d], minlength=nc) + np.bincount(nei[interior], fc[interior, d], minlength=nc)
    ca /= np.maximum(cnt, 1)[:, None]
    ref = np.where(interior[:, None], ca[np.where(interior, nei, 0)] - ca[own], fc - ca[own])
    bad = np.einsum("fd,fd->f", S, ref) < 0
    S[bad] *= -1.0
    vol = np.zeros(nc)
    mom = np.zeros((nc, dim))
    frac = 2.0 / 3.0 if dim == 2 else 0.75
    for cells, sign, faces in ((own, 1.0, slice(None)), (nei[interior], -1.0, np.nonzero(interior)[0])):
        h = fc[faces] - ca[cells]
        v = np.einsum("fd,fd->f", S[faces] * sign, h) / dim
        vc = (v[:, None] * (ca[cells] + frac * h)).T
        vol += np.bincount(cells, v, minlength=nc)
        for d in range(dim):
            mom[:, d] += np.bincount(cells, vc[d], minlength=nc)
    return fc, S, mom / vol[:, None], vol


def _batched_inverse(G):
    """``flowtrace/unstructured/fvmesh.py:25-39``."""
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


# ------------------------------------------------------------------------------------------- native
def load_native(path: Optional[str] = None):
    """The reference's C++ kernels compiled from its sources (``oracle/_ref``), bound with the
    signatures of ``flowtrace/native/__init__.py:97-113``; None when the library is absent."""
    path = path or os.path.join(HERE, "_ref", "libft_ref.so")
    if not os.path.exists(path):
        return None
    lib = ctypes.CDLL(path)
    P, I64, I = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int
    sig = {"ft_abi_version": ([], I), "ft_max_threads": ([], I), "ft_csr_spmm": ([I64, I64] + [P] * 5, None),
           "ft_face_interp": ([I64, I64] + [P] * 5, None), "ft_ls_gradient": ([I64, I64] + [P] * 14, None),
           "ft_gg_gradient": ([I64, I64] + [P] * 16, None), "ft_assemble": ([I64, I64, I64] + [P] * 7, None),
           "ft_bicgstab_jacobi": ([I64, P, P, P, P, P, P, ctypes.c_double, I64, I, P, P, P], I)}
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes, fn.restype = args, res
    return lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class _NativeCSR:
    """CSR matrix whose ``@`` runs ``ft_csr_spmm`` (``flowtrace/native/__init__.py:178-217``)."""

    def __init__(self, lib, data, indices, indptr, shape):
        self.lib = lib
        self.data = np.ascontiguousarray(data, dtype=np.float64)
        self.indices = np.ascontiguousarray(indices, dtype=np.int32)
        self.indptr = np.ascontiguousarray(indptr, dtype=np.int32)
        self.shape = shape
        self.csr = sp.csr_matrix((self.data, self.indices, self.indptr), shape=shape)

    def __matmul__(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        k = 1 if x.ndim == 1 else x.shape[1]
        y = np.empty((self.shape[0],) if x.ndim == 1 else (self.shape[0], k))
        self.lib.ft_csr_spmm(self.shape[0], k, _p(self.indptr), _p(self.indices), _p(self.data), _p(x), _p(y))
        return y

    def diagonal(self):
        return self.csr.diagonal()

    def toarray(self):
        return self.csr.toarray()


# ------------------------------------------------------------------------------------------- FV mesh
class OracleFV:
    """Finite-volume data of a mesh (``flowtrace/unstructured/fvmesh.py:60-356``)."""

    def __init__(self, mesh, native=None):
        if getattr(mesh, "periodic", None):
            raise NotImplementedError("periodic meshes are outside the oracle's scope")
        self.mesh = mesh
        self.dim = dim = mesh.dim
        fc, Sall, xc, vol = compute_geometry(mesh)
        self.nc = nc = mesh.n_cells
        interior = mesh.neighbour >= 0
        boundary = ~interior
        self.if_idx = np.nonzero(interior)[0]
        self.bf_idx = np.nonzero(boundary)[0]
        P = mesh.owner[interior].astype(np.int64)
        N = mesh.neighbour[interior].astype(np.int64)
        Pb = mesh.owner[boundary].astype(np.int64)
        self.n_if, self.n_bf = P.size, Pb.size
        S, Sb = Sall[interior], Sall[boundary]
        xf, xfb = fc[interior], fc[boundary]
        xN = xc[N]
        d = xN - xc[P]                                                        # fvmesh.py:109
        db = xfb - xc[Pb]
        dd = np.einsum("fd,fd->f", d, d)
        w = np.clip(np.einsum("fd,fd->f", xN - xf, d) / dd, 0.0, 1.0)         # fvmesh.py:112
        Sd = np.einsum("fd,fd->f", S, d)
        Sdb = np.einsum("fd,fd->f", Sb, db)
        SS = np.einsum("fd,fd->f", S, S)
        SSb = np.einsum("fd,fd->f", Sb, Sb)
        alpha, alpha_b = SS / Sd, SSb / Sdb                                   # fvmesh.py:117-118
        Tvec = S - alpha[:, None] * d
        self.non_orthogonality_deg = float(np.degrees(np.arccos(np.clip(Sd / np.sqrt(SS * dd), -1, 1))).max()) \
            if P.size else 0.0
        wl = 1.0 / dd                                                         # fvmesh.py:124-136
        wlb = 1.0 / np.einsum("fd,fd->f", db, db)
        Gm = np.zeros((nc, dim, dim))
        for a in range(dim):
            for b in range(a, dim):
                o = wl * d[:, a] * d[:, b]
                Gm[:, a, b] = (np.bincount(P, o, minlength=nc) + np.bincount(N, o, minlength=nc)
                               + np.bincount(Pb, wlb * db[:, a] * db[:, b], minlength=nc))
                Gm[:, b, a] = Gm[:, a, b]
        Ginv = _batched_inverse(Gm)
        ones = np.ones(P.size)
        self.Cown = sp.csr_matrix((ones, (P, np.arange(P.size))), shape=(nc, P.size))       # fvmesh.py:140-145
        self.Cnei = sp.csr_matrix((ones, (N, np.arange(N.size))), shape=(nc, N.size))
        self.Cb = sp.csr_matrix((np.ones(Pb.size), (Pb, np.arange(Pb.size))), shape=(nc, Pb.size))
        self.Cdiff = (self.Cown - self.Cnei).tocsr()
        rows = np.concatenate([np.arange(nc), P, N])                          # fvmesh.py:148-162
        cols = np.concatenate([np.arange(nc), N, P])
        pat = sp.csr_matrix((np.ones(rows.size, dtype=np.int8), (rows, cols)), shape=(nc, nc))
        pat.sum_duplicates()
        pat.sort_indices()
        row_of = np.repeat(np.arange(nc), np.diff(pat.indptr))
        keys = row_of.astype(np.int64) * nc + pat.indices
        self.nnz = pat.nnz
        self.slot_diag = np.searchsorted(keys, np.arange(nc, dtype=np.int64) * nc + np.arange(nc)).astype(np.int32)
        self.slot_PN = np.searchsorted(keys, P * nc + N).astype(np.int32)
        self.slot_NP = np.searchsorted(keys, N * nc + P).astype(np.int32)
        self.indptr, self.indices = pat.indptr.astype(np.int32), pat.indices.astype(np.int32)
        self.bzone = mesh.face_zone[boundary]
        self.P, self.N, self.Pb = P, N, Pb
        self.S, self.Sb, self.d, self.db, self.w = S, Sb, d, db, w
        self.alpha, self.alpha_b, self.Tvec = alpha, alpha_b, Tvec
        self.Sb_mag = np.sqrt(SSb)
        self.nb = Sb / np.sqrt(SSb)[:, None]
        self.db_t = db - np.einsum("fd,fd->f", db, self.nb)[:, None] * self.nb
        self.vol, self.xc, self.xfb = vol, xc, xfb
        self.face_centre, self.face_area_vec = fc, Sall
        self.yb = np.abs(np.einsum("fd,fd->f", db, Sb)) / np.sqrt(SSb)
        self.wl, self.wlb, self.Ginv = wl, wlb, Ginv
        self.dP_f = xf - xc[P]
        self.dN_f = xf - xN
        self.dxm = xf - (w[:, None] * xc[P] + (1.0 - w)[:, None] * xN)      # fvmesh.py:191
        self.cell_centre = xc
        self.lib = native
        if native is not None:
            cd, cb = self.Cdiff, self.Cb
            cd.sort_indices()
            cb.sort_indices()
            self._n = {"iptr": cd.indptr.astype(np.int32), "iidx": cd.indices.astype(np.int32),
                       "isgn": np.ascontiguousarray(cd.data, dtype=np.float64),
                       "bptr": cb.indptr.astype(np.int32), "bidx": cb.indices.astype(np.int32)}
            self._nat = {k: np.ascontiguousarray(v) for k, v in (
                ("P", P), ("N", N), ("w", w), ("wl", wl), ("d", d), ("wlb", wlb), ("db", db), ("Ginv", Ginv),
                ("S", S), ("Sb", Sb), ("vol", vol), ("dxm", self.dxm))}

    # ---- operators -----------------------------------------------------------------------------
    def scatter(self, f_int=None, f_nei=None, f_bnd=None):
        """``fvmesh.py:254-262``."""
        out = None
        for C, v in ((self.Cown, f_int), (self.Cnei, f_nei), (self.Cb, f_bnd)):
            if v is None:
                continue
            t = C @ v
            out = t if out is None else out + t
        return out

    def net_outflow(self, F, Fb):
        """``fvmesh.py:264-266``."""
        return self.Cdiff @ F + self.Cb @ Fb

    def gradient(self, phi, phi_b):
        """Least-squares gradient (``fvmesh.py:268-286``; native ``fvm_kernels.cpp:81-105``)."""
        if self.lib is not None:
            n, a = self._n, self._nat
            phi, phi_b = np.ascontiguousarray(phi, dtype=np.float64), np.ascontiguousarray(phi_b, dtype=np.float64)
            out = np.empty((self.nc, self.dim))
            self.lib.ft_ls_gradient(self.nc, self.dim, _p(n["iptr"]), _p(n["iidx"]), _p(n["bptr"]), _p(n["bidx"]),
                                    _p(a["P"]), _p(a["N"]), _p(a["wl"]), _p(a["d"]), _p(a["wlb"]), _p(a["db"]),
                                    _p(a["Ginv"]), _p(phi), _p(phi_b), _p(out))
            return out
        dphi = phi[self.N] - phi[self.P]
        dphib = phi_b - phi[self.Pb]
        r = (self.Cown @ ((self.wl * dphi)[:, None] * self.d) + self.Cnei @ ((self.wl * dphi)[:, None] * self.d)
             + self.Cb @ ((self.wlb * dphib)[:, None] * self.db))
        return np.einsum("cab,cb->ca", self.Ginv, r)

    def gradient_gg(self, phi, phi_b, grad=None):
        """Green-Gauss gradient with skewness correction (``fvmesh.py:288-309``)."""
        if self.lib is not None:
            n, a = self._n, self._nat
            phi, phi_b = np.ascontiguousarray(phi, dtype=np.float64), np.ascontiguousarray(phi_b, dtype=np.float64)
            g = np.ascontiguousarray(grad, dtype=np.float64) if grad is not None else None
            out = np.empty((self.nc, self.dim))
            self.lib.ft_gg_gradient(self.nc, self.dim, _p(n["iptr"]), _p(n["iidx"]), _p(n["isgn"]), _p(n["bptr"]),
                                    _p(n["bidx"]), _p(a["P"]), _p(a["N"]), _p(a["w"]), _p(a["S"]), _p(a["Sb"]),
                                    _p(a["vol"]), _p(a["dxm"]), _p(phi), _p(phi_b), _p(g) if g is not None else None,
                                    _p(out))
            return out
        pf = self.face_interp(phi)
        if grad is not None:
            pf = pf + np.sum(self.face_interp_vec(grad) * self.dxm, axis=1)
        s = self.Cdiff @ (pf[:, None] * self.S) + self.Cb @ (phi_b[:, None] * self.Sb)
        return s / self.vol[:, None]

    def face_interp(self, phi):
        """``fvmesh.py:318-323``."""
        return self.w * phi[self.P] + (1.0 - self.w) * phi[self.N]

    def face_interp_vec(self, g):
        """``fvmesh.py:325-330``."""
        return self.w[:, None] * g[self.P] + (1.0 - self.w)[:, None] * g[self.N]

    def matrix(self, diag, a_PN, a_NP):
        """CSR with a fixed pattern through the slot maps (``fvmesh.py:332-348``)."""
        if self.lib is not None:
            diag, a_PN, a_NP = (np.ascontiguousarray(v, dtype=np.float64) for v in (diag, a_PN, a_NP))
            data = np.empty(self.nnz)
            self.lib.ft_assemble(self.nnz, self.nc, self.n_if, _p(self.slot_diag), _p(self.slot_PN),
                                 _p(self.slot_NP), _p(diag), _p(a_PN), _p(a_NP), _p(data))
            return _NativeCSR(self.lib, data, self.indices, self.indptr, (self.nc, self.nc))
        data = np.zeros(self.nnz)
        data[self.slot_diag] = diag
        data += np.bincount(self.slot_PN, weights=a_PN, minlength=self.nnz)
        data += np.bincount(self.slot_NP, weights=a_NP, minlength=self.nnz)
        return sp.csr_matrix((data, self.indices, self.indptr), shape=(self.nc, self.nc))

    def matrix_like(self, data):
        """``fvmesh.py:350-356``."""
        return sp.csr_matrix((data, self.indices, self.indptr), shape=(self.nc, self.nc))


# ------------------------------------------------------------------------------------------- Krylov
@dataclass
class KrylovInfo:
    """``flowtrace/linalg/krylov.py:14-18``."""

    iterations: int
    residual: float
    converged: bool


def _dot(a, b):
    return float(np.vdot(a, b).real)


def pcg(A: Callable, b, M: Optional[Callable] = None, x0=None, tol=1e-8, maxiter=500, project=None):
    """Preconditioned CG (``flowtrace/linalg/krylov.py:25-65``)."""
    x = np.zeros_like(b) if x0 is None else x0.copy()
    r = b - A(x) if x0 is not None else b.copy()
    if project is not None:
        r = project(r)
    bnorm = float(np.linalg.norm(b)) or 1.0
    rnorm = float(np.linalg.norm(r))
    if rnorm / bnorm < tol:
        return x, KrylovInfo(0, rnorm / bnorm, True)
    z = M(r) if M is not None else r
    if project is not None:
        z = project(z)
    p = z.copy()
    rz = _dot(r, z)
    for k in range(1, maxiter + 1):
        Ap = A(p)
        pAp = _dot(p, Ap)
        if pAp <= 0.0:
            return x, KrylovInfo(k, rnorm / bnorm, False)
        alpha = rz / pAp
        x += alpha * p
        r -= alpha * Ap
        rnorm = float(np.linalg.norm(r))
        if rnorm / bnorm < tol:
            return x, KrylovInfo(k, rnorm / bnorm, True)
        z = M(r) if M is not None else r
        if project is not None:
            z = project(z)
        rz_new = _dot(r, z)
        if rz == 0.0:
            return x, KrylovInfo(k, rnorm / bnorm, False)
        beta = rz_new / rz
        rz = rz_new
        p = z + beta * p
    return x, KrylovInfo(maxiter, rnorm / bnorm, False)


def bicgstab(A: Callable, b, M: Optional[Callable] = None, x0=None, tol=1e-8, maxiter=500, relative_to_initial=False):
    """Right-preconditioned BiCGSTAB (``flowtrace/linalg/krylov.py:68-121``)."""
    x = np.zeros_like(b) if x0 is None else x0.copy()
    r = b - A(x) if x0 is not None else b.copy()
    rnorm = float(np.linalg.norm(r))
    b_abs = float(np.linalg.norm(b))
    bnorm = (rnorm if relative_to_initial else b_abs) or 1.0
    if rnorm / bnorm < tol or rnorm <= 1e-14 * b_abs:
        return x, KrylovInfo(0, rnorm / bnorm, True)
    r_hat = r.copy()
    rho = alpha = omega = 1.0
    v = np.zeros_like(b)
    p = np.zeros_like(b)
    k = 0
    for k in range(1, maxiter + 1):
        rho_new = _dot(r_hat, r)
        if rho_new == 0.0:
            break
        beta = (rho_new / rho) * (alpha / omega)
        rho = rho_new
        p = r + beta * (p - omega * v)
        phat = M(p) if M is not None else p
        v = A(phat)
        denom = _dot(r_hat, v)
        if denom == 0.0:
            break
        alpha = rho / denom
        s = r - alpha * v
        snorm = float(np.linalg.norm(s))
        if snorm / bnorm < tol:
            x += alpha * phat
            return x, KrylovInfo(k, snorm / bnorm, True)
        shat = M(s) if M is not None else s
        t = A(shat)
        tt = _dot(t, t)
        omega = _dot(t, s) / tt if tt > 0 else 0.0
        x_new = x + alpha * phat + omega * shat
        r = s - omega * t
        rnorm = float(np.linalg.norm(r))
        if not math.isfinite(rnorm):
            return x, KrylovInfo(k, float("nan"), False)
        x = x_new
        if rnorm / bnorm < tol or rnorm <= 1e-14 * b_abs:
            return x, KrylovInfo(k, rnorm / bnorm, True)
        if omega == 0.0:
            break
    return x, KrylovInfo(k, rnorm / bnorm, False)


def bicgstab_native(lib, A, b, x0, inv, tol, maxiter):
    """``ft_bicgstab_jacobi`` through its C ABI (``flowtrace/native/__init__.py:220-237``)."""
    n = A.shape[0]
    b, inv = np.ascontiguousarray(b, dtype=np.float64), np.ascontiguousarray(inv, dtype=np.float64)
    x = np.array(x0, dtype=np.float64, copy=True, order="C")
    work = np.empty(7 * n)
    it, res = ctypes.c_int64(0), ctypes.c_double(0.0)
    ok = lib.ft_bicgstab_jacobi(n, _p(A.indptr), _p(A.indices), _p(A.data), _p(b), _p(inv), _p(x), float(tol),
                                int(maxiter), 1, _p(work), ctypes.byref(it), ctypes.byref(res))
    return x, KrylovInfo(int(it.value), float(res.value), bool(ok))


# ------------------------------------------------------------------------------------------- SA-AMG
def _aggregate_py(indptr, indices, n):
    """Greedy three-pass aggregation (``flowtrace/linalg/amg.py:25-57``)."""
    agg = -np.ones(n, dtype=np.int64)
    na = 0
    for i in range(n):
        if agg[i] >= 0:
            continue
        free = True
        for k in range(indptr[i], indptr[i + 1]):
            if agg[indices[k]] >= 0:
                free = False
                break
        if free:
            agg[i] = na
            for k in range(indptr[i], indptr[i + 1]):
                agg[indices[k]] = na
            na += 1
    for i in range(n):
        if agg[i] >= 0:
            continue
        for k in range(indptr[i], indptr[i + 1]):
            j = indices[k]
            if agg[j] >= 0:
                agg[i] = agg[j]
                break
    for i in range(n):
        if agg[i] < 0:
            agg[i] = na
            na += 1
    return agg, na


try:  # the reference JIT-compiles the same loop with numba when present
    from numba import njit as _njit

    _aggregate = _njit(cache=False)(_aggregate_py)
except Exception:  # pragma: no cover
    _aggregate = _aggregate_py


def strength(A, theta):
    """``flowtrace/linalg/amg.py:60-66``."""
    A = A.tocoo()
    d = np.abs(A.diagonal())
    mask = (A.row != A.col) & (np.abs(A.data) >= theta * np.sqrt(d[A.row] * d[A.col]))
    S = sp.csr_matrix((np.ones(mask.sum()), (A.row[mask], A.col[mask])), shape=A.shape)
    S.sort_indices()
    return S


def spectral_radius(M, iters=15, seed=0):
    """``flowtrace/linalg/amg.py:69-77``."""
    rng = np.random.default_rng(seed)
    x = rng.standard_normal(M.shape[0])
    lam = 1.0
    for _ in range(iters):
        y = M @ x
        lam = np.linalg.norm(y) / max(np.linalg.norm(x), 1e-300)
        x = y / max(np.linalg.norm(y), 1e-300)
    return lam


class SmoothedAggregationAMG:
    """``flowtrace/linalg/amg.py:80-146`` (setup on the host, V-cycle with damped Jacobi)."""

    def __init__(self, A, theta=0.08, max_coarse=300, max_levels=20, smooth_sweeps=2, omega=0.8, singular=False):
        self.omega, self.sweeps = omega, smooth_sweeps
        A = sp.csr_matrix(A, dtype=np.float64)
        self.levels = []
        self.aggregates = []
        while A.shape[0] > max_coarse and len(self.levels) < max_levels - 1:
            S = strength(A, theta)
            agg, na = _aggregate(S.indptr.astype(np.int64), S.indices.astype(np.int64), A.shape[0])
            if na >= A.shape[0] * 0.9:
                break
            T = sp.csr_matrix((np.ones(A.shape[0]), (np.arange(A.shape[0]), agg)), shape=(A.shape[0], na))
            cnt = np.asarray(T.sum(axis=0)).ravel()
            T = T @ sp.diags(1.0 / np.sqrt(cnt))
            Dinv = 1.0 / A.diagonal()
            DA = sp.diags(Dinv) @ A
            rho = spectral_radius(DA)
            P = (T - (4.0 / 3.0 / rho) * (DA @ T)).tocsr()
            Ac = (P.T @ A @ P).tocsr()
            self.levels.append((A, P, P.T.tocsr(), Dinv))
            self.aggregates.append(np.asarray(agg))
            A = Ac
        self.coarse_n = A.shape[0]
        Ad = A.toarray()
        if singular:
            Ad = Ad + 1e-10 * np.abs(np.diag(Ad)).mean() * np.eye(Ad.shape[0])
        try:
            self.coarse_inv = np.linalg.inv(Ad)
        except np.linalg.LinAlgError:
            self.coarse_inv = np.linalg.pinv(Ad)

    @property
    def n_levels(self):
        return len(self.levels) + 1

    def _cycle(self, k, b):
        if k == len(self.levels):
            return self.coarse_inv @ b
        A, P, R, Dinv = self.levels[k]
        w = self.omega
        x = w * Dinv * b
        for _ in range(self.sweeps - 1):
            x = x + w * Dinv * (b - A @ x)
        r = b - A @ x
        x = x + P @ self._cycle(k + 1, R @ r)
        for _ in range(self.sweeps):
            x = x + w * Dinv * (b - A @ x)
        return x

    def __call__(self, b):
        return self._cycle(0, b.astype(np.float64))


# ------------------------------------------------------------------------------------------- solver
def auto_relax_p(non_orthogonality_deg):
    """``flowtrace/unstructured/simple.py:53-64``."""
    return 1.0 if non_orthogonality_deg <= 5.0 else 0.8


class OracleSimple:
    """Steady SIMPLE/SIMPLEC outer iteration (``flowtrace/unstructured/simple.py:71-1072``)."""

    GUARD_GROWTH, GUARD_ROUNDOFF, GUARD_EVERY = 20.0, 1e-6, 20                      # simple.py:706-712
    GUARD_FACTOR, GUARD_MIN_RELAX, GUARD_FALLBACK, GUARD_MIN_RELAX_U = 0.6, 0.1, True, 0.2

    def __init__(self, mesh, case, native=None, porosity=None, amg_theta=0.08):
        if case.turbulence not in ("laminar", "k-omega-sst"):
            raise NotImplementedError(f"turbulence={case.turbulence!r} is outside the oracle's scope")
        if case.radiation != "off":
            raise NotImplementedError(f"radiation={case.radiation!r} is outside the oracle's scope")
        if case.unsteady or case.species or case.mrf or case.solids or case.periodic:
            raise NotImplementedError("transient, species, MRF, solids and periodic cases are outside the oracle's scope")
        self.case, self.mesh = case, mesh
        self.amg_theta = float(amg_theta)
        self.native = native
        self.fv = fv = OracleFV(mesh, native)
        self.dim = dim = mesh.dim
        self.nc = mesh.n_cells
        self.energy = case.energy
        self.timers: Dict[str, float] = defaultdict(float)
        self.iteration = self.step_count = 0
        self.converged = False
        self._res_max5: Dict[str, float] = {}
        self._amg, self._amg_age, self.amg_rebuild = None, 10 ** 9, 10                 # simple.py:96-98
        self.last_linear = {}
        self._gp = self._gU = self._gT = None
        self.relax_p = float(case.relax_p) if case.relax_p is not None else auto_relax_p(fv.non_orthogonality_deg)
        self.porosity = None if porosity is None else np.asarray(porosity, dtype=np.float64)
        self._build_boundaries()
        U0 = np.zeros((self.nc, dim))
        U0[:] = (list(case.init_velocity) + [0.0] * 3)[:dim]
        self.U = U0
        self.p = np.zeros(self.nc)
        self.T = np.full(self.nc, case.init_T, dtype=np.float64) if self.energy else None
        ub = self._velocity_bvals(self.U)
        self.F = case.density * np.sum(fv.face_interp_vec(self.U) * fv.S, axis=1)
        self.Fb = self._boundary_flux_fixed(ub)
        self.mom_source = None
        self.energy_source = None
        self.turb = None
        if case.turbulence == "k-omega-sst":                                           # simple.py:115-117
            from .sst_oracle import OracleSST

            self.turb = OracleSST(self)
        self.guard_enabled = case.relax_p is None
        self._capture = None
        self._reset_guard()

    # ---- set-up ------------------------------------------------------------------------------
    def _build_boundaries(self):
        """``simple.py:185-240`` (no MRF or rotating walls)."""
        fv, case, dim = self.fv, self.case, self.dim
        n = fv.n_bf
        kind = np.zeros(n, dtype=np.int64)
        ub = np.zeros((n, dim))
        pb = np.zeros(n)
        tk = np.zeros(n, dtype=np.int64)
        tv = np.zeros(n)
        self.zone_specs = {}
        for z in self.mesh.boundary_zones():
            spec = case.boundaries.get(z.name)
            if spec is None:
                spec = _Spec(FLUENT_TO_KIND.get(z.type, "wall"))
                if spec.kind == "inlet":
                    spec.normal_speed = 1.0
            self.zone_specs[z.name] = spec
            m = fv.bzone == z.id
            kind[m] = _KIND_CODE[spec.kind]
            if spec.kind in ("wall", "inlet"):
                if spec.velocity is not None:
                    ub[m] = (list(spec.velocity) + [0.0, 0.0, 0.0])[:dim]
                elif spec.normal_speed is not None:
                    ub[m] = -spec.normal_speed * fv.nb[m]
            pb[m] = spec.pressure
            if spec.kind == "wall":
                tk[m] = {"adiabatic": T_ADIABATIC, "temperature": T_FIXED, "flux": T_FLUX}[spec.thermal]
            elif spec.kind in ("inlet", "pressure"):
                tk[m] = T_FIXED
            tv[m] = spec.value
        self.bkind = kind
        self.ub_fixed, self.pb_fixed, self.tkind, self.tval = ub, pb, tk, tv
        self.m_wall = (kind == WALL).astype(np.float64)
        self.m_inlet = (kind == INLET).astype(np.float64)
        self.m_pres = ((kind == OUTLET) | (kind == PRESSURE)).astype(np.float64)
        self.m_sym = (kind == SYMMETRY).astype(np.float64)
        self.m_dirvel = ((kind == WALL) | (kind == INLET) | (kind == SYMMETRY)).astype(np.float64)
        self.singular_p = not bool(((kind == OUTLET) | (kind == PRESSURE)).any())

    def initialize(self, fields: dict):
        """``simple.py:140-162``."""
        U = self.U.copy()
        for k, name in enumerate(("x-velocity", "y-velocity", "z-velocity")[:self.dim]):
            if name in fields:
                U[:, k] = np.asarray(fields[name], dtype=np.float64)
        self.U = U
        if "pressure" in fields:
            p = np.asarray(fields["pressure"], dtype=np.float64)
            self.p = p - p.mean() if self.singular_p else p
        if self.energy and "temperature" in fields:
            self.T = np.asarray(fields["temperature"], dtype=np.float64)
        ub = self._velocity_bvals(self.U)
        self.F = self.case.density * np.sum(self.fv.face_interp_vec(self.U) * self.fv.S, axis=1)
        self.Fb = self._boundary_flux_fixed(ub)
        self._gp = self._gU = self._gT = None
        self._capture = None
        self._reset_guard()

    def set_sources(self, momentum=None, energy=None):
        """``simple.py:164-182``."""
        self.mom_source = None if momentum is None else \
            np.asarray(momentum, dtype=np.float64).reshape(self.nc, self.dim) * self.fv.vol[:, None]
        self.energy_source = None if energy is None else \
            np.asarray(energy, dtype=np.float64).reshape(self.nc) * self.fv.vol / self.case.cp

    # ---- boundary values -------------------------------------------------------------------------
    def _velocity_bvals(self, U, gU=None):
        """``simple.py:305-316``."""
        fv = self.fv
        UP = U[fv.Pb]
        if gU is not None:
            UP = UP + np.stack([np.sum(g[fv.Pb] * fv.db_t, axis=1) for g in gU], axis=1)
        un = np.sum(UP * fv.nb, axis=1)
        sym = UP - un[:, None] * fv.nb
        fixed = (self.m_wall + self.m_inlet)[:, None]
        return fixed * self.ub_fixed + self.m_sym[:, None] * sym + self.m_pres[:, None] * UP

    def _pressure_bvals(self, p, gp=None):
        """``simple.py:318-325``."""
        fv = self.fv
        pP = p[fv.Pb]
        if gp is not None:
            pP = pP + np.sum(gp[fv.Pb] * fv.db, axis=1)
        return self.m_pres * self.pb_fixed + (1.0 - self.m_pres) * pP

    def _boundary_flux_fixed(self, ub):
        """``simple.py:327-330``."""
        flux = self.case.density * np.sum(ub * self.fv.Sb, axis=1)
        return flux * (self.m_inlet + self.m_pres)

    # ---- discretisation --------------------------------------------------------------------------
    @staticmethod
    def _split_gamma(gamma):
        """A diffusivity as (interior-face, boundary-face) values; a scalar serves both
        (``simple.py:333-338``)."""
        return gamma if isinstance(gamma, tuple) else (gamma, gamma)

    def _coefficients(self, gamma, dirichlet):
        """``simple.py:340-353``."""
        fv, F, Fb = self.fv, self.F, self.Fb
        gf, gb = self._split_gamma(gamma)
        D = gf * fv.alpha
        aPN = -(D + np.maximum(-F, 0.0))
        aNP = -(D + np.maximum(F, 0.0))
        Db = gb * fv.alpha_b * dirichlet
        diag = fv.scatter(D + np.maximum(F, 0.0), D + np.maximum(-F, 0.0), Db + np.maximum(Fb, 0.0))
        return diag, aPN, aNP, Db

    def _rhs(self, gamma, phi, grad, phi_b, Db, extra=None, scheme=None):
        """``simple.py:355-374``."""
        fv, F, Fb = self.fv, self.F, self.Fb
        gface, _ = self._split_gamma(gamma)
        rhs = fv.Cb @ ((Db + np.maximum(-Fb, 0.0)) * phi_b)
        gf = fv.face_interp_vec(grad)
        rhs = rhs + fv.Cdiff @ (gface * np.sum(gf * fv.Tvec, axis=1))
        if (scheme or self.case.scheme) == "second-order":
            P, N = fv.P, fv.N
            phP, phN = phi[P], phi[N]
            hoP = phP + np.sum(grad[P] * fv.dP_f, axis=1)
            hoN = phN + np.sum(grad[N] * fv.dN_f, axis=1)
            up = F >= 0
            ho = np.clip(np.where(up, hoP, hoN), np.minimum(phP, phN), np.maximum(phP, phN))
            rhs = rhs - fv.Cdiff @ (F * (ho - np.where(up, phP, phN)))
        if extra is not None:
            rhs = rhs + extra
        return rhs

    def _residual(self, A, diag, x, b):
        """``simple.py:376-380``."""
        r = float(np.sum(np.abs(b - A @ x)))
        s = float(np.sum(np.abs(diag * x)))
        return r / s if s > 0 else r

    def _solve(self, A, b, x0, diag, tol=0.1, maxiter=30):
        """``simple.py:489-497``."""
        inv = 1.0 / diag
        if self.native is not None:
            return bicgstab_native(self.native, A, b, x0, inv, tol, maxiter)
        return bicgstab(lambda v: A @ v, b, M=lambda v: inv * v, x0=x0, tol=tol, maxiter=maxiter,
                        relative_to_initial=True)

    # ---- the outer iteration ---------------------------------------------------------------------
    @property
    def finished(self):
        return self.converged or self.iteration >= self.case.max_iter

    def step(self) -> float:
        """One outer iteration (``simple.py:500-703``)."""
        if self.finished:
            return 0.0
        self._capture = None
        c, fv = self.case, self.fv
        rho, mu, dim = c.density, c.viscosity, self.dim
        U, p = self.U, self.p
        ub = self._velocity_bvals(U, self._gU)
        pb = self._pressure_bvals(p, self._gp)
        gp_ls = fv.gradient(p, pb)
        gp = gp_ls
        if c.pressure_gradient == "green-gauss":
            gp = fv.gradient_gg(p, pb, gp_ls)
        gU = [fv.gradient(U[:, k], ub[:, k]) for k in range(dim)]
        self._gp, self._gU = gp, gU
        src = -gp * fv.vol[:, None]                                                    # simple.py:526-536
        if self.energy and any(c.buoyancy[:dim]):
            src = src + (fv.vol * (self.T - c.t_ref))[:, None] * np.asarray(c.buoyancy[:dim], dtype=np.float64)[None, :]
        drive = np.asarray(c.body_force[:dim], dtype=np.float64)
        if np.any(drive):
            src = src + fv.vol[:, None] * drive[None, :]
        if self.mom_source is not None:
            src = src + self.mom_source
        gm = mu
        if self.turb is not None:                                                      # simple.py:545-548
            gm = self.turb.momentum_viscosity(U)
            src = src + self.turb.transpose_stress(gU)
        res = {}
        Ustar = np.empty_like(U)
        au = self.relax_u
        diag, aPN, aNP, Db = self._coefficients(gm, self.m_dirvel)
        if self.porosity is not None:  # implicit Brinkman drag alpha V (not in the reference)
            diag = diag + self.porosity * fv.vol
        rhs_all = [self._rhs(gm, U[:, k], gU[k], ub[:, k], Db, src[:, k]) for k in range(dim)]
        A = fv.matrix(diag, aPN, aNP)
        num = [float(np.sum(np.abs(rhs_all[k] - A @ U[:, k]))) for k in range(dim)]     # simple.py:565-569
        den = [float(np.sum(np.abs(diag * U[:, k]))) for k in range(dim)]
        floor = 1e-3 * max(max(den), 1e-300)
        for k, name in enumerate(("x-velocity", "y-velocity", "z-velocity")[:dim]):
            res[name] = num[k] / max(den[k], floor)
        diag_r = diag / au
        Ar = fv.matrix(diag_r, aPN, aNP)
        its, brs, infos = [], [], []
        for k in range(dim):
            b = rhs_all[k] + ((1.0 - au) / au) * diag * U[:, k]
            x, info = self._solve(Ar, b, U[:, k], diag_r)
            Ustar[:, k] = x
            its.append(info.iterations)
            brs.append(b)
            infos.append(info)
        if self.algo == "SIMPLEC":                                                     # simple.py:584-590
            sum_nb = fv.scatter(-aPN, -aNP)
            denom = diag_r - sum_nb
            denom = np.where(denom > 1e-12 * diag_r, denom, diag_r)
        else:
            denom = diag_r
        dP = fv.vol / denom
        dF = fv.face_interp(dP)
        gpf = fv.face_interp_vec(gp)
        P, N, Pb = fv.P, fv.N, fv.Pb
        Fst = rho * (np.sum(fv.face_interp_vec(Ustar) * fv.S, axis=1)                 # simple.py:598-599
                     - dF * fv.alpha * (p[N] - p[P] - np.sum(gpf * fv.d, axis=1)))
        Fb_in = rho * np.sum(self.ub_fixed * fv.Sb, axis=1) * self.m_inlet             # simple.py:610-613
        Fb_pr = rho * (np.sum(Ustar[Pb] * fv.Sb, axis=1)
                       - dP[Pb] * fv.alpha_b * (self.pb_fixed - p[Pb] - np.sum(gp[Pb] * fv.db, axis=1)))
        Fbst = Fb_in + Fb_pr * self.m_pres
        cf = rho * dF * fv.alpha                                                       # simple.py:616-621
        cb = rho * dP[Pb] * fv.alpha_b * self.m_pres
        diag_p = fv.scatter(cf, cf, cb)
        Ap = fv.matrix(diag_p, -cf, -cf)
        mass = fv.net_outflow(Fst, Fbst)
        res["continuity"] = float(np.sum(np.abs(mass)))
        if self._amg is None or self._amg_age >= self.amg_rebuild:                     # simple.py:624-628
            Ah = Ap.csr if hasattr(Ap, "csr") else Ap
            self._amg = SmoothedAggregationAMG(Ah, theta=self.amg_theta, singular=self.singular_p)
            self._amg_age = 0
        self._amg_age += 1
        project = (lambda v: v - v.mean()) if self.singular_p else None
        pp, pinfo = pcg(lambda v: Ap @ v, -mass, M=self._amg, tol=c.pressure_tol, maxiter=200, project=project)
        self.F = Fst + cf * (pp[P] - pp[N])                                            # simple.py:639-646
        self.Fb = Fbst + cb * pp[Pb]
        self.p = p + self.relax_p * pp
        if self.singular_p:
            self.p = self.p - self.p.mean()
        ppb = (1.0 - self.m_pres) * pp[Pb]
        gpp = fv.gradient(pp, ppb)
        self.U = Ustar - dP[:, None] * gpp
        cap = {"U_old": U, "p_old": p, "A": A, "b": rhs_all, "Ar": Ar, "br": brs, "U_star": Ustar,
               "mom_info": infos, "alpha_u": au, "Fst": Fst, "Fbst": Fbst, "mass": mass, "Ap": Ap, "pp": pp,
               "p_info": pinfo, "F": self.F, "Fb": self.Fb, "U_new": self.U, "p_new": self.p,
               "dP": dP, "gp": gp, "gU": gU}
        if self.energy:
            res["energy"] = self._energy()
            cap["energy"] = self._energy_capture
        if self.turb is not None:                                                      # simple.py:662-669
            ubc = self._velocity_bvals(self.U, gU)
            gUc = [fv.gradient(self.U[:, k], ubc[:, k]) for k in range(dim)]
            k_old, w_old = self.turb.k, self.turb.w
            res.update(self.turb.solve(gUc))
            cap["turbulence"] = {"k": (k_old, self.turb.k), "omega": (w_old, self.turb.w)}
        self.iteration += 1
        self.step_count = self.iteration
        self.last_linear = {"momentum_iters": its, "pressure_iters": pinfo.iterations,
                            "pressure_residual": pinfo.residual}
        prev = getattr(self, "_last_res", {}), getattr(self, "_last_raw", {})
        self._last_raw = dict(res)
        if self.iteration <= 5:
            self._res_max5["continuity"] = max(self._res_max5.get("continuity", 0.0), res["continuity"], 1e-300)
        flux_scale = float(np.sum(np.abs(self.F))) + float(np.sum(np.abs(self.Fb)))     # simple.py:687-688
        res["continuity"] /= max(self._res_max5["continuity"], 1e-3 * flux_scale)
        self._last_res = res
        cap["iteration"] = self.iteration
        rolled_back = self._stability_guard(self._last_raw["continuity"], flux_scale)
        cap["rolled_back"] = rolled_back
        self._capture = cap
        if rolled_back:
            self._last_res, self._last_raw = prev
            return 1.0
        if self.iteration > 5 and max(res.values()) < c.tol:
            self.converged = True
        return 1.0

    def _energy(self):
        """``simple.py:778-813`` (laminar, no radiation)."""
        c, fv = self.case, self.fv
        gam = c.conductivity / c.cp
        if self.turb is not None:
            gam = self.turb.energy_diffusivity(gam)                                    # simple.py:781-782
        T = self.T
        TP = T[fv.Pb]
        fixed = self.tkind == T_FIXED
        flux = self.tkind == T_FLUX
        out = self.bkind == OUTLET
        if self._gT is not None:
            TP = TP + np.sum(self._gT[fv.Pb] * fv.db_t, axis=1)
        Tb = np.where(fixed, self.tval, TP)
        Tb = np.where(out & (self.Fb < 0), self.tval, Tb)
        gT = fv.gradient(T, Tb)
        self._gT = gT
        q_in = fv.Cb @ (flux * self.tval * fv.Sb_mag / c.cp)
        if self.energy_source is not None:
            q_in = q_in + self.energy_source
        diag, aPN, aNP, Db = self._coefficients(gam, fixed.astype(np.float64))
        rhs = self._rhs(gam, T, gT, Tb, Db, q_in, scheme=c.scalar_scheme)
        A = fv.matrix(diag, aPN, aNP)
        r = self._residual(A, diag, T, rhs)
        aT = c.relax_T
        dr = diag / aT
        Ar = fv.matrix(dr, aPN, aNP)
        b = rhs + ((1.0 - aT) / aT) * diag * T
        self.T, info = self._solve(Ar, b, T, dr, tol=1e-3, maxiter=60)
        self._energy_capture = {"A": A, "b": rhs, "T_old": T, "Ar": Ar, "br": b, "T_new": self.T, "alpha": aT,
                                "info": info}
        return r

    # ---- guard and state -------------------------------------------------------------------------
    def _reset_guard(self):
        """``simple.py:714-720``."""
        self.guard_events = []
        self.algo = self.case.algorithm
        self.relax_u = self.case.relax_u
        self.guard_exhausted_at = None
        self._guard_min = float("inf")
        self._guard_snap = (self.state_dict(), float("inf")) if self.guard_enabled else None

    def _stability_guard(self, r, flux_scale):
        """``simple.py:722-776``."""
        if not self.guard_enabled:
            return False
        ref = max(self._guard_min, self.GUARD_ROUNDOFF * flux_scale)
        bad = not math.isfinite(r) or (self.iteration > 10 and r > self.GUARD_GROWTH * ref)
        if bad and self._guard_snap is not None and self.relax_p * self.GUARD_FACTOR >= self.GUARD_MIN_RELAX:
            snap, snap_r = self._guard_snap
            at = self.iteration
            self.load_state(snap)
            self.iteration = self.step_count = at
            self.relax_p *= self.GUARD_FACTOR
            self._amg_age = 10 ** 9
            self._guard_min = snap_r
            self.guard_events.append({"detected_at": at, "restored_to": int(snap["iteration"]),
                                      "relax_p": round(self.relax_p, 4), "continuity": r})
            return True
        stage2 = self.GUARD_FALLBACK and (self.algo == "SIMPLEC" or self.relax_u * 0.7 >= self.GUARD_MIN_RELAX_U - 1e-12)
        if bad and self._guard_snap is not None and stage2:
            snap, snap_r = self._guard_snap
            at = self.iteration
            self.load_state(snap)
            self.iteration = self.step_count = at
            if self.algo == "SIMPLEC":
                self.algo, self.relax_u, self.relax_p = "SIMPLE", min(self.relax_u, 0.3), 0.3
            else:
                self.relax_u *= 0.7
            self._amg_age = 10 ** 9
            self._guard_min = snap_r
            self.guard_events.append({"detected_at": at, "restored_to": int(snap["iteration"]), "algorithm": self.algo,
                                      "relax_p": round(self.relax_p, 4), "relax_u": round(self.relax_u, 4),
                                      "continuity": r})
            return True
        if bad and self.guard_exhausted_at is None:
            self.guard_exhausted_at = self.iteration
        if math.isfinite(r) and self.iteration > 5:
            self._guard_min = min(self._guard_min, r)
            if self.iteration % self.GUARD_EVERY == 0 and r <= 2.0 * self._guard_min:
                self._guard_snap = (self.state_dict(), r)
        return False

    def residuals(self):
        """``simple.py:822-833``."""
        r = dict(getattr(self, "_last_res", {}))
        return {"raw": dict(getattr(self, "_last_raw", r)), "scaled": r, "normalized": r}

    def fields(self):
        """``simple.py:862-880``."""
        out = {"x-velocity": self.U[:, 0].copy(), "y-velocity": self.U[:, 1].copy()}
        if self.dim == 3:
            out["z-velocity"] = self.U[:, 2].copy()
        out["velocity-magnitude"] = np.linalg.norm(self.U, axis=1)
        out["pressure"] = self.p.copy()
        if self.energy:
            out["temperature"] = self.T.copy()
        if self.turb is not None:
            out.update(self.turb.fields())
        return out

    def _wall_viscosity(self):
        """Boundary-face viscosity of the momentum equation (``simple.py:900-904``)."""
        if self.turb is not None:
            return self.turb.momentum_viscosity(self.U)[1]
        return np.full(self.fv.n_bf, float(self.case.viscosity))

    def wall_forces(self):
        """Pressure and viscous force on every wall zone (``simple.py:970-1001``)."""
        fv = self.fv
        pb = self._pressure_bvals(self.p, self._gp)
        mu_b = self._wall_viscosity()
        du = self.U[fv.Pb] - self.ub_fixed
        du_t = du - np.einsum("fd,fd->f", du, fv.nb)[:, None] * fv.nb
        f_p = pb[:, None] * fv.Sb
        f_v = (mu_b * fv.alpha_b)[:, None] * du_t
        out = {}
        for z in self.mesh.boundary_zones():
            m = (fv.bzone == z.id) & (self.bkind == WALL)
            if m.any():
                fp, fvis = f_p[m].sum(axis=0), f_v[m].sum(axis=0)
                out[z.name] = {"pressure": fp.tolist(), "viscous": fvis.tolist(), "total": (fp + fvis).tolist()}
        return out

    def _wall_shear(self):
        """Wall shear stress vector per boundary face, mu_w (u_P - u_w)_t / y_b."""
        fv = self.fv
        rel = self.U[fv.Pb] - self.ub_fixed
        rel_t = rel - np.sum(rel * fv.nb, axis=1)[:, None] * fv.nb
        return self._wall_viscosity()[:, None] * rel_t / fv.yb[:, None], rel_t

    def wall_report(self):
        """Per wall zone: area, forces, Cd/Cl, y+, skin friction, conducted heat
        (``simple.py:906-950``, no radiation)."""
        fv, c = self.fv, self.case
        rho, mu = c.density, c.viscosity
        tau_vec, _ = self._wall_shear()
        tau = np.sqrt(np.sum(tau_vec * tau_vec, axis=1))
        yplus = fv.yb * np.sqrt(tau / rho) * rho / mu
        forces = self.wall_forces()
        qconv = None
        if self.energy:
            Tw = np.where(self.tkind == T_FIXED, self.tval, self.T[fv.Pb])
            qconv = (c.conductivity * fv.alpha_b * (Tw - self.T[fv.Pb]) * (self.tkind == T_FIXED)
                     + np.where(self.tkind == T_FLUX, self.tval * fv.Sb_mag, 0.0))
        qdyn = 0.5 * rho * c.ref_velocity ** 2
        out = {}
        for z in self.mesh.boundary_zones():
            if z.name not in forces:
                continue
            m = fv.bzone == z.id
            A = fv.Sb_mag[m]
            f = forces[z.name]
            Ft = np.asarray(f["total"])
            rep = {"area": float(A.sum()), "force_pressure": f["pressure"], "force_viscous": f["viscous"],
                   "force_total": f["total"], "cd": float(Ft[0] / (qdyn * c.ref_area)),
                   "cl": float(Ft[1] / (qdyn * c.ref_area)),
                   "yplus_avg": float((yplus[m] * A).sum() / A.sum()), "yplus_max": float(yplus[m].max()),
                   "cf_avg": float((tau[m] * A).sum() / A.sum() / qdyn)}
            if qconv is not None:
                rep["heat_flow_conv"] = float(qconv[m].sum())
            out[z.name] = rep
        return out

    def wall_profile(self, zone):
        """Face-wise x, y, Cf, Cp, y+ on one wall zone, sorted by x (``simple.py:952-968``)."""
        fv, c = self.fv, self.case
        z = self.mesh.zone_by_name(zone)
        m = fv.bzone == z.id
        rho, mu = c.density, c.viscosity
        _, rel_t = self._wall_shear()
        tau = self._wall_viscosity() * np.sqrt(np.sum(rel_t * rel_t, axis=1)) / fv.yb
        qdyn = 0.5 * rho * c.ref_velocity ** 2
        xfb = fv.xfb[m]
        order = np.argsort(xfb[:, 0])
        return {"x": xfb[order, 0], "y": xfb[order, 1], "cf": tau[m][order] / qdyn,
                "cp": self._pressure_bvals(self.p, self._gp)[m][order] / qdyn,
                "yplus": (fv.yb * np.sqrt(tau / rho) * rho / mu)[m][order]}

    def state_dict(self):
        """``simple.py:1033-1046``."""
        st = {"U": self.U.copy(), "p": self.p.copy(), "F": self.F.copy(), "Fb": self.Fb.copy(),
              "iteration": self.iteration}
        if self.energy:
            st["T"] = self.T.copy()
        if getattr(self, "turb", None) is not None:
            st.update(self.turb.state())
        st["time"], st["time_step"] = 0.0, 0
        st["res_continuity_norm"] = self._res_max5.get("continuity", 0.0)
        return st

    def load_state(self, st):
        """``simple.py:1048-1072``."""
        self.U = np.array(st["U"], dtype=np.float64)
        self.p = np.array(st["p"], dtype=np.float64)
        self.F = np.array(st["F"], dtype=np.float64)
        self.Fb = np.array(st["Fb"], dtype=np.float64)
        if self.energy and "T" in st:
            self.T = np.array(st["T"], dtype=np.float64)
        self.iteration = int(st.get("iteration", 0))
        self._gp = self._gU = self._gT = None
        self._capture = None
        if self.turb is not None:
            self.turb.load(st)
        if float(st.get("res_continuity_norm", 0.0)) > 0:
            self._res_max5["continuity"] = float(st["res_continuity_norm"])


class _Spec:
    """Default spec of a zone that the case does not name (``simple.py:199-203``)."""

    def __init__(self, kind):
        self.kind, self.velocity, self.normal_speed, self.pressure = kind, None, None, 0.0
        self.thermal, self.value = "adiabatic", 0.0
        self.turb_intensity = self.turb_viscosity_ratio = self.k = self.omega = None
