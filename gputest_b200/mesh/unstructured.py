"""Face-based unstructured mesh: the host-side input format of the SIMPLEC path.

The data model is Fluent's, as FlowTrace keeps it (``flowtrace/mesh/unstructured.py:29-129``):
a list of faces, each with its node loop, an owner cell and a neighbour cell (-1 on the
boundary), a face-zone id per face and a cell-zone id per cell. Area vectors point from
owner to neighbour, and out of the domain on boundary faces.

``compute_geometry`` restates the reference's face/cell geometry
(``flowtrace/mesh/unstructured.py:171-261``): fan-triangulated face centres and areas about
the node mean, a left-handed-face repair pass against approximate cell centres, and a
pyramid decomposition for volumes and centroids. It runs once, on the host, at set-up.

The generators reproduce the reference's node, cell and face numbering exactly where the
reference has the same generator (``cartesian_mesh_2d`` single-diagonal, ``extrude_to_3d``),
so a mesh built here is the same array set the reference builds. Two generators the
reference lacks are added: alternating-diagonal triangulation and a 3-D hexahedral box with
interior-node jitter in all three directions.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

BC_CODES = {
    2: "interior", 3: "wall", 4: "pressure-inlet", 5: "pressure-outlet", 7: "symmetry",
    8: "periodic-shadow", 9: "pressure-far-field", 10: "velocity-inlet", 12: "periodic",
    14: "fan", 20: "mass-flow-inlet", 24: "interface", 31: "parent", 36: "outflow", 37: "axis",
}


@dataclass
class Zone:
    """A face or cell zone (``flowtrace/mesh/unstructured.py:29-40``)."""

    id: int
    name: str
    type: str
    kind: str  # "face" or "cell"
    first: int = 0
    last: int = -1

    @property
    def count(self) -> int:
        return self.last - self.first + 1


@dataclass
class UnstructuredMesh:
    """Face-based mesh (``flowtrace/mesh/unstructured.py:43-129``)."""

    dim: int
    nodes: np.ndarray
    face_ptr: np.ndarray
    face_nodes: np.ndarray
    owner: np.ndarray
    neighbour: np.ndarray
    face_zone: np.ndarray
    n_cells: int
    cell_zone: np.ndarray
    zones: Dict[int, Zone] = field(default_factory=dict)
    name: str = "mesh"
    periodic: List[dict] = field(default_factory=list)

    @property
    def n_faces(self) -> int:
        return int(self.owner.shape[0])

    @property
    def n_nodes(self) -> int:
        return int(self.nodes.shape[0])

    def face_zones(self) -> List[Zone]:
        return [z for z in self.zones.values() if z.kind == "face"]

    def periodic_zone_ids(self) -> set:
        return {p["zone_a"] for p in self.periodic} | {p["zone_b"] for p in self.periodic}

    def boundary_zones(self) -> List[Zone]:
        per = self.periodic_zone_ids()
        return [z for z in self.face_zones() if z.type != "interior" and z.id not in per]

    def cell_zones(self) -> List[Zone]:
        return [z for z in self.zones.values() if z.kind == "cell"]

    def zone_by_name(self, name: str) -> Optional[Zone]:
        for z in self.zones.values():
            if z.name == name:
                return z
        return None

    def faces_of_zone(self, zid: int) -> np.ndarray:
        return np.flatnonzero(self.face_zone == zid)

    def summary(self) -> dict:
        nb = int((self.neighbour < 0).sum())
        return {"name": self.name, "dim": self.dim, "nodes": self.n_nodes, "faces": self.n_faces,
                "interior_faces": self.n_faces - nb, "boundary_faces": nb, "cells": self.n_cells,
                "zones": [{"id": z.id, "name": z.name, "type": z.type, "kind": z.kind, "count": z.count}
                          for z in sorted(self.zones.values(), key=lambda z: z.id)]}

    def cell_polygons_2d(self):
        """Counter-clockwise node loop of every 2-D cell, as (ptr, nodes).

        A 2-D face n0 -> n1 has its owner on the left, so around the owner the edge runs
        n0 -> n1 and around the neighbour n1 -> n0; chaining the edges of a cell gives its loop
        (``flowtrace/mesh/unstructured.py:103-129``).
        """
        if self.dim != 2:
            raise ValueError("cell polygons are only defined for 2-D meshes")
        n0 = self.face_nodes[self.face_ptr[:-1]]
        n1 = self.face_nodes[self.face_ptr[:-1] + 1]
        inner = self.neighbour >= 0
        cells = np.concatenate([self.owner, self.neighbour[inner]])
        tail = np.concatenate([n0, n1[inner]])
        head = np.concatenate([n1, n0[inner]])
        order = np.argsort(cells, kind="stable")
        cells, tail, head = cells[order], tail[order], head[order]
        ptr = np.concatenate([[0], np.cumsum(np.bincount(cells, minlength=self.n_cells))])
        loops = np.empty(tail.shape[0], dtype=np.int64)
        for c in range(self.n_cells):
            s, e = ptr[c], ptr[c + 1]
            succ = dict(zip(tail[s:e].tolist(), head[s:e].tolist()))
            first = int(tail[s])
            cur = first
            for k in range(s, e):
                loops[k] = cur
                cur = succ.get(cur, first)
        return ptr, loops


@dataclass
class Geometry:
    face_centre: np.ndarray
    face_area_vec: np.ndarray
    face_area: np.ndarray
    cell_centre: np.ndarray
    cell_volume: np.ndarray
    flipped_faces: int = 0

    @property
    def total_volume(self) -> float:
        return float(self.cell_volume.sum())


def _host_arrays(mesh: UnstructuredMesh):
    i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)  # noqa: E731
    return (np.ascontiguousarray(mesh.nodes, dtype=np.float64), i32(mesh.face_ptr), i32(mesh.face_nodes))


def face_centres_and_areas(mesh: UnstructuredMesh):
    """Face centres and area vectors (``flowtrace/mesh/unstructured.py:171-212``), by the library's
    host loop over the same per-face code as the device set-up (``b2s_host_face_geometry``):
    2-D, the segment midpoint and S = (n1 - n0) x z; 3-D, each face fanned into triangles about
    its node mean, the centre the triangle centroids weighted by their areas projected on S."""
    from .. import _lib

    X, fptr, fnodes = _host_arrays(mesh)
    nf = mesh.n_faces
    fc, S = np.empty((nf, mesh.dim)), np.empty((nf, mesh.dim))
    bad = _lib.lib().b2s_host_face_geometry(mesh.dim, nf, X.ctypes.data, fptr.ctypes.data, fnodes.ctypes.data,
                                            fc.ctypes.data, S.ctypes.data)
    if bad < 0:
        raise ValueError("invalid mesh arrays")
    if bad:
        raise ValueError("2-D meshes must have 2-node faces" if mesh.dim == 2 else
                         "3-D faces must have 3 to 32 nodes")
    return fc, S


def compute_geometry(mesh: UnstructuredMesh, repair: bool = True) -> Geometry:
    """Face, cell and volume geometry (``flowtrace/mesh/unstructured.py:171-261``) by the library's
    host loops over the per-face and per-cell code of the device set-up (``b2s_host_geometry``):
    face centres and areas, approximate cell centres (the mean of the face centres), the
    orientation repair (``repair``: every S turned to point away from its owner) and cell volumes
    and centroids from the pyramids of the faces over the approximate centres, each cell's sums
    taken over its owned and then its neighbour faces in face order, as the reference's
    ``np.bincount`` sums."""
    from .. import _lib

    X, fptr, fnodes = _host_arrays(mesh)
    nf, nc, dim = mesh.n_faces, mesh.n_cells, mesh.dim
    own = np.ascontiguousarray(mesh.owner, dtype=np.int32)
    nei = np.ascontiguousarray(mesh.neighbour, dtype=np.int32)
    fc, S = np.empty((nf, dim)), np.empty((nf, dim))
    xc, vol = np.empty((nc, dim)), np.empty(nc)
    cnt = np.zeros(3, dtype=np.int32)
    rc = _lib.lib().b2s_host_geometry(dim, nc, nf, X.ctypes.data, fptr.ctypes.data, fnodes.ctypes.data,
                                      own.ctypes.data, nei.ctypes.data, int(bool(repair)), fc.ctypes.data,
                                      S.ctypes.data, xc.ctypes.data, vol.ctypes.data, cnt.ctypes.data)
    if rc != 0:
        raise ValueError("invalid mesh arrays")
    if cnt[0]:
        raise ValueError("2-D meshes must have 2-node faces" if dim == 2 else "3-D faces must have 3 to 32 nodes")
    if cnt[2]:
        raise ValueError(f"{int(cnt[2])} cells have non-positive volume")
    return Geometry(face_centre=fc, face_area_vec=S, face_area=np.linalg.norm(S, axis=1), cell_centre=xc,
                    cell_volume=vol, flipped_faces=int(cnt[1]))


# ----------------------------------------------------------------------------------------------
# generators
# ----------------------------------------------------------------------------------------------
def _assemble_mesh(dim, nodes, families, n_cells, bzones, name):
    """Concatenate face families into a mesh: interior families first (zone 3), then the
    boundary zones in order, each a (face_nodes (m, k), owner) pair; cell zone 2 = fluid."""
    loops, owner, neigh, fzone = [], [], [], []
    for fn, o, n in families:
        loops.append(fn)
        owner.append(o)
        neigh.append(n)
        fzone.append(np.full(len(o), 3))
    n_int = int(sum(len(o) for o in owner))
    zones = {2: Zone(2, "fluid", "fluid", "cell", 0, n_cells - 1),
             3: Zone(3, "interior-fluid", "interior", "face", 0, n_int - 1)}
    start = n_int
    for k, (zname, ztype, fn, o) in enumerate(bzones):
        zid = 4 + k
        loops.append(fn)
        owner.append(o)
        neigh.append(np.full(len(o), -1))
        fzone.append(np.full(len(o), zid))
        zones[zid] = Zone(zid, zname, ztype, "face", start, start + len(o) - 1)
        start += len(o)
    width = loops[0].shape[1]
    fnodes = np.concatenate(loops).astype(np.int64)
    return UnstructuredMesh(
        dim=dim, nodes=nodes, face_ptr=np.arange(0, width * fnodes.shape[0] + 1, width, dtype=np.int64),
        face_nodes=fnodes.ravel(), owner=np.concatenate(owner).astype(np.int64),
        neighbour=np.concatenate(neigh).astype(np.int64), face_zone=np.concatenate(fzone).astype(np.int64),
        n_cells=n_cells, cell_zone=np.full(n_cells, 2, dtype=np.int64), zones=zones, name=name)


def cartesian_mesh_2d(nx: int, ny: int, lx: float = 1.0, ly: float = 1.0,
                      names=("left", "right", "bottom", "top"), types=("wall", "wall", "wall", "wall"),
                      triangulate=False, jitter: float = 0.0, seed: int = 0, x0: float = 0.0, y0: float = 0.0,
                      warp: float = 0.0, xs=None, ys=None) -> UnstructuredMesh:
    """Quad or triangle mesh of a rectangle with four boundary zones.

    Same numbering and options as ``flowtrace/mesh/unstructured.py:430-556``: node (i, j) is
    ``i (ny+1) + j``, quad (i, j) is ``i ny + j``; interior vertical faces, then interior
    horizontal faces, then the left/right/bottom/top zones; ``jitter`` moves interior nodes by
    U(-jitter, jitter) spacings from ``default_rng(seed)`` (x draws, then y draws); ``warp`` is
    the smooth sinusoidal distortion. ``triangulate=True`` (or ``"single"``) splits every
    quad along its (i, j)-(i+1, j+1) diagonal as the reference does; ``"alternating"`` uses
    that diagonal where i + j is even and the (i+1, j)-(i, j+1) diagonal where it is odd.
    """
    if xs is not None:
        xs = np.asarray(xs, dtype=float)
        nx, lx = xs.size - 1, float(xs[-1] - xs[0])
    else:
        xs = x0 + np.linspace(0, lx, nx + 1)
    if ys is not None:
        ys = np.asarray(ys, dtype=float)
        ny, ly = ys.size - 1, float(ys[-1] - ys[0])
    else:
        ys = y0 + np.linspace(0, ly, ny + 1)
    X, Y = np.meshgrid(xs, ys, indexing="ij")
    if jitter:
        rng = np.random.default_rng(seed)
        X[1:-1, 1:-1] += rng.uniform(-jitter, jitter, (nx - 1, ny - 1)) * (lx / nx)
        Y[1:-1, 1:-1] += rng.uniform(-jitter, jitter, (nx - 1, ny - 1)) * (ly / ny)
    if warp:
        sx = (X - xs[0]) / (xs[-1] - xs[0])
        sy = (Y - ys[0]) / (ys[-1] - ys[0])
        dw = warp * np.sin(2 * np.pi * sx) * np.sin(2 * np.pi * sy)
        X = X + dw * (xs[-1] - xs[0])
        Y = Y + dw * (ys[-1] - ys[0])
    nodes = np.stack([X.ravel(), Y.ravel()], axis=1)
    node = lambda i, j: i * (ny + 1) + j  # noqa: E731

    def grid(ilo, ihi, jlo, jhi):
        I, J = np.meshgrid(np.arange(ilo, ihi), np.arange(jlo, jhi), indexing="ij")
        return I.ravel(), J.ravel()

    mode = {False: None, None: None, True: "single", "single": "single", "alternating": "alternating"}[triangulate]
    if mode is None:
        quad = lambda i, j: i * ny + j  # noqa: E731
        right_of = left_of = top_of = bottom_of = quad
        n_cells = nx * ny
        diag = []
    else:
        # two triangles per quad: 2 q + t. With the (i,j)-(i+1,j+1) diagonal, t = 0 is the
        # lower-right triangle (bottom and right edges), t = 1 the upper-left one (top, left).
        # With the (i+1,j)-(i,j+1) diagonal, t = 0 is lower-left (bottom, left) and t = 1
        # upper-right (top, right).
        anti = (lambda i, j: (i + j) % 2 == 1) if mode == "alternating" else (lambda i, j: np.zeros_like(i, bool))
        tri = lambda i, j, t: 2 * (i * ny + j) + t  # noqa: E731
        bottom_of = lambda i, j: tri(i, j, 0)  # noqa: E731
        top_of = lambda i, j: tri(i, j, 1)  # noqa: E731
        right_of = lambda i, j: tri(i, j, np.where(anti(i, j), 1, 0))  # noqa: E731
        left_of = lambda i, j: tri(i, j, np.where(anti(i, j), 0, 1))  # noqa: E731
        n_cells = 2 * nx * ny
        I, J = grid(0, nx, 0, ny)
        a = anti(I, J)
        # the diagonal's area vector (dy, -dx) points from the upper triangle to the lower
        # one for the main diagonal, and from lower-left to upper-right for the anti-diagonal
        dnodes = np.where(a[:, None], np.stack([node(I + 1, J), node(I, J + 1)], axis=1),
                          np.stack([node(I, J), node(I + 1, J + 1)], axis=1))
        downer = np.where(a, tri(I, J, 0), tri(I, J, 1))
        dneigh = np.where(a, tri(I, J, 1), tri(I, J, 0))
        diag = [(dnodes, downer, dneigh)]
    I, J = grid(1, nx, 0, ny)
    vert = (np.stack([node(I, J), node(I, J + 1)], axis=1), right_of(I - 1, J), left_of(I, J))
    I, J = grid(0, nx, 1, ny)
    horiz = (np.stack([node(I + 1, J), node(I, J)], axis=1), top_of(I, J - 1), bottom_of(I, J))
    j, i = np.arange(ny), np.arange(nx)
    zero_j, zero_i = np.zeros_like(j), np.zeros_like(i)
    sides = {
        "left": (np.stack([node(0, j + 1), node(0, j)], axis=1), left_of(zero_j, j)),
        "right": (np.stack([node(nx, j), node(nx, j + 1)], axis=1), right_of(zero_j + nx - 1, j)),
        "bottom": (np.stack([node(i, 0), node(i + 1, 0)], axis=1), bottom_of(i, zero_i)),
        "top": (np.stack([node(i + 1, ny), node(i, ny)], axis=1), top_of(i, zero_i + ny - 1)),
    }
    bz = [(names[k], types[k]) + sides[s] for k, s in enumerate(("left", "right", "bottom", "top"))]
    suffix = {None: "", "single": "-tri", "alternating": "-alt"}[mode]
    return _assemble_mesh(2, nodes, diag + [vert, horiz], n_cells, bz, f"rect{nx}x{ny}{suffix}")


def box_mesh_3d(nx: int, ny: int, nz: int, lx: float = 1.0, ly: float = 1.0, lz: float = 1.0,
                jitter: float = 0.0, seed: int = 0,
                names=("xmin", "xmax", "ymin", "ymax", "zmin", "zmax"),
                types=("wall", "wall", "wall", "wall", "wall", "wall")) -> UnstructuredMesh:
    """Hexahedral box [0,lx]x[0,ly]x[0,lz] with six boundary zones (zones that share a name are
    merged). Interior nodes move by U(-jitter, jitter) spacings in x, y and z (draws from
    ``default_rng(seed)``: x, then y, then z). Node (i,j,k) = (i (ny+1) + j)(nz+1) + k and
    cell (i,j,k) = (i ny + j) nz + k; interior x-, y-, then z-faces, then the boundary zones."""
    xs, ys, zs = (np.linspace(0, L, n + 1) for L, n in ((lx, nx), (ly, ny), (lz, nz)))
    X, Y, Z = np.meshgrid(xs, ys, zs, indexing="ij")
    if jitter:
        rng = np.random.default_rng(seed)
        shape = (nx - 1, ny - 1, nz - 1)
        X[1:-1, 1:-1, 1:-1] += rng.uniform(-jitter, jitter, shape) * (lx / nx)
        Y[1:-1, 1:-1, 1:-1] += rng.uniform(-jitter, jitter, shape) * (ly / ny)
        Z[1:-1, 1:-1, 1:-1] += rng.uniform(-jitter, jitter, shape) * (lz / nz)
    nodes = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    node = lambda i, j, k: (i * (ny + 1) + j) * (nz + 1) + k  # noqa: E731
    cell = lambda i, j, k: (i * ny + j) * nz + k  # noqa: E731

    def grid(ri, rj, rk):
        I, J, K = np.meshgrid(np.arange(*ri), np.arange(*rj), np.arange(*rk), indexing="ij")
        return I.ravel(), J.ravel(), K.ravel()

    # node loops whose right-hand normal is +x, +y or +z
    xloop = lambda i, j, k: np.stack([node(i, j, k), node(i, j + 1, k), node(i, j + 1, k + 1), node(i, j, k + 1)], 1)  # noqa: E731,E501
    yloop = lambda i, j, k: np.stack([node(i, j, k), node(i, j, k + 1), node(i + 1, j, k + 1), node(i + 1, j, k)], 1)  # noqa: E731,E501
    zloop = lambda i, j, k: np.stack([node(i, j, k), node(i + 1, j, k), node(i + 1, j + 1, k), node(i, j + 1, k)], 1)  # noqa: E731,E501
    I, J, K = grid((1, nx), (0, ny), (0, nz))
    fx = (xloop(I, J, K), cell(I - 1, J, K), cell(I, J, K))
    I, J, K = grid((0, nx), (1, ny), (0, nz))
    fy = (yloop(I, J, K), cell(I, J - 1, K), cell(I, J, K))
    I, J, K = grid((0, nx), (0, ny), (1, nz))
    fz = (zloop(I, J, K), cell(I, J, K - 1), cell(I, J, K))
    sides = []
    I, J, K = grid((0, 1), (0, ny), (0, nz))
    sides.append((xloop(I, J, K)[:, ::-1], cell(I, J, K)))
    sides.append((xloop(I + nx, J, K), cell(I + nx - 1, J, K)))
    I, J, K = grid((0, nx), (0, 1), (0, nz))
    sides.append((yloop(I, J, K)[:, ::-1], cell(I, J, K)))
    sides.append((yloop(I, J + ny, K), cell(I, J + ny - 1, K)))
    I, J, K = grid((0, nx), (0, ny), (0, 1))
    sides.append((zloop(I, J, K)[:, ::-1], cell(I, J, K)))
    sides.append((zloop(I, J, K + nz), cell(I, J, K + nz - 1)))
    merged: Dict[str, list] = {}
    order: List[str] = []
    for k, (fn, o) in enumerate(sides):
        if names[k] not in merged:
            merged[names[k]] = [types[k], [], []]
            order.append(names[k])
        merged[names[k]][1].append(fn)
        merged[names[k]][2].append(o)
    bz = [(nm, merged[nm][0], np.concatenate(merged[nm][1]), np.concatenate(merged[nm][2])) for nm in order]
    return _assemble_mesh(3, nodes, [fx, fy, fz], nx * ny * nz, bz, f"box{nx}x{ny}x{nz}")


def extrude_to_3d(mesh2d: UnstructuredMesh, nz: int, lz: float,
                  front=("front", "symmetry"), back=("back", "symmetry")) -> UnstructuredMesh:
    """Extrude a 2-D mesh into prisms/hexes along z (``flowtrace/mesh/unstructured.py:647-711``):
    per layer the side faces (a,k)(b,k)(b,k+1)(a,k+1) of every 2-D face, then the cap faces
    between layers (interior) and at z = 0 (``back``) and z = lz (``front``); faces are then
    sorted by zone."""
    if mesh2d.dim != 2:
        raise ValueError("need a 2-D mesh")
    nn2, nc2 = mesh2d.n_nodes, mesh2d.n_cells
    zs = np.linspace(0.0, lz, nz + 1)
    nodes = np.concatenate([np.column_stack([mesh2d.nodes, np.full(nn2, z)]) for z in zs])
    a = mesh2d.face_nodes[mesh2d.face_ptr[:-1]]
    b = mesh2d.face_nodes[mesh2d.face_ptr[:-1] + 1]
    side_loops, side_own, side_nei, side_zone = [], [], [], []
    inner2 = mesh2d.neighbour >= 0
    for k in range(nz):
        side_loops.append(np.stack([a + k * nn2, b + k * nn2, b + (k + 1) * nn2, a + (k + 1) * nn2], axis=1))
        side_own.append(mesh2d.owner + k * nc2)
        side_nei.append(np.where(inner2, np.maximum(mesh2d.neighbour, 0) + k * nc2, -1))
        side_zone.append(mesh2d.face_zone)
    side = np.concatenate(side_loops)
    counts = [np.full(side.shape[0], 4)]
    fnodes = [side.ravel()]
    own, nei, fz = [np.concatenate(side_own)], [np.concatenate(side_nei)], [np.concatenate(side_zone)]
    ptr2, loops2 = mesh2d.cell_polygons_2d()
    cnt2 = np.diff(ptr2)
    zmax = max(mesh2d.zones) + 1
    zones = dict(mesh2d.zones)
    int_zone = next(z.id for z in mesh2d.face_zones() if z.type == "interior")
    cells2 = np.arange(nc2)
    rev = np.concatenate([np.arange(ptr2[c + 1] - 1, ptr2[c] - 1, -1) for c in range(nc2)]) if nc2 else np.zeros(0, int)
    for k in range(nz + 1):
        layer = loops2 + k * nn2
        if k == 0:
            fnodes.append(layer[rev])
            own.append(cells2)
            nei.append(np.full(nc2, -1))
            fz.append(np.full(nc2, zmax))
        elif k == nz:
            fnodes.append(layer)
            own.append(cells2 + (nz - 1) * nc2)
            nei.append(np.full(nc2, -1))
            fz.append(np.full(nc2, zmax + 1))
        else:
            fnodes.append(layer)
            own.append(cells2 + (k - 1) * nc2)
            nei.append(cells2 + k * nc2)
            fz.append(np.full(nc2, int_zone))
        counts.append(cnt2)
    for z in mesh2d.cell_zones():
        idx = np.flatnonzero(np.tile(mesh2d.cell_zone, nz) == z.id)
        zones[z.id] = Zone(z.id, z.name, z.type, "cell", int(idx[0]), int(idx[-1]))
    zones[zmax] = Zone(zmax, back[0], back[1], "face")
    zones[zmax + 1] = Zone(zmax + 1, front[0], front[1], "face")
    counts = np.concatenate(counts)
    m = UnstructuredMesh(dim=3, nodes=nodes, face_ptr=np.concatenate([[0], np.cumsum(counts)]).astype(np.int64),
                         face_nodes=np.concatenate(fnodes).astype(np.int64), owner=np.concatenate(own).astype(np.int64),
                         neighbour=np.concatenate(nei).astype(np.int64), face_zone=np.concatenate(fz).astype(np.int64),
                         n_cells=nc2 * nz, cell_zone=np.tile(mesh2d.cell_zone, nz), zones=zones,
                         name=mesh2d.name + f"-x{nz}")
    return sort_faces_by_zone(m)


def set_cell_zone(mesh: UnstructuredMesh, where, name: str, type: str = "fluid") -> UnstructuredMesh:
    """A new mesh with the cells whose centres satisfy ``where(xc)`` in a new cell zone ``name``
    (id: the largest zone id + 1) of Fluent type ``type`` (``flowtrace/mesh/unstructured.py:611-644``).
    Cells are renumbered by a stable sort on their zone id, so that every cell zone is a
    contiguous range of cells (as Fluent files store them); zones left without cells are
    dropped. Raises ValueError when no cell matches."""
    sel = np.asarray(where(compute_geometry(mesh).cell_centre), dtype=bool)
    if not sel.any():
        raise ValueError("no cell matches the zone condition")
    zid = max(mesh.zones) + 1
    cz = np.where(sel, zid, mesh.cell_zone)
    zones = dict(mesh.zones)
    zones[zid] = Zone(zid, name, type, "cell")
    old_of_new = np.argsort(cz, kind="stable")
    new_of_old = np.empty_like(old_of_new)
    new_of_old[old_of_new] = np.arange(old_of_new.size)
    cz = cz[old_of_new]
    present = set(np.unique(cz).tolist())
    out = {}
    for k, z in zones.items():
        if z.kind != "cell":
            out[k] = z
        elif k in present:
            idx = np.flatnonzero(cz == k)
            out[k] = Zone(z.id, z.name, z.type, "cell", int(idx[0]), int(idx[-1]))
    nei = np.where(mesh.neighbour >= 0, new_of_old[np.maximum(mesh.neighbour, 0)], -1)
    return UnstructuredMesh(dim=mesh.dim, nodes=mesh.nodes, face_ptr=mesh.face_ptr, face_nodes=mesh.face_nodes,
                            owner=new_of_old[mesh.owner], neighbour=nei, face_zone=mesh.face_zone,
                            n_cells=mesh.n_cells, cell_zone=cz, zones=out, name=mesh.name,
                            periodic=list(mesh.periodic))


def extract_cells(mesh: UnstructuredMesh, keep, interface_type: str = "wall"):
    """The sub-mesh of the cells where ``keep`` is True (``flowtrace/mesh/unstructured.py:714-779``):
    the fluid part of a conjugate heat-transfer mesh. Faces between a kept and a dropped cell
    become boundary faces of new zones ``interface-<dropped cell zone>`` (ids after the mesh's
    largest, in order of the first face met), oriented out of the kept cell (a face kept through
    its neighbour has its node loop reversed). Faces are then sorted by zone (interior zones
    first, then by id). Returns (sub-mesh, face map: the original index of every sub-mesh face,
    -(index + 1) where the loop was reversed, cell map: the original index of every sub-mesh
    cell)."""
    keep = np.asarray(keep, dtype=bool)
    if mesh.periodic:
        raise NotImplementedError("extracting cells from a mesh with periodic zones is not supported")
    cmap = np.flatnonzero(keep)
    new_id = np.full(mesh.n_cells, -1, dtype=np.int64)
    new_id[cmap] = np.arange(cmap.size)
    own, nei = mesh.owner, mesh.neighbour
    ko = keep[own]
    kn = (nei >= 0) & keep[np.maximum(nei, 0)]
    whole = ko & (kn | (nei < 0))          # kept as it is (interior of the kept cells, or boundary)
    iface = (ko ^ kn) & (nei >= 0)         # between a kept and a dropped cell
    sel = np.flatnonzero(whole | iface)    # in face order
    flip = iface[sel] & ~ko[sel]           # kept through the neighbour: reverse, neighbour becomes owner
    dropped = np.where(ko[sel], np.maximum(nei[sel], 0), own[sel])
    zones = {zid: z for zid, z in mesh.zones.items() if z.kind == "face"}
    for z in mesh.cell_zones():
        if np.any(keep[mesh.cell_zone == z.id]):
            zones[z.id] = Zone(z.id, z.name, z.type, "cell")
    fzone = mesh.face_zone[sel].copy()
    is_if = iface[sel]
    next_id = max(mesh.zones) + 1
    iface_id = {}
    for dz in mesh.cell_zone[dropped[is_if]].tolist():  # new zone ids in order of first appearance
        if dz not in iface_id:
            oz = mesh.zones[int(dz)]
            iface_id[dz] = next_id
            zones[next_id] = Zone(next_id, f"interface-{oz.name}", interface_type, "face")
            next_id += 1
    if is_if.any():
        fzone[is_if] = np.array([iface_id[dz] for dz in mesh.cell_zone[dropped[is_if]].tolist()], dtype=np.int64)
    owner = np.where(flip, new_id[np.maximum(nei[sel], 0)], new_id[own[sel]])
    neighbour = np.where(is_if | (nei[sel] < 0), -1, new_id[np.maximum(nei[sel], 0)])
    counts = np.diff(mesh.face_ptr)[sel]
    ptr = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    f_of = np.repeat(np.arange(sel.size), counts)
    pos = np.arange(int(counts.sum())) - ptr[f_of]
    src = mesh.face_ptr[sel][f_of] + np.where(flip[f_of], counts[f_of] - 1 - pos, pos)
    fmap = np.where(flip, -(sel + 1), sel)
    present = set(fzone.tolist())
    zones = {k: z for k, z in zones.items() if z.kind == "cell" or k in present}
    sub = UnstructuredMesh(dim=mesh.dim, nodes=mesh.nodes, face_ptr=ptr, face_nodes=mesh.face_nodes[src],
                           owner=owner.astype(np.int64), neighbour=neighbour.astype(np.int64), face_zone=fzone,
                           n_cells=int(cmap.size), cell_zone=mesh.cell_zone[cmap], zones=zones,
                           name=mesh.name + "-fluid")
    zorder = sorted(sub.face_zones(), key=lambda z: (z.type != "interior", z.id))
    rank = {z.id: r for r, z in enumerate(zorder)}
    perm = np.argsort(np.array([rank[z] for z in fzone.tolist()]), kind="stable")
    sub = sort_faces_by_zone(sub)
    for z in sub.cell_zones():
        w = np.flatnonzero(sub.cell_zone == z.id)
        z.first, z.last = int(w[0]), int(w[-1])
    return sub, fmap[perm], cmap


def sort_faces_by_zone(mesh: UnstructuredMesh) -> UnstructuredMesh:
    """Faces reordered so each face zone is contiguous, interior zones first, then by zone id
    (stable within a zone); ``flowtrace/mesh/unstructured.py:783-810``."""
    zorder = sorted(mesh.face_zones(), key=lambda z: (z.type != "interior", z.id))
    rank = {z.id: r for r, z in enumerate(zorder)}
    perm = np.argsort(np.array([rank[z] for z in mesh.face_zone.tolist()]), kind="stable")
    counts = np.diff(mesh.face_ptr)[perm]
    starts = mesh.face_ptr[:-1][perm]
    new_ptr = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    idx = np.repeat(starts - new_ptr[:-1], counts) + np.arange(int(counts.sum()))
    fz = mesh.face_zone[perm]
    zones = dict(mesh.zones)
    for z in zorder:
        where = np.flatnonzero(fz == z.id)
        zones[z.id] = Zone(z.id, z.name, z.type, "face", int(where[0]), int(where[-1]))
    inv = np.empty(perm.size, dtype=np.int64)
    inv[perm] = np.arange(perm.size)
    periodic = [dict(p, faces_a=inv[p["faces_a"]], faces_b=inv[p["faces_b"]]) for p in mesh.periodic]
    return UnstructuredMesh(dim=mesh.dim, nodes=mesh.nodes, face_ptr=new_ptr, face_nodes=mesh.face_nodes[idx],
                            owner=mesh.owner[perm], neighbour=mesh.neighbour[perm], face_zone=fz,
                            n_cells=mesh.n_cells, cell_zone=mesh.cell_zone, zones=zones, name=mesh.name,
                            periodic=periodic)


def union_mesh(meshes: List[UnstructuredMesh], prefixes: Optional[List[str]] = None,
               name: str = "batch") -> UnstructuredMesh:
    """Disjoint union of meshes of one dimension: the block-diagonal batch of independent cases.

    Cells, faces and nodes of mesh i follow those of meshes 0..i-1; every zone is kept, renamed
    ``prefixes[i] + name`` (default ``"c{i}/"``) with a fresh id, and the faces are then sorted by
    zone (interior zones first). ``union_groups`` gives the mesh each union cell came from."""
    if not meshes:
        raise ValueError("no meshes")
    dim = meshes[0].dim
    if any(m.dim != dim for m in meshes):
        raise ValueError("meshes of different dimensions")
    if any(m.periodic for m in meshes):
        raise NotImplementedError("periodic meshes cannot be batched")
    prefixes = prefixes or [f"c{i}/" for i in range(len(meshes))]
    nodes, fptr, fnodes, own, nei, fz, cz, zones = [], [np.zeros(1, dtype=np.int64)], [], [], [], [], [], {}
    n_off = c_off = fn_off = 0
    zid = 1
    for m, pre in zip(meshes, prefixes):
        remap = {}
        for z in sorted(m.zones.values(), key=lambda z: z.id):
            remap[z.id] = zid
            zones[zid] = Zone(zid, pre + z.name, z.type, z.kind)
            zid += 1
        lut = np.zeros(max(m.zones) + 1, dtype=np.int64)
        for old, new in remap.items():
            lut[old] = new
        nodes.append(m.nodes)
        fptr.append(m.face_ptr[1:] + fn_off)
        fnodes.append(m.face_nodes + n_off)
        own.append(m.owner + c_off)
        nei.append(np.where(m.neighbour >= 0, m.neighbour + c_off, -1))
        fz.append(lut[m.face_zone])
        cz.append(lut[m.cell_zone])
        n_off += m.n_nodes
        c_off += m.n_cells
        fn_off += int(m.face_ptr[-1])
    cell_zone = np.concatenate(cz)
    for z in zones.values():
        if z.kind == "cell":
            where = np.flatnonzero(cell_zone == z.id)
            if where.size:
                z.first, z.last = int(where[0]), int(where[-1])
    u = UnstructuredMesh(dim=dim, nodes=np.concatenate(nodes), face_ptr=np.concatenate(fptr).astype(np.int64),
                         face_nodes=np.concatenate(fnodes), owner=np.concatenate(own), neighbour=np.concatenate(nei),
                         face_zone=np.concatenate(fz), n_cells=c_off, cell_zone=cell_zone, zones=zones, name=name)
    return sort_faces_by_zone(u)


def union_groups(meshes: List[UnstructuredMesh]) -> np.ndarray:
    """Index of the source mesh of every cell of ``union_mesh(meshes)``."""
    return np.repeat(np.arange(len(meshes)), [m.n_cells for m in meshes])
