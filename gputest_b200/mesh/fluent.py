"""Ansys Fluent mesh files (.msh, legacy .cas; ASCII or binary sections; optionally gzipped).

``read_fluent_mesh`` is the input step of the path: a Fluent mesh file becomes the
``UnstructuredMesh`` that ``SimpleSolver`` takes (and from it the device mesh). It reads the
sections the reference's reader reads (``flowtrace/mesh/fluent_msh.py:173-418``) and builds the
same arrays from them, so a solve of a file matches the reference's solve of it:

    (0 / 1 "...")                comment / header, skipped
    (2 d)                        dimension
    (10 / 2010 / 3010 ...)       nodes: header (zone first last type [dim]) in hexadecimal, then
                                 ASCII reals, or binary float32 (2010) / float64 (3010)
    (12 / 2012 / 3012 ...)       cell zones (zone first last type [element type])
    (13 / 2013 / 3013 ...)       faces: header (zone first last bc-type face-type); records of
                                 node indices then the two cells c0 c1 (1-based, 0 = none),
                                 fixed length for face types 2, 3, 4, count-prefixed otherwise;
                                 binary sections hold int32
    (18 / 2018 ...)              periodic shadow face pairs
    (39 / 45 (id type name) ..)  zone names and types (decimal id)

Anything else is skipped (balanced parentheses; binary sections up to their "End of Binary
Section" trailer). The arrays follow the reference's conventions: faces in order of their
Fluent index; a face stored with only c1 gets its node loop reversed and c1 as owner; in 3-D
every face loop is reversed (Fluent's right-hand normal points toward c0, the mesh model's out of
the owner); owner = c0 - 1, neighbour = c1 - 1 or -1. An unreadable file raises
``FluentMeshError`` (a ``ValueError``) naming the file; a missing one ``FileNotFoundError``.

``write_fluent_mesh`` writes a mesh as an ASCII (or binary-section) Fluent file.
"""

from __future__ import annotations

import gzip
import os
import zlib
from typing import Dict, List, Tuple

import numpy as np

from .unstructured import BC_CODES, UnstructuredMesh, Zone, face_centres_and_areas

_SPACE = b" \t\r\n\f\v"
_DELIM = _SPACE + b"()"


class FluentMeshError(ValueError):
    """A file that is not a readable Fluent mesh."""


class _Buf:
    """A cursor over the file's bytes with the few lexical steps the format needs."""

    def __init__(self, data: bytes):
        self.b, self.p, self.n = data, 0, len(data)

    def ws(self):
        b, p, n = self.b, self.p, self.n
        while p < n and b[p] in _SPACE:
            p += 1
        self.p = p

    def at(self) -> int:
        self.ws()
        return self.b[self.p] if self.p < self.n else -1

    def take(self, ch: int):
        if self.at() != ch:
            got = chr(self.b[self.p]) if self.p < self.n else "end of file"
            raise FluentMeshError(f"expected '{chr(ch)}' at byte {self.p}, found {got!r}")
        self.p += 1

    def token(self) -> bytes:
        self.ws()
        b, s, n = self.b, self.p, self.n
        e = s
        while e < n and b[e] not in _DELIM:
            e += 1
        self.p = e
        return b[s:e]

    def string(self):
        """Skip a double-quoted string (backslash escapes)."""
        self.take(ord('"'))
        b, p, n = self.b, self.p, self.n
        while p < n and b[p] != ord('"'):
            p += 2 if b[p] == ord("\\") else 1
        self.p = p + 1

    def skip_group(self):
        """Skip one balanced parenthesised group starting at '(' (strings respected)."""
        self.take(ord("("))
        depth, b, n = 1, self.b, self.n
        while depth and self.p < n:
            c = b[self.p]
            if c == ord('"'):
                self.string()
                continue
            depth += (c == ord("(")) - (c == ord(")"))
            self.p += 1
        if depth:
            raise FluentMeshError("unbalanced parentheses")

    def header(self) -> List[bytes]:
        self.take(ord("("))
        toks = []
        while self.at() != ord(")"):
            t = self.token()
            if not t:
                raise FluentMeshError(f"bad section header at byte {self.p}")
            toks.append(t)
        self.p += 1
        return toks

    def ascii_data(self) -> bytes:
        """The body of an ASCII data group '( ... )' (numbers only, no nested groups)."""
        self.take(ord("("))
        e = self.b.find(b")", self.p)
        if e < 0:
            raise FluentMeshError("unterminated data block")
        data = self.b[self.p:e]
        self.p = e + 1
        return data

    def binary_data(self, nbytes: int) -> bytes:
        self.take(ord("("))
        if self.p + nbytes > self.n:
            raise FluentMeshError("binary data block runs past the end of the file")
        data = self.b[self.p:self.p + nbytes]
        self.p += nbytes
        self.take(ord(")"))
        return data

    def binary_trailer(self, index: int):
        """'End of Binary Section <index>' and the closing parenthesis."""
        for word in (b"End", b"of", b"Binary", b"Section"):
            if self.token() != word:
                raise FluentMeshError(f"binary section {index} lacks its trailer")
        self.token()
        self.take(ord(")"))

    def skip_binary_section(self, index: int):
        q = self.b.find(b"End of Binary Section", self.p)
        if q < 0:
            raise FluentMeshError(f"cannot skip binary section {index}")
        self.p = q
        self.binary_trailer(index)


def _hex(t: bytes) -> int:
    return int(t, 16)


def _hex_array(data: bytes) -> np.ndarray:
    toks = data.split()
    return np.array([int(t, 16) for t in toks], dtype=np.int64)


def _face_records(vals: np.ndarray, nf: int, ftype: int):
    """(node counts, node indices, c0, c1, integers used) of nf face records."""
    if ftype in (2, 3, 4):
        k = ftype
        rec = vals[: nf * (k + 2)].reshape(nf, k + 2)
        return np.full(nf, k, dtype=np.int64), rec[:, :k].reshape(-1), rec[:, k].copy(), rec[:, k + 1].copy(), nf * (k + 2)
    counts = np.empty(nf, dtype=np.int64)
    starts = np.empty(nf, dtype=np.int64)
    p = 0
    for f in range(nf):  # count-prefixed (mixed / polygonal) records
        k = int(vals[p])
        counts[f], starts[f] = k, p + 1
        p += k + 3
    idx = np.repeat(starts, counts) + (np.arange(int(counts.sum())) - np.repeat(np.cumsum(counts) - counts, counts))
    last = starts + counts
    return counts, vals[idx], vals[last], vals[last + 1], p


def _load(path_or_bytes, name):
    if isinstance(path_or_bytes, (bytes, bytearray)):
        data, name = bytes(path_or_bytes), name or "mesh"
    else:
        with open(path_or_bytes, "rb") as fh:
            data = fh.read()
        name = name or os.path.basename(str(path_or_bytes))
    if data[:2] == b"\x1f\x8b":
        data = gzip.decompress(data)
    return data, name


def read_fluent_mesh(path_or_bytes, name: str = None) -> UnstructuredMesh:
    """Read a Fluent mesh (a path, or the file's bytes) into an ``UnstructuredMesh``."""
    try:
        data, name = _load(path_or_bytes, name)
        return _parse(data, name)
    except FluentMeshError as exc:
        where = "" if isinstance(path_or_bytes, (bytes, bytearray)) else f"{path_or_bytes}: "
        raise FluentMeshError(f"{where}{exc}") from None
    except (ValueError, IndexError, KeyError, EOFError, gzip.BadGzipFile, zlib.error) as exc:
        where = "" if isinstance(path_or_bytes, (bytes, bytearray)) else f"{path_or_bytes}: "
        raise FluentMeshError(f"{where}not a readable Fluent mesh ({type(exc).__name__}: {exc})") from exc


def _parse(data: bytes, name: str) -> UnstructuredMesh:
    r = _Buf(data)
    dim = None
    nodes_decl = cells_decl = 0
    node_blocks: List[Tuple[int, np.ndarray]] = []
    face_blocks = []  # (zone, first, bc type, counts, nodes, c0, c1)
    cell_blocks = []  # (zone, first, last, type)
    zone_info: Dict[int, Tuple[str, str]] = {}
    periodic = []
    while True:
        c = r.at()
        if c < 0:
            break
        if c != ord("("):  # stray text between sections: skip the line
            e = r.b.find(b"\n", r.p)
            r.p = r.n if e < 0 else e + 1
            continue
        start = r.p
        r.p += 1
        tok = r.token()
        if not tok.isdigit():
            r.p = start
            r.skip_group()
            continue
        index = int(tok)
        if index in (0, 1):
            r.p = start
            r.skip_group()
        elif index == 2:
            dim = int(r.token())
            r.take(ord(")"))
        elif index in (10, 2010, 3010):
            h = [_hex(t) for t in r.header()]
            zid, first, last = h[0], h[1], h[2]
            nd = h[4] if len(h) > 4 else (dim or 3)
            dim = dim or nd
            if zid == 0 or r.at() == ord(")"):
                if zid == 0:
                    nodes_decl = max(last - first + 1, 0)
                r.take(ord(")"))
                continue
            count = last - first + 1
            if index == 10:
                xyz = np.array(r.ascii_data().split(), dtype=np.float64)
                r.take(ord(")"))
            else:
                dt = np.dtype(np.float32 if index == 2010 else np.float64)
                xyz = np.frombuffer(r.binary_data(count * nd * dt.itemsize), dtype=dt).astype(np.float64)
                r.binary_trailer(index)
            if xyz.size != count * nd:
                raise FluentMeshError(f"node zone {zid}: expected {count * nd} coordinates, found {xyz.size}")
            node_blocks.append((first, xyz.reshape(count, nd)))
        elif index in (12, 2012, 3012):
            h = [_hex(t) for t in r.header()]
            zid, first, last, ztype = (h + [0, 0, 0, 0])[:4]
            if zid == 0:
                cells_decl = max(last - first + 1, 0)
                r.take(ord(")"))
                continue
            if r.at() == ord("("):  # per-cell element types of a mixed zone: not needed
                if index == 12:
                    r.ascii_data()
                    r.take(ord(")"))
                else:
                    r.binary_data(4 * (last - first + 1))
                    r.binary_trailer(index)
            else:
                r.take(ord(")"))
            cell_blocks.append((zid, first, last, ztype))
        elif index in (13, 2013, 3013):
            h = [_hex(t) for t in r.header()]
            zid, first, last, bctype, ftype = (h + [0] * 5)[:5]
            if zid == 0 or r.at() == ord(")"):
                r.take(ord(")"))
                continue
            nf = last - first + 1
            if index == 13:
                vals = _hex_array(r.ascii_data())
                r.take(ord(")"))
            else:
                if ftype in (2, 3, 4):
                    vals = np.frombuffer(r.binary_data(4 * nf * (ftype + 2)), dtype=np.int32).astype(np.int64)
                else:  # count-prefixed records: walk them to find the block's length
                    r.take(ord("("))
                    p0, p = r.p, r.p
                    for _ in range(nf):
                        k = int(np.frombuffer(r.b, dtype=np.int32, count=1, offset=p)[0])
                        p += 4 * (k + 3)
                    vals = np.frombuffer(r.b[p0:p], dtype=np.int32).astype(np.int64)
                    r.p = p
                    r.take(ord(")"))
                r.binary_trailer(index)
            counts, fnodes, c0, c1, used = _face_records(vals, nf, ftype)
            if used != vals.size:
                raise FluentMeshError(f"face zone {zid}: expected {used} integers, found {vals.size}")
            face_blocks.append((zid, first, bctype, counts, fnodes, c0, c1))
        elif index in (18, 2018):
            h = r.header()
            if r.at() == ord("("):
                if index == 18:
                    vals = _hex_array(r.ascii_data())
                    r.take(ord(")"))
                else:
                    n2 = 2 * (_hex(h[1]) - _hex(h[0]) + 1)
                    vals = np.frombuffer(r.binary_data(4 * n2), dtype=np.int32).astype(np.int64)
                    r.binary_trailer(index)
                periodic.append((h, vals.reshape(-1, 2) - 1))
            else:
                r.take(ord(")"))
        elif index in (39, 45):
            r.take(ord("("))
            e = r.b.find(b")", r.p)
            toks = r.b[r.p:e].split()
            r.p = e + 1
            zid = int(toks[0])
            ztype = toks[1].decode(errors="replace")
            zname = toks[2].decode(errors="replace") if len(toks) > 2 else f"zone-{zid}"
            zone_info[zid] = (ztype, zname)
            while r.at() == ord("("):
                r.skip_group()
            r.take(ord(")"))
        elif index >= 2000:
            r.skip_binary_section(index)
        else:
            r.p = start
            r.skip_group()

    if dim is None or not node_blocks or not face_blocks:
        raise FluentMeshError("file does not contain a complete Fluent mesh (nodes/faces missing)")
    n_nodes = max(nodes_decl, max(first + xyz.shape[0] - 1 for first, xyz in node_blocks))
    nodes = np.zeros((n_nodes, dim))
    for first, xyz in node_blocks:
        nodes[first - 1:first - 1 + xyz.shape[0]] = xyz[:, :dim]
    face_blocks.sort(key=lambda fb: fb[1])  # faces in order of their Fluent index
    counts = np.concatenate([fb[3] for fb in face_blocks])
    fnodes = np.concatenate([fb[4] for fb in face_blocks]) - 1
    c0 = np.concatenate([fb[5] for fb in face_blocks])
    c1 = np.concatenate([fb[6] for fb in face_blocks])
    fzone = np.concatenate([np.full(fb[3].size, fb[0], dtype=np.int64) for fb in face_blocks])
    ptr = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    # reversed loops: faces stored with only c1 (made owner), and every face in 3-D
    rev = (c0 == 0) & (c1 != 0)
    c0, c1 = np.where(rev, c1, c0), np.where(rev, 0, c1)
    if dim == 3:
        rev = ~rev
    if rev.any():
        f_of = np.repeat(np.arange(counts.size), counts)
        pos = np.arange(fnodes.size) - ptr[f_of]
        src = np.where(rev[f_of], ptr[f_of] + counts[f_of] - 1 - pos, np.arange(fnodes.size))
        fnodes = fnodes[src]
    owner = c0 - 1
    neighbour = np.where(c1 > 0, c1 - 1, -1)
    if owner.size and owner.min() < 0:
        raise FluentMeshError("a face has no cell on either side")
    n_cells = max(cells_decl, int(owner.max()) + 1, int(neighbour.max()) + 1)
    zones: Dict[int, Zone] = {}
    pos = 0
    for zid, _first, bctype, cnt, *_ in face_blocks:
        ztype, zname = zone_info.get(zid, (BC_CODES.get(bctype, "wall"), f"zone-{zid}"))
        zones[zid] = Zone(zid, zname, ztype, "face", pos, pos + cnt.size - 1)
        pos += cnt.size
    cell_zone = np.zeros(n_cells, dtype=np.int64)
    for zid, first, last, ztype in cell_blocks:
        cell_zone[first - 1:last] = zid
        zt, zn = zone_info.get(zid, ("fluid" if ztype == 1 else "solid", f"zone-{zid}"))
        zones[zid] = Zone(zid, zn, zt, "cell", first - 1, last - 1)
    if not cell_blocks:
        zones[1] = Zone(1, "fluid", "fluid", "cell", 0, n_cells - 1)
        cell_zone[:] = 1
    mesh = UnstructuredMesh(dim=dim, nodes=nodes, face_ptr=ptr, face_nodes=fnodes.astype(np.int64),
                            owner=owner.astype(np.int64), neighbour=neighbour.astype(np.int64), face_zone=fzone,
                            n_cells=n_cells, cell_zone=cell_zone, zones=zones, name=name)
    if periodic:
        fc, _ = face_centres_and_areas(mesh)
        for h, pairs in periodic:
            fa, fb = pairs[:, 0], pairs[:, 1]
            if fa.size == 0 or fa.max() >= mesh.n_faces or fb.max() >= mesh.n_faces:
                raise FluentMeshError("periodic face pairs refer to faces outside the mesh")
            mesh.periodic.append({"zone_a": _hex(h[2]), "zone_b": _hex(h[3]), "faces_a": fa, "faces_b": fb,
                                  "translation": (fc[fb] - fc[fa]).mean(axis=0)})
    return mesh


# ------------------------------------------------------------------------------------------ writer
_FLUENT_BC = {v: k for k, v in BC_CODES.items()}


def write_fluent_mesh(mesh: UnstructuredMesh, path: str, binary: bool = False, title: str = "b2s") -> None:
    """Write ``mesh`` as a Fluent mesh file (ASCII sections, or binary node and face sections);
    ``read_fluent_mesh`` of the file gives back the same arrays and zones. Face and cell zones
    must be contiguous ranges (as the generators, ``sort_faces_by_zone`` and ``set_cell_zone``
    leave them); otherwise ValueError."""
    dim, nn, nc, nf = mesh.dim, mesh.n_nodes, mesh.n_cells, mesh.n_faces
    counts = np.diff(mesh.face_ptr)
    fnodes = mesh.face_nodes.copy()
    if dim == 3:  # back to Fluent's orientation (right-hand normal toward c0)
        f_of = np.repeat(np.arange(nf), counts)
        pos = np.arange(fnodes.size) - mesh.face_ptr[f_of]
        fnodes = fnodes[mesh.face_ptr[f_of] + counts[f_of] - 1 - pos]
    out = [f'(0 "{title}")\n'.encode(), f"(2 {dim})\n".encode(), f"(10 (0 1 {nn:x} 0 {dim:x}))\n".encode()]
    if binary:
        out += [f"(3010 (1 1 {nn:x} 1 {dim:x})(".encode(), np.ascontiguousarray(mesh.nodes, dtype=np.float64).tobytes(),
                b")End of Binary Section 3010)\n"]
    else:
        out.append(f"(10 (1 1 {nn:x} 1 {dim:x})(\n".encode())
        out.append("".join(" ".join(f"{v:.17g}" for v in row) + "\n" for row in mesh.nodes).encode())
        out.append(b"))\n")
    out.append(f"(12 (0 1 {nc:x} 0))\n".encode())
    for z in sorted(mesh.cell_zones(), key=lambda z: z.first):
        if z.last < z.first or not np.all(mesh.cell_zone[z.first:z.last + 1] == z.id) or \
                np.count_nonzero(mesh.cell_zone == z.id) != z.last - z.first + 1:
            raise ValueError(f"cell zone {z.name!r} is not a contiguous range of cells (set_cell_zone renumbers "
                             "cells so that it is)")
        out.append(f"(12 ({z.id:x} {z.first + 1:x} {z.last + 1:x} 1 0))\n".encode())
    out.append(f"(13 (0 1 {nf:x} 0))\n".encode())
    for z in sorted(mesh.face_zones(), key=lambda z: z.first):
        f0, f1 = z.first, z.last + 1
        if not np.all(mesh.face_zone[f0:f1] == z.id):
            raise ValueError(f"face zone {z.name!r} is not a contiguous range of faces")
        k = np.unique(counts[f0:f1])
        ftype = int(k[0]) if k.size == 1 and int(k[0]) in (2, 3, 4) else 5
        c0 = mesh.owner[f0:f1] + 1
        c1 = np.where(mesh.neighbour[f0:f1] >= 0, mesh.neighbour[f0:f1] + 1, 0)
        bc = _FLUENT_BC.get(z.type, 3)
        recs = []
        for f in range(f0, f1):
            loop = fnodes[mesh.face_ptr[f]:mesh.face_ptr[f + 1]] + 1
            head = [] if ftype != 5 else [loop.size]
            recs.append(head + loop.tolist() + [int(c0[f - f0]), int(c1[f - f0])])
        hdr = f"{z.id:x} {f0 + 1:x} {f1:x} {bc:x} {ftype:x}"
        if binary:
            flat = np.array([v for rec in recs for v in rec], dtype=np.int32)
            out += [f"(3013 ({hdr})(".encode(), flat.tobytes(), b")End of Binary Section 3013)\n"]
        else:
            out.append(f"(13 ({hdr})(\n".encode())
            out.append("".join(" ".join(f"{v:x}" for v in rec) + "\n" for rec in recs).encode())
            out.append(b"))\n")
    for z in sorted(mesh.zones.values(), key=lambda z: z.id):
        out.append(f"(45 ({z.id} {z.type} {z.name})())\n".encode())
    with open(path, "wb") as fh:
        fh.write(b"".join(out))
