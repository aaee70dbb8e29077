"""The generated Fluent files and the mesh digest shared by ``make_fluent_golden.py`` and
``tests/test_fluent.py``."""

from __future__ import annotations

import hashlib
import os

import numpy as np

ARRAYS = ("nodes", "face_ptr", "face_nodes", "owner", "neighbour", "face_zone", "cell_zone")


def digest(mesh) -> dict:
    """Sizes, SHA-256 of every array (float64 / int64, C order) and the zone table of a mesh."""
    out = {"dim": int(mesh.dim), "n_cells": int(mesh.n_cells), "n_faces": int(mesh.face_ptr.size - 1),
           "n_nodes": int(mesh.nodes.shape[0])}
    for k in ARRAYS:
        a = np.asarray(getattr(mesh, k))
        a = np.ascontiguousarray(a, dtype=np.float64 if a.dtype.kind == "f" else np.int64)
        out[k] = hashlib.sha256(a.tobytes()).hexdigest()
    out["zones"] = sorted([int(z.id), z.name, z.type, z.kind, int(z.first), int(z.last)] for z in mesh.zones.values())
    return out


def generated_meshes():
    from gputest_b200.mesh.unstructured import box_mesh_3d, cartesian_mesh_2d, extrude_to_3d

    return {"tri2d": cartesian_mesh_2d(12, 9, triangulate="alternating", jitter=0.2, seed=3),
            "hex3d": box_mesh_3d(5, 4, 3, jitter=0.1, seed=1),
            "prism3d": extrude_to_3d(cartesian_mesh_2d(4, 3, triangulate=True), 2, 0.5)}


def generated_cases(directory) -> dict:
    """Write every generated mesh as ASCII and as binary Fluent files under ``directory``."""
    from gputest_b200.mesh.fluent import write_fluent_mesh

    out = {}
    for name, m in generated_meshes().items():
        for binary in (False, True):
            key = f"{name}_{'binary' if binary else 'ascii'}"
            path = os.path.join(directory, key + ".msh")
            write_fluent_mesh(m, path, binary=binary)
            out[key] = path
    return out
