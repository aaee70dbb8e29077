"""Meshes with a solid cell zone, shared by ``make_extract_golden.py`` and ``tests/test_host.py``:
each generated mesh gets a second cell zone (type solid) for the cells whose centre satisfies a
predicate; the keep mask is its complement (the fluid)."""

from __future__ import annotations

import hashlib

import numpy as np


def with_solid_zone(mesh, predicate, name="solid"):
    """The mesh's cells whose centre satisfies ``predicate`` moved to a new solid cell zone."""
    from gputest_b200.mesh.unstructured import Zone, compute_geometry

    xc = compute_geometry(mesh).cell_centre
    sel = predicate(xc)
    zid = max(mesh.zones) + 1
    mesh.cell_zone = np.where(sel, zid, mesh.cell_zone).astype(np.int64)
    mesh.zones[zid] = Zone(zid, name, "solid", "cell", 0, -1)
    return mesh, ~sel


def zoned_meshes():
    from gputest_b200.mesh.unstructured import box_mesh_3d, cartesian_mesh_2d

    return {
        "quad_lower_half": with_solid_zone(cartesian_mesh_2d(8, 6), lambda x: x[:, 1] < 0.5),
        "tri_disc": with_solid_zone(cartesian_mesh_2d(12, 12, triangulate=True, jitter=0.1, seed=4),
                                    lambda x: (x[:, 0] - 0.5) ** 2 + (x[:, 1] - 0.5) ** 2 < 0.09, "heater"),
        "hex_slab": with_solid_zone(box_mesh_3d(5, 4, 3, jitter=0.1, seed=2), lambda x: x[:, 0] < 0.45, "wall-block"),
    }


def extract_digest(sub, fmap, cmap) -> dict:
    from tests.golden.fluent_cases import digest

    out = digest(sub)
    out["face_map"] = hashlib.sha256(np.ascontiguousarray(fmap, dtype=np.int64).tobytes()).hexdigest()
    out["cell_map"] = hashlib.sha256(np.ascontiguousarray(cmap, dtype=np.int64).tobytes()).hexdigest()
    out["name"] = sub.name
    return out


def cell_zone_cases(cartesian_mesh_2d, extrude_to_3d, set_cell_zone):
    """Meshes built with ``set_cell_zone`` (once or twice) from generated meshes; the generators
    and ``set_cell_zone`` are passed in, so that the reference's and this package's build them."""
    m1 = cartesian_mesh_2d(30, 3, 3.0, 1.0)
    m1 = set_cell_zone(m1, lambda x: x[:, 0] < 1.0, "a", "solid")
    m1 = set_cell_zone(m1, lambda x: x[:, 0] > 2.0, "b", "solid")
    return {
        "quad_lower_half": set_cell_zone(cartesian_mesh_2d(8, 6), lambda x: x[:, 1] < 0.5, "solid", "solid"),
        "tri_disc": set_cell_zone(cartesian_mesh_2d(12, 12, triangulate=True, jitter=0.1, seed=4),
                                  lambda x: (x[:, 0] - 0.5) ** 2 + (x[:, 1] - 0.5) ** 2 < 0.09, "heater", "solid"),
        "hex_slab": set_cell_zone(extrude_to_3d(cartesian_mesh_2d(5, 4, jitter=0.1, seed=2), 3, 1.0),
                                  lambda x: x[:, 0] < 0.45, "wall-block", "solid"),
        "composite_two_zones": m1,
    }
