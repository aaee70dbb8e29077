"""Generates ``tests/golden/extract_digests.json``: what the reference's ``extract_cells``
(``flowtrace/mesh/unstructured.py:714-779``) builds from the meshes of ``mesh_cases.py`` (each
with a solid cell zone; the fluid cells kept), as digests of the sub-mesh, the face map and the
cell map.

    python tests/golden/make_extract_golden.py [--reference /root/reference]
"""

from __future__ import annotations

import argparse
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from tests.golden.mesh_cases import extract_digest, zoned_meshes  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    args = ap.parse_args()
    sys.path.insert(0, args.reference)
    from flowtrace.mesh import unstructured as ref

    out = {}
    for key, (m, keep) in zoned_meshes().items():
        # the reference's own mesh type, built from the same arrays
        rm = ref.UnstructuredMesh(dim=m.dim, nodes=m.nodes, face_ptr=m.face_ptr, face_nodes=m.face_nodes,
                                  owner=m.owner, neighbour=m.neighbour, face_zone=m.face_zone, n_cells=m.n_cells,
                                  cell_zone=m.cell_zone,
                                  zones={k: ref.Zone(z.id, z.name, z.type, z.kind, z.first, z.last)
                                         for k, z in m.zones.items()}, name=m.name)
        out[key] = extract_digest(*ref.extract_cells(rm, keep))
    with open(os.path.join(HERE, "extract_digests.json"), "w") as fh:
        json.dump(out, fh, indent=1, sort_keys=True)
    print(f"wrote {len(out)} digests")


if __name__ == "__main__":
    main()
