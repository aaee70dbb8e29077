"""Generates ``tests/golden/cellzone_digests.json``: digests of the meshes the reference's
``set_cell_zone`` (``flowtrace/mesh/unstructured.py:611-644``) builds for the cases of
``mesh_cases.cell_zone_cases``.

    python tests/golden/make_cellzone_golden.py [--reference /root/reference]
"""

from __future__ import annotations

import argparse
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from tests.golden.fluent_cases import digest  # noqa: E402
from tests.golden.mesh_cases import cell_zone_cases  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    args = ap.parse_args()
    sys.path.insert(0, args.reference)
    from flowtrace.mesh import unstructured as ref

    out = {k: digest(m) for k, m in cell_zone_cases(ref.cartesian_mesh_2d, ref.extrude_to_3d, ref.set_cell_zone).items()}
    with open(os.path.join(HERE, "cellzone_digests.json"), "w") as fh:
        json.dump(out, fh, indent=1, sort_keys=True)
    print(f"wrote {len(out)} digests")


if __name__ == "__main__":
    main()
