"""Generates ``tests/golden/fluent_digests.json``: what the reference's own Fluent reader
(``flowtrace/mesh/fluent_msh.py:173-418``) builds from

* the Fluent mesh files the reference ships (``tests/data/SquareCylinder-Coarse.msh`` and
  ``examples/*.msh*``; read in place, not copied), and
* files written by ``gputest_b200.mesh.fluent.write_fluent_mesh`` from three generated meshes
  (2-D triangles, 3-D hexahedra, 3-D prisms with mixed face types), with ASCII and with binary
  sections,

recorded as digests (sizes, SHA-256 of every array, the zone table), so that the tests can pin
``read_fluent_mesh`` against the reference without the reference present.

    python tests/golden/make_fluent_golden.py [--reference /root/reference]
"""

from __future__ import annotations

import argparse
import glob
import json
import os
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from tests.golden.fluent_cases import digest, generated_cases  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    args = ap.parse_args()
    sys.path.insert(0, args.reference)
    from flowtrace.mesh.fluent_msh import read_fluent_mesh as ref_read

    out = {"shipped": {}, "generated": {}}
    files = [os.path.join(args.reference, "tests", "data", "SquareCylinder-Coarse.msh")]
    files += sorted(glob.glob(os.path.join(args.reference, "examples", "*.msh*")))
    for f in files:
        rel = os.path.relpath(f, args.reference)
        out["shipped"][rel] = digest(ref_read(f))
    with tempfile.TemporaryDirectory() as d:
        for key, path in generated_cases(d).items():
            out["generated"][key] = digest(ref_read(path))
    with open(os.path.join(HERE, "fluent_digests.json"), "w") as fh:
        json.dump(out, fh, indent=1, sort_keys=True)
    print(f"wrote {len(out['shipped'])} shipped and {len(out['generated'])} generated digests")


if __name__ == "__main__":
    main()
