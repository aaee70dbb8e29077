"""Generates ``tests/golden/report_fixtures.npz``: the reference's wall reports
(``wall_forces``, ``wall_report``, ``wall_profile``; ``flowtrace/unstructured/simple.py:906-1001``)
after a number of outer iterations on the cases of ``tests/golden/report_cases.py``, with the
fields they were computed from.

    python tests/golden/make_report_golden.py [--reference /root/reference]
"""

from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from tests.golden.report_cases import REPORT_CASES  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    args = ap.parse_args()
    sys.path.insert(0, args.reference)
    from flowtrace import native
    from flowtrace.hardware.backend import get_backend
    from flowtrace.mesh.unstructured import cartesian_mesh_2d, extrude_to_3d
    from flowtrace.unstructured.case import BoundarySpec, UnstructuredCase
    from flowtrace.unstructured.simple import SimpleSolver

    cpu = get_backend("numpy")
    out = {}
    with native.disabled():
        for name, (build, kw, n, zone) in REPORT_CASES.items():
            bnd = {z: BoundarySpec(**spec) for z, spec in kw["boundaries"].items()}
            s = SimpleSolver(build(cartesian_mesh_2d, extrude_to_3d),
                             UnstructuredCase(backend="numpy", **{**kw, "boundaries": bnd}), cpu)
            for _ in range(n):
                s.step()
            p = f"rep|{name}|"
            for k, v in s.fields().items():
                out[p + "field|" + k] = np.asarray(v, dtype=np.float64)
            rep = {"wall_forces": s.wall_forces(), "wall_report": s.wall_report()}
            out[p + "json"] = np.frombuffer(json.dumps(rep, sort_keys=True).encode(), dtype=np.uint8)
            for k, v in s.wall_profile(zone).items():
                out[p + "profile|" + k] = np.asarray(v, dtype=np.float64)
    path = os.path.join(HERE, "report_fixtures.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {len(out)} arrays to {path} ({os.path.getsize(path)} bytes)")


if __name__ == "__main__":
    main()
