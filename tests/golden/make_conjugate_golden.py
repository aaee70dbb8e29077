"""Generates ``tests/golden/conjugate_fixtures.npz`` by running the reference's conjugate heat
transfer solver (``flowtrace/unstructured/conjugate.py``).

    python tests/golden/make_conjugate_golden.py [--reference /root/reference]

Imports FlowTrace from the reference checkout (its NumPy path, native kernels disabled). For
every case of ``tests/golden/conjugate_cases.py`` (meshes built here and handed to the reference
as its own mesh type, from the same arrays) it records the harmonic face diffusivities, the
solid heat sources and, after a number of outer iterations, every field (fluid fields on the full
mesh, zero in the solids; the temperature everywhere), the residuals, the linear-solver counts
and the heat flows per zone and across the fluid-solid interfaces.
"""

from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from tests.golden.conjugate_cases import CONJUGATE_CASES  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    ap.add_argument("--out", default=os.path.join(HERE, "conjugate_fixtures.npz"))
    args = ap.parse_args()
    sys.path.insert(0, args.reference)
    from flowtrace import native
    from flowtrace.hardware.backend import get_backend
    from flowtrace.mesh import unstructured as ref
    from flowtrace.unstructured.case import BoundarySpec, UnstructuredCase
    from flowtrace.unstructured.conjugate import ConjugateSolver

    cpu = get_backend("numpy")
    out = {}
    with native.disabled():
        for name, (build, kw, n) in CONJUGATE_CASES.items():
            m = build()
            rm = ref.UnstructuredMesh(dim=m.dim, nodes=m.nodes, face_ptr=m.face_ptr, face_nodes=m.face_nodes,
                                      owner=m.owner, neighbour=m.neighbour, face_zone=m.face_zone,
                                      n_cells=m.n_cells, cell_zone=m.cell_zone,
                                      zones={k: ref.Zone(z.id, z.name, z.type, z.kind, z.first, z.last)
                                             for k, z in m.zones.items()}, name=m.name)
            bnd = {z: BoundarySpec(**spec) for z, spec in kw["boundaries"].items()}
            s = ConjugateSolver(rm, UnstructuredCase(backend="numpy", **{**kw, "boundaries": bnd}), cpu)
            p = f"cht|{name}|"
            gf, gb = s._face_gamma()
            out[p + "gamma_face"], out[p + "gamma_bface"] = np.asarray(gf), np.asarray(gb)
            out[p + "q_cell"] = np.asarray(s.q_cell)
            out[p + "cell_map"] = np.asarray(s.cell_map)
            for _ in range(n):
                s.step()
            for k, v in s.fields().items():
                out[p + "field|" + k] = np.asarray(v, dtype=np.float64)
            for k, v in s.residuals()["scaled"].items():
                out[p + "res|" + k] = np.array([v])
            out[p + "linear"] = np.array(list(s.last_linear["momentum_iters"]) + [s.last_linear["pressure_iters"]])
            out[p + "iterations"] = np.array([s.iteration])
            hf = s.heat_flow()
            out[p + "heat_flow"] = np.frombuffer(json.dumps(hf, sort_keys=True).encode(), dtype=np.uint8)
    np.savez_compressed(args.out, **out)
    print(f"wrote {len(out)} arrays to {args.out} ({os.path.getsize(args.out)} bytes)")


if __name__ == "__main__":
    main()
