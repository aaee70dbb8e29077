"""Generates ``tests/golden/sst_fixtures.npz`` by running the reference's k-omega SST solver.

    python tests/golden/make_sst_golden.py [--reference /root/reference]

Imports FlowTrace from the reference checkout (its NumPy path, native kernels disabled) and
records, for the turbulent cases of ``SST_CASES`` (``tests/golden/sst_cases.py``):

* the wall distance of every cell and the inlet/initial turbulence values;
* after a number of outer iterations: every field the solver reports (velocity, pressure,
  k, omega, mu_t, the viscosity ratio, y+ and, with energy, temperature), the scaled residuals
  (k and omega included) and the linear-solver iteration counts;
* the face viscosities of the momentum equations (mu + mu_t inside, the wall-function viscosity on
  walls) and the transpose-stress source at the state reached;
* Spalding's u+ on a set of wall Reynolds numbers.

The fixtures are small and committed, so the tests need no reference to run.
"""

from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from tests.golden.sst_cases import RE_Y, SST_CASES  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    ap.add_argument("--out", default=os.path.join(HERE, "sst_fixtures.npz"))
    args = ap.parse_args()
    sys.path.insert(0, args.reference)
    from flowtrace import native
    from flowtrace.hardware.backend import get_backend
    from flowtrace.mesh.unstructured import cartesian_mesh_2d, extrude_to_3d
    from flowtrace.unstructured.case import BoundarySpec, UnstructuredCase
    from flowtrace.unstructured.simple import SimpleSolver
    from flowtrace.unstructured.turbulence import spalding_uplus

    cpu = get_backend("numpy")
    out = {"spalding|re_y": RE_Y, "spalding|uplus": spalding_uplus(RE_Y)}
    with native.disabled():
        for name, (mesh_fn, kw, n) in SST_CASES.items():
            mesh = mesh_fn(cartesian_mesh_2d, extrude_to_3d)
            bnd = {z: BoundarySpec(**spec) for z, spec in kw["boundaries"].items()}
            case = UnstructuredCase(backend="numpy", **{**kw, "boundaries": bnd})
            s = SimpleSolver(mesh, case, cpu)
            t = s.turb
            p = f"sst|{name}|"
            out[p + "wall_distance"] = np.asarray(t.y, dtype=np.float64)
            out[p + "kb_in"], out[p + "sb_in"] = t.kb_in, t.sb_in
            out[p + "k0"], out[p + "w0"] = np.asarray(t.k), np.asarray(t.w)
            for _ in range(n):
                s.step()
            for k, v in s.fields().items():
                out[p + "field|" + k] = np.asarray(v, dtype=np.float64)
            for k, v in s.residuals()["scaled"].items():
                out[p + "res|" + k] = np.array([v])
            out[p + "linear"] = np.array(list(s.last_linear["momentum_iters"]) + [s.last_linear["pressure_iters"]])
            gf, gb = t.momentum_viscosity(s.U)
            out[p + "mu_face"], out[p + "mu_bface"] = np.asarray(gf), np.asarray(gb)
            out[p + "transpose_stress"] = np.asarray(t.transpose_stress(s._gU))
            out[p + "iterations"] = np.array([s.iteration])
    np.savez_compressed(args.out, **out)
    print(f"wrote {len(out)} arrays to {args.out} ({os.path.getsize(args.out)} bytes)")


if __name__ == "__main__":
    main()
