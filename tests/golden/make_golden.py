"""Generates the golden fixtures of ``tests/golden/`` by running the reference itself.

    python tests/golden/make_golden.py [--reference /root/reference]

Imports FlowTrace from the reference checkout (its NumPy path, native kernels disabled) and
records, on the meshes and seeded inputs of the reference's own tests
(``tests/test_native.py:23-64``, ``tests/test_gpu_real.py:92-107``, ``tests/test_diagnostics.py:52-75``):

* hashes of generated meshes (node, face and zone arrays);
* finite-volume operators on two meshes: face interpolation, least-squares and Green-Gauss
  gradients, matrix assembly and the incidence products;
* Jacobi-BiCGSTAB results for three (tol, maxiter) pairs;
* the smoothed-aggregation hierarchy and one V-cycle of a captured pressure matrix;
* SIMPLEC fields, residuals and linear-solver counts after a number of outer iterations, and the
  systems captured in one iteration.

The fixtures are small (.npz) and committed; the tests compare the oracle (CPU) and the CUDA
path (GPU) against them, so the reference is not needed to run the tests.
"""

from __future__ import annotations

import argparse
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def mesh_digest(m) -> str:
    h = hashlib.sha256()
    for a in (m.nodes, m.face_ptr, m.face_nodes, m.owner, m.neighbour, m.face_zone, m.cell_zone):
        h.update(np.ascontiguousarray(a).tobytes())
    for k in sorted(m.zones):
        z = m.zones[k]
        h.update(f"{z.id}|{z.name}|{z.type}|{z.kind}|{z.first}|{z.last}".encode())
    return h.hexdigest()


MESH_CASES = {
    "quad5x4": dict(nx=5, ny=4),
    "tri20x16w": dict(nx=20, ny=16, triangulate=True, warp=0.05),
    "tri32j": dict(nx=32, ny=32, triangulate=True, jitter=0.2),
    "quad6x5j3": dict(nx=6, ny=5, jitter=0.1, seed=3),
    "chan7x3": dict(nx=7, ny=3, lx=4.0, ly=1.0, names=("inlet", "outlet", "bottom", "top"),
                    types=("velocity-inlet", "pressure-outlet", "wall", "wall")),
}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    args = ap.parse_args()
    sys.path.insert(0, args.reference)
    from flowtrace import native
    from flowtrace.hardware.backend import get_backend
    from flowtrace.linalg.amg import SmoothedAggregationAMG
    from flowtrace.linalg.krylov import bicgstab
    from flowtrace.mesh.unstructured import cartesian_mesh_2d, extrude_to_3d
    from flowtrace.unstructured.case import BoundarySpec, UnstructuredCase
    from flowtrace.unstructured.fvmesh import FVMesh
    from flowtrace.unstructured.simple import SimpleSolver

    cpu = get_backend("numpy")
    out = {}
    # ---- mesh generators
    for name, kw in MESH_CASES.items():
        out[f"mesh|{name}"] = np.frombuffer(mesh_digest(cartesian_mesh_2d(**kw)).encode(), dtype=np.uint8)
    out["mesh|extrude6x5w"] = np.frombuffer(mesh_digest(extrude_to_3d(cartesian_mesh_2d(6, 5, warp=0.05), 4, 0.5)).encode(),
                                            dtype=np.uint8)
    # ---- operators (tests/test_native.py:23-48)
    meshes = {"tri2d": cartesian_mesh_2d(20, 16, triangulate=True, warp=0.05),
              "hex3d": extrude_to_3d(cartesian_mesh_2d(6, 5, warp=0.05), 4, 0.5)}
    with native.disabled():
        for name, mesh in meshes.items():
            fv = FVMesh(mesh, cpu)
            rng = np.random.default_rng(0)
            phi, phib = rng.standard_normal(fv.nc), rng.standard_normal(fv.n_bf)
            g = rng.standard_normal((fv.nc, fv.dim))
            F, G = rng.standard_normal(fv.n_if), rng.standard_normal((fv.n_if, fv.dim))
            d = 4 + rng.random(fv.nc)
            a1, a2 = -rng.random(fv.n_if), -rng.random(fv.n_if)
            p = f"op|{name}|"
            out[p + "interp"] = fv.face_interp(phi)
            out[p + "interp_vec"] = fv.face_interp_vec(g)
            out[p + "ls"] = fv.gradient(phi, phib)
            out[p + "gg"] = fv.gradient_gg(phi, phib)
            out[p + "gg_corr"] = fv.gradient_gg(phi, phib, g)
            out[p + "cdiff_F"] = fv.Cdiff_d @ F
            out[p + "cown_G"] = fv.Cown_d @ G
            A = fv.matrix(d, a1, a2)
            out[p + "matrix_data"] = A.data
            out[p + "matrix_indptr"] = A.indptr
            out[p + "matrix_indices"] = A.indices
        # ---- BiCGSTAB (tests/test_native.py:51-64)
        fv = FVMesh(cartesian_mesh_2d(24, 24, triangulate=True, warp=0.05), cpu)
        rng = np.random.default_rng(2)
        d = 4 + rng.random(fv.nc)
        A = fv.matrix(d, -rng.random(fv.n_if), -rng.random(fv.n_if))
        b, x0, inv = rng.standard_normal(fv.nc), rng.standard_normal(fv.nc), 1.0 / d
        for tol, maxiter in ((0.1, 30), (1e-10, 500), (1e-10, 3)):
            x, info = bicgstab(lambda v: A @ v, b, np, M=lambda v: inv * v, x0=x0, tol=tol, maxiter=maxiter,
                               relative_to_initial=True)
            p = f"bicg|{tol}|{maxiter}|"
            out[p + "x"] = x
            out[p + "info"] = np.array([info.iterations, info.residual, float(info.converged)])
        # ---- SIMPLEC runs
        top = {"top": BoundarySpec("wall", velocity=[1.0, 0.0])}
        runs = {
            "tri16": (cartesian_mesh_2d(16, 16, triangulate=True, warp=0.05),
                      dict(boundaries=top, viscosity=0.01, max_iter=40, tol=0.0, pressure_tol=1e-9), 40),
            "cavity64": (cartesian_mesh_2d(64, 64),
                         dict(boundaries=top, viscosity=0.01, scheme="upwind", pressure_tol=1e-8, max_iter=300, tol=0.0), 30),
            "channel_energy": (cartesian_mesh_2d(24, 8, 3.0, 1.0, names=("in", "out", "bottom", "top"), warp=0.03),
                               dict(boundaries={"in": BoundarySpec("inlet", velocity=[1.0, 0.0], value=1.0),
                                                "out": BoundarySpec("outlet"),
                                                "bottom": BoundarySpec("wall", thermal="temperature", value=0.0),
                                                "top": BoundarySpec("wall", thermal="flux", value=2.0)},
                                    energy=True, viscosity=0.01, conductivity=0.02, max_iter=50, tol=0.0), 30),
        }
        for name, (mesh, kw, n) in runs.items():
            s = SimpleSolver(mesh, UnstructuredCase(backend="numpy", **kw), cpu)
            for _ in range(n):
                s.step()
            p = f"simplec|{name}|"
            for k, v in s.fields().items():
                out[p + "field|" + k] = v
            for k, v in s.residuals()["scaled"].items():
                out[p + "res|" + k] = np.array([v])
            out[p + "linear"] = np.array(list(s.last_linear["momentum_iters"]) + [s.last_linear["pressure_iters"]])
            if name == "tri16":
                cap = s._capture
                out[p + "cap|A"] = cap["A"].data
                out[p + "cap|Ar"] = cap["Ar"].data
                out[p + "cap|Ap"] = cap["Ap"].data
                out[p + "cap|b"] = np.stack(cap["b"], axis=1)
                out[p + "cap|br"] = np.stack(cap["br"], axis=1)
                out[p + "cap|mass"] = cap["mass"]
                out[p + "cap|U_old"] = cap["U_old"]
                out[p + "cap|Fst"] = cap["Fst"]
        # ---- SA-AMG on the captured pressure matrix of the 48x48 triangle cavity
        s = SimpleSolver(cartesian_mesh_2d(48, 48, triangulate=True, jitter=0.2),
                         UnstructuredCase(backend="numpy", boundaries=top, viscosity=0.01, max_iter=10, tol=0.0), cpu)
        for _ in range(3):
            s.step()
        Ap = s._capture["Ap"]
        amg = SmoothedAggregationAMG(Ap, cpu, singular=True)
        rb = np.random.default_rng(7).standard_normal(Ap.shape[0])
        rb -= rb.mean()
        out["amg|Ap_data"], out["amg|Ap_indptr"], out["amg|Ap_indices"] = Ap.data, Ap.indptr, Ap.indices
        out["amg|sizes"] = np.array([lv[0].shape[0] for lv in amg.levels] + [amg.coarse_n])
        out["amg|b"] = rb
        out["amg|vcycle"] = amg(rb)
    path = os.path.join(HERE, "reference_fixtures.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: {len(out)} arrays, {os.path.getsize(path) / 1e6:.2f} MB")


if __name__ == "__main__":
    main()
