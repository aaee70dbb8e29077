"""Benchmark of the B200 SIMPLEC outer iteration (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config c2] [--impl ours|reference]

Metric: SIMPLEC cell-iterations/s (cells x outer iterations / device time of ``step()``).
A "step" is one outer iteration of the hot path over the workload's mesh. Workload (default):
the 2-D cavity on a 256 x 256 quad grid cut into 131,072 triangles along alternating
diagonals, interior nodes jittered by +-0.2h (seed 0), Re 1000, linear-upwind convection with
non-orthogonal correction, aggregation-AMG pressure solve, FP64 (synthetic mesh and fields).

Timed region: W untimed warm-up steps (the first builds the AMG hierarchy), then exactly K
steps, each bracketed by CUDA events on the solver's stream; L2 is flushed (a 512 MiB write)
between timed steps, outside the events. ``value`` sums the K step times; with N > 1 every
rank runs an independent replica (the path does not shard: replicas only), the time is the
max over ranks and ``value`` the aggregate. ``e2e`` is the same metric through the public API
from host data: constructing ``SimpleSolver`` from the host mesh (its host->device copies),
W + K steps (each reads its residual report back) and the final ``fields()`` read.

``--impl reference`` times the reference's CPU path on the host's cores: the oracle driver
with the reference's own C++/OpenMP kernels (built from its sources into ``oracle/_ref``) or,
without that library, the NumPy oracle; rank 0 only.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "SIMPLEC cell-iters/s to 1e-6 residual vs plain FP64 GPU path; HBM % of peak"
UNIT = "cell-iters/s"


# ---------------------------------------------------------------------------------- workloads
def make_workload(name):
    import numpy as np

    from gputest_b200.mesh.unstructured import box_mesh_3d, cartesian_mesh_2d
    from gputest_b200.unstructured.case import BoundarySpec, UnstructuredCase

    if name == "c1":
        mesh = cartesian_mesh_2d(64, 64)
        case = UnstructuredCase(boundaries={"top": BoundarySpec("wall", velocity=[1.0, 0.0])}, viscosity=0.01,
                                scheme="upwind", pressure_tol=1e-8, max_iter=300, tol=1e-6)
        desc = {"workload": "cavity 64x64 quads (4,096 cells), Re 100, upwind, PCG 1e-8", "cells": mesh.n_cells}
        return mesh, case, desc, None, {}
    if name == "c2":
        mesh = cartesian_mesh_2d(256, 256, triangulate="alternating", jitter=0.2, seed=0)
        case = UnstructuredCase(boundaries={"top": BoundarySpec("wall", velocity=[1.0, 0.0])}, viscosity=1e-3,
                                scheme="second-order", max_iter=100000, tol=1e-6)
        desc = {"workload": "cavity 256x256 alternating-diagonal triangles (131,072 cells), jitter 0.2h seed 0, "
                            "Re 1000, linear-upwind + non-orthogonal correction, SA-AMG PCG", "cells": mesh.n_cells}
        return mesh, case, desc, None, {}
    if name == "c3":
        names = ("inlet", "outlet", "wall", "wall", "wall", "wall")
        mesh = box_mesh_3d(128, 64, 64, 4.0, 1.0, 1.0, jitter=0.1, seed=1, names=names,
                           types=("velocity-inlet", "pressure-outlet", "wall", "wall", "wall", "wall"))
        mu = 1.0 / 500.0
        case = UnstructuredCase(boundaries={"inlet": BoundarySpec("inlet", velocity=[1.0, 0.0, 0.0], value=0.0),
                                            "outlet": BoundarySpec("outlet", pressure=0.0),
                                            "wall": BoundarySpec("wall", thermal="flux", value=5e3)},
                                viscosity=mu, energy=True, cp=1.0, conductivity=mu / 0.71, max_iter=100000, tol=1e-6)

        def inlet(solver):
            z = mesh.zone_by_name("inlet")
            fc = solver.fv.boundary_centres_host()[solver.fv.bzone == z.id]
            u = 36.0 * fc[:, 1] * (1 - fc[:, 1]) * fc[:, 2] * (1 - fc[:, 2])
            solver.set_boundary_velocity("inlet", np.stack([u, 0 * u, 0 * u], axis=1))
            solver.initialize({})

        # smoothed aggregation with the strength rule of pyamg's defaults (theta 0): the reference's
        # own theta 0.08 needs ~150 CG iterations per solve on this anisotropic mesh already at 65k
        # cells (operator complexity 6.5); theta 0 needs 4 (complexity 1.5)
        desc = {"workload": "3-D duct 4x1x1, 128x64x64 hexes (524,288 cells), jitter 0.1h seed 1, parabolic inlet "
                            "Re 500, heated walls 5e3 W/m2, Pr 0.71; SA-AMG strength theta 0", "cells": mesh.n_cells}
        return mesh, case, desc, inlet, {"amg_theta": 0.0}
    if name == "sst":
        # turbulent channel, k-omega SST with Spalding wall viscosity; nodes clustered to both walls
        eta = np.linspace(0.0, 1.0, 257)
        ys = 0.5 * (1.0 + np.tanh(2.5 * (2.0 * eta - 1.0)) / np.tanh(2.5))
        mesh = cartesian_mesh_2d(512, 256, 8.0, 1.0, names=("inlet", "outlet", "bottom", "top"),
                                 types=("velocity-inlet", "pressure-outlet", "wall", "wall"), ys=ys)
        case = UnstructuredCase(boundaries={"inlet": BoundarySpec("inlet", velocity=[1.0, 0.0]),
                                            "outlet": BoundarySpec("outlet", pressure=0.0)},
                                viscosity=1e-4, turbulence="k-omega-sst", scheme="second-order",
                                max_iter=100000, tol=1e-6)
        desc = {"workload": "turbulent channel 8x1, 512x256 quads (131,072 cells) clustered to the walls (tanh 2.5), "
                            "Re_h 1e4, k-omega SST with Spalding wall viscosity, linear-upwind U, upwind k/omega, "
                            "SA-AMG PCG", "cells": mesh.n_cells}
        return mesh, case, desc, None, {}
    raise SystemExit(f"unknown config {name!r}")


def make_batch_workload(ncase=256, seed=2, lo=1e3, hi=6.4e4):
    """The batched sweep: ncase independent 2-D cases from ``default_rng(seed)``; per case a fair
    coin picks a lid-driven cavity (unit square) or a 4 x 1 channel, the cell count is log-uniform
    in [lo, hi] (nearest grid), interior nodes jittered by +-0.15h, Re uniform in [100, 2000],
    lid/inlet speed U uniform in [0.5, 2], viscosity U L / Re (L = 1)."""
    import numpy as np

    from gputest_b200.mesh.unstructured import cartesian_mesh_2d
    from gputest_b200.unstructured.case import BoundarySpec, UnstructuredCase

    rng = np.random.default_rng(seed)
    meshes, cases, kinds = [], [], []
    for i in range(ncase):
        cavity = rng.random() < 0.5
        nc = float(np.exp(rng.uniform(np.log(lo), np.log(hi))))
        re = float(rng.uniform(100.0, 2000.0))
        u = float(rng.uniform(0.5, 2.0))
        if cavity:
            n = max(4, int(round(np.sqrt(nc))))
            m = cartesian_mesh_2d(n, n, jitter=0.15, seed=i)
            b = {"top": BoundarySpec("wall", velocity=[u, 0.0])}
        else:
            ny = max(2, int(round(np.sqrt(nc / 4.0))))
            m = cartesian_mesh_2d(4 * ny, ny, 4.0, 1.0, names=("in", "out", "bottom", "top"), jitter=0.15, seed=i)
            b = {"in": BoundarySpec("inlet", velocity=[u, 0.0]), "out": BoundarySpec("outlet"),
                 "bottom": BoundarySpec("wall"), "top": BoundarySpec("wall")}
        meshes.append(m)
        cases.append(UnstructuredCase(boundaries=b, viscosity=u / re, tol=1e-6, max_iter=100000))
        kinds.append("cavity" if cavity else "channel")
    return meshes, cases, kinds


def make_adjoint_workload(nx=512, ny=128, seed=3, corr=0.1):
    """The adjoint workload: a 4 x 1 channel of nx x ny quads, Re 200 (u_in 1, viscosity 1/200),
    upwind convection, SIMPLE with relaxation 0.3 / 0.3 (the relaxation the stability guard
    settles on for porosity contrasts of 1e4); Brinkman porosity alpha = 1e4 sigmoid(8 g), g a
    Gaussian random field of correlation length ``corr`` (white noise from default_rng(seed),
    filtered by exp(-k^2 corr^2 / 2) in Fourier space, unit variance) sampled at the cell centres."""
    import numpy as np

    from gputest_b200.mesh.unstructured import cartesian_mesh_2d, compute_geometry
    from gputest_b200.unstructured.case import BoundarySpec, UnstructuredCase

    mesh = cartesian_mesh_2d(nx, ny, 4.0, 1.0, names=("in", "out", "bottom", "top"))
    case = UnstructuredCase(boundaries={"in": BoundarySpec("inlet", velocity=[1.0, 0.0]), "out": BoundarySpec("outlet"),
                                        "bottom": BoundarySpec("wall"), "top": BoundarySpec("wall")},
                            viscosity=1.0 / 200.0, scheme="upwind", tol=1e-12, max_iter=200000, algorithm="SIMPLE",
                            relax_u=0.3, relax_p=0.3)
    rng = np.random.default_rng(seed)
    white = rng.standard_normal((ny, nx))
    kx = 2 * np.pi * np.fft.fftfreq(nx, d=4.0 / nx)
    ky = 2 * np.pi * np.fft.fftfreq(ny, d=1.0 / ny)
    K2 = ky[:, None] ** 2 + kx[None, :] ** 2
    g = np.real(np.fft.ifft2(np.fft.fft2(white) * np.exp(-0.5 * K2 * corr ** 2)))
    g = (g - g.mean()) / g.std()
    xc = compute_geometry(mesh).cell_centre
    i = np.clip((xc[:, 0] / (4.0 / nx)).astype(int), 0, nx - 1)
    j = np.clip((xc[:, 1] / (1.0 / ny)).astype(int), 0, ny - 1)
    por = 1e4 / (1.0 + np.exp(-8.0 * g[j, i]))
    return mesh, case, por


def run_adjoint(args):
    """dJ/d(porosity) and dJ/du_in by the discrete adjoint against central differences along
    ``args.fd_dirs`` random directions (step 1e-6; porosity directions relative to alpha)."""
    import numpy as np
    import torch

    from gputest_b200.unstructured.adjoint import PorousChannel

    nx, ny = (int(v) for v in args.adj_grid.split("x"))
    mesh, case, por = make_adjoint_workload(nx, ny)
    prob = PorousChannel(mesh, case, "in", "out")
    prob.method = args.adj_method
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    s = prob.solve(por, 1.0)
    e1.record()
    torch.cuda.synchronize()
    primal_ms, its = e0.elapsed_time(e1), s.iteration
    log = lambda *a: print("[c5]", *a, file=sys.stderr, flush=True)  # noqa: E731
    log(f"primal: {its} iterations, {primal_ms / 1e3:.1f} s")
    t0 = time.perf_counter()
    J, d_por, d_uin, info = prob.gradient(tol=args.adj_tol)
    torch.cuda.synchronize()
    adj_s = time.perf_counter() - t0
    log(f"adjoint ({info['method']}): {adj_s:.1f} s, residual {info['residual']:.2e}")
    rng = np.random.default_rng(11)
    h, errs, fd_its = 1e-6, [], []
    for _ in range(args.fd_dirs):
        d = rng.standard_normal(por.size) * por
        d /= np.abs(d / por).max()
        prob.solve(por + h * d, 1.0)
        fd_its.append(prob.solver.iteration)
        Jp = prob.J()
        prob.solve(por - h * d, 1.0)
        Jm = prob.J()
        fd = (Jp - Jm) / (2 * h)
        errs.append(abs(float(d_por @ d) - fd) / max(abs(fd), 1e-300))
        log(f"direction {len(errs)}: adjoint {float(d_por @ d):.12e} fd {fd:.12e} rel {errs[-1]:.2e}")
    prob.solve(por, 1.0 + h)
    Jp = prob.J()
    prob.solve(por, 1.0 - h)
    Jm = prob.J()
    fd_u = (Jp - Jm) / (2 * h)
    return {"J": J, "primal_ms": primal_ms, "primal_iterations": its, "adjoint_seconds": adj_s,
            "method": info["method"], "iterations": info["iterations"], "residual": info["residual"],
            "direct": {k: info[k] for k in ("assemble_s", "factor_s", "solve_s", "jacobian_nnz", "lu_fill",
                                            "eliminated_gradients", "residuals") if k in info},
            "vjp_calls": info["vjp_calls"], "fd_rel_errors_porosity": errs, "dJ_du_in": d_uin, "fd_dJ_du_in": fd_u,
            "fd_rel_error_u_in": abs(d_uin - fd_u) / max(abs(fd_u), 1e-300), "fd_warm_iterations": fd_its,
            "cells": mesh.n_cells}


def run_probe(args):
    """HBM bandwidth probe (``--config probe``) on a 4,194,304-cell 3-D duct (256 x 128 x 128
    jittered hexahedra, inlet / outlet / walls, Re 500: ~350 MB of CSR, several times L2) where
    the data cannot stay in L2: the drop-in solver's own stage kernels through the C ABI - the
    momentum assembly and the pressure-correction assembly (from the initial state, with the
    solver's buffers), the SpMV of the momentum matrix and the fused least-squares gradient of
    1 + dim fields. K timed launches each after W untimed, CUDA events on the launching stream;
    achieved = algorithmic bytes (``stage_bytes``: every array a kernel reads or writes, once) /
    time."""
    import ctypes

    import numpy as np
    import torch

    from gputest_b200 import _lib
    from gputest_b200.mesh.unstructured import box_mesh_3d
    from gputest_b200.unstructured.case import BoundarySpec, UnstructuredCase
    from gputest_b200.unstructured.simple import SimpleSolver

    nx, ny, nz = (int(v) for v in args.probe_grid.split("x"))
    t0 = time.perf_counter()
    mesh = box_mesh_3d(nx, ny, nz, 2.0, 1.0, 1.0, jitter=0.1, seed=1,
                       names=("inlet", "outlet", "wall", "wall", "wall", "wall"),
                       types=("velocity-inlet", "pressure-outlet", "wall", "wall", "wall", "wall"))
    case = UnstructuredCase(boundaries={"inlet": BoundarySpec("inlet", velocity=[1.0, 0.0, 0.0]),
                                        "outlet": BoundarySpec("outlet", pressure=0.0), "wall": BoundarySpec("wall")},
                            viscosity=1.0 / 500.0, tol=0.0, max_iter=1)
    sv = SimpleSolver(mesh, case)
    setup_s = time.perf_counter() - t0
    fv = sv.fv
    L, s = _lib.lib(), _lib.stream_ptr()
    nc, nf, nb, d, nnz = fv.nc, fv.n_if, fv.n_bf, fv.dim, fv.nnz
    g = torch.Generator(device="cuda").manual_seed(0)
    x = torch.rand(nc, dtype=torch.float64, device="cuda", generator=g)
    y = torch.empty_like(x)
    k = 1 + d
    phi = torch.rand(k, nc, dtype=torch.float64, device="cuda", generator=g)
    phib = torch.rand(k, nb, dtype=torch.float64, device="cuda", generator=g)
    grad = torch.empty(k, d, nc, dtype=torch.float64, device="cuda")
    m, bc = fv.cmesh_ref, ctypes.byref(sv.cbc)
    prm = sv._params()
    pr = ctypes.byref(prm)
    Up, F, Fb = sv._Up[sv._cur], sv._F[sv._cur], sv._Fb[sv._cur]
    part = sv.part
    pt = lambda q: part.data_ptr() + 8 * q * sv.nblk  # noqa: E731

    def mom():
        _lib.check(L.b2s_momentum_assemble_d(m, bc, pr, Up.data_ptr(), sv.gUp.data_ptr(), sv.gpf.data_ptr(),
                                             sv.bUp.data_ptr(), F.data_ptr(), Fb.data_ptr(), None, None,
                                             sv.val_A.data_ptr(), sv.diag.data_ptr(), sv.inv.data_ptr(),
                                             sv.dP.data_ptr(), sv.bmom.data_ptr(), sv.brmom.data_ptr(),
                                             pt(sv.Q_MOM), s), "b2s_momentum_assemble_d")

    def pre():
        _lib.check(L.b2s_pressure_assemble_d(m, bc, pr, sv.Ustar.data_ptr(), Up.data_ptr(), sv.gpf.data_ptr(),
                                             sv.dP.data_ptr(), sv.Fst.data_ptr(), sv.cf.data_ptr(),
                                             sv.Fbst.data_ptr(), sv.cb.data_ptr(), sv.val_P.data_ptr(),
                                             sv.rhs_p.data_ptr(), pt(sv.Q_CONT), s), "b2s_pressure_assemble_d")

    _lib.check(L.b2s_flow_bvals_d(m, bc, Up.data_ptr(), None, None, sv.bUp.data_ptr(), s), "b2s_flow_bvals_d")
    mom()
    sv.Ustar.copy_(Up[1:])

    def timed(fn):
        for _ in range(max(args.warmup, 3)):
            fn()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        torch.cuda.synchronize()
        for a, b in ev:
            a.record()
            fn()
            b.record()
        torch.cuda.synchronize()
        return float(np.median([a.elapsed_time(b) for a, b in ev])) / 1e3

    spmv = lambda: _lib.check(L.b2s_spmv_d(nc, 1, fv.rowptr.data_ptr(), fv.col.data_ptr(), sv.val_A.data_ptr(),  # noqa: E731
                                           x.data_ptr(), y.data_ptr(), s), "b2s_spmv_d")
    lsg = lambda: _lib.check(L.b2s_ls_gradient_d(fv.cmesh_ref, k, phi.data_ptr(), phib.data_ptr(),  # noqa: E731
                                                 grad.data_ptr(), s), "b2s_ls_gradient_d")
    sz = 8
    bytes_spmv = nnz * (sz + 4) + 4 * (nc + 1) + 2 * nc * sz
    geom = 8 * nf + nf * sz * (1 + d) + nb * (4 + sz * (1 + d)) + nc * sz * d * d + 4 * 3 * (nc + 1) + 4 * nf
    bytes_lsg = geom + k * (nc + nb) * sz + k * nc * d * sz
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    out = {}
    for name, fn, byts in (("momentum_assembly", mom, stage_bytes(sv, "momentum_assembly", None)),
                           ("pressure_assembly", pre, stage_bytes(sv, "pressure_assembly", None)),
                           ("spmv", spmv, bytes_spmv), ("ls_gradient_4_fields", lsg, bytes_lsg)):
        t = timed(fn)
        out[name] = {"ms": t * 1e3, "algorithmic_bytes": byts, "achieved_gbs": byts / t / 1e9,
                     "frac": byts / t / 1e9 / hbm}
    return {"cells": nc, "faces": nf, "nnz": nnz, "setup_s": setup_s, "kernels": out, "peak": hbm,
            "peak_source": "measured" if "hbm_gbs" in peaks else "fallback"}


# ---------------------------------------------------------------------------------- byte models
def stage_bytes(solver, stage, step_info):
    """Algorithmic DRAM bytes of one launch of a stage: every array the stage's kernels read
    or write, counted once per pass over it (FP64 values 8 B, indices 4 B)."""
    fv = solver.fv
    nc, nf, nb, d, nnz = fv.nc, fv.n_if, fv.n_bf, fv.dim, fv.nnz
    csr = nnz * 12 + (nc + 1) * 4
    face_topo = nf * 4 * 3 + (nc + 1) * 8 + nf * 4  # fP, fN, forig, own/nei ptr, nei_face
    if stage == "momentum_assembly":
        faces = face_topo + nf * 8 * (2 + 3 * d) + nf * 4 * 2  # alpha, F, w, Tv, dPf, dNf, slot_PN/NP
        cells = nc * 8 * (d + d * d + d + 1) + nc * 8 * (3 + 2 * d) + nc * 4 * 2  # U, gU, gp, vol; outputs; slot_diag, bptr
        bnd = nb * 8 * (3 + d) + nb * 4
        return faces + cells + bnd + csr + nnz * 8  # CSR read for the residual, values written
    if stage == "turbulence_terms":  # b2s_sst_momentum_terms_d: face viscosities, wall law, transpose stress
        energy = getattr(solver, "energy", False)
        faces = face_topo + nf * 8 * (1 + d) + nf * 8 * (2 if energy else 1)  # w, S; mu_f (+ kT_f) out
        cells = nc * 8 * (1 + d + d * d) + nc * 8 * d + (nc + 1) * 4  # mu_t, U, grad U; tsrc out; bptr
        bnd = nb * 8 * (1 + 1 + 2 * d) + nb * 8 * (3 if energy else 2)  # m_wall, yb, ub, n; mu_b, y+ (+ kT_b)
        return faces + cells + bnd
    if stage == "pressure_assembly":
        faces = face_topo + nf * 8 * (3 + 2 * d) + nf * 8 * 2 + nf * 4 * 2  # w, alpha, S, d; Fst, cf out; slots
        cells = nc * 8 * (d + 1 + d + 1) + nc * 8 * 2 + nnz * 8
        bnd = nb * 8 * (4 + 3 * d) + nb * 4
        return faces + cells + bnd
    if stage == "momentum_solve":
        import numpy as np

        its = int(np.max(step_info["momentum_iters"]))
        k = d
        init = csr + nc * 8 * k * 6
        per_it = 2 * (csr + nc * 8 * k * 2) + nc * 8 * k * 14 + nc * 8 * 2
        return init + its * per_it
    if stage == "pressure_solve":
        import numpy as np

        amg = solver._amg
        its = int(np.max(step_info["pressure_iters"]))
        init = nc * 8 * 3
        per_it = (csr + nc * 8 * 2) + nc * 8 * 9
        vc = 0
        h = amg.c
        for l in range(h.nlevels):
            lv = h.levels[l]
            a = lv.nnz * 12 + (lv.n + 1) * 4
            pr = lv.p_nnz * 12 + (lv.n + 1) * 4
            rr = lv.p_nnz * 12 + (lv.nc + 1) * 4
            vc += 4 * a + lv.n * 8 * (3 + 3 + 2 + 2 + 8) + pr + rr + lv.nc * 8 * 2
        vc += amg.coarse_n * amg.coarse_n * 8 + amg.coarse_n * 16
        return init + its * (per_it + vc) + vc
    return None


def _smi_target(dev_index):
    """The nvidia-smi id of torch device ``dev_index``: its entry of CUDA_VISIBLE_DEVICES (an
    index or a UUID) when that is set, else the index itself."""
    vis = [v.strip() for v in os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",") if v.strip()]
    return vis[dev_index] if dev_index < len(vis) else str(dev_index)


class ClockSampler:
    """nvidia-smi samples of the SM clock, the power draw, the utilisation and the throttle
    reasons of one GPU every 100 ms, from ``start()`` to ``stop()``, into a temporary file."""

    QUERY = ("clocks.sm,clocks.max.sm,power.draw,utilization.gpu,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, dev_index):
        import tempfile

        self.target = _smi_target(dev_index)
        fd, self.path = tempfile.mkstemp(prefix="b2s_clocks_", suffix=".csv")
        os.close(fd)
        self.proc = None

    def start(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", self.target, f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def stop(self):
        """Stop sampling; the median SM clock over the samples taken under load (utilisation
        above 0), the maximum clock and every throttle reason seen active."""
        if self.proc is None:
            return None
        self.proc.terminate()
        self.proc.wait()
        self.fh.close()
        sm, loaded, mx, reasons = [], [], None, set()
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 8:
                continue
            try:
                clk, mx = float(f[0]), float(f[1])
            except ValueError:
                continue
            sm.append(clk)
            try:
                if float(f[3]) > 0:
                    loaded.append(clk)
            except ValueError:
                pass
            for n, v in zip(self.NAMES, f[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        try:
            os.unlink(self.path)
        except OSError:
            pass
        use = loaded or sm
        return {"sm_mhz": statistics.median(use) if use else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "samples_under_load": len(loaded)}


# ---------------------------------------------------------------------------------- CPU reference
def cpu_reference(mesh, case, inlet, steps, warmup, budget_s=None, amg_theta=0.08):
    """Time the reference's CPU path (oracle driver + the reference's C++ kernels when built)."""
    import numpy as np

    from oracle.simplec_oracle import OracleSimple, load_native

    lib = load_native()
    threads = int(lib.ft_max_threads()) if lib is not None else 1
    o = OracleSimple(mesh, case, native=lib, amg_theta=amg_theta)
    if inlet is not None:
        z = mesh.zone_by_name("inlet")
        fc = o.fv.xfb[o.fv.bzone == z.id]
        u = 36.0 * fc[:, 1] * (1 - fc[:, 1]) * fc[:, 2] * (1 - fc[:, 2])
        ub = o.ub_fixed.copy()
        ub[o.fv.bzone == z.id] = np.stack([u, 0 * u, 0 * u], axis=1)
        o.ub_fixed = ub
        o.initialize({})
    case.tol = 0.0
    for _ in range(warmup):
        o.step()
    t0 = time.perf_counter()
    n = 0
    while n < steps and (budget_s is None or time.perf_counter() - t0 < budget_s or n < 3):
        o.step()
        n += 1
    dt = time.perf_counter() - t0
    kind = "reference" if lib is not None else "port"
    return {"value": mesh.n_cells * n / dt, "unit": UNIT, "cores": threads, "kind": kind, "iterations": n,
            "seconds": dt, "sample": f"{n} outer iterations after {warmup} warm-up of the same workload; "
            + ("oracle driver with the reference's own C++/OpenMP kernels built from its sources"
               if lib is not None else "NumPy/SciPy oracle (reference C++ kernels not built)")}


# ---------------------------------------------------------------------------------- replicas
def max_over_ranks(ms: float, world: int, device=None) -> float:
    """The slowest rank's time: every rank runs an independent replica, so the job takes as long
    as its slowest replica (all-reduce MAX; NCCL on CUDA tensors, gloo on CPU ones)."""
    if world <= 1:
        return ms
    import torch
    import torch.distributed as dist

    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------------- batched sweep
def deal_cases(cells, world):
    """Greedy cells-balanced deal of independent cases to ``world`` ranks: largest case first,
    each to the rank with the fewest cells so far (ties to the lowest rank). Returns, per rank,
    its case indices in increasing order. Every case goes to exactly one rank; the spread of
    the ranks' cell totals is at most the largest case's cell count."""
    import numpy as np

    order = np.argsort([-int(c) for c in cells], kind="stable")
    load = np.zeros(world)
    out = [[] for _ in range(world)]
    for i in order:
        r = int(np.argmin(load))
        load[r] += int(cells[i])
        out[r].append(int(i))
    return [sorted(o) for o in out]


def run_batch(args, rank, world):
    """The batched sweep (``--config c4``): all cases as one ``BatchSimpleSolver`` (the timed arm)
    against the same cases solved one at a time by ``MixedSimpleSolver`` (same arithmetic), on a
    stratified sample of cases whose per-step times are interpolated over the cell count. With
    N > 1 ranks the cases are dealt to ranks by cell count (replicas of the batch mechanism,
    no collective in the data path)."""
    import numpy as np
    import torch

    from gputest_b200.unstructured.batch import BatchSimpleSolver
    from gputest_b200.unstructured.mixed import MixedSimpleSolver

    meshes, cases, kinds = make_batch_workload(args.batch_cases)
    mine = deal_cases([m.n_cells for m in meshes], world)[rank]
    meshes, cases, kinds = [meshes[i] for i in mine], [cases[i] for i in mine], [kinds[i] for i in mine]
    ncell = int(sum(m.n_cells for m in meshes))
    K, W = args.steps, max(args.warmup, 3)
    t0 = time.perf_counter()
    bs = BatchSimpleSolver(meshes, [__import__("copy").deepcopy(c) for c in cases])
    for c in bs.cases + [bs.case]:
        c.tol = 0.0
    setup_s = time.perf_counter() - t0
    tuning = bs.autotune()  # team shapes of the per-case Krylov solves, timed on this batch
    for _ in range(W):  # after the tuning: the graphs are captured with the chosen shapes
        bs.step()
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    l0 = bs.kernel_launches
    torch.cuda.synchronize()
    for k in range(K):
        flush.zero_()
        ev[k][0].record()
        bs.step()
        ev[k][1].record()
    torch.cuda.synchronize()
    launches = bs.kernel_launches - l0
    ms = sum(a.elapsed_time(b) for a, b in ev)
    bs.profile_stages = True
    bs.stage_times.clear()
    infos = []
    for _ in range(K):
        flush.zero_()
        bs.step()
        infos.append(dict(bs.last_linear))
    bs.profile_stages = False
    torch.cuda.synchronize()
    times = dict(bs.stage_times)
    # one case at a time, same arithmetic: a stratified sample by cell count
    idx = np.argsort([m.n_cells for m in meshes], kind="stable")
    sample = sorted(set(int(idx[int(j)]) for j in np.linspace(0, len(idx) - 1, min(args.batch_sample, len(idx))).round()))
    samp = []
    for i in sample:
        c = __import__("copy").deepcopy(cases[i])
        c.tol = 0.0
        s1 = MixedSimpleSolver(meshes[i], c)
        for _ in range(W):
            s1.step()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(K):
            s1.step()
        e1.record()
        torch.cuda.synchronize()
        samp.append((meshes[i].n_cells, e0.elapsed_time(e1) / K))
        del s1
    xs = np.log([a for a, _ in samp])
    ys = np.array([b for _, b in samp])
    seq_ms = float(sum(np.interp(np.log(m.n_cells), xs, ys) for m in meshes))
    one = ncell / (seq_ms / 1e3)
    ms_max = max_over_ranks(ms, world, "cuda")
    tot = torch.tensor([float(ncell) * K], dtype=torch.float64, device="cuda")
    if world > 1:
        import torch.distributed as dist

        dist.all_reduce(tot)
    value = float(tot.item()) / (ms_max / 1e3)
    conv = None
    if args.converge:
        cc = [__import__("copy").deepcopy(c) for c in cases]
        for c in cc:
            c.max_iter = args.batch_converge_max_iter
        bc = BatchSimpleSolver(meshes, cc)
        c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        c0.record()
        bc.run()
        c1.record()
        torch.cuda.synchronize()
        cms = c0.elapsed_time(c1)
        conv = {"all_converged": bool(bc.converged), "iterations": bc.iteration, "seconds": cms / 1e3,
                "case_iterations": {"min": int(bc.case_converged_at.min()), "median": float(np.median(bc.case_converged_at)),
                                    "max": int(bc.case_converged_at.max())},
                "useful_cell_iters_per_s": float(np.dot(bs.case_cells, np.maximum(bc.case_converged_at, 0)) / (cms / 1e3)),
                "value": ncell * bc.iteration / (cms / 1e3)}
    return {"value": value, "ms": ms_max, "ncell": ncell, "ncase": len(meshes), "setup_s": setup_s,
            "launches": launches, "times": times, "infos": infos, "one_at_a_time": one, "seq_ms": seq_ms,
            "sample": samp, "solver": bs, "converge": conv,
            "autotune": {"momentum": list(tuning["momentum"]), "pressure": list(tuning["pressure"]),
                         "fields": ["cluster_blocks", "block_threads", "wide_row"],
                         "ms_momentum_pressure": {"x".join(map(str, k)): v for k, v in tuning["ms"].items()}},
            "kinds": {"cavity": kinds.count("cavity"), "channel": kinds.count("channel")}}


def batch_cpu_reference(args):
    """The reference's CPU path on the batched sweep: the cases run one after another (as the
    reference's batch runner does), timed on a stratified sample of 8 cases for a bounded time
    each and extrapolated over the cell count of all cases."""
    import numpy as np

    meshes, cases, kinds = make_batch_workload(args.batch_cases)
    idx = np.argsort([m.n_cells for m in meshes], kind="stable")
    sample = sorted(set(int(idx[int(j)]) for j in np.linspace(0, len(idx) - 1, 8).round()))
    pts, cores, kind = [], 1, "port"
    for i in sample:
        r = cpu_reference(meshes[i], __import__("copy").deepcopy(cases[i]), None, steps=1000, warmup=1, budget_s=3.0)
        pts.append((meshes[i].n_cells, 1e3 * r["seconds"] / r["iterations"]))
        cores, kind = r["cores"], r["kind"]
    xs, ys = np.log([a for a, _ in pts]), np.array([b for _, b in pts])
    ncell = sum(m.n_cells for m in meshes)
    seq_ms = float(sum(np.interp(np.log(m.n_cells), xs, ys) for m in meshes))
    value = ncell / (seq_ms / 1e3)
    ref = {"value": value, "unit": UNIT, "cores": cores, "kind": kind, "iterations": 1, "seconds": seq_ms / 1e3,
           "sample": f"{len(sample)} of {len(meshes)} cases, one after another, >= 3 s each after 1 warm-up "
                     "iteration; per-iteration time interpolated over the cell count of every case"}
    return ref, batch_desc(args)


def batch_desc(args):
    """Workload description of the whole batched sweep (every case, whatever the rank count)."""
    meshes, _, _ = make_batch_workload(args.batch_cases)
    ncell = sum(m.n_cells for m in meshes)
    return {"workload": f"batched sweep: {len(meshes)} 2-D cavity/channel cases, 1k-64k cells log-uniform, jitter "
                        f"0.15h, Re 100-2000, seed 2 ({ncell:,} cells)", "cells": ncell}


def main_batch(args, rank, world, dev):
    import torch

    smi = ClockSampler(dev).start()
    t_e2e = time.perf_counter()
    r = run_batch(args, rank, world)
    clocks = smi.stop()
    bs, K = r["solver"], args.steps
    torch.cuda.synchronize()
    f = bs.fields()
    e2e_s = time.perf_counter() - t_e2e
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    times = r["times"]
    dom = max((k for k in ("momentum_assembly", "pressure_assembly") if k in times), key=lambda k: times[k])
    byts = sum(stage_bytes(bs, dom, inf) for inf in r["infos"])
    achieved = byts / (times[dom] / 1e3) / 1e9
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
        ref, _ = batch_cpu_reference(args)
        cpu = {k: ref[k] for k in ("value", "unit", "cores", "kind", "sample")}
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    W = max(args.warmup, 3)
    nall = r["ncell"] * world
    line = {"metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": r["ms"] / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 systems, f64 residuals", "data": "synthetic",
            "config": workload_config(batch_desc(args)), "cases": r["kinds"], "cells_rank0": r["ncell"],
            "precision": "mixed", "l2": "flushed between timed steps (512 MiB write)",
            "parallelism": f"cases dealt to {world} ranks" if world > 1 else "single GPU",
            "one_at_a_time": {"value": r["one_at_a_time"], "unit": UNIT, "ratio": r["value"] / world / r["one_at_a_time"],
                              "sample": f"{len(r['sample'])} cases timed alone with MixedSimpleSolver "
                                        f"({K} steps each), per-step time interpolated over the cell count"},
            "e2e": {"value": nall * (W + 2 * K) / e2e_s, "unit": UNIT,
                    "h2d_bytes_per_step": sum(v.numel() * v.element_size() for v in bs.fv.t.values()) / (W + 2 * K),
                    "d2h_bytes_per_step": (bs.report_g.numel() * (W + 2 * K) + sum(v.nbytes for v in f.values()))
                    / (W + 2 * K),
                    "includes": "host set-up of the batch (union mesh, device mesh, AMG), W+2K steps, fields()"},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                         "traffic": None, "algorithmic_bytes_per_launch": byts / K,
                         "stage_ms_per_step": {k: v / K for k, v in sorted(times.items(), key=lambda kv: -kv[1])}},
            "cpu_baseline": cpu, "clocks": clocks, "gpu_launches": r["launches"], "setup_seconds": r["setup_s"],
            "autotune": r["autotune"], "to_convergence": r["converge"]}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------- main
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--config", default="c2")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"],
                    help="fp64: the drop-in SimpleSolver; mixed: MixedSimpleSolver (float systems, double residuals)")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--converge", action="store_true", help="c4: also run the batch to the 1e-6 residual")
    ap.add_argument("--no-amg-setup", action="store_true",
                    help="skip the AMG set-up block (device vs host set-up, re-aggregation policy)")
    ap.add_argument("--no-converge", action="store_true", help="skip the to-convergence runs (FP64 and mixed)")
    ap.add_argument("--no-c3", action="store_true", help="c2: skip the 524,288-cell duct block (FP64 vs mixed)")
    ap.add_argument("--batch-cases", type=int, default=256, help="c4: cases in the sweep")
    ap.add_argument("--batch-sample", type=int, default=24, help="c4: cases timed one at a time")
    ap.add_argument("--converge-max-iter", type=int, default=40000, help="outer-iteration cap of the to-convergence runs")
    ap.add_argument("--batch-converge-max-iter", type=int, default=6000, help="c4: outer-iteration cap of --converge")
    ap.add_argument("--fd-dirs", type=int, default=16, help="c5: random finite-difference directions")
    ap.add_argument("--adj-grid", default="512x128", help="c5: channel grid nx x ny")
    ap.add_argument("--probe-grid", default="256x128x128", help="probe: duct grid nx x ny x nz")
    ap.add_argument("--adj-tol", type=float, default=1e-11,
                    help="adjoint solve tolerance (relative residual; the GMRES solve on the 512x128 channel "
                         "needs about 1e-9, above the products' rounding floor)")
    ap.add_argument("--adj-method", default="direct", choices=("direct", "gmres"),
                    help="c5: adjoint solve (sparse LU of the assembled Jacobian, or preconditioned GMRES)")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
        if args.config == "c4":
            ref, desc = batch_cpu_reference(args)
        else:
            mesh, case, desc, inlet, skw = make_workload(args.config)
            ref = cpu_reference(mesh, case, inlet, args.steps, args.warmup, amg_theta=skw.get("amg_theta", 0.08))
        line = {"metric": METRIC, "value": ref["value"], "unit": UNIT, "n_gpus": args.gpus, "steps": ref["iterations"],
                "warmup": args.warmup, "ms_per_step": 1e3 * ref["seconds"] / ref["iterations"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": workload_config(desc), "parallelism": "host cores", "impl": "reference",
                "cpu_baseline": {k: ref[k] for k in ("value", "unit", "cores", "kind", "sample")},
                "e2e": {"value": ref["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    import torch
    import torch.distributed as dist

    if world > 1:
        import datetime

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    else:
        torch.cuda.set_device(0)
    from gputest_b200.unstructured.mixed import MixedSimpleSolver
    from gputest_b200.unstructured.simple import SimpleSolver

    dev = torch.cuda.current_device()
    if args.config == "c4":
        return main_batch(args, rank, world, dev)
    if args.config == "probe":
        r = run_probe(args)
        if rank == 0:
            line = {"metric": "HBM bandwidth probe: momentum assembly achieved / measured copy bandwidth",
                    "value": r["kernels"]["momentum_assembly"]["frac"],
                    "unit": "fraction", "n_gpus": world, "steps": args.steps, "warmup": max(args.warmup, 3),
                    "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                    "data": "synthetic", "config": {"workload": f"3-D duct 2x1x1, {args.probe_grid} hexahedra "
                                                                f"({r['cells']:,} cells), jitter 0.1h seed 1, Re 500",
                                                    "l2": "inputs larger than L2"},
                    "kernels": r["kernels"], "peak_gbs": r["peak"], "peak_source": r["peak_source"],
                    "setup_seconds": r["setup_s"]}
            print(json.dumps(line), flush=True)
        return
    if args.config == "c5":
        r = run_adjoint(args)
        if rank == 0:
            worst = max(r["fd_rel_errors_porosity"] + [r["fd_rel_error_u_in"]])
            line = {"metric": "adjoint dJ/d(porosity, u_in) max relative error vs central FD", "value": worst,
                    "unit": "relative error", "n_gpus": world, "steps": r["primal_iterations"], "warmup": 0,
                    "ms_per_step": r["primal_ms"] / max(r["primal_iterations"], 1), "higher_is_better": False,
                    "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                    "config": {"workload": f"porous channel 4x1, {args.adj_grid} quads ({r['cells']:,} cells), Re 200, "
                                           "Brinkman alpha = 1e4 sigmoid(8 g), g a Gaussian random field (corr 0.1, "
                                           "seed 3), J = p_in - p_out + viscous dissipation",
                               "fd": f"{args.fd_dirs} random directions + u_in, central, step 1e-6"},
                    "primal_cell_iters_per_s": r["cells"] * r["primal_iterations"] / (r["primal_ms"] / 1e3),
                    "adjoint": {k: r[k] for k in ("adjoint_seconds", "method", "iterations", "residual", "direct",
                                                  "vjp_calls")},
                    "dJ_du_in": r["dJ_du_in"], "fd_dJ_du_in": r["fd_dJ_du_in"],
                    "fd_rel_errors_porosity": r["fd_rel_errors_porosity"], "J": r["J"],
                    "gpu_launches": None}
            print(json.dumps(line), flush=True)
        return
    mesh, case, desc, inlet, skw = make_workload(args.config)
    Solver = MixedSimpleSolver if args.precision == "mixed" else SimpleSolver
    mk = lambda c: Solver(mesh, c, **skw)  # noqa: E731
    nc = mesh.n_cells
    K, W = args.steps, max(args.warmup, 1)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    smi = ClockSampler(dev).start()  # over every GPU phase below: warm-up to the last solve
    # ---- device-timed run
    run_case = __import__("copy").deepcopy(case)
    run_case.tol = 0.0  # K steps regardless of convergence
    s = mk(run_case)
    if inlet is not None:
        inlet(s)
    for _ in range(W):
        s.step()
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    launches0 = s.kernel_launches
    ev = []
    infos = []

    def before():  # L2 flush between timed iterations, outside their events
        flush.zero_()
        ev.append((torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)))
        ev[-1][0].record()

    def after():
        ev[-1][1].record()

    barrier()
    s.run(max_steps=K, hooks=(before, after, lambda: infos.append(dict(s.last_linear))))
    barrier()
    launches = s.kernel_launches - launches0
    step_ms = [a.elapsed_time(b) for a, b in ev]
    graphs = bool(s.use_graphs and s._graphs)
    # per-stage kernel times: K more steps enqueued stage by stage with CUDA events between the
    # stages (graph replay leaves no room for events), same flush between steps
    s.profile_stages = True
    s.stage_times.clear()
    for k in range(K):
        flush.zero_()
        s.step()
        infos.append(dict(s.last_linear))
    s.profile_stages = False
    torch.cuda.synchronize()
    total_ms = max_over_ranks(sum(step_ms), world, "cuda")
    value = world * nc * K / (total_ms / 1e3)

    # ---- roofline of the dominant stage (stage events over the timed region)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    times = dict(s.stage_times)
    dom = max((k for k in times if stage_bytes(s, k, infos[0]) is not None), key=lambda k: times[k])
    byts = sum(stage_bytes(s, dom, inf) for inf in infos[K:])
    achieved = byts / (times[dom] / 1e3) / 1e9
    traffic = None
    try:  # DRAM bytes per launch from the committed ncu capture of this workload's kernel
        traffic = json.load(open(os.path.join(ROOT, "profiles", "traffic.json"))).get(args.config, {}).get(dom)
    except Exception:
        pass
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                "traffic": traffic, "algorithmic_bytes_per_launch": byts / K,
                "kernel_timing": "CUDA events between stages over K stage-by-stage steps right after the timed region",
                "stage_ms_per_step": {k: v / K for k, v in sorted(times.items(), key=lambda kv: -kv[1])}}
    del s

    # ---- end to end through the public API, from host data (after one untimed pass of the same
    # calls, as the timed steps follow warm-up steps)
    s2 = mk(run_case)
    if inlet is not None:
        inlet(s2)
    s2.run(max_steps=2)
    s2.fields()
    del s2
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    t_host = time.perf_counter()
    s2 = mk(run_case)
    if inlet is not None:
        inlet(s2)
    setup_s = time.perf_counter() - t_host
    s2.run(max_steps=W + K)
    f = s2.fields()
    e1.record()
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1), world, "cuda")
    h2d = s2.fv.h2d_bytes + sum(v.numel() * v.element_size() for v in s2._bc_t.values()) + (1 + s2.dim) * nc * 8
    d2h = s2.report.numel() * (W + K) + sum(v.nbytes for v in f.values())
    e2e = {"value": world * nc * (W + K) / (e2e_ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": h2d / (W + K),
           "d2h_bytes_per_step": d2h / (W + K), "includes": "solver construction from the host mesh, W+K steps, "
           "fields() read back; after one untimed pass of the same calls", "setup_seconds": setup_s, "seconds": e2e_ms / 1e3}
    del s2

    # ---- the metric's "to 1e-6" half: fresh solvers run to the 1e-6 scaled residual
    converge = None
    if not args.no_converge and args.config in ("c1", "c2", "c3", "sst"):
        barrier()
        converge = {"fp64": solve_to_convergence(SimpleSolver, mesh, case, inlet, skw, args.converge_max_iter)}
        if args.config != "sst":
            converge["mixed"] = solve_to_convergence(MixedSimpleSolver, mesh, case, inlet, skw, args.converge_max_iter)
            converge["mixed_over_fp64"] = mixed_over_fp64(converge["fp64"], converge["mixed"])
        for v in converge.values():
            v.pop("fields", None)

    # ---- the AMG set-up: device against host, and the reference's re-aggregation policy
    amg_setup = None
    if not args.no_amg_setup and args.config in ("c1", "c2", "c3"):
        barrier()
        amg_setup = amg_setup_block(mesh, case, inlet, skw, steps=100 if args.config != "c3" else 30)

    # ---- the metric's "vs plain FP64 GPU path" half on the 524,288-cell duct
    c3 = None
    if args.config == "c2" and not args.no_c3:
        barrier()
        c3 = c3_block(args)
    clocks = smi.stop()

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
        cb_case = __import__("copy").deepcopy(case)
        cpu = cpu_reference(mesh, cb_case, inlet, steps=1000, warmup=2, budget_s=15.0,
                            amg_theta=skw.get("amg_theta", 0.08))
        cpu = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": total_ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f32 systems, f64 residuals", "data": "synthetic",
            "config": workload_config(desc), "precision": args.precision,
            "l2": "flushed between timed steps (512 MiB write)",
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
            "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu, "clocks": clocks, "gpu_launches": launches,
            "linear_iterations_last": infos[K - 1], "cuda_graphs": graphs, "to_convergence": converge, "c3": c3,
            "amg_setup": amg_setup}
    print(json.dumps(line), flush=True)


def amg_setup_block(mesh, case, inlet, skw, steps):
    """The hierarchy's set-up from the pressure-correction matrix of the third iteration: on the
    device (``AMGHierarchy.on_device``, median of 3) and on the host (SciPy + the C++ greedy,
    then the device rebuild), whether both give the same aggregates; then fresh solvers timed
    over ``steps`` iterations after 12, with the first set-up's aggregates kept (the default) and
    with the reference's policy (``reaggregate``: a device set-up from the first level whose
    strength graph changed, at every rebuild where one did)."""
    import statistics

    import torch

    from gputest_b200.linalg.amg import AMGHierarchy
    from gputest_b200.unstructured.simple import SimpleSolver

    c = __import__("copy").deepcopy(case)
    c.tol = 0.0
    s = SimpleSolver(mesh, c, **skw)
    if inlet:
        inlet(s)
    for _ in range(3):
        s.step()
    fv = s.fv
    perm = torch.as_tensor(fv.perm, device="cuda")

    def timed(fn):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out = fn()
        torch.cuda.synchronize()
        return out, time.perf_counter() - t0

    dev_s, hd = [], None
    for _ in range(3):
        hd, dt = timed(lambda: AMGHierarchy.on_device(perm, fv.rowptr, fv.col, fv.t["slot_diag"], s.val_P,
                                                      singular=s.singular_p, max_coarse=s.max_coarse,
                                                      theta=s.amg_theta))
        dev_s.append(dt)

    def host():
        h = AMGHierarchy(fv.matrix_to_host(s.val_P), fv.perm, fv.rowptr, fv.col, fv.t["slot_diag"], s.val_P,
                         fv.slot_ref, singular=s.singular_p, max_coarse=s.max_coarse, theta=s.amg_theta)
        h.rebuild()
        return h

    hh, host_s = timed(host)
    same = hd.sizes == hh.sizes and all(torch.equal(hd._keep[2 * l]["agg"], hh._keep[2 * l]["agg"])
                                        for l in range(hh.n_levels - 1))
    sizes = list(hd.sizes)
    del s, hd, hh
    runs = {}
    for name, reagg in (("fixed", False), ("reaggregate", True)):
        s = SimpleSolver(mesh, c, **skw)
        if inlet:
            inlet(s)
        s.reaggregate = reagg
        for _ in range(12):
            s.step()
        n0 = s.amg_setups
        _, dt = timed(lambda: s.run(max_steps=steps))
        runs[name] = {"ms_per_step": dt / steps * 1e3, "setups": s.amg_setups - n0}
        del s
    return {"device_ms": statistics.median(dev_s) * 1e3, "host_ms": host_s * 1e3, "same_aggregates": bool(same),
            "level_sizes": sizes, "steps": steps, **runs}


def workload_config(desc):
    """The ``config`` object of both arms: the workload and its size, nothing arm-specific."""
    return {"workload": desc["workload"], "cells": desc["cells"]}


def solve_to_convergence(Solver, mesh, case, inlet, skw, max_iter):
    """A fresh solver from the host mesh run to the case's tolerance (1e-6 scaled residual) with
    ``run()``; seconds by CUDA events around ``run()`` (construction excluded, reported apart).
    The first outer iteration includes the AMG host set-up; ``steady`` is the same metric over
    the iterations after it (an event recorded on the stream just before the second iteration
    is enqueued)."""
    import copy

    import torch

    c = copy.deepcopy(case)
    c.max_iter = int(max_iter)
    t0 = time.perf_counter()
    s = Solver(mesh, c, **skw)
    if inlet is not None:
        inlet(s)
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e_first = torch.cuda.Event(enable_timing=True)
    enq = []

    def before_each():
        if len(enq) == 1:
            e_first.record()
        enq.append(True)

    e0.record()
    s.run(hooks=(before_each, None, None))
    e1.record()
    torch.cuda.synchronize()
    sec = e0.elapsed_time(e1) / 1e3
    rest = e_first.elapsed_time(e1) / 1e3 if len(enq) > 1 else sec
    its = int(s.iteration)
    out = {"converged": bool(s.converged), "iterations": its, "seconds": sec,
           "value": mesh.n_cells * its / sec, "ms_per_step": 1e3 * sec / max(its, 1),
           "first_iteration_seconds": sec - rest,
           "steady": {"value": mesh.n_cells * (its - 1) / rest if its > 1 else None,
                      "ms_per_step": 1e3 * rest / max(its - 1, 1)},
           "setup_seconds": setup_s, "tol": float(c.tol),
           "residuals": {k: float(v) for k, v in s.residuals()["scaled"].items()},
           "amg_setups": int(s.amg_setups), "fields": s.fields()}
    del s
    torch.cuda.empty_cache()
    return out


def mixed_over_fp64(a, b):
    """Mixed over FP64: cell-iterations/s ratio, seconds-to-convergence ratio and the largest
    relative field difference of the two converged runs (max |mixed - fp64| / max |fp64|)."""
    import numpy as np

    diff = {}
    for k, v in a["fields"].items():
        if k in b["fields"]:
            ref = np.asarray(v)
            diff[k] = float(np.abs(np.asarray(b["fields"][k]) - ref).max() / max(np.abs(ref).max(), 1e-300))
    steady = (b["steady"]["value"] / a["steady"]["value"]) if a["steady"]["value"] and b["steady"]["value"] else None
    return {"cell_iters_per_s_ratio": b["value"] / a["value"], "time_to_tol_ratio": a["seconds"] / b["seconds"],
            "steady_cell_iters_per_s_ratio": steady,
            "iterations": [a["iterations"], b["iterations"]], "field_max_rel_diff": diff}


def c3_block(args):
    """The 524,288-cell heated duct: FP64 ``SimpleSolver`` and ``MixedSimpleSolver`` from fresh
    solvers to the 1e-6 scaled residual; seconds, cell-iterations/s, their ratio and the
    converged fields' difference."""
    from gputest_b200.unstructured.mixed import MixedSimpleSolver
    from gputest_b200.unstructured.simple import SimpleSolver

    mesh, case, desc, inlet, skw = make_workload("c3")
    a = solve_to_convergence(SimpleSolver, mesh, case, inlet, skw, args.converge_max_iter)
    b = solve_to_convergence(MixedSimpleSolver, mesh, case, inlet, skw, args.converge_max_iter)
    out = {"workload": desc["workload"], "cells": desc["cells"], "fp64": a, "mixed": b,
           "mixed_over_fp64": mixed_over_fp64(a, b)}
    a.pop("fields")
    b.pop("fields")
    return out


if __name__ == "__main__":
    main()
