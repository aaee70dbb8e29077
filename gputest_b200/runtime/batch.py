"""Many independent cases from mesh files, solved on the B200 as block-diagonal batches.

Counterpart of ``flowtrace/runtime/batch.py:142-222`` (``run_batch``), with the same job
description (``BatchJob``) and per-job result records. The reference runs every case in a
process of its own (one GPU worker, one CPU worker per core); here the cases are read and
grouped, and every group of cases that can share one iteration - the same dimension, the
settings ``BatchSimpleSolver`` requires them to share, no energy equation - is solved as
block-diagonal batches of at most ``max_batch_cells`` cells (largest cases first) in one
``BatchSimpleSolver`` each (one set of launches per stage for all its cases). A case that cannot
share (energy, a setting of its own, ``precision="fp64"``) is solved alone by ``SimpleSolver``, or
by ``ConjugateSolver`` when it has solid zones.
As in the reference, each case's boundaries start from its mesh's zone types
(``default_boundaries``) with the job's overrides, a case that fails is reported with its
error and does not stop the others, and every result names the device it ran on.
"""

from __future__ import annotations

import os
import time
import traceback
from dataclasses import dataclass, field
from typing import Callable, Dict, List

import numpy as np

__all__ = ["BatchJob", "plan_batch", "run_batch"]


@dataclass
class BatchJob:
    name: str
    mesh: str  # path of a Fluent mesh/case file (.msh, .cas, optionally gzipped)
    case: dict = field(default_factory=dict)  # UnstructuredCase keyword arguments (boundaries as dicts)
    out_dir: str = ""  # if set: <out_dir>/<name>.npz with the cell centres and fields
    solver: str = "pressure-based"


def _prepare(job: BatchJob):
    """(mesh, case) of a job, as the reference's worker builds them (``batch.py:66-72``)."""
    from ..mesh.fluent import read_fluent_mesh
    from ..unstructured.case import UnstructuredCase, default_boundaries

    if job.solver != "pressure-based":
        raise NotImplementedError(f"solver {job.solver!r} is not implemented on the B200 path")
    mesh = read_fluent_mesh(job.mesh)
    kw = dict(job.case or {})
    kw.pop("backend", None)
    bnd = default_boundaries(mesh)
    for k, v in (kw.pop("boundaries", None) or {}).items():
        if k not in bnd:
            raise ValueError(f"zone {k!r} is not a boundary zone of {job.mesh} ({', '.join(sorted(bnd))})")
        bnd[k] = v
    return mesh, UnstructuredCase(boundaries=bnd, **kw)


def _group_key(mesh, case, precision):
    from ..unstructured.batch import _SHARED

    if precision != "mixed" or case.energy:
        return None
    return (mesh.dim,) + tuple(repr(getattr(case, k)) for k in _SHARED)


def plan_batch(jobs: List[BatchJob], max_batch_cells: int = 4_000_000, precision: str = "mixed") -> dict:
    """Read every job and decide how it runs (no solving): {"batches": [[job names]], "single":
    [job names], "errors": {name: message}, "jobs": [{"name", "cells", "batch"}]}; the prepared
    (mesh, case) pairs are kept under "_prepared"."""
    if len({j.name for j in jobs}) != len(jobs):
        raise ValueError("job names must be unique")
    if precision not in ("mixed", "fp64"):
        raise ValueError("precision is 'mixed' (batched) or 'fp64' (one case at a time)")
    prepared, errors = {}, {}
    for j in jobs:
        try:
            prepared[j.name] = _prepare(j)
        except Exception as exc:  # one unreadable case must not stop the batch
            errors[j.name] = f"{type(exc).__name__}: {exc}"
    groups: Dict[tuple, List[str]] = {}
    single = []
    for j in jobs:
        if j.name not in prepared:
            continue
        key = _group_key(*prepared[j.name], precision)
        if key is None:
            single.append(j.name)
        else:
            groups.setdefault(key, []).append(j.name)
    batches = []
    for names in groups.values():
        names = sorted(names, key=lambda n: -prepared[n][0].n_cells)
        cur, cells = [], 0
        for n in names:  # largest first, packed up to max_batch_cells
            c = prepared[n][0].n_cells
            if cur and cells + c > max_batch_cells:
                batches.append(cur)
                cur, cells = [], 0
            cur.append(n)
            cells += c
        batches.append(cur)
    single += [b[0] for b in batches if len(b) == 1]
    batches = [b for b in batches if len(b) > 1]
    where = {n: k for k, b in enumerate(batches) for n in b}
    rows = [{"name": j.name, "cells": prepared[j.name][0].n_cells if j.name in prepared else None,
             "batch": where.get(j.name)} for j in jobs]
    return {"batches": batches, "single": single, "errors": errors, "jobs": rows, "_prepared": prepared}


def _save(job: BatchJob, mesh, fields: dict) -> str:
    from ..mesh.unstructured import compute_geometry

    os.makedirs(job.out_dir, exist_ok=True)
    path = os.path.join(job.out_dir, job.name + ".npz")
    np.savez_compressed(path, centres=compute_geometry(mesh).cell_centre, **fields)
    return path


def run_batch(jobs: List[BatchJob], max_batch_cells: int = 4_000_000, precision: str = "mixed",
              autotune: bool = False, log: Callable[[str], None] = print) -> dict:
    """Solve every job; returns {"plan": .., "results": [..] (in job order), "wall_seconds": ..}.
    ``precision="mixed"`` batches the cases that can share an iteration (float systems, double
    residuals and refinement: the fixed point of the double iteration); ``"fp64"`` solves every
    case alone with the double ``SimpleSolver``. ``autotune`` times the batch team shapes first."""
    import torch

    from ..unstructured.batch import BatchSimpleSolver
    from ..unstructured.conjugate import make_solver

    t0 = time.perf_counter()
    plan = plan_batch(jobs, max_batch_cells, precision)
    prepared = plan.pop("_prepared")
    by_name = {j.name: j for j in jobs}
    device = f"cuda:{torch.cuda.current_device()}" if torch.cuda.is_available() else "none"
    results: Dict[str, dict] = {n: {"name": n, "mesh": by_name[n].mesh, "backend": "b200", "error": e}
                                for n, e in plan["errors"].items()}
    log(f"Batch: {len(jobs)} cases, {len(plan['batches'])} device batch(es), {len(plan['single'])} alone, "
        f"{len(plan['errors'])} unreadable")
    for k, names in enumerate(plan["batches"]):
        tb = time.perf_counter()
        try:
            bs = BatchSimpleSolver([prepared[n][0] for n in names], [prepared[n][1] for n in names])
            if autotune:
                bs.autotune()
            bs.run()
            secs = time.perf_counter() - tb
            for i, n in enumerate(names):
                job, mesh = by_name[n], prepared[n][0]
                at = int(bs.case_converged_at[i])
                res = {"name": n, "mesh": job.mesh, "backend": "b200-batch", "device": device, "error": None,
                       "cells": mesh.n_cells, "iterations": at if at >= 0 else bs.iteration, "converged": at >= 0,
                       "solve_seconds": secs, "batch": k, "batch_cases": len(names),
                       "residuals": bs.case_residuals(i),
                       "stability_rollbacks": len(bs.case_guard_events[i])}
                if job.out_dir:
                    res["npz"] = _save(job, mesh, bs.case_fields(i))
                results[n] = res
            log(f"  batch {k}: {len(names)} cases, {sum(prepared[n][0].n_cells for n in names):,} cells, "
                f"{bs.iteration} iterations, {int((bs.case_converged_at >= 0).sum())} converged, {secs:.1f} s")
        except Exception as exc:  # a failing batch reports the error on each of its cases
            err = f"{type(exc).__name__}: {exc}"
            for n in names:
                results[n] = {"name": n, "mesh": by_name[n].mesh, "backend": "b200-batch", "error": err,
                              "traceback": traceback.format_exc()[-3000:]}
            log(f"  FAILED batch {k}: {err}")
    for n in plan["single"]:
        job, (mesh, case) = by_name[n], prepared[n]
        t1 = time.perf_counter()
        res = {"name": n, "mesh": job.mesh, "backend": "b200", "device": device, "error": None}
        try:
            s = make_solver(mesh, case)  # a conjugate solver for cases with solid zones (batch.py:74)
            s.run()
            res.update({"cells": mesh.n_cells, "iterations": s.iteration, "converged": bool(s.converged),
                        "solve_seconds": time.perf_counter() - t1, "residuals": s.residuals()["scaled"],
                        "mass_balance": s.mass_balance(), "wall_forces": s.wall_forces(),
                        "heat_flow": s.heat_flow() if case.energy else {},
                        "stability_rollbacks": len(s.guard_events)})
            if job.out_dir:
                res["npz"] = _save(job, mesh, s.fields())
            log(f"  done  {n}: {s.iteration} its, {'converged' if s.converged else 'NOT converged'}")
        except Exception as exc:  # one failing case must not stop the batch
            res["error"] = f"{type(exc).__name__}: {exc}"
            res["traceback"] = traceback.format_exc()[-3000:]
            log(f"  FAILED {n}: {res['error']}")
        results[n] = res
    wall = time.perf_counter() - t0
    log(f"Batch finished in {wall:.1f} s")
    return {"plan": plan, "results": [results[j.name] for j in jobs], "wall_seconds": wall}
