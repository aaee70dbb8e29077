"""``gputest_b200.runtime.batch`` (the counterpart of the reference's ``run_batch``): planning on
the host (grouping of the cases that can share an iteration, packing by cells, unreadable jobs
reported) and, on the GPU, mesh-file jobs solved as device batches to the fields of the same
cases solved alone, with a failing job reported and the others unaffected."""

import numpy as np
import pytest

from gputest_b200.mesh.fluent import write_fluent_mesh
from gputest_b200.mesh.unstructured import cartesian_mesh_2d
from gputest_b200.runtime.batch import BatchJob, plan_batch


def _jobs(tmp_path):
    meshes = {"cav_a": cartesian_mesh_2d(14, 14, jitter=0.1, seed=1),
              "cav_b": cartesian_mesh_2d(10, 10, jitter=0.1, seed=2),
              "chan": cartesian_mesh_2d(24, 6, 4.0, 1.0, names=("in", "out", "bottom", "top"),
                                        types=("velocity-inlet", "pressure-outlet", "wall", "wall"), jitter=0.1)}
    paths = {}
    for k, m in meshes.items():
        paths[k] = str(tmp_path / f"{k}.msh")
        write_fluent_mesh(m, paths[k])
    common = {"tol": 1e-9, "max_iter": 5000}
    jobs = [BatchJob("cav_a", paths["cav_a"], {"viscosity": 0.01, "boundaries": {"top": {"kind": "wall", "velocity": [1.0, 0.0]}}, **common}),
            BatchJob("cav_b", paths["cav_b"], {"viscosity": 0.02, "boundaries": {"top": {"kind": "wall", "velocity": [0.5, 0.0]}}, **common}),
            BatchJob("chan", paths["chan"], {"viscosity": 0.02, "boundaries": {"in": {"kind": "inlet", "velocity": [1.0, 0.0]}}, **common}),
            BatchJob("bad_zone", paths["cav_b"], {"boundaries": {"lid": {"kind": "wall"}}}),
            BatchJob("missing", str(tmp_path / "nope.msh"))]
    return jobs


def test_plan_groups_the_cases_that_can_share_an_iteration(tmp_path):
    jobs = _jobs(tmp_path)
    plan = plan_batch(jobs)
    assert plan["batches"] == [["cav_a", "chan", "cav_b"]] and plan["single"] == []
    assert [r["cells"] for r in plan["jobs"][:3]] == [196, 100, 144]
    assert set(plan["errors"]) == {"bad_zone", "missing"} and "not a boundary zone" in plan["errors"]["bad_zone"]
    # a cell budget splits the group (largest first: 196 | 144 + 100); a batch of one runs alone
    small = plan_batch(jobs, max_batch_cells=300)
    assert small["batches"] == [["chan", "cav_b"]] and small["single"] == ["cav_a"]
    assert plan_batch(jobs, precision="fp64")["batches"] == []
    with pytest.raises(ValueError):
        plan_batch(jobs + [jobs[0]])


@pytest.mark.gpu
def test_run_batch_solves_each_case_like_the_case_alone(tmp_path):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gputest_b200.runtime.batch import _prepare, run_batch
    from gputest_b200.unstructured.simple import SimpleSolver

    jobs = _jobs(tmp_path)
    for j in jobs:
        j.out_dir = str(tmp_path / "out")
    out = run_batch(jobs, log=lambda *_: None)
    res = {r["name"]: r for r in out["results"]}
    assert res["bad_zone"]["error"] and res["missing"]["error"]
    for n in ("cav_a", "cav_b", "chan"):
        r = res[n]
        assert r["error"] is None and r["converged"] and r["backend"] == "b200-batch", r
        mesh, case = _prepare(next(j for j in jobs if j.name == n))
        s = SimpleSolver(mesh, case)
        s.run()
        got = np.load(r["npz"])
        for k, v in s.fields().items():
            assert float(np.abs(got[k] - v).max()) <= 1e-6 * max(float(np.abs(v).max()), 1e-300), (n, k)


def test_a_case_with_a_solid_zone_is_planned_alone(tmp_path):
    """A mesh file with a solid cell zone (``set_cell_zone``) and the solid's conductivity in the
    case: read back with its zones, planned to run alone (``run_batch`` hands it to
    ``make_solver``, which builds a ``ConjugateSolver``), beside a batch of plain cases."""
    from gputest_b200.mesh.unstructured import set_cell_zone
    from gputest_b200.runtime.batch import _prepare

    m = cartesian_mesh_2d(30, 10, 4.0, 1.25, names=("inlet", "outlet", "bottom", "top"),
                          types=("velocity-inlet", "pressure-outlet", "wall", "wall"), y0=-0.25)
    m = set_cell_zone(m, lambda x: x[:, 1] < 0.0, "heater", "solid")
    path = str(tmp_path / "heated.msh")
    write_fluent_mesh(m, path)
    job = BatchJob("heated", path, {"energy": True, "conductivity": 0.05, "viscosity": 0.05,
                                    "solids": {"heater": {"conductivity": 2.0, "source": 4.0}},
                                    "boundaries": {"inlet": {"kind": "inlet", "normal_speed": 1.0}}})
    mesh, case = _prepare(job)
    assert any(z.type == "solid" for z in mesh.cell_zones()) and case.solids
    plan = plan_batch(_jobs(tmp_path)[:3] + [job])
    assert plan["single"] == ["heated"] and plan["batches"] == [["cav_a", "chan", "cav_b"]]
