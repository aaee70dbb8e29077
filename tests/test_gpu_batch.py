"""Block-diagonal batches of independent cases (``BatchSimpleSolver``): every case of a batch
converges to the fields of the same case solved alone, and the per-case Krylov solves keep each
case's own scalars (same iteration counts as the single-system float solver)."""

import numpy as np
import pytest

from gputest_b200.mesh.unstructured import cartesian_mesh_2d
from gputest_b200.unstructured.case import BoundarySpec, UnstructuredCase

pytestmark = pytest.mark.gpu

FIELD_TOL = 1e-6


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


def _cases(tol=1e-9, max_iter=5000):
    spec = [("cavity", 20, 20, 0.01, 1.0), ("channel", 30, 8, 0.02, 1.5), ("cavity", 12, 12, 0.005, 0.7),
            ("channel", 16, 6, 0.01, 0.8)]
    meshes, cases = [], []
    for k, (kind, nx, ny, mu, u) in enumerate(spec):
        if kind == "cavity":
            m = cartesian_mesh_2d(nx, ny, jitter=0.15, seed=k)
            b = {"top": BoundarySpec("wall", velocity=[u, 0.0])}
        else:
            m = cartesian_mesh_2d(nx, ny, 4.0, 1.0, names=("in", "out", "bottom", "top"), jitter=0.15, seed=k)
            b = {"in": BoundarySpec("inlet", velocity=[u, 0.0]), "out": BoundarySpec("outlet"),
                 "bottom": BoundarySpec("wall"), "top": BoundarySpec("wall")}
        meshes.append(m)
        cases.append(UnstructuredCase(boundaries=b, viscosity=mu, tol=tol, max_iter=max_iter))
    return meshes, cases


def test_batched_cases_converge_to_their_single_case_fields():
    from gputest_b200.unstructured.batch import BatchSimpleSolver
    from gputest_b200.unstructured.simple import SimpleSolver

    meshes, cases = _cases()
    bs = BatchSimpleSolver(meshes, cases)
    assert list(bs.case_singular) == [True, False, True, False]
    bs.run()
    assert bs.converged and np.all(bs.case_converged_at > 5)
    for i, (m, c) in enumerate(zip(meshes, cases)):
        s = SimpleSolver(m, c)
        s.run()
        assert s.converged
        ref, got = s.fields(), bs.case_fields(i)
        for k in ref:
            assert _rel(got[k], ref[k]) <= FIELD_TOL, (i, k, _rel(got[k], ref[k]))


def test_batched_iterations_match_single_case_float_solves():
    """The first outer iteration (zero fields, the same start for both): per case, the momentum
    BiCGSTAB counts and every scaled residual equal those of the case solved alone in float; the
    pressure-correction solves differ only through the preconditioner (the batch's hierarchy)."""
    from gputest_b200.unstructured.batch import BatchSimpleSolver
    from gputest_b200.unstructured.mixed import MixedSimpleSolver

    meshes, cases = _cases(tol=0.0, max_iter=10)
    bs = BatchSimpleSolver(meshes, cases)
    bs.step()
    for i, (m, c) in enumerate(zip(meshes, cases)):
        s = MixedSimpleSolver(m, c)
        s.step()
        assert list(bs.last_linear["momentum_iters"][i]) == list(s.last_linear["momentum_iters"]), i
        assert bs.last_linear["pressure_residual"][i] < c.pressure_tol
        rb, rs = bs.case_residuals(i), s.residuals()["scaled"]
        for k in rs:
            assert rb[k] == pytest.approx(rs[k], rel=1e-6, abs=1e-12), (i, k)


def test_batch_rejects_cases_that_differ_in_shared_settings():
    from gputest_b200.unstructured.batch import BatchSimpleSolver

    meshes, cases = _cases()
    cases[1].scheme = "upwind"
    with pytest.raises(ValueError):
        BatchSimpleSolver(meshes, cases)


def test_batch_stability_guard_rolls_back_one_case_only():
    """A case driven to divergence (planted in its state on the host side: its fluxes scaled up)
    is rolled back and relaxed by its own guard; the other cases are untouched by it."""
    import torch

    from gputest_b200.unstructured.batch import BatchSimpleSolver

    meshes, cases = _cases(tol=0.0, max_iter=100)
    bs = BatchSimpleSolver(meshes, cases)
    ref = BatchSimpleSolver(meshes, cases)
    for _ in range(25):
        bs.step()
        ref.step()
    (a, b), (fa, fb), _ = bs._case_slices(1)
    bs._F[bs._cur][fa:fb] *= 1e6  # wreck case 1's mass fluxes
    bs.step()
    ref.step()
    assert bs.case_guard_events[1] and not any(bs.case_guard_events[g] for g in (0, 2, 3))
    assert bs.case_relax_p[1] < ref.case_relax_p[1]
    for g in (0, 2, 3):
        assert bs.case_residuals(g) == ref.case_residuals(g)
    for _ in range(5):
        bs.step()
    assert np.isfinite(bs.case_residuals(1)["continuity"])


@pytest.mark.parametrize("team", [(2, 512, 16), (8, 1024, 0)])
def test_other_team_shapes_converge_to_the_same_fields(team):
    """Non-default team shapes (blocks per cluster, threads per block, rows-per-warp switch; 0
    never walks a row by a warp) solve every case to the fields of the case solved alone."""
    from gputest_b200 import _lib
    from gputest_b200.unstructured.batch import BatchSimpleSolver
    from gputest_b200.unstructured.simple import SimpleSolver

    meshes, cases = _cases()
    bs = BatchSimpleSolver(meshes, cases)
    bs.team = _lib.TeamConfig(*team, 0)
    bs.team_momentum = _lib.TeamConfig(*team, 0)
    bs.run()
    assert bs.converged
    for i, (m, c) in enumerate(zip(meshes, cases)):
        s = SimpleSolver(m, c)
        s.run()
        ref, got = s.fields(), bs.case_fields(i)
        for k in ref:
            assert _rel(got[k], ref[k]) <= FIELD_TOL, (team, i, k)


def test_autotune_times_the_candidates_and_keeps_the_fastest():
    from gputest_b200.unstructured.batch import BatchSimpleSolver

    meshes, cases = _cases(tol=0.0, max_iter=20)
    bs = BatchSimpleSolver(meshes, cases)
    cands = [(2, 512, 16), (4, 1024, 24), (8, 1024, 48)]
    tuned = bs.autotune(candidates=cands, reps=2, margin=0.0)
    ms = {k: v for k, v in tuned["ms"].items() if v is not None}
    assert set(tuned["ms"]) == set(cands) and ms
    assert tuned["momentum"] == min(ms, key=lambda k: ms[k][0])
    assert tuned["pressure"] == min(ms, key=lambda k: ms[k][1])
    assert (bs.team.cluster_blocks, bs.team.block_threads, bs.team.wide_row) == tuned["pressure"]
    m = bs.team_momentum
    assert (m.cluster_blocks, m.block_threads, m.wide_row) == tuned["momentum"]
    it = bs.iteration
    f0 = bs.fields()
    bs.run(max_steps=3)
    assert bs.iteration == it + 3 and all(np.all(np.isfinite(v)) for v in bs.fields().values())
    assert f0.keys() == bs.fields().keys()
