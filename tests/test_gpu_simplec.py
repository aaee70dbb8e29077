"""The B200 SimpleSolver against the oracle, iterate by iterate (``tests/test_native.py:67-103``
and ``tests/test_gpu_real.py:92-107,174-191`` of the reference are the models)."""

import numpy as np
import pytest

from gputest_b200.mesh.unstructured import box_mesh_3d, cartesian_mesh_2d, extrude_to_3d
from gputest_b200.unstructured.case import BoundarySpec, UnstructuredCase
from oracle.simplec_oracle import OracleSimple

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


def _pair(mesh, case, n, max_coarse=300, amg_theta=0.08):
    from gputest_b200.unstructured.simple import SimpleSolver

    o = OracleSimple(mesh, case, amg_theta=amg_theta)
    s = SimpleSolver(mesh, case, max_coarse=max_coarse, amg_theta=amg_theta)
    s.reaggregate = True  # the reference re-aggregates at every rebuild
    for _ in range(n):
        o.step()
        s.step()
    return o, s


def _cavity_case(dim=2, **kw):
    top = [1.0, 0.0] if dim == 2 else [1.0, 0.0, 0.0]
    return UnstructuredCase(boundaries={"top": BoundarySpec("wall", velocity=top)}, **kw)


# Iterate-by-iterate comparisons use a tight pressure-correction tolerance, as the reference's
# own GPU-versus-CPU test does (``tests/test_gpu_real.py:92-107``): on a closed domain the
# pressure matrix is singular and the reference inverts its coarsest AMG matrix shifted by
# 1e-10 mean|diag| (condition ~1e10), so with a loose tolerance round-off differences of the
# two inversions are amplified into the iterates (not into the converged solution).
TIGHT = 1e-9


def test_simplec_iterates_equal_oracle_on_skewed_triangles():
    """40 SIMPLEC iterations on skewed triangles, not converged (``test_native.py:79-87``)."""
    o, s = _pair(cartesian_mesh_2d(16, 16, triangulate=True, warp=0.05),
                 _cavity_case(viscosity=0.01, max_iter=40, tol=0.0, pressure_tol=TIGHT), 40)
    fo, fs = o.fields(), s.fields()
    for k in ("x-velocity", "y-velocity", "pressure"):
        assert _rel(fs[k], fo[k]) < 1e-10, k
    assert s.last_linear["momentum_iters"] == o.last_linear["momentum_iters"]
    assert abs(s.last_linear["pressure_iters"] - o.last_linear["pressure_iters"]) <= 1
    for k, v in o.residuals()["scaled"].items():
        assert s.residuals()["scaled"][k] == pytest.approx(v, rel=1e-6), k


def test_simplec_lid_driven_cavity_upwind_tight_pressure():
    """The 64 x 64 cavity of the CPU-runnable configuration, 30 iterations."""
    case = _cavity_case(viscosity=0.01, scheme="upwind", pressure_tol=1e-8, max_iter=300, tol=0.0)
    o, s = _pair(cartesian_mesh_2d(64, 64), case, 30)
    fo, fs = o.fields(), s.fields()
    for k in ("x-velocity", "y-velocity", "pressure"):
        assert _rel(fs[k], fo[k]) < 1e-9, k


def test_simplec_alternating_triangles_second_order():
    """Alternating-diagonal jittered triangles, linear-upwind, Re 1000 (the large 2-D config's
    mesh type and scheme, at a size the oracle finishes in seconds)."""
    case = _cavity_case(viscosity=1e-3, max_iter=100, tol=0.0, pressure_tol=TIGHT)
    o, s = _pair(cartesian_mesh_2d(32, 32, triangulate="alternating", jitter=0.2, seed=0), case, 30)
    fo, fs = o.fields(), s.fields()
    for k in ("x-velocity", "y-velocity", "pressure"):
        assert _rel(fs[k], fo[k]) < 1e-8, k


def test_simplec_channel_with_energy():
    m = cartesian_mesh_2d(24, 8, 3.0, 1.0, names=("in", "out", "bottom", "top"), warp=0.03)
    case = UnstructuredCase(boundaries={"in": BoundarySpec("inlet", velocity=[1.0, 0.0], value=1.0),
                                        "out": BoundarySpec("outlet"),
                                        "bottom": BoundarySpec("wall", thermal="temperature", value=0.0),
                                        "top": BoundarySpec("wall", thermal="flux", value=2.0)},
                            energy=True, viscosity=0.01, conductivity=0.02, max_iter=50, tol=0.0)
    o, s = _pair(m, case, 30)
    fo, fs = o.fields(), s.fields()
    for k in ("x-velocity", "y-velocity", "pressure", "temperature"):
        assert _rel(fs[k], fo[k]) < 1e-8, k
    mb_s = s.mass_balance()
    for z in m.boundary_zones():  # per-zone boundary mass flow equals the oracle's
        ref = float(o.Fb[o.fv.bzone == z.id].sum())
        assert mb_s[z.name] == pytest.approx(ref, rel=1e-8, abs=1e-12), z.name


def test_simplec_3d_extruded_and_jittered_box():
    o, s = _pair(extrude_to_3d(cartesian_mesh_2d(6, 5, warp=0.05), 4, 0.5),
                 _cavity_case(dim=3, viscosity=0.01, max_iter=40, tol=0.0, pressure_tol=TIGHT), 20)
    for k in ("x-velocity", "y-velocity", "z-velocity", "pressure"):
        assert _rel(s.fields()[k], o.fields()[k]) < 1e-10, k
    m = box_mesh_3d(12, 6, 6, 4.0, 1.0, 1.0, jitter=0.1, seed=1, names=("inlet", "outlet", "wall", "wall", "wall", "wall"))
    case = UnstructuredCase(boundaries={"inlet": BoundarySpec("inlet", normal_speed=1.0), "outlet": BoundarySpec("outlet"),
                                        "wall": BoundarySpec("wall")}, viscosity=0.02, max_iter=40, tol=0.0)
    o, s = _pair(m, case, 15)
    for k in ("x-velocity", "y-velocity", "z-velocity", "pressure"):
        assert _rel(s.fields()[k], o.fields()[k]) < 1e-9, k


def test_converged_cavity_equals_the_oracle_solution():
    """At the default pressure tolerance the iterates differ at round-off level, the converged
    solution does not: both runs converge to the 1e-6 scaled residual and agree."""
    case = _cavity_case(viscosity=0.01, max_iter=3000, tol=1e-6)
    mesh = cartesian_mesh_2d(24, 24, triangulate=True, jitter=0.2)
    from gputest_b200.unstructured.simple import SimpleSolver

    o = OracleSimple(mesh, case)
    while not o.finished:
        o.step()
    s = SimpleSolver(mesh, case)
    s.run()
    assert o.converged and s.converged
    assert abs(s.iteration - o.iteration) <= max(5, 0.05 * o.iteration)
    for k in ("x-velocity", "y-velocity"):
        assert _rel(s.fields()[k], o.fields()[k]) < 1e-4, k


def test_state_round_trip_and_guard_snapshot():
    from gputest_b200.unstructured.simple import SimpleSolver

    mesh = cartesian_mesh_2d(12, 12, triangulate=True, warp=0.05)
    s = SimpleSolver(mesh, _cavity_case(viscosity=0.01, max_iter=100, tol=0.0))
    for _ in range(5):
        s.step()
    st = s.state_dict()
    f5 = s.fields()
    for _ in range(3):
        s.step()
    s.load_state(st)
    assert s.iteration == 5
    for k, v in f5.items():
        assert np.array_equal(s.fields()[k], v), k
    assert s.captured_systems() is None


def test_assembly_per_entry_from_the_same_state():
    """FP64 assembly within 1e-12 per entry: both solvers restart from the oracle's state after 8
    iterations (``load_state`` clears the lagged gradients in both) and take one step; every
    captured system entry agrees."""
    from gputest_b200.unstructured.simple import SimpleSolver

    mesh = cartesian_mesh_2d(24, 24, triangulate="alternating", jitter=0.2)
    case = _cavity_case(viscosity=1e-3, max_iter=100, tol=0.0)
    o = OracleSimple(mesh, case)
    for _ in range(8):
        o.step()
    st = o.state_dict()
    s = SimpleSolver(mesh, case)
    s.load_state(st)
    o.load_state(st)
    o.step()
    s.step()
    co, cs = o._capture, s.captured_systems()
    pairs = {"A": (cs["A"].data, co["A"].data), "Ar": (cs["Ar"].data, co["Ar"].data),
             "Ap": (cs["Ap"].data, co["Ap"].data), "b": (np.stack(cs["b"], 1), np.stack(co["b"], 1)),
             "br": (np.stack(cs["br"], 1), np.stack(co["br"], 1)), "mass": (cs["mass"], co["mass"]),
             "Fst": (cs["Fst"], co["Fst"]), "Fbst": (cs["Fbst"], co["Fbst"])}
    for k, (ours, ref) in pairs.items():
        assert np.abs(ours - ref).max() <= 1e-12 * np.abs(ref).max(), k


def test_simplec_iterates_equal_oracle_with_pyamg_strength_rule():
    """The AMG with strength threshold 0 (pyamg's default rule) on a jittered 3-D duct with an
    outlet: iterates against the oracle configured the same way."""
    names = ("inlet", "outlet", "wall", "wall", "wall", "wall")
    mesh = box_mesh_3d(12, 6, 6, 4.0, 1.0, 1.0, jitter=0.1, seed=1, names=names,
                       types=("velocity-inlet", "pressure-outlet", "wall", "wall", "wall", "wall"))
    case = UnstructuredCase(boundaries={"inlet": BoundarySpec("inlet", velocity=[1.0, 0.0, 0.0]),
                                        "outlet": BoundarySpec("outlet", pressure=0.0),
                                        "wall": BoundarySpec("wall")},
                            viscosity=0.02, max_iter=30, tol=0.0, pressure_tol=TIGHT)
    o, s = _pair(mesh, case, 15, amg_theta=0.0)
    fo, fs = o.fields(), s.fields()
    for k in fo:
        assert _rel(fs[k], fo[k]) < 1e-9, k
    assert s._amg.sizes == [lv[0].shape[0] for lv in o._amg.levels] + [o._amg.coarse_inv.shape[0]]


def test_coarse_inverse_of_every_shared_memory_size():
    """Coarse levels of 70 rows (a 20 x 20 jittered cavity with max_coarse 150): the dense
    inverse's shared memory plus the kernel's static buffers exceed the default 48 KB."""
    o, s = _pair(cartesian_mesh_2d(20, 20, jitter=0.15, seed=0),
                 _cavity_case(viscosity=0.01, max_iter=10, tol=0.0, pressure_tol=TIGHT), 5, max_coarse=150)
    assert s._amg.sizes[-1] > 64
    fo, fs = o.fields(), s.fields()
    for k in ("x-velocity", "y-velocity", "pressure"):
        assert _rel(fs[k], fo[k]) < 1e-9, k


def test_porous_channel_iterates_equal_oracle():
    """Brinkman porosity (alpha V on the momentum diagonal, also in the SIMPLE coefficient) with
    SIMPLE and fixed relaxation, the adjoint workload's setting."""
    from gputest_b200.unstructured.simple import SimpleSolver

    m = cartesian_mesh_2d(24, 8, 4.0, 1.0, names=("in", "out", "bottom", "top"))
    case = UnstructuredCase(boundaries={"in": BoundarySpec("inlet", velocity=[1.0, 0.0]), "out": BoundarySpec("outlet"),
                                        "bottom": BoundarySpec("wall"), "top": BoundarySpec("wall")},
                            viscosity=1 / 200, scheme="upwind", tol=0.0, max_iter=100, algorithm="SIMPLE",
                            relax_u=0.3, relax_p=0.3, pressure_tol=TIGHT)
    por = 1e4 / (1 + np.exp(-8 * np.random.default_rng(0).standard_normal(m.n_cells)))
    o = OracleSimple(m, case, porosity=por)
    s = SimpleSolver(m, case, max_coarse=300)
    s.set_porosity(por)
    s.reaggregate = True  # the reference re-aggregates at every rebuild
    for it in range(40):
        o.step()
        s.step()
    fo, fs = o.fields(), s.fields()
    for k in ("x-velocity", "y-velocity", "pressure"):
        assert _rel(fs[k], fo[k]) < 1e-9, k


@pytest.mark.parametrize("mixed", [False, True])
def test_pipelined_run_equals_stepping(mixed):
    """``run()`` enqueues iteration k+1 before reading iteration k's report; its iterates, the
    iteration it converges at and the state it leaves (including the lagged gradients a
    discarded speculative iteration overwrote) equal those of plain ``step()`` calls: the fields
    agree bit for bit after the first run and after a continued run with a tighter tolerance."""
    from gputest_b200.unstructured.mixed import MixedSimpleSolver
    from gputest_b200.unstructured.simple import SimpleSolver

    cls = MixedSimpleSolver if mixed else SimpleSolver
    mesh = cartesian_mesh_2d(20, 20, triangulate=True, jitter=0.15)
    case = _cavity_case(viscosity=0.01, max_iter=2000, tol=1e-4)
    a, b = cls(mesh, case), cls(mesh, case)
    a.run()
    while not b.finished:
        b.step()
    assert a.converged and b.converged and a.iteration == b.iteration
    for k, v in b.fields().items():
        assert np.array_equal(a.fields()[k], v), k
    assert a.residuals() == b.residuals()
    for s in (a, b):
        s.case.tol = 1e-6
        s.converged = False
    a.run(max_steps=37)
    for _ in range(37):
        b.step()
    assert a.iteration == b.iteration
    for k, v in b.fields().items():
        assert np.array_equal(a.fields()[k], v), k
