"""The oracle's conjugate heat transfer (``oracle/conjugate_oracle.py``) against the reference's
``ConjugateSolver``, through ``tests/golden/conjugate_fixtures.npz`` (made by
``tests/golden/make_conjugate_golden.py`` on the cases of ``tests/golden/conjugate_cases.py``): a
1-D composite wall of two solids around a fluid slab, a channel over a heated solid block, and a
lid-driven triangulated cavity around a heated solid disc. Also the product's host set-up of the
same solver (``gputest_b200.unstructured.conjugate.conjugate_setup``)."""

import json
import os

import numpy as np
import pytest

from gputest_b200.unstructured.case import BoundarySpec, UnstructuredCase
from oracle.conjugate_oracle import OracleConjugate
from tests.golden.conjugate_cases import CONJUGATE_CASES

GOLD = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "conjugate_fixtures.npz"))


def _rel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _case(name):
    build, kw, n = CONJUGATE_CASES[name]
    bnd = {z: BoundarySpec(**spec) for z, spec in kw["boundaries"].items()}
    return build(), UnstructuredCase(**{**kw, "boundaries": bnd}), n


@pytest.mark.parametrize("name", sorted(CONJUGATE_CASES))
def test_oracle_conjugate_equals_the_reference(name):
    mesh, case, n = _case(name)
    o = OracleConjugate(mesh, case)
    p = f"cht|{name}|"
    gf, gb = o.face_gamma()
    assert np.array_equal(gf, GOLD[p + "gamma_face"]) and np.array_equal(gb, GOLD[p + "gamma_bface"])
    assert np.array_equal(o.q_cell, GOLD[p + "q_cell"]) and np.array_equal(o.cell_map, GOLD[p + "cell_map"])
    for _ in range(n):
        o.step()
    assert o.iteration == int(GOLD[p + "iterations"][0])
    f = o.fields()
    for k in (k.split("|", 3)[3] for k in GOLD.files if k.startswith(p + "field|")):
        assert _rel(f[k], GOLD[p + "field|" + k]) <= 1e-12, k
    for k, v in o.residuals()["scaled"].items():
        assert v == pytest.approx(float(GOLD[p + "res|" + k][0]), rel=1e-8, abs=1e-300), k
    assert list(o.last_linear["momentum_iters"]) + [o.last_linear["pressure_iters"]] == list(GOLD[p + "linear"])
    ref = json.loads(bytes(GOLD[p + "heat_flow"]).decode())
    ours = o.heat_flow()
    assert set(ours) == set(ref)
    for k, v in ref.items():
        assert ours[k] == pytest.approx(v, rel=1e-9, abs=1e-12), k


def test_composite_wall_is_exact():
    """The reference's own check (``tests/test_zones.py:92-105``): with harmonic face
    conductivities the 1-D composite wall is solved exactly."""
    mesh, case, _ = _case("composite")
    o = OracleConjugate(mesh, case)
    for _ in range(60):
        o.step()
    x, T = o.fv.xc[:, 0], o.fields()["temperature"]
    q = 1 / 3.2
    Te = np.where(x < 1, 1 - q * x / 5, np.where(x < 2, 1 - q / 5 - q * (x - 1), 1 - 1.2 * q - 2 * q * (x - 2)))
    assert np.abs(T - Te).max() < 1e-10


@pytest.mark.parametrize("name", sorted(CONJUGATE_CASES))
def test_product_conjugate_setup_equals_the_reference(name):
    """The B200 path's host set-up (``conjugate_setup``): harmonic face diffusivities, sources,
    the fluid sub-mesh's cell map, the flux maps and the thermal boundary arrays."""
    from gputest_b200.unstructured.conjugate import conjugate_setup

    mesh, case, _ = _case(name)
    hs = conjugate_setup(mesh, case)
    p = f"cht|{name}|"
    if case.turbulence == "laminar":  # with turbulence the reference's face values include mu_t / Pr_t
        assert np.array_equal(hs["gamma_face"], GOLD[p + "gamma_face"])
        assert np.array_equal(hs["gamma_bface"], GOLD[p + "gamma_bface"])
    assert np.array_equal(hs["q_cell"], GOLD[p + "q_cell"]) and np.array_equal(hs["cell_map"], GOLD[p + "cell_map"])
    o = OracleConjugate(mesh, case)
    for k in ("if_dst", "bf_src", "bf_dst"):
        assert np.array_equal(hs[k], getattr(o, "_" + k)), k
    assert np.array_equal(hs["tkind"], o.tkind) and np.array_equal(hs["tval"], o.tval)
    assert np.array_equal(hs["is_outlet"], o.is_outlet)
    assert not hs["flow_case"].solids and not hs["flow_case"].energy


def test_conjugate_setup_rejects_what_the_reference_rejects():
    """``tests/test_zones.py:108-111``: a solid zone without a conductivity, and no energy."""
    from gputest_b200.unstructured.conjugate import conjugate_setup

    mesh, case, _ = _case("heated")
    with pytest.raises(ValueError):
        conjugate_setup(mesh, UnstructuredCase(energy=True))
    with pytest.raises(ValueError):
        conjugate_setup(mesh, UnstructuredCase(energy=False, solids=dict(case.solids)))


def test_conjugate_temperatures_are_set_to_what_the_gpu_test_asks():
    """How far the reference's own temperature moves when the cell conductivities are perturbed by
    1e-15 relative: below 1e-10 on the composite wall and the heated channel, ~1e-7 on the
    triangulated cavity (an energy BiCGSTAB solve at tolerance 1e-4 changes its iteration count),
    where the energy residual moves by up to ~1.5e-4 and the heat flows by ~6e-6. The CUDA test
    compares temperatures at 1e-8 and 1e-5, that residual at 1e-3 and those heat flows at 1e-4
    for that reason."""
    worst, res_worst, hf_worst = {}, 0.0, 0.0
    g = float(GOLD["cht|tri_disc|res|energy"][0])
    hf_ref = json.loads(bytes(GOLD["cht|tri_disc|heat_flow"]).decode())
    for name in sorted(CONJUGATE_CASES):
        for seed in range(2):
            mesh, case, n = _case(name)
            o = OracleConjugate(mesh, case)
            o.gam_cell = o.gam_cell * (1 + 1e-15 * np.random.default_rng(seed).standard_normal(o.nc))
            for _ in range(n):
                o.step()
            d = _rel(o.fields()["temperature"], GOLD[f"cht|{name}|field|temperature"])
            worst[name] = max(worst.get(name, 0.0), d)
            if name == "tri_disc":
                res_worst = max(res_worst, abs(o.residuals()["scaled"]["energy"] / g - 1))
                hf = o.heat_flow()
                hf_worst = max(hf_worst, *(abs(hf[k] - v) / abs(v) for k, v in hf_ref.items() if v != 0))
    assert worst["composite"] < 1e-10 and worst["heated"] < 1e-10
    assert worst["tri_disc"] < 1e-5 and worst["heated_sst"] < 1e-5
    assert 1e-5 < res_worst < 1e-3
    assert 1e-7 < hf_worst < 1e-4


@pytest.mark.parametrize("name", sorted(CONJUGATE_CASES))
def test_device_flux_maps_scatter_like_the_reference(name):
    """The index maps ``ConjugateSolver`` builds (``device_flux_maps``) to move the fluid's face fluxes (in the fluid
    sub-mesh's device face order) into the full mesh's device face order, applied on the host to
    the device layouts (``FVMesh`` built on the CPU): in range, one-to-one, and equal after
    conversion to the reference's order to the oracle's ``_full_fluxes`` (``conjugate.py:136-144``)."""
    import torch

    from gputest_b200.unstructured.conjugate import conjugate_setup, device_flux_maps
    from gputest_b200.unstructured.fvmesh import FVMesh

    mesh, case, _ = _case(name)
    hs = conjugate_setup(mesh, case)
    fv, sfv = FVMesh(mesh, torch.device("cpu")), FVMesh(hs["sub"], torch.device("cpu"))
    if_dst, bf_src, bf_dst = device_flux_maps(hs, fv, sfv)
    assert if_dst.min() >= 0 and if_dst.max() < fv.n_if and np.unique(if_dst).size == if_dst.size
    assert bf_src.max() < sfv.n_bf and bf_dst.max() < fv.n_bf and np.unique(bf_dst).size == bf_dst.size
    o = OracleConjugate(mesh, case)
    rng = np.random.default_rng(0)
    o.flow.F, o.flow.Fb = rng.standard_normal(o.flow.fv.n_if), rng.standard_normal(o.flow.fv.n_bf)
    F_ref, Fb_ref = o._full_fluxes()
    F_dev = np.zeros(fv.n_if)
    F_dev[if_dst] = o.flow.F[sfv.face_ref]
    Fb_dev = np.zeros(fv.n_bf)
    Fb_dev[bf_dst] = o.flow.Fb[sfv.bface_ref][bf_src]
    assert np.array_equal(F_dev, F_ref[fv.face_ref]) and np.array_equal(Fb_dev, Fb_ref[fv.bface_ref])


def test_turbulent_face_diffusivities_on_the_device_layout():
    """What ``ConjugateSolver`` computes every iteration with the SST model, run on the host on the
    device layouts (``FVMesh`` built on the CPU): the flow's mu_t scattered to the full mesh's
    fluid cells, k/cp + mu_t/Pr_t, then ``harmonic_face_gamma``; equal to the oracle's face
    diffusivities (``conjugate.py:146-159``) bit for bit after three iterations."""
    import torch

    from gputest_b200.unstructured.conjugate import PR_T, conjugate_setup, harmonic_face_gamma
    from gputest_b200.unstructured.fvmesh import FVMesh

    mesh, case, _ = _case("heated_sst")
    o = OracleConjugate(mesh, case)
    for _ in range(3):
        o.step()
    hs = conjugate_setup(mesh, case)
    fv, sfv = FVMesh(mesh, torch.device("cpu")), FVMesh(hs["sub"], torch.device("cpu"))
    idx = torch.as_tensor(fv.iperm[hs["cell_map"][sfv.perm]], dtype=torch.long)
    mut_full = torch.zeros(fv.nc, dtype=torch.float64)
    mut_full.index_copy_(0, idx, torch.as_tensor(o.flow.turb.mut[sfv.perm]))
    g = fv.cells_to_device(hs["gam_cell"]) + mut_full / PR_T
    gf, gb = harmonic_face_gamma(g, fv.t["w"], fv.t["fP"].long(), fv.t["fN"].long(), fv.t["bP"].long())
    ogf, ogb = o.face_gamma()
    assert np.array_equal(gf.numpy(), ogf[fv.face_ref]) and np.array_equal(gb.numpy(), ogb[fv.bface_ref])
    assert not np.array_equal(ogf, hs["gamma_face"])  # mu_t did change them
