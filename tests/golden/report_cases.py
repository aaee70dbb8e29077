"""Cases of the wall-report fixtures: a laminar channel with a heated (fixed temperature) and a
flux wall, and the k-omega SST channel of ``sst_cases.py``. Each is (mesh builder taking the
generators ``(cartesian_mesh_2d, extrude_to_3d)``, case keywords with boundaries as dicts,
outer iterations, the wall zone whose profile is recorded)."""

from tests.golden.sst_cases import SST_CASES


def _channel(cm, ex):
    return cm(24, 8, 3.0, 1.0, names=("in", "out", "bottom", "top"), warp=0.03)


REPORT_CASES = {
    "channel_energy": (_channel,
                       dict(boundaries={"in": {"kind": "inlet", "velocity": [1.0, 0.0], "value": 1.0},
                                        "out": {"kind": "outlet"},
                                        "bottom": {"kind": "wall", "thermal": "temperature", "value": 0.0},
                                        "top": {"kind": "wall", "thermal": "flux", "value": 2.0}},
                            energy=True, viscosity=0.01, conductivity=0.02, max_iter=50, tol=0.0,
                            ref_velocity=1.5, ref_area=0.5), 30, "bottom"),
    "sst_chan2d": SST_CASES["chan2d"] + ("top",),
}
