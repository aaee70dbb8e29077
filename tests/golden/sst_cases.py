"""Turbulent (k-omega SST) cases shared by the fixture generator and the tests.

Each case is (mesh builder, case keywords with boundaries as dicts, outer iterations). A mesh
builder takes the two generators ``(cartesian_mesh_2d, extrude_to_3d)``, so that the reference's
generators and this package's (which build identical arrays) make the same mesh.
"""

import numpy as np

RE_Y = np.array([0.0, 1e-6, 0.3, 4.0, 25.0, 119.9, 120.1, 900.0, 1.2e4, 3.0e5, 8.0e6])

_CHAN = ("in", "out", "bottom", "top")


def _chan2d(cm, ex):
    return cm(40, 16, 4.0, 1.0, names=_CHAN)


def _tri2d(cm, ex):
    return cm(24, 10, 3.0, 1.0, names=_CHAN, triangulate=True, jitter=0.15, seed=1)


def _duct3d(cm, ex):
    return ex(cm(12, 6, 3.0, 1.0, names=_CHAN), 6, 1.0)


_WALLS = {"bottom": {"kind": "wall"}, "top": {"kind": "wall"}}

SST_CASES = {
    "chan2d": (_chan2d,
               dict(boundaries={"in": {"kind": "inlet", "velocity": [1.0, 0.0]}, "out": {"kind": "outlet"}, **_WALLS},
                    turbulence="k-omega-sst", viscosity=1e-4, max_iter=100, tol=0.0, pressure_tol=1e-9), 25),
    "tri2d_energy": (_tri2d,
                     dict(boundaries={"in": {"kind": "inlet", "velocity": [1.0, 0.0], "value": 1.0,
                                             "turb_intensity": 0.08, "turb_viscosity_ratio": 20.0},
                                      "out": {"kind": "outlet"},
                                      "bottom": {"kind": "wall", "thermal": "temperature", "value": 0.0},
                                      "top": {"kind": "wall", "velocity": [0.2, 0.0]}},
                          turbulence="k-omega-sst", energy=True, viscosity=2e-4, conductivity=3e-4,
                          max_iter=100, tol=0.0, pressure_tol=1e-9), 20),
    "duct3d": (_duct3d,
               dict(boundaries={"in": {"kind": "inlet", "velocity": [1.0, 0.0, 0.0], "k": 2e-3, "omega": 5.0},
                                "out": {"kind": "outlet"}, **_WALLS,
                                "back": {"kind": "wall"}, "front": {"kind": "wall"}},
                    turbulence="k-omega-sst", viscosity=5e-4, max_iter=100, tol=0.0, pressure_tol=1e-9), 15),
}
