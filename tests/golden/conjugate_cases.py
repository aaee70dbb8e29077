"""Conjugate heat transfer cases shared by the fixture generator and the tests.

Each case is (mesh builder, case keywords with boundaries as dicts, outer iterations). The
builders use this package's generators (which build the reference's arrays) and move cells
into solid cell zones by their centres, as the reference's ``set_cell_zone`` does.
"""

from tests.golden.mesh_cases import with_solid_zone


def _composite():
    from gputest_b200.mesh.unstructured import cartesian_mesh_2d

    m = cartesian_mesh_2d(30, 3, 3.0, 1.0)
    m, _ = with_solid_zone(m, lambda x: x[:, 0] < 1.0, "a")
    m, _ = with_solid_zone(m, lambda x: x[:, 0] > 2.0, "b")
    return m


def _heated():
    from gputest_b200.mesh.unstructured import cartesian_mesh_2d

    m = cartesian_mesh_2d(30, 10, 4.0, 1.25, names=("inlet", "outlet", "bottom", "top"),
                          types=("velocity-inlet", "pressure-outlet", "wall", "wall"), y0=-0.25)
    m, _ = with_solid_zone(m, lambda x: x[:, 1] < 0.0, "heater")
    return m


def _tri_disc():
    from gputest_b200.mesh.unstructured import cartesian_mesh_2d

    m = cartesian_mesh_2d(16, 16, triangulate=True, jitter=0.1, seed=4)
    m, _ = with_solid_zone(m, lambda x: (x[:, 0] - 0.5) ** 2 + (x[:, 1] - 0.45) ** 2 < 0.06, "heater")
    return m


CONJUGATE_CASES = {
    "composite": (_composite,
                  dict(energy=True, conductivity=1.0,
                       solids={"a": {"conductivity": 5.0}, "b": {"conductivity": 0.5}},
                       boundaries={"left": {"kind": "wall", "thermal": "temperature", "value": 1.0},
                                   "right": {"kind": "wall", "thermal": "temperature", "value": 0.0}},
                       max_iter=300, tol=0.0, pressure_tol=1e-9), 30),
    "heated": (_heated,
               dict(energy=True, conductivity=0.05, viscosity=0.05,
                    solids={"heater": {"conductivity": 2.0, "source": 4.0}},
                    boundaries={"inlet": {"kind": "inlet", "normal_speed": 1.0, "value": 0.0},
                                "outlet": {"kind": "outlet"}},
                    max_iter=300, tol=0.0, pressure_tol=1e-9), 30),
    "heated_sst": (_heated,
                   dict(energy=True, conductivity=0.002, viscosity=2e-3, turbulence="k-omega-sst",
                        solids={"heater": {"conductivity": 2.0, "source": 4.0}},
                        boundaries={"inlet": {"kind": "inlet", "normal_speed": 1.0, "value": 0.0},
                                    "outlet": {"kind": "outlet"}},
                        max_iter=300, tol=0.0, pressure_tol=1e-9), 20),
    "tri_disc": (_tri_disc,
                 dict(energy=True, conductivity=0.02, viscosity=0.01,
                      solids={"heater": {"conductivity": 3.0, "source": 2.0}},
                      boundaries={"top": {"kind": "wall", "velocity": [1.0, 0.0], "thermal": "temperature",
                                          "value": 0.0},
                                  "bottom": {"kind": "wall", "thermal": "temperature", "value": 1.0}},
                      max_iter=300, tol=0.0, pressure_tol=1e-9), 25),
}
