"""Case and boundary-condition objects of the unstructured SIMPLEC solver.

Same fields, defaults and validation as ``flowtrace/unstructured/case.py:9-188`` so that a
case written for the reference runs here unchanged. The k-omega SST model and solid zones (through
``conjugate.make_solver``) are implemented; fields of the models that are not (the k-epsilon
models, radiation, species, MRF, periodic pairs, transient) are kept so such cases still parse,
and ``SimpleSolver`` rejects them with ``NotImplementedError``.
"""

from __future__ import annotations

from dataclasses import asdict, dataclass, field
from typing import Dict, List, Optional

FLUENT_TO_KIND = {
    "wall": "wall",
    "velocity-inlet": "inlet",
    "mass-flow-inlet": "inlet",
    "pressure-inlet": "pressure",
    "pressure-outlet": "outlet",
    "outflow": "outlet",
    "pressure-far-field": "outlet",
    "outlet-vent": "outlet",
    "exhaust-fan": "outlet",
    "inlet-vent": "pressure",
    "intake-fan": "pressure",
    "symmetry": "symmetry",
    "axis": "symmetry",
    "periodic": "periodic",
    "periodic-shadow": "periodic",
}
KINDS = ("wall", "inlet", "outlet", "pressure", "symmetry", "periodic")
RADIATION_MODELS = ("off", "p1")
TURBULENCE_MODELS = ("laminar", "k-omega-sst", "k-epsilon-realizable", "k-epsilon-standard")
TURBULENCE_ALIASES = {"sst": "k-omega-sst", "kw-sst": "k-omega-sst", "k-omega": "k-omega-sst", "none": "laminar"}


@dataclass
class BoundarySpec:
    """Boundary condition of one face zone.

    wall: ``velocity`` (default no-slip at rest), ``thermal`` 'adiabatic' | 'temperature' |
    'flux' with ``value``; inlet: ``velocity`` or ``normal_speed`` (> 0 into the domain), T =
    ``value``; outlet: static gauge ``pressure``, zero-gradient velocity and temperature;
    pressure: an opening at ``pressure``; symmetry: slip, no normal flux.
    """

    kind: str = "wall"
    velocity: Optional[List[float]] = None
    normal_speed: Optional[float] = None
    pressure: float = 0.0
    thermal: str = "adiabatic"
    value: float = 0.0
    turb_intensity: Optional[float] = None
    turb_viscosity_ratio: Optional[float] = None
    k: Optional[float] = None
    omega: Optional[float] = None
    epsilon: Optional[float] = None
    rotation: Optional[dict] = None
    emissivity: float = 1.0
    species: Optional[Dict[str, float]] = None

    def __post_init__(self):
        if self.kind not in KINDS:
            raise ValueError(f"unknown boundary kind {self.kind!r}")


@dataclass
class UnstructuredCase:
    name: str = "unstructured case"
    mesh_file: str = ""
    boundaries: Dict[str, BoundarySpec] = field(default_factory=dict)
    density: float = 1.0
    viscosity: float = 0.01
    energy: bool = False
    conductivity: float = 0.01
    cp: float = 1.0
    buoyancy: List[float] = field(default_factory=lambda: [0.0, 0.0, 0.0])
    t_ref: float = 0.0
    body_force: List[float] = field(default_factory=lambda: [0.0, 0.0, 0.0])
    algorithm: str = "SIMPLEC"
    relax_u: float = 0.7
    relax_p: Optional[float] = None
    relax_T: float = 1.0
    scheme: str = "second-order"
    scalar_scheme: Optional[str] = None
    pressure_gradient: str = "green-gauss"
    pressure_tol: float = 0.1
    turbulence: str = "laminar"
    turb_intensity: float = 0.05
    turb_viscosity_ratio: float = 10.0
    turb_reference_velocity: Optional[float] = None
    turb_init: Optional[Dict[str, float]] = None
    relax_k: Optional[float] = None
    relax_w: Optional[float] = None
    relax_mut: float = 1.0
    turb_scheme: str = "upwind"
    mrf: Dict[str, dict] = field(default_factory=dict)
    solids: Dict[str, dict] = field(default_factory=dict)
    max_iter: int = 2000
    tol: float = 1e-5
    init_velocity: List[float] = field(default_factory=lambda: [0.0, 0.0, 0.0])
    init_T: float = 0.0
    backend: str = "auto"
    precision: str = "fp64"
    monitor_interval: int = 1
    periodic: List[List[str]] = field(default_factory=list)
    periodic_pressure_gradient: List[float] = field(default_factory=lambda: [0.0, 0.0, 0.0])
    unsteady: bool = False
    dt: float = 0.01
    t_end: float = 1.0
    time_scheme: str = "bdf2"
    inner_iterations: int = 20
    inner_tol: float = 1e-4
    radiation: str = "off"
    absorption: float = 1.0
    scattering: float = 0.0
    species: List[str] = field(default_factory=list)
    species_diffusivity: float = 1e-5
    schmidt_turbulent: float = 0.7
    prandtl_turbulent: float = 0.85
    ref_velocity: float = 1.0
    ref_area: float = 1.0

    def __post_init__(self):
        self.boundaries = {k: (BoundarySpec(**v) if isinstance(v, dict) else v) for k, v in self.boundaries.items()}
        if self.algorithm.upper() not in ("SIMPLE", "SIMPLEC"):
            raise ValueError("algorithm must be SIMPLE or SIMPLEC")
        self.algorithm = self.algorithm.upper()
        if self.relax_p is None and self.algorithm == "SIMPLE":
            self.relax_p = 0.3
        self.turbulence = TURBULENCE_ALIASES.get(str(self.turbulence).lower(), str(self.turbulence).lower())
        if self.turbulence not in TURBULENCE_MODELS:
            raise ValueError(f"turbulence must be one of {TURBULENCE_MODELS}")
        if self.pressure_gradient not in ("green-gauss", "least-squares"):
            raise ValueError("pressure_gradient must be 'green-gauss' or 'least-squares'")
        self.radiation = str(self.radiation).lower()
        if self.radiation not in RADIATION_MODELS:
            raise ValueError(f"radiation must be one of {RADIATION_MODELS}")
        if self.radiation != "off" and not self.energy:
            raise ValueError("the radiation model needs the energy equation (energy=True)")
        if self.time_scheme not in ("euler", "bdf2"):
            raise ValueError("time_scheme must be 'euler' or 'bdf2'")
        if self.precision not in ("fp64", "fp32", "mixed"):
            raise ValueError("precision must be 'fp64', 'fp32' or 'mixed'")
        self.periodic = [list(p) for p in self.periodic]

    @property
    def turbulent(self) -> bool:
        return self.turbulence != "laminar"

    def to_dict(self) -> dict:
        return asdict(self)

    @classmethod
    def from_dict(cls, d: dict) -> "UnstructuredCase":
        return cls(**d)


def default_boundaries(mesh) -> Dict[str, BoundarySpec]:
    """A boundary spec per boundary zone from its Fluent type; inlets get normal speed 1."""
    out = {}
    for z in mesh.boundary_zones():
        kind = FLUENT_TO_KIND.get(z.type, "wall")
        spec = BoundarySpec(kind=kind)
        if kind == "inlet":
            spec.normal_speed = 1.0
        out[z.name] = spec
    return out
