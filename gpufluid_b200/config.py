"""Scene-TOML schema of the reference (src/gpufluid/cli/config.py:60-518).

The sections and keys a FLIP/PIC/APIC scene uses parse exactly as in the
reference, with the same defaults, into dataclasses of the same names.  The
keys are [domain], [fluid], [[fluids]], [[obstacle]] (sphere, box,
cylinder_y, plane), [[inflow]], [[outflow]], [simulation] and [output].  Problems raise
``BlockError("C7.1", ...)`` as the reference does (config.py:297-300, :382,
:390).

Added optional [simulation] keys (reference defaults when absent):
``pressure_tol`` (1e-4), ``pcg_rhs_sign`` (-1: physical sign; +1: the
reference PCG's), ``pcg_check_every`` (10), ``pcg_preconditioner``
("jacobi", the reference's, or "tile_sgs"), ``pcg_sgs_sweeps`` (2) and
``pcg_coarse`` (false).

Sections outside this build parse, but a scene that uses them is rejected
with BlockError("C7.1") when the solver is built: mesh fluids and obstacles,
obstacle motion, and an MPM solver.
"""
from __future__ import annotations

import tomllib
from dataclasses import dataclass, field
from pathlib import Path
from typing import List, Optional, Sequence, Tuple, Union


class BlockError(RuntimeError):
    """Error tagged with the reference's block id ("[C7.1] message")."""

    def __init__(self, block_id: str, message: str):
        self.block_id = block_id
        self.message = message
        super().__init__(f"[{block_id}] {message}")


@dataclass
class DomainCfg:
    resolution: Tuple[int, int, int] = (64, 64, 64)
    dx: Optional[float] = None


@dataclass
class FluidBoxCfg:
    type: str = "box"
    lo: Tuple[float, float, float] = (0.05, 0.05, 0.05)
    hi: Tuple[float, float, float] = (0.40, 0.70, 0.40)
    ppc: int = 8
    color: Optional[Tuple[float, float, float]] = None
    temperature: Optional[float] = None


@dataclass
class FluidMeshCfg:
    type: str = "mesh"
    path: str = ""
    scale: float = 1.0
    translate: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    rotate_deg: Optional[Tuple[float, float, float]] = None
    ppc: int = 8
    color: Optional[Tuple[float, float, float]] = None
    temperature: Optional[float] = None


@dataclass
class ObstacleSphereCfg:
    type: str
    center: Tuple[float, float, float]
    radius: float


@dataclass
class ObstacleBoxCfg:
    type: str
    center: Tuple[float, float, float]
    half_size: Tuple[float, float, float]


@dataclass
class ObstacleCylinderYCfg:
    type: str
    center: Tuple[float, float, float]
    radius: float
    half_height: float


@dataclass
class ObstacleMeshCfg:
    type: str
    path: str
    scale: float = 1.0
    translate: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    rotate_deg: Optional[Tuple[float, float, float]] = None


@dataclass
class ObstaclePlaneCfg:
    type: str
    point: Tuple[float, float, float]
    normal: Tuple[float, float, float]
    bbox_lo: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    bbox_hi: Tuple[float, float, float] = (1.0, 1.0, 1.0)


ObstacleCfg = Union[ObstacleSphereCfg, ObstacleBoxCfg, ObstacleCylinderYCfg, ObstacleMeshCfg,
                    ObstaclePlaneCfg]


@dataclass
class SimulationCfg:
    solver: str = "flip"
    dt: float = 0.005
    pressure_iters: int = 60
    pressure_solver: str = "jacobi"
    cfl: bool = False
    cfl_factor: float = 0.5
    cfl_max_substeps: int = 16
    flip_blend: float = 0.95
    gravity: float = -9.81
    rho: float = 1.0
    viscosity: float = 0.0
    viscosity_iters: int = 12
    surface_tension: float = 0.0
    csf_smoothing_passes: int = 2
    transfer_mode: str = "flip"
    reseed: bool = False
    reseed_every_n_frames: int = 5
    reseed_min_per_cell: int = 4
    reseed_max_per_cell: int = 16
    frames: int = 100
    fps: int = 24
    pressure_tol: float = 1e-4
    pcg_rhs_sign: int = -1
    pcg_check_every: int = 10
    pcg_preconditioner: str = "jacobi"
    pcg_sgs_sweeps: int = 2
    pcg_coarse: bool = False


@dataclass
class OutputCfg:
    cache_dir: str = "out/sim"
    mesh: bool = True
    iso_level: float = 0.6
    smooth_passes: int = 2
    mesh_smooth_passes: int = 0
    mesh_smooth_method: str = "taubin"
    decimate_ratio: float = 1.0
    wall_margin_cells: int = 0
    mesh_method: str = "trilinear"
    cubic_radius_cells: float = 2.0
    sdf_particle_radius_cells: float = 1.0
    sdf_search_radius_cells: float = 4.0
    particles: bool = False
    usd: bool = False
    whitewater: bool = False


@dataclass
class InflowCfg:
    """config.py:140-158 (``keyframes`` moves MPM emitters only; FLIP ignores it)."""
    lo: Tuple[float, float, float]
    hi: Tuple[float, float, float]
    velocity: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    rate_per_sec: float = 5000.0
    frame_start: int = 0
    frame_end: int = 1_000_000
    keyframes: List[List[float]] = field(default_factory=list)
    color: Optional[Tuple[float, float, float]] = None
    temperature: Optional[float] = None


@dataclass
class OutflowCfg:
    """config.py:161-166."""
    lo: Tuple[float, float, float]
    hi: Tuple[float, float, float]
    frame_start: int = 0
    frame_end: int = 1_000_000


@dataclass
class SceneCfg:
    domain: DomainCfg = field(default_factory=DomainCfg)
    fluid: object = field(default_factory=FluidBoxCfg)
    fluids: List[object] = field(default_factory=list)
    obstacle: List[ObstacleCfg] = field(default_factory=list)
    obstacle_motion: List[Optional[dict]] = field(default_factory=list)
    inflow: List[InflowCfg] = field(default_factory=list)
    outflow: List[OutflowCfg] = field(default_factory=list)
    simulation: SimulationCfg = field(default_factory=SimulationCfg)
    output: OutputCfg = field(default_factory=OutputCfg)
    config_dir: Optional[Path] = None

    @property
    def dx(self) -> float:
        if self.domain.dx is not None:
            return self.domain.dx
        return 1.0 / max(self.domain.resolution)

    @property
    def domain_size(self) -> Tuple[float, float, float]:
        nx, ny, nz = self.domain.resolution
        return (nx * self.dx, ny * self.dx, nz * self.dx)


def _tuple(seq, n, name):
    if not isinstance(seq, Sequence) or isinstance(seq, str) or len(seq) != n:
        raise BlockError("C7.1", f"{name}: expected list of {n}; got {seq!r}")
    return tuple(seq)


def _parse_inflow(d: dict) -> InflowCfg:
    """config.py:319-333."""
    try:
        return InflowCfg(
            lo=_tuple(d["lo"], 3, "inflow.lo"), hi=_tuple(d["hi"], 3, "inflow.hi"),
            velocity=_tuple(d.get("velocity", [0, 0, 0]), 3, "inflow.velocity"),
            rate_per_sec=float(d.get("rate_per_sec", 5000.0)),
            frame_start=int(d.get("frame_start", 0)),
            frame_end=int(d.get("frame_end", 1_000_000)),
            keyframes=[[float(v) for v in row] for row in d.get("keyframes", [])],
            color=_tuple(d["color"], 3, "inflow.color") if "color" in d else None,
            temperature=float(d["temperature"]) if "temperature" in d else None)
    except KeyError as e:
        raise BlockError("C7.1", f"inflow: missing key {e.args[0]!r}") from None


def _parse_outflow(d: dict) -> OutflowCfg:
    """config.py:336-342."""
    try:
        return OutflowCfg(lo=_tuple(d["lo"], 3, "outflow.lo"), hi=_tuple(d["hi"], 3, "outflow.hi"),
                          frame_start=int(d.get("frame_start", 0)),
                          frame_end=int(d.get("frame_end", 1_000_000)))
    except KeyError as e:
        raise BlockError("C7.1", f"outflow: missing key {e.args[0]!r}") from None


def _parse_fluid(fl: dict) -> object:
    ftype = fl.get("type", "box")
    color = _tuple(fl["color"], 3, "fluid.color") if "color" in fl else None
    temperature = float(fl["temperature"]) if "temperature" in fl else None
    if ftype == "box":
        return FluidBoxCfg(type="box", lo=_tuple(fl.get("lo", [0.05, 0.05, 0.05]), 3, "fluid.lo"),
                           hi=_tuple(fl.get("hi", [0.40, 0.70, 0.40]), 3, "fluid.hi"),
                           ppc=int(fl.get("ppc", 8)), color=color, temperature=temperature)
    if ftype == "mesh":
        return FluidMeshCfg(type="mesh", path=str(fl.get("path", "")),
                            scale=float(fl.get("scale", 1.0)),
                            translate=_tuple(fl.get("translate", [0, 0, 0]), 3, "fluid.translate"),
                            rotate_deg=(_tuple(fl["rotate_deg"], 3, "fluid.rotate_deg")
                                        if "rotate_deg" in fl else None),
                            ppc=int(fl.get("ppc", 8)), color=color, temperature=temperature)
    raise BlockError("C7.1", f"unknown fluid type: {ftype!r}")


def _parse_obstacle(d: dict) -> ObstacleCfg:
    t = d.get("type")
    try:
        if t == "sphere":
            return ObstacleSphereCfg("sphere", _tuple(d["center"], 3, "obstacle.center"),
                                     float(d["radius"]))
        if t == "box":
            return ObstacleBoxCfg("box", _tuple(d["center"], 3, "obstacle.center"),
                                  _tuple(d["half_size"], 3, "obstacle.half_size"))
        if t == "cylinder_y":
            return ObstacleCylinderYCfg("cylinder_y", _tuple(d["center"], 3, "obstacle.center"),
                                        float(d["radius"]), float(d["half_height"]))
        if t == "plane":
            return ObstaclePlaneCfg("plane", _tuple(d["point"], 3, "obstacle.point"),
                                    _tuple(d["normal"], 3, "obstacle.normal"),
                                    _tuple(d.get("bbox_lo", [0, 0, 0]), 3, "obstacle.bbox_lo"),
                                    _tuple(d.get("bbox_hi", [1, 1, 1]), 3, "obstacle.bbox_hi"))
        if t == "mesh":
            return ObstacleMeshCfg("mesh", str(d["path"]), float(d.get("scale", 1.0)),
                                   _tuple(d.get("translate", [0, 0, 0]), 3, "obstacle.translate"),
                                   (_tuple(d["rotate_deg"], 3, "obstacle.rotate_deg")
                                    if "rotate_deg" in d else None))
    except KeyError as e:
        raise BlockError("C7.1", f"obstacle {t!r}: missing key {e.args[0]!r}") from None
    raise BlockError("C7.1", f"unknown obstacle type: {t!r}")


def load_scene(path: Union[str, Path]) -> SceneCfg:
    """Load and validate a TOML scene config (config.py:386-518)."""
    p = Path(path)
    if not p.exists():
        raise BlockError("C7.1", f"config not found: {p}")
    try:
        with open(p, "rb") as f:
            raw = tomllib.load(f)
    except tomllib.TOMLDecodeError as e:
        raise BlockError("C7.1", f"invalid TOML in {p}: {e}") from None
    dom = raw.get("domain", {})
    domain = DomainCfg(
        resolution=tuple(int(x) for x in _tuple(dom.get("resolution", [64, 64, 64]), 3,
                                                 "domain.resolution")),
        dx=float(dom["dx"]) if "dx" in dom else None)
    fluid = _parse_fluid(raw.get("fluid", {}))
    fluids = [_parse_fluid(f) for f in raw.get("fluids", [])]
    obstacles, motions = [], []
    for d in raw.get("obstacle", []):
        obstacles.append(_parse_obstacle(d))
        motions.append(d.get("motion"))
    sim = raw.get("simulation", {})
    defaults = SimulationCfg()
    kw = {}
    for name, default in defaults.__dict__.items():
        if name in sim:
            v = sim[name]
            kw[name] = type(default)(v) if not isinstance(default, bool) else bool(v)
    simulation = SimulationCfg(**kw)
    out = raw.get("output", {})
    od = OutputCfg()
    okw = {}
    for name, default in od.__dict__.items():
        if name in out:
            v = out[name]
            okw[name] = type(default)(v) if not isinstance(default, bool) else bool(v)
    output = OutputCfg(**okw)
    return SceneCfg(domain=domain, fluid=fluid, fluids=fluids, obstacle=obstacles,
                    obstacle_motion=motions,
                    inflow=[_parse_inflow(d) for d in raw.get("inflow", [])],
                    outflow=[_parse_outflow(d) for d in raw.get("outflow", [])],
                    simulation=simulation, output=output,
                    config_dir=p.parent.resolve())
