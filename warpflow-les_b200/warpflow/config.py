"""YAML case files -> typed configuration.

Same schema, defaults and validation as the reference loader
(warpflow/config.py:15-132): one dataclass per YAML section, ``physics.sgs``
flattened into ``sgs_enabled/sgs_model/sgs_cw``, and every grid axis must
divide by the domain count and by 2**(mg_levels-1).

Two additions: ``numerics.mg_precision`` selects the multigrid arithmetic,
``"fp64"`` (default, the reference's) or ``"mixed"`` (FP32 V-cycles inside
an FP64 defect correction); ``numerics.mg_coarse`` selects how the coarsest
level's n_coarse sweeps run, ``"operator"`` (default: the same linear map
applied as one precomputed matrix-vector product, where the coarsest edge is
4..24 in steps of 4) or ``"sweeps"``.
"""
from __future__ import annotations

from dataclasses import dataclass, field, fields
from pathlib import Path

import yaml


@dataclass
class DomainCfg:
    lx: float = 1.0
    ly: float = 1.0
    lz: float = 1.0


@dataclass
class GridCfg:
    nx: int = 80
    ny: int = 80
    nz: int = 80


@dataclass
class PhysicsCfg:
    reynolds: float = 400.0
    sgs_enabled: bool = True
    sgs_model: str = "wale"
    sgs_cw: float = 0.46


@dataclass
class InitialCfg:
    type: str = "rest"
    noise: float = 0.01


@dataclass
class BoundaryCfg:
    west: str = "wall"
    east: str = "wall"
    south: str = "slip"
    north: str = "slip"
    bottom: str = "wall"
    top: str = "moving_lid"
    lid_velocity: float = 1.0


@dataclass
class NumericsCfg:
    time_scheme: str = "rk2"
    convection: str = "cds4"
    diffusion: str = "explicit4"
    pressure_solver: str = "multigrid"
    mg_levels: int = 3
    max_outer_iters: int = 30
    div_tolerance: float = 1.0e-6
    ghost_layers: int = 3
    mg_precision: str = "fp64"
    mg_coarse: str = "operator"


@dataclass
class TimeCfg:
    n_steps: int = 1000
    variable_dt: bool = True
    dt_init: float = 3.0e-4
    safety_factor: float = 0.8
    dt_growth: float = 1.1


@dataclass
class OutputCfg:
    n_out: int = 1500
    log_interval: int = 20
    outdir: str = "output"


@dataclass
class MpiCfg:
    domains: tuple = (1, 1, 1)


@dataclass
class CaseConfig:
    name: str = "cavity"
    domain: DomainCfg = field(default_factory=DomainCfg)
    grid: GridCfg = field(default_factory=GridCfg)
    physics: PhysicsCfg = field(default_factory=PhysicsCfg)
    initial: InitialCfg = field(default_factory=InitialCfg)
    boundaries: BoundaryCfg = field(default_factory=BoundaryCfg)
    numerics: NumericsCfg = field(default_factory=NumericsCfg)
    time: TimeCfg = field(default_factory=TimeCfg)
    output: OutputCfg = field(default_factory=OutputCfg)
    mpi: MpiCfg = field(default_factory=MpiCfg)


_SECTIONS = {"domain": DomainCfg, "grid": GridCfg, "initial": InitialCfg,
             "boundaries": BoundaryCfg, "numerics": NumericsCfg, "time": TimeCfg,
             "output": OutputCfg, "mpi": MpiCfg}


def _section(cls, raw):
    """Build a section dataclass; unknown keys raise TypeError as in the
    reference (which passes the mapping straight to the constructor)."""
    raw = dict(raw or {})
    known = {f.name for f in fields(cls)}
    extra = set(raw) - known
    if extra:
        raise TypeError("%s got unexpected keys %s" % (cls.__name__, sorted(extra)))
    return cls(**raw)


def case_from_dict(raw: dict) -> CaseConfig:
    cfg = CaseConfig(name=raw.get("case", "cavity"))
    for key, cls in _SECTIONS.items():
        setattr(cfg, key, _section(cls, raw.get(key, {})))
    phys = dict(raw.get("physics", {}) or {})
    sgs = dict(phys.pop("sgs", {}) or {})
    cfg.physics = PhysicsCfg(reynolds=phys.get("reynolds", 400.0),
                             sgs_enabled=sgs.get("enabled", True),
                             sgs_model=sgs.get("model", "wale"),
                             sgs_cw=sgs.get("cw", 0.46))
    if cfg.numerics.mg_precision not in ("fp64", "mixed"):
        raise ValueError("numerics.mg_precision must be 'fp64' or 'mixed', got %r"
                         % (cfg.numerics.mg_precision,))
    if cfg.numerics.mg_coarse not in ("operator", "sweeps"):
        raise ValueError("numerics.mg_coarse must be 'operator' or 'sweeps', got %r"
                         % (cfg.numerics.mg_coarse,))
    ncell = (cfg.grid.nx, cfg.grid.ny, cfg.grid.nz)
    div = 2 ** (cfg.numerics.mg_levels - 1)
    for axis, (n, m) in enumerate(zip(ncell, cfg.mpi.domains)):
        if n % m:
            raise ValueError(f"grid axis {axis} ({n} cells) not divisible by "
                             f"mpi domains ({m})")
        if (n // m) % div:
            raise ValueError(f"sub-domain cells on axis {axis} ({n // m}) must be "
                             f"divisible by 2**(mg_levels-1)={div}")
    return cfg


def load_case(path: str | Path) -> CaseConfig:
    """Read a YAML case file (reference config.py:101-132)."""
    return case_from_dict(yaml.safe_load(Path(path).read_text()) or {})
