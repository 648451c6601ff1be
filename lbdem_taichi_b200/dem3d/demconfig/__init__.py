"""DEM configuration objects (API of src/dem3d/demconfig/)."""
from __future__ import annotations

from abc import ABC, abstractmethod
from dataclasses import dataclass, field
from typing import Optional

from ...vector import Vector3


class ContactModelConfig(ABC):
    @abstractmethod
    def get_model_name(self) -> str: ...

    @abstractmethod
    def validate(self): ...


@dataclass
class LinearContactConfig(ContactModelConfig):
    """Linear spring-dashpot parameters (contact_model.py:22-40)."""
    stiffness_normal: float
    stiffness_tangential: float
    damping_normal: float
    damping_tangential: float
    pp_friction: float
    pw_friction: float

    def get_model_name(self) -> str:
        return "linear"

    def validate(self):
        if self.stiffness_normal <= 0 or self.stiffness_tangential <= 0:
            raise ValueError("Stiffness values must be positive")
        if self.damping_normal < 0 or self.damping_tangential < 0:
            raise ValueError("Damping values must be non-negative")
        if not (0 <= self.pp_friction <= 1) or not (0 <= self.pw_friction <= 1):
            raise ValueError("Friction coefficients must be between 0 and 1")


@dataclass
class HertzContactConfig(ContactModelConfig):
    """Hertz-Mindlin parameters (contact_model.py:43-61)."""
    pp_friction: float
    pw_friction: float
    pp_restitution: float
    pw_restitution: float

    def get_model_name(self) -> str:
        return "hertz"

    def validate(self):
        if not (0 <= self.pp_friction <= 1) or not (0 <= self.pw_friction <= 1):
            raise ValueError("Friction coefficients must be between 0 and 1")
        if not (0 <= self.pp_restitution <= 1) or not (0 <= self.pw_restitution <= 1):
            raise ValueError("Restitution coefficients must be between 0 and 1")


@dataclass
class DomainBounds:
    xmin: float
    xmax: float
    ymin: float
    ymax: float
    zmin: float
    zmax: float

    def __post_init__(self):
        for a in "xyz":
            lo, hi = getattr(self, a + "min"), getattr(self, a + "max")
            if lo >= hi:
                raise ValueError(f"{a}min ({lo}) must be < {a}max ({hi})")

    def get_extended_bounds(self):
        return Vector3(self.xmin, self.ymin, self.zmin), Vector3(self.xmax, self.ymax, self.zmax)


@dataclass
class ParticleProperties:
    elastic_modulus: float = 0
    poisson_ratio: float = 0
    density: float = 0
    max_coordinate_number: int = 0


@dataclass
class WallProperties:
    density: float = 0
    elastic_modulus: float = 0
    poisson_ratio: float = 0.0


class DEMSolverConfig:
    """Solver configuration (demconfig.py:7-149): domain, dt, gravity, contact
    model, particle/wall properties, six axis-aligned walls, periodicity."""
    BOUNDARY_TYPE_WALL = 0
    BOUNDARY_TYPE_PERIODIC = 1

    def __init__(self, domain: DomainBounds, dt: float, gravity, contact_model: ContactModelConfig,
                 init_particles: Optional[object] = None):
        if dt <= 0:
            raise ValueError(f"Time step dt must be positive, got {dt}")
        contact_model.validate()
        self.domain = domain
        self.dt = dt
        self.gravity = Vector3(*gravity)
        self.init_particles = init_particles
        self.contact_model = contact_model
        self.particle_props = ParticleProperties()
        self.wall_props = WallProperties()
        self.domain_min, self.domain_max = domain.get_extended_bounds()
        self._setup_walls()

    def _setup_walls(self):
        self.wall_normals = [Vector3(1.0, 0.0, 0.0), Vector3(-1.0, 0.0, 0.0), Vector3(0.0, 1.0, 0.0),
                             Vector3(0.0, -1.0, 0.0), Vector3(0.0, 0.0, 1.0), Vector3(0.0, 0.0, -1.0)]
        d = self.domain
        self.wall_distances = [d.xmax, -d.xmin, d.ymax, -d.ymin, d.zmax, -d.zmin]
        self.boundaryType = [self.BOUNDARY_TYPE_WALL] * 6

    def set_particle_properties(self, **kwargs) -> "DEMSolverConfig":
        for k, v in kwargs.items():
            if not hasattr(self.particle_props, k):
                raise ValueError(f"Unknown particle property: {k}")
            setattr(self.particle_props, k, v)
        return self

    def set_wall_properties(self, **kwargs) -> "DEMSolverConfig":
        for k, v in kwargs.items():
            if not hasattr(self.wall_props, k):
                raise ValueError(f"Unknown wall property: {k}")
            setattr(self.wall_props, k, v)
        return self

    def set_periodic_boundaries(self, x_periodic=False, y_periodic=False, z_periodic=False):
        for axis, flag in enumerate((x_periodic, y_periodic, z_periodic)):
            if flag:
                self.boundaryType[2 * axis] = self.BOUNDARY_TYPE_PERIODIC
                self.boundaryType[2 * axis + 1] = self.BOUNDARY_TYPE_PERIODIC
        return self

    def update_contact_model(self, **kwargs) -> "DEMSolverConfig":
        for k, v in kwargs.items():
            if not hasattr(self.contact_model, k):
                raise ValueError(f"Unknown parameter '{k}' for {self.contact_model.get_model_name()} contact model")
            setattr(self.contact_model, k, v)
        self.contact_model.validate()
        return self

    def summary(self) -> str:
        m = self.contact_model
        s = (f"\nDEM Solver Configuration:\n========================\n"
             f"Domain: [{self.domain.xmin}, {self.domain.xmax}] \u00d7 [{self.domain.ymin}, {self.domain.ymax}] \u00d7 "
             f"[{self.domain.zmin}, {self.domain.zmax}]\nTime step: {self.dt} s\n"
             f"Gravity: ({self.gravity.x}, {self.gravity.y}, {self.gravity.z}) m/s\u00b2\n\n"
             f"Particle Properties:\n- Elastic modulus: {self.particle_props.elastic_modulus} Pa\n"
             f"- Poisson ratio: {self.particle_props.poisson_ratio}\n- Density: {self.particle_props.density} kg/m\u00b3\n\n"
             f"Wall Properties:\n- Density: {self.wall_props.density} kg/m\u00b3\n"
             f"- Elastic modulus: {self.wall_props.elastic_modulus} Pa\n"
             f"- Poisson ratio: {self.wall_props.poisson_ratio}\n\nContact Model: {m.get_model_name().upper()}\n")
        if isinstance(m, LinearContactConfig):
            s += (f"- Normal stiffness: {m.stiffness_normal} N/m\n- Tangential stiffness: {m.stiffness_tangential} N/m\n"
                  f"- Normal damping: {m.damping_normal}\n- Tangential damping: {m.damping_tangential}\n")
        else:
            s += f"- P-P restitution: {m.pp_restitution}\n- P-W restitution: {m.pw_restitution}\n"
        s += (f"- P-P friction: {m.pp_friction}\n- P-W friction: {m.pw_friction}\n"
              f"- Max coordination number: {self.particle_props.max_coordinate_number}\n")
        return s


__all__ = ["ContactModelConfig", "LinearContactConfig", "HertzContactConfig", "DomainBounds",
           "ParticleProperties", "WallProperties", "DEMSolverConfig"]
