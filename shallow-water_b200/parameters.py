"""Simulation parameters (reference src/parameters.rs:8-92), read from YAML."""
import math
from dataclasses import dataclass, field


@dataclass
class Numerical:
    grid_resolution: int = 32
    vertical_layers: int = 4
    time_step: float = 1.0 / 32.0
    duration: float = 25.0
    save_interval: float = 0.25
    max_pressure_difference: float = 1.0e-9
    strip_width: float = 0.4
    a2: float = 0.02
    a3: float = -0.01


@dataclass
class Physical:
    coriolis_frequency: float = 4.0 * math.pi
    gravity_wave_speed: float = 2.0 * math.pi
    mean_fluid_depth: float = 0.4
    damping: float = 10.0
    nnu: float = 3.0


@dataclass
class Environment:
    threads: int = 0
    output_directory: str = "./out"


@dataclass
class Parameters:
    numerical: Numerical = field(default_factory=Numerical)
    physical: Physical = field(default_factory=Physical)
    environment: Environment = field(default_factory=Environment)

    @classmethod
    def from_yaml(cls, path):
        import yaml
        with open(path) as f:
            d = yaml.safe_load(f) or {}
        return cls(Numerical(**d.get("numerical", {})), Physical(**d.get("physical", {})),
                   Environment(**d.get("environment", {})))
