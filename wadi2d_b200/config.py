"""The configuration records the step reads, with the reference's names and defaults
(wadi2d/config/schema.py:422-519, wadi2d/config/constants.py:3-7). Plain dataclasses: validation ranges are the
reference's, checked by ``validate``; ``Numerics(cfl=0.9)`` is allowed, as ``Numerics.model_construct`` is there."""

from __future__ import annotations

from dataclasses import dataclass

G = 9.80665
CRITICAL_WEIR_COEFF = 1.7046


@dataclass(frozen=True)
class Tables:
    rows: int = 16
    face_depth_max: float = 16.0
    face_depth_min: float = 8.0
    face_conveyance: str = "local_radius"
    local_radius_beta: float = 9.0
    crest_tolerance: float = 0.05


@dataclass(frozen=True)
class Numerics:
    cfl: float = 0.45
    limiter: str = "minmod"
    sheet_flow: bool = True
    mirror_dry_faces: bool = True
    face_depth_carry: bool = True
    e_wet: float = 1e-4
    h_cfl: float = 0.01
    u_max: float = 25.0
    dt_max: float = 5.0
    dt_min: float = 1e-3
    dt_every: int = 8
    wave_floor: float = 3.0
    plan_min: float = 0.02
    active_every: int = 16
    local_time_stepping: bool = False
    lts_levels: int = 3
    level_fp64: bool = False
    """Invert the near-dry bottom interval of each cell table in FP64 (not in the reference; off reproduces it)."""
    arithmetic: str = "exact"
    """The build of the step's face and update passes (not in the reference): "exact" is the reference's float32
    arithmetic, its CPU twin's bits; "fast" adds FMA contraction and the hardware's approximate division, square root
    and cube root in the face pass."""

    def validate(self) -> Numerics:
        """The reference's bounds (wadi2d/config/schema.py:457-519); cfl up to 0.7."""
        checks = [
            (0.05 <= self.cfl <= 0.7, "cfl"), (self.limiter in ("none", "minmod"), "limiter"),
            (1e-6 <= self.e_wet <= 0.1, "e_wet"), (1e-4 <= self.h_cfl <= 1.0, "h_cfl"),
            (1.0 <= self.u_max <= 100.0, "u_max"), (1e-3 <= self.dt_max <= 600.0, "dt_max"),
            (1e-6 <= self.dt_min <= 1.0, "dt_min"), (1 <= self.dt_every <= 64, "dt_every"),
            (0.1 <= self.wave_floor <= 30.0, "wave_floor"), (1e-4 <= self.plan_min <= 1.0, "plan_min"),
            (1 <= self.active_every <= 32, "active_every"), (self.arithmetic in ("exact", "fast"), "arithmetic"),
        ]  # fmt: skip
        bad = [n for ok, n in checks if not ok]
        if bad:
            raise ValueError(f"Numerics out of range: {bad}")
        return self


@dataclass(frozen=True)
class Outputs:
    """The envelope settings of wadi2d/config/schema.py:988-1066."""

    maxima_every: int = 4
    arrival_depth: float = 0.1
    speed_depth: float = 0.05
