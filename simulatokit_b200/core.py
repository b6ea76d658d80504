"""Core types of the host side: beam, grid, antialias sizes, waves, structures (Sources/SimulatoCore/).

These mirror SimulatoKit's value types so that callers and tests read like the reference's; every array result of the
hot path comes from libsimulato_cuda."""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from ._lib import InvalidArgument, SIMK_ERR_INVALID


def _refuse(msg: str):
    raise InvalidArgument(SIMK_ERR_INVALID, msg)


# CODATA 2014 as ASE 3.29 / abTEM 1.0.10 (Sources/SimulatoCore/PhysicalConstants.swift:8-31)
PLANCK = 6.62607004e-34
ELECTRON_MASS = 9.10938356e-31
SPEED_OF_LIGHT = 299792458.0
ELEMENTARY_CHARGE = 1.6021766208e-19
_ASE_KG, _ASE_COULOMB, _ASE_SECOND, _ASE_JOULE = 6.0221408585491615e26, 6.241509125883258e18, 98226947884640.62, \
    6.241509125883258e18


@dataclass(frozen=True)
class ElectronBeam:
    """Sources/SimulatoCore/ElectronBeam.swift:10-44."""
    energy: float

    def __post_init__(self):
        if not (math.isfinite(self.energy) and self.energy > 0):
            _refuse(f"invalid energy {self.energy}")

    @property
    def wavelength(self) -> float:
        c2 = SPEED_OF_LIGHT * SPEED_OF_LIGHT
        return PLANCK * SPEED_OF_LIGHT / math.sqrt(self.energy * (2 * ELECTRON_MASS * c2 / ELEMENTARY_CHARGE +
                                                                  self.energy)) / ELEMENTARY_CHARGE * 1.0e10

    @property
    def interaction_parameter(self) -> float:
        mass = (1 + ELEMENTARY_CHARGE * self.energy / (ELECTRON_MASS * SPEED_OF_LIGHT ** 2)) * ELECTRON_MASS
        hsj = PLANCK * _ASE_SECOND * _ASE_JOULE
        return 2 * math.pi * mass * _ASE_KG * ELEMENTARY_CHARGE * _ASE_COULOMB * self.wavelength / (hsj * hsj)


@dataclass(frozen=True)
class Grid:
    """nx x ny points over extent_x x extent_y [A], x first, row-major (Sources/SimulatoCore/Grid.swift:8-91)."""
    nx: int
    ny: int
    extent_x: float
    extent_y: float

    def __post_init__(self):
        for n in (self.nx, self.ny):
            if not (isinstance(n, (int, np.integer)) and n >= 2):
                _refuse(f"unsupported grid length {n}")
        if not (math.isfinite(self.extent_x) and math.isfinite(self.extent_y) and self.extent_x > 0
                and self.extent_y > 0):
            _refuse(f"invalid extent {self.extent_x} x {self.extent_y}")

    @staticmethod
    def from_sampling(extent_x, extent_y, sampling_x, sampling_y=None) -> "Grid":
        """abTEM's _adjust_gpts: ceil(extent / sampling) points (Grid.swift:31-41)."""
        sampling_y = sampling_x if sampling_y is None else sampling_y
        if not (math.isfinite(sampling_x) and math.isfinite(sampling_y) and sampling_x > 0 and sampling_y > 0):
            _refuse("invalid sampling")
        return Grid(int(math.ceil(extent_x / sampling_x)), int(math.ceil(extent_y / sampling_y)), extent_x, extent_y)

    @property
    def sampling_x(self):
        return self.extent_x / self.nx

    @property
    def sampling_y(self):
        return self.extent_y / self.ny

    @property
    def count(self):
        return self.nx * self.ny

    def matches(self, other: "Grid", rtol: float = 1e-12) -> bool:
        """Grid.matches (Grid.swift:69-80)."""
        def close(a, b):
            return a == b or abs(a - b) <= rtol * max(abs(a), abs(b))
        return self.nx == other.nx and self.ny == other.ny and close(self.extent_x, other.extent_x) and \
            close(self.extent_y, other.extent_y)

    def c(self):
        from ._lib import Grid_t
        return Grid_t(self.nx, self.ny, float(self.extent_x), float(self.extent_y))


class Antialias:
    """Sources/SimulatoCore/Antialias.swift:11-58."""
    cutoff = 0.6666666
    taper = 0.01

    @staticmethod
    def cutoff_pattern_size(grid: Grid):
        kcut = 2.0 / 3.0 / max(grid.sampling_x, grid.sampling_y)

        def size(n, extent):
            m = int(math.floor(np.round(kcut * extent, 7)))
            if m % 2 != n % 2:
                m += 1
            if m % 2 == 0:
                m += 1
            return m
        return size(grid.nx, grid.nx * grid.sampling_x), size(grid.ny, grid.ny * grid.sampling_y)


@dataclass
class Waves:
    """A wave on a grid with its beam (Sources/SimulatoCore/Waves.swift:8-97). field: complex128 [nx, ny].
    normalization: "values" (a plane wave) or "reciprocal_space" (a probe)."""
    field: np.ndarray
    grid: Grid
    beam: ElectronBeam
    normalization: str = "values"
    tilt: tuple = (0.0, 0.0)

    @staticmethod
    def plane_wave(beam: ElectronBeam, grid: Grid, tilt=(0.0, 0.0)) -> "Waves":
        return Waves(np.ones((grid.nx, grid.ny), dtype=np.complex128), grid, beam, "values", tuple(tilt))

    planeWave = plane_wave

    def intensity(self) -> np.ndarray:
        return self.field.real ** 2 + self.field.imag ** 2

    @property
    def total_intensity(self) -> float:
        return float(self.intensity().sum())


@dataclass
class AtomicStructure:
    """An orthogonal box with atoms (Sources/SimulatoCore/AtomicStructure.swift:9-55)."""
    box: tuple
    numbers: np.ndarray
    positions: np.ndarray

    def __post_init__(self):
        self.box = tuple(float(b) for b in self.box)
        if not all(math.isfinite(b) and b > 0 for b in self.box):
            _refuse(f"invalid box {self.box}")
        self.numbers = np.asarray(self.numbers, dtype=np.int64).reshape(-1)
        self.positions = np.asarray(self.positions, dtype=np.float64).reshape(-1, 3)
        if len(self.numbers) != len(self.positions):
            _refuse("numbers and positions differ in length")
        bad = ~np.isfinite(self.positions).all(axis=1)
        if bad.any():
            _refuse(f"invalid position of atom {int(np.argmax(bad))}")

    def repeated(self, nx: int, ny: int, nz: int) -> "AtomicStructure":
        """ASE's repeat order: x outermost, then y, then z, the atoms innermost (AtomicStructure.swift:40-54)."""
        shifts = np.array([(mx * self.box[0], my * self.box[1], mz * self.box[2])
                           for mx in range(nx) for my in range(ny) for mz in range(nz)])
        pos = (shifts[:, None, :] + self.positions[None, :, :]).reshape(-1, 3)
        nums = np.tile(self.numbers, len(shifts))
        return AtomicStructure((self.box[0] * nx, self.box[1] * ny, self.box[2] * nz), nums, pos)
