"""Detectors and the STEM driver on the CUDA backend (Sources/SimulatoDetector/Detectors.swift, STEM.swift).

Every detector runs on the device on |FFT2(exit)|^2 of each position, accumulated in float64, averaged over the
potentials (frozen-phonon configurations)."""

from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from .core import Grid, Waves, _refuse
from .engine import Engine, ExecutionOptions
from .multislice import Backend


class AnnularDetector:
    """sum P over inner^2 <= alpha^2 < outer^2 [mrad]; outer None: floor(min cutoff angles) (Detectors.swift:91-136)."""

    def __init__(self, inner: float = 0.0, outer: float | None = None):
        if not (math.isfinite(inner) and inner >= 0):
            _refuse("inner must be finite and >= 0")
        if outer is not None and not (math.isfinite(outer) and outer >= inner):
            _refuse(f"outer must be finite and >= inner, got {outer}")
        self.inner, self.outer = float(inner), outer

    def c(self):
        return L.Detector_t(L.DET_ANNULAR, 0, 0, 0 if self.outer is None else 1, 0, 0, self.inner,
                            0.0 if self.outer is None else float(self.outer), 0.0)


_MAX_ANGLE = {"cutoff": L.MAXANGLE_CUTOFF, "valid": L.MAXANGLE_VALID, "full": L.MAXANGLE_FULL}


class PixelatedDetector:
    """The pattern cropped (cutoff / valid / full) and fftshifted (Detectors.swift:140-168)."""

    def __init__(self, max_angle: str = "valid"):
        if max_angle not in _MAX_ANGLE:
            _refuse(f"unknown max angle {max_angle!r}")
        self.max_angle = max_angle

    def c(self):
        return L.Detector_t(L.DET_PIXELATED, _MAX_ANGLE[self.max_angle], 0, 0, 0, 0, 0.0, 0.0, 0.0)


class CenterOfMassDetector:
    """sum P alpha over a pixelated region, not divided by sum P; units "mrad" or "inverse" (Detectors.swift:172-206)."""

    def __init__(self, max_angle: str = "valid", units: str = "inverse"):
        if max_angle not in _MAX_ANGLE or units not in ("mrad", "inverse"):
            _refuse("unknown max angle or units")
        self.max_angle, self.units = max_angle, units

    def c(self):
        u = L.UNITS_MRAD if self.units == "mrad" else L.UNITS_INV_ANGSTROM
        return L.Detector_t(L.DET_COM, _MAX_ANGLE[self.max_angle], u, 0, 0, 0, 0.0, 0.0, 0.0)


class SegmentedDetector:
    """n_r x n_phi polar bins between inner and outer [mrad], azimuth from rotation [rad] (Detectors.swift:210-263)."""

    def __init__(self, radial_bins: int, azimuthal_bins: int, inner: float, outer: float, rotation: float = 0.0):
        if radial_bins < 1 or azimuthal_bins < 1:
            _refuse("bins must be at least 1")
        if not (math.isfinite(inner) and math.isfinite(outer) and inner >= 0 and outer > inner
                and math.isfinite(rotation)):
            _refuse("need 0 <= inner < outer, finite, and a finite rotation")
        self.nr, self.nphi, self.inner, self.outer, self.rotation = radial_bins, azimuthal_bins, inner, outer, rotation

    def c(self):
        return L.Detector_t(L.DET_SEGMENTED, 0, 0, 1, self.nr, self.nphi, float(self.inner), float(self.outer),
                            float(self.rotation))


class BinnedPixelatedDetector:
    """The pattern on a uniform gpts[0] x gpts[1] grid of angles over [-max_angle, max_angle) mrad per axis, bin 0 at
    -max_angle: each k-space pixel's intensity goes to the bins its square overlaps, in proportion to the overlap area.
    The reference's PixelatedDetector has no numeric-angle mode (Detectors.swift:140-168; only cutoff / valid / full),
    so this rule is this library's own: 4D-STEM patterns "cropped to 128 x 128 up to 60 mrad"."""

    def __init__(self, max_angle: float, gpts=(128, 128)):
        if not (math.isfinite(max_angle) and max_angle > 0):
            _refuse("the maximum angle must be finite and positive")
        if len(gpts) != 2 or min(gpts) < 1 or max(gpts) > 4096:
            _refuse("bins must be in 1..4096 per axis")
        self.max_angle, self.gpts = float(max_angle), (int(gpts[0]), int(gpts[1]))

    def c(self):
        return L.Detector_t(L.DET_BINNED, 0, 0, 1, self.gpts[0], self.gpts[1], 0.0, self.max_angle, 0.0)


class WavesDetector:
    """The complex exit wave at every position (abTEM's WavesDetector; WavesDetector.swift:35-67): on the simulation grid,
    or resampled in Fourier space to rows x columns points over the same extent (Waves.resampled,
    WavesResample.swift:16-43)."""

    def __init__(self, rows: int | None = None, columns: int | None = None):
        if (rows is None) != (columns is None):
            _refuse("give both rows and columns, or neither")
        for n in (rows, columns):
            if n is not None and not (isinstance(n, (int, np.integer)) and n >= 2):
                _refuse(f"unsupported grid length {n}")
        self.rows, self.columns = rows, columns

    @staticmethod
    def required_bytes(positions: int, rows: int, columns: int) -> int:
        """complex float64 waves: 16 bytes a point (WavesDetector.requiredBytes)."""
        return positions * rows * columns * 16


def _physical_memory_half() -> int:
    try:
        return os.sysconf("SC_PAGE_SIZE") * os.sysconf("SC_PHYS_PAGES") // 2
    except (ValueError, OSError, AttributeError):
        return 1 << 62


@dataclass
class ScanWaves:
    """The exit waves of a scan (ScanWaves, WavesDetector.swift:71-106): values[position][row][column], positions
    row-major over (scan x, scan y), on `grid` (the detector's rows x columns over the simulation extent)."""
    scan_shape: list
    grid: Grid
    beam: object
    values: np.ndarray

    def __getitem__(self, ix_iy) -> Waves:
        ix, iy = ix_iy
        return Waves(self.values[ix * self.scan_shape[1] + iy], self.grid, self.beam, "reciprocal_space")

    def array(self) -> np.ndarray:
        return self.values.reshape(tuple(self.scan_shape) + (self.grid.nx, self.grid.ny))


def _waves_scan(probe, potential, scan, detector: WavesDetector, engine: Engine) -> ScanWaves:
    rows = detector.rows or probe.grid.nx
    columns = detector.columns or probe.grid.ny
    positions = np.ascontiguousarray(scan.positions, dtype=np.float64)
    n = len(positions)
    re = np.zeros(n * rows * columns)
    im = np.zeros(n * rows * columns)
    p = probe.c()
    h = potential.handle(engine).handle
    L.check(engine.lib.simk_scan_waves(engine.handle, C.byref(p), h, n, L.dptr(positions), detector.rows or 0,
                                       detector.columns or 0, L.dptr(re), L.dptr(im)))
    grid = Grid(rows, columns, probe.grid.extent_x, probe.grid.extent_y)
    return ScanWaves(list(scan.shape), grid, probe.beam, (re + 1j * im).reshape(n, rows, columns))


def _check_waves_memory(probe, scan, detector: WavesDetector, configurations: int, limit: int | None):
    rows = detector.rows or probe.grid.nx
    columns = detector.columns or probe.grid.ny
    positions = len(scan.positions) * configurations
    need = WavesDetector.required_bytes(positions, rows, columns)
    limit = _physical_memory_half() if limit is None else limit
    if need > limit:
        _refuse(f"{positions} exit waves of {rows} x {columns} points need {need} bytes, more than the {limit} bytes "
                f"allowed (half of the physical memory); scan fewer positions or configurations, or detect on a "
                f"smaller rows x columns")


def detector_shape(detector, grid: Grid, energy: float):
    g = grid.c()
    d = detector.c()
    nd = C.c_int32(0)
    sh = (C.c_int32 * 2)()
    L.check(L.lib().simk_detector_shape(C.byref(g), energy, C.byref(d), C.byref(nd), sh))
    return [] if nd.value == 0 else [sh[0]] if nd.value == 1 else [sh[0], sh[1]]


@dataclass
class ScanMeasurement:
    """One detector's values over a scan, row-major (scan x, scan y, value shape) (STEM.swift:14-43)."""
    scan_shape: list
    value_shape: list
    values: np.ndarray

    def __getitem__(self, ixy):
        ix, iy = ixy
        n = int(np.prod(self.value_shape)) if self.value_shape else 1
        base = (ix * self.scan_shape[1] + iy) * n
        return self.values.reshape(-1)[base:base + n]

    def array(self) -> np.ndarray:
        return self.values.reshape(tuple(self.scan_shape) + tuple(self.value_shape))


class STEM:
    """STEM.scan (STEM.swift:49-150) on the device."""

    @staticmethod
    def scan(probe, potentials, scan, detectors, backend: Backend = Backend.cuda,
             options: ExecutionOptions | None = None, engine: Engine | None = None, memory_limit: int | None = None):
        """`detectors`: a list of measurement detectors (-> one ScanMeasurement each, averaged over the potentials), or
        a WavesDetector (-> ScanWaves of the single potential; memory_limit defaults to half the physical memory)."""
        if isinstance(detectors, WavesDetector):
            # STEM.scan(probe:potentials:scan:detector: WavesDetector) (WavesDetector.swift:115-137): one potential
            if len(potentials) != 1:
                _refuse(f"the waves detector takes one potential, got {len(potentials)}"
                        + ("" if not potentials else ": averaging complex waves over configurations is not "
                           "meaningful; scan the configurations with STEM.scanFrozenPhonons"))
            if not potentials[0].grid.matches(probe.grid):
                _refuse("grid mismatch")
            _check_waves_memory(probe, scan, detectors, 1, memory_limit)
            e = engine or Engine.require()
            e.apply(options)
            return _waves_scan(probe, potentials[0], scan, detectors, e)
        if not potentials:
            _refuse("no potential")
        for p in potentials:
            if not p.grid.matches(probe.grid):
                _refuse("grid mismatch")
        positions = np.ascontiguousarray(scan.positions, dtype=np.float64)
        shape = list(scan.shape)
        if not (1 <= len(shape) <= 2) or int(np.prod(shape)) != len(positions):
            _refuse("the scan shape must have one or two axes whose product is the number of positions")
        e = engine or Engine.require()
        e.apply(options)
        shapes = [detector_shape(d, probe.grid, probe.beam.energy) for d in detectors]
        counts = [int(np.prod(s)) if s else 1 for s in shapes]
        outs = [np.zeros(len(positions) * c) for c in counts]
        handles = [p.handle(e) for p in potentials]
        harr = (C.c_void_p * len(handles))(*[h.handle for h in handles])
        darr = (L.Detector_t * max(1, len(detectors)))(*[d.c() for d in detectors])
        oarr = (L.PD * max(1, len(outs)))(*[L.dptr(o) for o in outs])
        p = probe.c()
        L.check(e.lib.simk_scan(e.handle, C.byref(p), len(handles), harr, len(positions), L.dptr(positions),
                                len(detectors), darr, oarr))
        return [ScanMeasurement(shape, s, o) for s, o in zip(shapes, outs)]

    @staticmethod
    def scanFrozenPhonons(probe, phonons, nx, ny, slice_thickness, scan, detectors, parameterization=None,
                          options: ExecutionOptions | None = None, engine: Engine | None = None,
                          memory_limit: int | None = None):
        """The scan averaged over every configuration of a FrozenPhonons ensemble; with a WavesDetector, one ScanWaves
        per configuration instead (complex waves are not averaged, WavesDetector.swift:141-173)."""
        pots = phonons.lazy_potentials(nx, ny, slice_thickness, parameterization)
        if isinstance(detectors, WavesDetector):
            if not pots:
                _refuse("no potential")
            _check_waves_memory(probe, scan, detectors, len(pots), memory_limit)
            e = engine or Engine.require()
            e.apply(options)
            return [_waves_scan(probe, p, scan, detectors, e) for p in pots]
        return STEM.scan(probe, pots, scan, detectors, options=options, engine=engine)
