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

    @property
    def value_count(self) -> int:
        return int(np.prod(self.value_shape)) if self.value_shape else 1

    # ---- post-processing (ScanOperations.swift:12-117, IntegratedCenterOfMass.swift:11-41), on the device ----------

    def gaussianSourceSize(self, sigma: float | None = None, *, sigmaX: float | None = None,
                           sigmaY: float | None = None, samplingX: float, samplingY: float,
                           engine: Engine | None = None) -> "ScanMeasurement":
        """The scan with the finite source size of a Gaussian probe of standard deviation sigma [A] (or sigmaX,
        sigmaY): every value filtered periodically over the scan with scipy's kernel, the scan's pixel sizes
        samplingX, samplingY [A] (ScanOperations.swift:19-41). Bit-equal to the reference's float64 loop."""
        if sigma is not None:
            if sigmaX is not None or sigmaY is not None:
                _refuse("give sigma or sigmaX and sigmaY, not both")
            sigmaX = sigmaY = sigma
        if sigmaX is None or sigmaY is None:
            _refuse("give sigma or sigmaX and sigmaY")
        for v in (sigmaX, sigmaY):
            if not (math.isfinite(v) and v >= 0):
                _refuse(f"the source size must be finite and non-negative, got ({sigmaX}, {sigmaY}) A")
        for v in (samplingX, samplingY):
            if not (math.isfinite(v) and v > 0):
                _refuse(f"the scan sampling must be finite and positive, got ({samplingX}, {samplingY}) A")
        if len(self.scan_shape) != 2:
            _refuse("the source size filters a two-axis scan; a line scan has one axis")
        e = engine or Engine.require()
        vin = np.ascontiguousarray(self.values, dtype=np.float64).reshape(-1)
        out = np.empty_like(vin)
        L.check(e.lib.simk_gaussian_source_size(e.handle, self.scan_shape[0], self.scan_shape[1], self.value_count,
                                                float(sigmaX), float(sigmaY), float(samplingX), float(samplingY),
                                                L.dptr(vin), L.dptr(out)))
        return ScanMeasurement(list(self.scan_shape), list(self.value_shape), out.reshape(np.shape(self.values)))

    def poissonNoise(self, dose: float | None = None, *, dosePerArea: float | None = None,
                     samplingX: float | None = None, samplingY: float | None = None, samples: int | None = None,
                     seed: int = 0, stream: str = "values", engine: Engine | None = None):
        """Poisson noise for a total dose [electrons per pattern] or a dose per area [electrons / A^2] over scan pixels
        of samplingX x samplingY [A] (ScanOperations.swift:74-127): every value times the dose, clipped at 0, one
        Poisson draw each. With `samples`, a list of that many independent draws. A seed gives the same noise on every
        run. stream="values" (default): every value has a generator of its own, drawn in parallel; stream="reference":
        the reference's single generator stream in value order (one device thread), so a seed gives its draws."""
        if stream not in ("values", "reference"):
            _refuse(f"unknown Poisson stream {stream!r}: 'values' or 'reference'")
        if dosePerArea is not None:
            if dose is not None:
                _refuse("give dose or dosePerArea, not both")
            for v in (samplingX, samplingY):
                if v is None or not (math.isfinite(v) and v > 0):
                    _refuse(f"the scan sampling must be finite and positive, got ({samplingX}, {samplingY}) A")
            dose = samplingX * samplingY * dosePerArea
        if dose is None:
            _refuse("give dose or dosePerArea")
        n_samples = 1 if samples is None else int(samples)
        if n_samples < 1:
            _refuse(f"samples must be at least 1, got {n_samples}")
        vin = np.ascontiguousarray(self.values, dtype=np.float64).reshape(-1)
        if n_samples * vin.size * 8 > _physical_memory_half():
            _refuse(f"{n_samples} samples of {vin.size} values exceed half of the physical memory")
        if not (math.isfinite(dose) and dose >= 0):
            _refuse(f"the dose must be finite and non-negative, got {dose}")
        e = engine or Engine.require()
        out = np.empty(n_samples * vin.size)
        L.check(e.lib.simk_context_set_option(e.handle, L.OPT_POISSON_STREAM, 1 if stream == "reference" else 0))
        try:
            L.check(e.lib.simk_poisson_noise(e.handle, vin.size, L.dptr(vin), float(dose), n_samples,
                                             int(seed) & 0xFFFFFFFFFFFFFFFF, L.dptr(out)))
        finally:
            L.check(e.lib.simk_context_set_option(e.handle, L.OPT_POISSON_STREAM, 0))
        draws = [ScanMeasurement(list(self.scan_shape), list(self.value_shape),
                                 out[s * vin.size:(s + 1) * vin.size].reshape(np.shape(self.values)))
                 for s in range(n_samples)]
        return draws if samples is not None else draws[0]

    def gradientImages(self, samplingX: float, samplingY: float):
        """The x and y components of a two-value (centre-of-mass) measurement as two images over the scan
        (IntegratedCenterOfMass.swift:15-30)."""
        if list(self.value_shape) != [2]:
            _refuse(f"a centre-of-mass image needs two values per position (x, y), this measurement has shape "
                    f"{self.value_shape}")
        if len(self.scan_shape) != 2:
            _refuse(f"a centre-of-mass image needs a two-axis scan, this measurement has scan shape {self.scan_shape}")
        v = np.asarray(self.values, dtype=np.float64).reshape(self.scan_shape[0], self.scan_shape[1], 2)
        nx, ny = self.scan_shape
        return (RealField(nx, ny, v[..., 0].reshape(-1).copy(), samplingX, samplingY),
                RealField(nx, ny, v[..., 1].reshape(-1).copy(), samplingX, samplingY))

    def integratedCenterOfMass(self, samplingX: float, samplingY: float, engine: Engine | None = None) -> "RealField":
        """The integrated centre of mass (IntegratedCenterOfMass.swift:36-40): the Fourier-space integral of the
        centre-of-mass image, minimum 0, sampled as the scan."""
        gx, gy = self.gradientImages(samplingX, samplingY)
        return RealField.integratingGradient(gx, gy, engine=engine)


@dataclass
class RealField:
    """A real nx x ny image, row-major [ix * ny + iy], with its pixel sizes [A] (SimulatoCore's RealField)."""
    nx: int
    ny: int
    values: np.ndarray
    samplingX: float
    samplingY: float

    @staticmethod
    def integratingGradient(x: "RealField", y: "RealField", engine: Engine | None = None) -> "RealField":
        """The integral of a gradient field (ImageOperations.swift:31-48, 140-167; abTEM integrate_gradient):
        T^ = (kx g^x + ky g^y) / (2 pi i |k|^2), 0 at zero frequency, the real part of the inverse transform less its
        minimum, on the device in float64."""
        if (x.nx, x.ny, x.samplingX, x.samplingY) != (y.nx, y.ny, y.samplingX, y.samplingY):
            _refuse("the two gradient components must have the same shape and sampling")
        for v in (x.samplingX, x.samplingY):
            if not (math.isfinite(v) and v > 0):
                _refuse(f"invalid sampling ({x.samplingX}, {x.samplingY})")
        if x.nx < 2 or x.ny < 2:
            _refuse(f"the gradient's images need at least 2 points per axis, got {x.nx} x {x.ny}")
        e = engine or Engine.require()
        gx = np.ascontiguousarray(x.values, dtype=np.float64).reshape(-1)
        gy = np.ascontiguousarray(y.values, dtype=np.float64).reshape(-1)
        out = np.empty(x.nx * x.ny)
        L.check(e.lib.simk_integrate_gradient(e.handle, x.nx, x.ny, float(x.samplingX), float(x.samplingY),
                                              L.dptr(gx), L.dptr(gy), 1, L.dptr(out)))
        return RealField(x.nx, x.ny, out, x.samplingX, x.samplingY)


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
