"""Illumination, imaging and scan geometry (Sources/SimulatoProbe/): Aperture, Aberrations, Probe, GridScan,
ContrastTransferFunction."""

from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from .core import ElectronBeam, Grid, Waves, _refuse
from .engine import Engine

ABERRATION_SYMBOLS = ("C10", "C12", "phi12", "C21", "phi21", "C23", "phi23", "C30", "C32", "phi32", "C34", "phi34",
                      "C41", "phi41", "C43", "phi43", "C45", "phi45", "C50", "C52", "phi52", "C54", "phi54", "C56",
                      "phi56")


@dataclass(frozen=True)
class Aperture:
    """Semiangle cutoff [mrad] with abTEM's one-pixel soft edge (Probe.swift:11-48)."""
    semiangle_cutoff: float
    soft: bool = True

    def __post_init__(self):
        if not (self.semiangle_cutoff > 0) or math.isnan(self.semiangle_cutoff):
            _refuse(f"invalid aperture {self.semiangle_cutoff}")


class Aberrations:
    """Polar aberration coefficients in A and rad (Aberrations.swift:8-37); defocus = -C10, Cs = C30."""

    def __init__(self, **coefficients):
        self.values = {k: 0.0 for k in ABERRATION_SYMBOLS}
        for k, v in coefficients.items():
            if k == "defocus":
                self.values["C10"] = -float(v)
            elif k == "Cs":
                self.values["C30"] = float(v)
            elif k in self.values:
                self.values[k] = float(v)
            else:
                _refuse(f"unknown aberration {k}")
        if not all(math.isfinite(v) for v in self.values.values()):
            _refuse("every coefficient must be finite")

    def array(self):
        return [self.values[k] for k in ABERRATION_SYMBOLS]


class Probe:
    """A convergent probe (Probe.swift:51-157); built on the device."""

    def __init__(self, beam: ElectronBeam, grid: Grid, aperture: Aperture, aberrations: Aberrations | None = None,
                 tilt=(0.0, 0.0)):
        if not all(math.isfinite(t) for t in tilt):
            _refuse("the tilt must be finite")
        self.beam, self.grid, self.aperture = beam, grid, aperture
        self.aberrations = aberrations or Aberrations()
        self.tilt = (float(tilt[0]), float(tilt[1]))

    def c(self):
        ab = (C.c_double * 25)(*self.aberrations.array())
        return L.Probe_t(self.beam.energy, float(self.aperture.semiangle_cutoff), 1 if self.aperture.soft else 0, 0, ab,
                         self.tilt[0], self.tilt[1])

    def centred_spectrum(self, engine: Engine | None = None) -> np.ndarray:
        """Psi0 = aperture exp(-i chi) / norm, unshifted (Probe.swift:113-136), computed on the device in float64."""
        e = engine or Engine.require()
        re, im = np.empty((self.grid.nx, self.grid.ny)), np.empty((self.grid.nx, self.grid.ny))
        g, p = self.grid.c(), self.c()
        L.check(e.lib.simk_probe_spectrum(e.handle, C.byref(g), C.byref(p), L.dptr(re), L.dptr(im)))
        return re + 1j * im

    def build_many(self, positions, engine: Engine | None = None) -> list:
        """The probes at `positions` [(x, y)] built on the device: the gpuProbes hook (MetalMultislice.swift:113-117)."""
        e = engine or Engine.require()
        pos = np.ascontiguousarray(np.asarray(positions, dtype=np.float64).reshape(-1, 2))
        n = len(pos)
        re = np.empty((n, self.grid.nx, self.grid.ny))
        im = np.empty_like(re)
        g, p = self.grid.c(), self.c()
        L.check(e.lib.simk_build_probes(e.handle, C.byref(g), C.byref(p), n, L.dptr(pos), L.dptr(re), L.dptr(im)))
        return [Waves(re[k] + 1j * im[k], self.grid, self.beam, "reciprocal_space", self.tilt) for k in range(n)]

    def build(self, at, engine: Engine | None = None) -> Waves:
        """Probe.build(at:) (Probe.swift:72-109): centred at (x, y) [A], sum_k |Psi(k)|^2 = 1."""
        if not all(math.isfinite(v) for v in at):
            _refuse("invalid position 0")
        return self.build_many([at], engine)[0]


@dataclass(frozen=True)
class GridScan:
    """A rectangular grid of probe positions, x first (GridScan.swift:10-67)."""
    start: tuple
    end: tuple
    nx: int
    ny: int
    endpoint: bool = False

    def __post_init__(self):
        if self.nx < 1 or self.ny < 1:
            _refuse(f"gpts must be at least 1, got {self.nx} x {self.ny}")
        if not all(math.isfinite(v) for v in (*self.start, *self.end)):
            _refuse("start and end must be finite")
        if not (self.end[0] - self.start[0] > 0 or self.end[1] - self.start[1] > 0):
            _refuse("scan extent must be positive on at least one axis (abTEM's rule)")

    @staticmethod
    def linspace(a, b, n, endpoint):
        div = n - 1 if endpoint else n
        if div <= 0:
            return np.array([a])
        step = (b - a) / div
        out = np.arange(n) * step + a
        if endpoint and n > 1:
            out[-1] = b
        return out

    @property
    def shape(self):
        return [self.nx, self.ny]

    @property
    def positions(self) -> np.ndarray:
        xs = self.linspace(self.start[0], self.end[0], self.nx, self.endpoint)
        ys = self.linspace(self.start[1], self.end[1], self.ny, self.endpoint)
        return np.stack(np.meshgrid(xs, ys, indexing="ij"), axis=-1).reshape(-1, 2)


class ContrastTransferFunction:
    """An objective lens (abTEM's CTF; ContrastTransferFunction.swift:37-160): the aberration phase exp(-i chi), the
    spatial (angular spread beta [mrad]) and temporal (focal spread Delta [A]) envelopes of the quasi-coherent
    approximation, and the aperture (semiangle [mrad], inf for none). The kernel is computed in float64 on the device;
    `apply` is Waves.applying (IFFT(FFT(psi) H)) for a batch of waves, float32, returning the waves and the images."""

    def __init__(self, aberrations: Aberrations | None = None, semiangle_cutoff: float = math.inf,
                 soft_aperture: bool = True, focal_spread: float = 0.0, angular_spread: float = 0.0):
        if not (semiangle_cutoff > 0) or math.isnan(semiangle_cutoff):
            _refuse(f"invalid aperture {semiangle_cutoff}")
        if not (math.isfinite(focal_spread) and focal_spread >= 0):
            _refuse(f"focal spread must be finite and >= 0 A, got {focal_spread}")
        if not (math.isfinite(angular_spread) and angular_spread >= 0):
            _refuse(f"angular spread must be finite and >= 0 mrad, got {angular_spread}")
        self.aberrations = aberrations or Aberrations()
        self.semiangle_cutoff = float(semiangle_cutoff)
        self.soft_aperture = bool(soft_aperture)
        self.focal_spread = float(focal_spread)
        self.angular_spread = float(angular_spread)

    def c(self):
        return L.Ctf_t((C.c_double * 25)(*self.aberrations.array()), self.semiangle_cutoff,
                       1 if self.soft_aperture else 0, 0, self.focal_spread, self.angular_spread)

    def kernel(self, grid: Grid, energy: float, engine: Engine | None = None) -> np.ndarray:
        """H on the grid in FFT order (ContrastTransferFunction.kernel, :85-115)."""
        e = engine or Engine.require()
        re = np.zeros(grid.nx * grid.ny)
        im = np.zeros(grid.nx * grid.ny)
        g, c = grid.c(), self.c()
        L.check(e.lib.simk_ctf_kernel(e.handle, C.byref(g), float(energy), C.byref(c), L.dptr(re), L.dptr(im)))
        return (re + 1j * im).reshape(grid.nx, grid.ny)

    def apply(self, waves, engine: Engine | None = None):
        """Waves.applying (:146-161) on one Waves or a list of waves of one grid and beam: (waves, images)."""
        e = engine or Engine.require()
        many = isinstance(waves, (list, tuple))
        ws = list(waves) if many else [waves]
        if not ws:
            return ([], []) if many else (None, None)
        grid, beam = ws[0].grid, ws[0].beam
        for w in ws:
            if not w.grid.matches(grid) or w.beam.energy != beam.energy:
                _refuse("the waves must share one grid and beam")
        n = grid.nx * grid.ny
        stack = np.ascontiguousarray(np.stack([w.field for w in ws]).reshape(len(ws), n))
        re_in, im_in = np.ascontiguousarray(stack.real), np.ascontiguousarray(stack.imag)
        re, im, inten = np.zeros(len(ws) * n), np.zeros(len(ws) * n), np.zeros(len(ws) * n)
        g, c = grid.c(), self.c()
        L.check(e.lib.simk_apply_ctf(e.handle, C.byref(g), float(beam.energy), C.byref(c), len(ws), L.dptr(re_in),
                                     L.dptr(im_in), L.dptr(re), L.dptr(im), L.dptr(inten)))
        out = [Waves((re[k * n:(k + 1) * n] + 1j * im[k * n:(k + 1) * n]).reshape(grid.nx, grid.ny), grid, w.beam,
                     w.normalization) for k, w in enumerate(ws)]
        images = [inten[k * n:(k + 1) * n].reshape(grid.nx, grid.ny) for k in range(len(ws))]
        return (out, images) if many else (out[0], images[0])

    @staticmethod
    def scherzer_defocus(Cs: float, energy: float, factor: float = 1.5) -> float:
        """sign(Cs) sqrt(factor |Cs| lambda) [A] (:118-124)."""
        if not (math.isfinite(factor) and factor > 0):
            _refuse("the Scherzer factor must be finite and positive")
        lam = ElectronBeam(energy).wavelength
        s = 1.0 if Cs > 0 else (-1.0 if Cs < 0 else 0.0)
        return s * math.sqrt(factor * abs(Cs) * lam)

    @staticmethod
    def point_resolution(Cs: float, energy: float, divisor: float = 6.0) -> float:
        """(lambda^3 |Cs| / divisor)^(1/4) [A] (:127-131)."""
        if not (math.isfinite(divisor) and divisor > 0):
            _refuse("the divisor must be finite and positive")
        lam = ElectronBeam(energy).wavelength
        return math.pow(math.pow(lam, 3) * abs(Cs) / divisor, 1.0 / 4)

    @staticmethod
    def nyquist_sampling(semiangle_cutoff: float, energy: float, oversampling: float = 4.0) -> float:
        """1 / (oversampling alpha_c / lambda 1e-3) [A] (:134-142)."""
        if not (math.isfinite(semiangle_cutoff) and semiangle_cutoff > 0):
            _refuse(f"invalid aperture {semiangle_cutoff}")
        if not (math.isfinite(oversampling) and oversampling > 0):
            _refuse(f"invalid oversampling {oversampling}")
        lam = ElectronBeam(energy).wavelength
        return 1 / (oversampling * semiangle_cutoff / lam * 1e-3)
