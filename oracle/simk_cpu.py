"""TEST INFRASTRUCTURE: ctypes wrapper of oracle/cpu/simk_cpu.cpp, the C++ float64 restatement of the reference's
`.cpu` STEM scan path (Multislice.runCPU, Probe.build, DiffractionIntensity and the annular detectors, positions over
threads as runCPUParallel: Sources/SimulatoCore/Multislice.swift:132-157, Sources/SimulatoProbe/Probe.swift:113-156,
Sources/SimulatoDetector/Detectors.swift:28-36, 119-135, Sources/SimulatoCore/MetalMultislice.swift:28-47).

Besides the per-position loop it restates the per-potential set-up (Sources/SimulatoMultislice/ProjectedPotential.swift:
110-201, Multislice.swift:83-130, Sources/SimulatoProbe/Probe.swift:25-48, 113-136, Detectors.swift:39-44, 119-135,
FrozenPhonons.swift:14-58), so `ScanInputs.from_structure` builds a scan from atoms without the NumPy oracle; only the
Lobato table comes from the oracle's data file. Only the tests and the benchmark's CPU legs use it, as a checker and as
the timed CPU baseline; the CUDA library never does. The library is built by `make -C oracle/cpu` (or `build()` below) into oracle/_build/libsimk_cpu.so."""

import ctypes as C
import os
import subprocess

import numpy as np

from . import simk_oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libsimk_cpu.so")
_lib = None

_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)


def build(force: bool = False) -> str:
    """Compiles the C++ restatement (g++, no external libraries). Returns the library's path."""
    src = os.path.join(HERE, "cpu", "simk_cpu.cpp")
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", os.path.join(HERE, "cpu")] + (["-B"] if force else []), check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.simk_cpu_fft2.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _D, _D]
        L.simk_cpu_fft2.restype = C.c_int
        L.simk_cpu_stem_scan.argtypes = [C.c_int, C.c_int, C.c_int, _D, _D, _I, _D, _D, _D, _D, _D, _D, C.c_int, _D,
                                         C.c_int, _D, C.c_int, _D]
        L.simk_cpu_stem_scan.restype = C.c_int
        L.simk_cpu_fft_path.argtypes = [C.c_int]
        L.simk_cpu_fft_path.restype = C.c_int
        L.simk_cpu_factorization.argtypes = [C.c_int, _I, C.c_int]
        L.simk_cpu_factorization.restype = C.c_int
        L.simk_cpu_cost_guess.argtypes = [C.c_int]
        L.simk_cpu_cost_guess.restype = C.c_double
        L.simk_cpu_potential.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int, _D, C.c_int,
                                         _I, _D, C.c_int, _I, _D, _D, C.c_int, _D]
        L.simk_cpu_transmission.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, _D, _D, _D]
        L.simk_cpu_propagator.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                          C.c_double, C.c_double, _D, _D]
        L.simk_cpu_probe_spectrum.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                              C.c_int, _D, _D, _D]
        L.simk_cpu_annular_mask.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                            C.c_double, _D]
        L.simk_cpu_normals.argtypes = [C.c_uint64, C.c_int, _D]
        for f in ("simk_cpu_potential", "simk_cpu_transmission", "simk_cpu_propagator", "simk_cpu_probe_spectrum",
                  "simk_cpu_annular_mask", "simk_cpu_normals"):
            getattr(L, f).restype = C.c_int
        _lib = L
    return _lib


FFT_PATHS = {0: "direct", 1: "mixedRadix", 2: "bluestein"}


def fft_path(n: int) -> str:
    """The transform one axis of length n takes: 'direct' (the lengths the reference gives vDSP: f 2^m, f in
    {1, 3, 5, 15}, m >= 3), 'mixedRadix' or 'bluestein' (MixedRadixPlan.prefersBluestein)."""
    return FFT_PATHS[lib().simk_cpu_fft_path(int(n))]


def factorization(n: int):
    """MixedRadixPlan.factorization: 2 first, then the 4s, then the odd primes ascending; None below 2."""
    out = (C.c_int * 64)()
    k = lib().simk_cpu_factorization(int(n), out, 64)
    return list(out[:k]) if k else None


def cost_guess(n: int) -> float:
    """MixedRadixPlan.costGuess: n times the sum of the factors (4 for a 4, 1.1 p above 5)."""
    return lib().simk_cpu_cost_guess(int(n))


def _p(a):
    return a.ctypes.data_as(_D)


def fft2(a: np.ndarray, inverse: bool = False) -> np.ndarray:
    """NumPy's fft2 / ifft2 over the last two axes, by the C++ mixed-radix / Bluestein transform."""
    a = np.asarray(a, dtype=np.complex128)
    shape = a.shape
    nx, ny = shape[-2], shape[-1]
    count = int(np.prod(shape[:-2])) if len(shape) > 2 else 1
    re = np.ascontiguousarray(a.real).reshape(-1).copy()
    im = np.ascontiguousarray(a.imag).reshape(-1).copy()
    rc = lib().simk_cpu_fft2(nx, ny, count, 1 if inverse else 0, _p(re), _p(im))
    if rc != 0:
        raise ValueError(f"simk_cpu_fft2: bad arguments ({nx}, {ny}, {count})")
    return (re + 1j * im).reshape(shape)


def _check(rc: int, what: str):
    if rc != 0:
        raise ValueError(f"{what}: bad arguments (status {rc})")


def potential(s: "O.Structure", nx: int, ny: int, thicknesses, pi_choice: str = "exact") -> np.ndarray:
    """The projected potential of every slice [S][nx][ny] by the C++ restatement (wrap, slicing, bilinear deltas,
    f(k^2) / S(k) per element), with the Lobato table the oracle reads."""
    numbers = np.ascontiguousarray(s.numbers, dtype=np.int32)
    elements = sorted(set(int(z) for z in numbers))
    tz = np.array(elements, dtype=np.int32)
    ta = np.ascontiguousarray([O.lobato_parameters(z)[0] for z in elements], dtype=np.float64).reshape(-1)
    tb = np.ascontiguousarray([O.lobato_parameters(z)[1] for z in elements], dtype=np.float64).reshape(-1)
    t = np.ascontiguousarray(thicknesses, dtype=np.float64)
    xyz = np.ascontiguousarray(s.positions, dtype=np.float64).reshape(-1)
    out = np.zeros((len(t), nx, ny))
    _check(lib().simk_cpu_potential(nx, ny, s.box[0], s.box[1], s.box[2], len(t), _p(t), len(numbers),
                                    numbers.ctypes.data_as(_I), _p(xyz), len(tz), tz.ctypes.data_as(_I),
                                    _p(ta if ta.size else np.zeros(1)), _p(tb if tb.size else np.zeros(1)),
                                    1 if pi_choice == "abtem" else 0, _p(out)), "simk_cpu_potential")
    return out


def transmission(v: np.ndarray, energy: float, g: "O.Grid") -> np.ndarray:
    v = np.ascontiguousarray(v, dtype=np.float64)
    re, im = np.zeros_like(v), np.zeros_like(v)
    _check(lib().simk_cpu_transmission(g.nx, g.ny, g.extent_x, g.extent_y, energy, _p(v), _p(re), _p(im)),
           "simk_cpu_transmission")
    return re + 1j * im


def propagator(g: "O.Grid", energy: float, dz: float, tilt=(0.0, 0.0)) -> np.ndarray:
    re, im = np.zeros((g.nx, g.ny)), np.zeros((g.nx, g.ny))
    _check(lib().simk_cpu_propagator(g.nx, g.ny, g.extent_x, g.extent_y, energy, dz, float(tilt[0]), float(tilt[1]),
                                     _p(re), _p(im)), "simk_cpu_propagator")
    return re + 1j * im


def probe_spectrum(p: "O.ProbeSpec", g: "O.Grid") -> np.ndarray:
    ab = np.ascontiguousarray([float(p.aberrations.get(k, 0.0)) for k in O.ABERRATION_SYMBOLS], dtype=np.float64)
    re, im = np.zeros((g.nx, g.ny)), np.zeros((g.nx, g.ny))
    _check(lib().simk_cpu_probe_spectrum(g.nx, g.ny, g.extent_x, g.extent_y, p.energy, p.semiangle,
                                         1 if p.soft else 0, _p(ab), _p(re), _p(im)), "simk_cpu_probe_spectrum")
    return re + 1j * im


def annular_mask(g: "O.Grid", energy: float, inner: float, outer: float) -> np.ndarray:
    out = np.zeros((g.nx, g.ny))
    _check(lib().simk_cpu_annular_mask(g.nx, g.ny, g.extent_x, g.extent_y, energy, inner, outer, _p(out)),
           "simk_cpu_annular_mask")
    return out


def normals(seed: int, n: int) -> np.ndarray:
    """The first n outputs of GaussianGenerator(seed)."""
    out = np.zeros(n)
    _check(lib().simk_cpu_normals(int(seed) & 0xFFFFFFFFFFFFFFFF, n, _p(out)), "simk_cpu_normals")
    return out


class ScanInputs:
    """The per-potential inputs of the scan, built once by the float64 NumPy oracle (they are shared by all positions,
    as runBatch shares them): transmissions, one propagator per distinct slice thickness, the probe's centred spectrum
    and the detectors' masks."""

    def __init__(self, probe: "O.ProbeSpec", g: "O.Grid", transmissions, thicknesses, masks):
        self.g = g
        nx, ny = g.nx, g.ny
        t = np.asarray(transmissions, dtype=np.complex128).reshape(len(thicknesses), nx, ny)
        self.t_re, self.t_im = np.ascontiguousarray(t.real), np.ascontiguousarray(t.imag)
        dzs = []
        self.prop = np.zeros(len(thicknesses), dtype=np.int32)
        for j, dz in enumerate(thicknesses):
            if dz not in dzs:
                dzs.append(dz)
            self.prop[j] = dzs.index(dz)
        p = np.stack([O.propagator(g, probe.energy, dz, probe.tilt) for dz in dzs])
        self.p_re, self.p_im = np.ascontiguousarray(p.real), np.ascontiguousarray(p.imag)
        s = O.centred_spectrum(probe, g)
        self.s_re, self.s_im = np.ascontiguousarray(s.real), np.ascontiguousarray(s.imag)
        self.fx = O.fftfreq(nx, 1.0).astype(np.float64)
        self.fy = O.fftfreq(ny, 1.0).astype(np.float64)
        self.masks = np.ascontiguousarray(np.asarray(masks, dtype=np.float64).reshape(-1, nx, ny))
        self.n_slices = len(thicknesses)

    @classmethod
    def from_structure(cls, probe: "O.ProbeSpec", s: "O.Structure", nx: int, ny: int, thicknesses, detectors,
                       pi_choice: str = "exact") -> "ScanInputs":
        """Every input built by the C++ restatement: the potential, the transmissions, one propagator per distinct
        thickness, the probe spectrum and the annular masks ((inner, outer) [mrad]; outer already checked against
        the grid's largest angle)."""
        g = O.Grid(nx, ny, s.box[0], s.box[1])
        vs = potential(s, nx, ny, thicknesses, pi_choice)
        self = cls.__new__(cls)
        self.g = g
        t = np.stack([transmission(v, probe.energy, g) for v in vs])
        self.t_re, self.t_im = np.ascontiguousarray(t.real), np.ascontiguousarray(t.imag)
        dzs = []
        self.prop = np.zeros(len(thicknesses), dtype=np.int32)
        for j, dz in enumerate(thicknesses):
            if dz not in dzs:
                dzs.append(dz)
            self.prop[j] = dzs.index(dz)
        pr = np.stack([propagator(g, probe.energy, dz, probe.tilt) for dz in dzs])
        self.p_re, self.p_im = np.ascontiguousarray(pr.real), np.ascontiguousarray(pr.imag)
        sp = probe_spectrum(probe, g)
        self.s_re, self.s_im = np.ascontiguousarray(sp.real), np.ascontiguousarray(sp.imag)
        self.fx = O.fftfreq(nx, 1.0).astype(np.float64)
        self.fy = O.fftfreq(ny, 1.0).astype(np.float64)
        self.masks = np.ascontiguousarray(np.stack([annular_mask(g, probe.energy, a, b) for a, b in detectors]))
        self.n_slices = len(thicknesses)
        return self

    def scan(self, positions, threads: int = 1) -> np.ndarray:
        """Detector values [position][detector] at `positions` (Angstrom)."""
        g = self.g
        pos = np.asarray(positions, dtype=np.float64).reshape(-1, 2)
        pix = np.ascontiguousarray(np.stack([pos[:, 0] / g.sampling[0], pos[:, 1] / g.sampling[1]], axis=1))
        out = np.zeros((len(pix), len(self.masks)), dtype=np.float64)
        rc = lib().simk_cpu_stem_scan(g.nx, g.ny, self.n_slices, _p(self.t_re), _p(self.t_im),
                                      self.prop.ctypes.data_as(_I), _p(self.p_re), _p(self.p_im), _p(self.s_re),
                                      _p(self.s_im), _p(self.fx), _p(self.fy), len(pix), _p(pix), len(self.masks),
                                      _p(self.masks), max(1, int(threads)), _p(out))
        if rc != 0:
            raise ValueError("simk_cpu_stem_scan: bad arguments")
        return out


def annular_masks(g: "O.Grid", energy: float, detectors) -> np.ndarray:
    """0/1 masks of annular detectors given as (inner, outer) in mrad (Detectors.swift:119-135)."""
    return np.stack([O.annular_mask(g, energy, a, b).astype(np.float64) for a, b in detectors])
