"""TEST INFRASTRUCTURE: ctypes wrapper of oracle/cpu/simk_cpu.cpp, the C++ float64 restatement of the reference's
`.cpu` STEM scan path (Multislice.runCPU, Probe.build, DiffractionIntensity and the annular detectors, positions over
threads as runCPUParallel: Sources/SimulatoCore/Multislice.swift:132-157, Sources/SimulatoProbe/Probe.swift:113-156,
Sources/SimulatoDetector/Detectors.swift:28-36, 119-135, Sources/SimulatoCore/MetalMultislice.swift:28-47).

Only the tests and the benchmark's CPU legs use it, as a checker and as the timed CPU baseline; the CUDA library never
does. The library is built by `make -C oracle/cpu` (or `build()` below) into oracle/_build/libsimk_cpu.so."""

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
