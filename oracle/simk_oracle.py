"""CPU float64 oracle for the multislice hot path -- TEST INFRASTRUCTURE ONLY.

This module is the checker, never the product: only `tests/`, `__graft_entry__.smoke()` and `bench.py`'s CPU-baseline
leg may import it. The CUDA library (`libsimulato_cuda.so`) never calls it and has no CPU fallback.

It restates SimulatoKit 0.5.0's float64 `.cpu` path (a Swift port of abTEM 1.0.10) in NumPy, function by function,
following the reference sources cited in each docstring (paths relative to the SimulatoKit project) and the
formula-level recipes of its pin generator (`tools/pins/potential-multislice/pins.py:55-213`,
`tools/pins/stem-detectors/pins.py:71-168`). Its FFT is NumPy's pocketfft in float64, the engine the reference's
fixtures were generated with.

Parity is pinned: `tests/test_oracle_pins.py` checks it against the reference's own abTEM-generated fixtures
(copied as subsets into `tests/golden/` by `tests/golden/make_golden.py`) at the reference's own bounds
(V, t 1e-11; exit waves, patterns, detectors 1e-10 with abTEM's float32 pi; 1e-6 with the exact pi).
"""

from __future__ import annotations

import json
import math
import os
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_TABLE = os.path.join(_HERE, "..", "simulatokit_b200", "data", "lobato.json")

# ---------------------------------------------------------------------------------------------------------------------
# Constants (Sources/SimulatoCore/PhysicalConstants.swift:8-31): CODATA 2014 as ASE 3.29 / abTEM 1.0.10 use them.
# ---------------------------------------------------------------------------------------------------------------------
PLANCK = 6.62607004e-34
ELECTRON_MASS = 9.10938356e-31
SPEED_OF_LIGHT = 299792458.0
ELEMENTARY_CHARGE = 1.6021766208e-19
KAPPA = 0.0208865737082965
ASE_KG = 6.0221408585491615e26
ASE_COULOMB = 6.241509125883258e18
ASE_SECOND = 98226947884640.62
ASE_JOULE = 6.241509125883258e18

PI32 = float(np.float32(np.pi))               # LobatoParameterization.swift:47
PI2_32 = float(np.float32(np.pi * np.pi))     # LobatoParameterization.swift:48


def wavelength(energy: float) -> float:
    """lambda [A] (ElectronBeam.swift:38-43): h c / sqrt(E (2 m c^2 / e + E)) / e * 1e10."""
    c2 = SPEED_OF_LIGHT * SPEED_OF_LIGHT
    return PLANCK * SPEED_OF_LIGHT / math.sqrt(energy * (2 * ELECTRON_MASS * c2 / ELEMENTARY_CHARGE + energy)) \
        / ELEMENTARY_CHARGE * 1.0e10


def interaction_parameter(energy: float) -> float:
    """sigma [1/(V A)] in abTEM's evaluation order (ElectronBeam.swift:24-30)."""
    mass = (1 + ELEMENTARY_CHARGE * energy / (ELECTRON_MASS * (SPEED_OF_LIGHT * SPEED_OF_LIGHT))) * ELECTRON_MASS
    hsj = PLANCK * ASE_SECOND * ASE_JOULE
    return 2 * math.pi * mass * ASE_KG * ELEMENTARY_CHARGE * ASE_COULOMB * wavelength(energy) / (hsj * hsj)


# ---------------------------------------------------------------------------------------------------------------------
# Grid (Sources/SimulatoCore/Grid.swift:45-86)
# ---------------------------------------------------------------------------------------------------------------------

def fftfreq(n: int, d: float) -> np.ndarray:
    """NumPy's fftfreq, bit for bit (Grid.swift:82-86)."""
    val = 1.0 / (n * d)
    pos = (n - 1) // 2 + 1
    i = np.arange(n)
    return np.where(i < pos, i, i - n).astype(np.float64) * val


@dataclass(frozen=True)
class Grid:
    nx: int
    ny: int
    extent_x: float
    extent_y: float

    @property
    def sampling(self):
        return (self.extent_x / self.nx, self.extent_y / self.ny)

    @property
    def reciprocal_sampling(self):
        """1 / (n * (extent / n)) as abTEM computes it (Grid.swift:52-53)."""
        sx, sy = self.sampling
        return (1.0 / (self.nx * sx), 1.0 / (self.ny * sy))

    def kx(self):
        return fftfreq(self.nx, self.sampling[0])

    def ky(self):
        return fftfreq(self.ny, self.sampling[1])

    def k2(self):
        kx, ky = self.kx(), self.ky()
        return kx[:, None] ** 2 + ky[None, :] ** 2


def grid_from_sampling(extent_x, extent_y, sampling_x, sampling_y) -> Grid:
    """abTEM's Grid._adjust_gpts: ceil(extent / sampling) points (Grid.swift:31-41)."""
    return Grid(int(math.ceil(extent_x / sampling_x)), int(math.ceil(extent_y / sampling_y)), extent_x, extent_y)


# ---------------------------------------------------------------------------------------------------------------------
# Antialias aperture (Sources/SimulatoCore/Antialias.swift:18-52)
# ---------------------------------------------------------------------------------------------------------------------
ANTIALIAS_CUTOFF = 0.6666666
ANTIALIAS_TAPER = 0.01


def antialias_aperture(g: Grid) -> np.ndarray:
    dmax = max(g.sampling)
    kc = ANTIALIAS_CUTOFF / dmax / 2
    w = ANTIALIAS_TAPER / dmax
    r = np.sqrt(g.kx()[:, None] ** 2 + g.ky()[None, :] ** 2)
    out = np.ones((g.nx, g.ny))
    band = (r > kc - w) & (r <= kc)
    out[band] = 0.5 * (1 + np.cos(np.pi * (r[band] - kc + w) / w))
    out[r > kc] = 0.0
    return out


def _round_decimals(x: float, d: int) -> float:
    f = 10.0 ** d
    return float(np.round(x * f)) / f


def cutoff_pattern_size(g: Grid):
    """Odd-parity crop size of Waves.diffractionPattern(.cutoff) (Antialias.swift:43-52)."""
    kcut = 2.0 / 3.0 / max(g.sampling)

    def size(n, extent):
        m = int(math.floor(_round_decimals(kcut * extent, 7)))
        if m % 2 != n % 2:
            m += 1
        if m % 2 == 0:
            m += 1
        return m
    sx, sy = g.sampling
    return size(g.nx, g.nx * sx), size(g.ny, g.ny * sy)


def cutoff_gpts_same(g: Grid):
    """Detectors.swift:54-62 (abTEM's _antialias_cutoff_gpts, the grid's parity)."""
    kcut = 2.0 / 3.0 / max(g.sampling)

    def size(n, extent):
        m = int(math.floor(_round_decimals(kcut * extent, 7)))
        if m % 2 != n % 2:
            m += 1
        return m
    sx, sy = g.sampling
    return size(g.nx, g.nx * sx), size(g.ny, g.ny * sy)


def crop_indices(n: int, m: int) -> np.ndarray:
    """Waves.swift:90-96: the first floor(m/2)+1 (m odd) or m/2 (m even) frequencies, then the last floor(m/2)."""
    if m >= n:
        return np.arange(n)
    low = m // 2 + 1 if m % 2 == 1 else m // 2
    high = m // 2
    return np.r_[np.arange(low), np.arange(n - high, n)]


def crop_shift(values: np.ndarray, mx: int, my: int) -> np.ndarray:
    """DiffractionIntensity.cropped (Detectors.swift:70-80): crop in FFT order then fftshift."""
    sx, sy = crop_indices(values.shape[0], mx), crop_indices(values.shape[1], my)
    c = values[np.ix_(sx, sy)]
    return np.roll(np.roll(c, len(sx) // 2, axis=0), len(sy) // 2, axis=1)


# ---------------------------------------------------------------------------------------------------------------------
# Lobato parameterisation (Sources/SimulatoMultislice/LobatoParameterization.swift:38-69)
# ---------------------------------------------------------------------------------------------------------------------
_LOBATO = None


def lobato_parameters(z: int):
    global _LOBATO
    if _LOBATO is None:
        data = json.load(open(_TABLE))
        _LOBATO = {e["Z"]: (np.array(e["a"]), np.array(e["b"])) for e in data["elements"]}
    if z not in _LOBATO:
        raise ValueError(f"unsupported element Z={z}")
    return _LOBATO[z]


def scaled_parameters(z: int):
    """A = pi^2 a / b^1.5 / kappa, B = 2 pi / sqrt(b) (LobatoParameterization.swift:38-44)."""
    a, b = lobato_parameters(z)
    pi2 = math.pi * math.pi
    A = np.array([pi2 * a[i] / b[i] ** 1.5 / KAPPA for i in range(5)])
    B = np.array([2 * math.pi / math.sqrt(b[i]) for i in range(5)])
    return A, B


def projected_scattering_factor(z: int, k2, pi_choice: str = "exact") -> np.ndarray:
    """f(k^2) = 8 pi sum_i [A/B/(q+B^2) + A B/(q+B^2)^2], q = 4 pi^2 k^2, term by term
    (LobatoParameterization.swift:51-69). pi_choice 'exact' or 'abtem' (float32 pi)."""
    A, B = scaled_parameters(z)
    pi, pi2 = (PI32, PI2_32) if pi_choice == "abtem" else (math.pi, math.pi * math.pi)
    q = (4 * pi2) * np.asarray(k2, dtype=np.float64)
    s = np.zeros_like(q)
    for i in range(5):
        d = q + B[i] * B[i]
        s = s + (A[i] / B[i] / d + A[i] * B[i] / (d * d))
    return (8 * pi) * s


# ---------------------------------------------------------------------------------------------------------------------
# Structures, slicing, potential (Slicing.swift, Potential.swift, ProjectedPotential.swift)
# ---------------------------------------------------------------------------------------------------------------------

@dataclass
class Structure:
    box: tuple          # (Lx, Ly, Lz) [A]
    numbers: np.ndarray  # [n] int
    positions: np.ndarray  # [n, 3] float64

    def repeated(self, nx, ny, nz):
        """AtomicStructure.repeated (AtomicStructure.swift:40-54): x outermost, then y, z, atoms innermost."""
        nums, pos = [], []
        for mx in range(nx):
            for my in range(ny):
                for mz in range(nz):
                    shift = np.array([mx * self.box[0], my * self.box[1], mz * self.box[2]])
                    nums.append(self.numbers)
                    pos.append(self.positions + shift)
        return Structure((self.box[0] * nx, self.box[1] * ny, self.box[2] * nz),
                         np.concatenate(nums) if nums else np.zeros(0, int),
                         np.concatenate(pos) if pos else np.zeros((0, 3)))


def slice_thicknesses(depth: float, requested: float):
    """ceil(Lz / s) slices of Lz / n (Slicing.swift:17-25)."""
    n = int(math.ceil(depth / requested))
    return [depth / n] * n


def wrapped(s: Structure) -> np.ndarray:
    """Fractional mod 1, top-face rule (Slicing.swift:71-84)."""
    p = np.array(s.positions, dtype=np.float64).reshape(-1, 3).copy()
    for d in range(3):
        f = np.fmod(p[:, d] / s.box[d], 1.0)
        f = np.where(f < 0, f + 1.0, f)
        f = np.where(f == 1.0, 0.0, f)
        p[:, d] = f * s.box[d]
    p[p[:, 2] > s.box[2] - 1e-10, 2] = 0.0
    return p


def slice_indices(z: np.ndarray, thicknesses) -> np.ndarray:
    """digitize against the cumulative edges - 1e-12 (Slicing.swift:88-104)."""
    edges = []
    acc = 0.0
    for t in thicknesses:
        acc += t
        edges.append(acc)
    edges = np.array(edges) - 1e-12
    idx = np.searchsorted(edges, z, side="right")
    return np.minimum(idx, len(thicknesses) - 1)


def compensation(g: Grid) -> np.ndarray:
    """S = sin(kappa)/kappa dx dy, kappa in cycles per pixel, S(0) = dx dy (ProjectedPotential.swift:130-143)."""
    dx, dy = g.sampling
    a = g.kx()[:, None] * dx
    b = g.ky()[None, :] * dy
    k = np.sqrt(a * a + b * b)
    k[0, 0] = 1.0
    s = np.sin(k) / k * (dx * dy)
    s[0, 0] = dx * dy
    return s


def superpose_deltas(xy_pix: np.ndarray, nx: int, ny: int) -> np.ndarray:
    """Bilinear weights at 4 pixels mod the grid, weight by weight, atom by atom
    (ProjectedPotential.swift:178-201)."""
    arr = np.zeros(nx * ny)
    if len(xy_pix) == 0:
        return arr.reshape(nx, ny)
    px, py = xy_pix[:, 0], xy_pix[:, 1]
    r = np.floor(px).astype(np.int64)
    c = np.floor(py).astype(np.int64)
    x = px - r
    y = py - c
    xy = x * y
    w = [1 + xy - y - x, x - xy, y - xy, xy]
    for k in range(4):
        i = np.mod(r + (1 if k in (1, 3) else 0), nx)
        j = np.mod(c + (1 if k >= 2 else 0), ny)
        np.add.at(arr, i * ny + j, w[k])
    return arr.reshape(nx, ny)


@dataclass
class Potential:
    """The lazy potential (Potential.swift:12-92): wrapped atoms with their slice index."""
    grid: Grid
    thicknesses: list
    numbers: np.ndarray
    positions: np.ndarray   # wrapped
    slice_of_atom: np.ndarray
    pi_choice: str = "exact"

    @staticmethod
    def from_structure(s: Structure, nx, ny, slice_thickness=None, thicknesses=None, pi_choice="exact"):
        g = Grid(nx, ny, s.box[0], s.box[1])
        t = thicknesses if thicknesses is not None else slice_thicknesses(s.box[2], slice_thickness)
        p = wrapped(s)
        return Potential(g, list(t), np.asarray(s.numbers, dtype=int), p, slice_indices(p[:, 2], t), pi_choice)

    def kernel(self, z: int) -> np.ndarray:
        """f(k^2) / S(k) (ProjectedPotential.swift:146-153)."""
        return projected_scattering_factor(z, self.grid.k2(), self.pi_choice) / compensation(self.grid)

    def slice_values(self, j: int) -> np.ndarray:
        """V of slice j: elements in increasing Z, Re IFFT(FFT(deltas) f / S) (ProjectedPotential.swift:156-174)."""
        g = self.grid
        v = np.zeros((g.nx, g.ny))
        sel = self.slice_of_atom == j
        nums = self.numbers[sel]
        pos = self.positions[sel]
        for z in sorted(set(int(n) for n in nums)):
            xy = pos[nums == z][:, :2] / np.array(g.sampling)
            d = superpose_deltas(xy, g.nx, g.ny).astype(np.complex128)
            f = np.fft.fft2(d) * self.kernel(z)
            v = v + np.fft.ifft2(f).real
        return v

    def build(self) -> list:
        return [self.slice_values(j) for j in range(len(self.thicknesses))]


# ---------------------------------------------------------------------------------------------------------------------
# Multislice (Sources/SimulatoMultislice/Multislice.swift:83-166)
# ---------------------------------------------------------------------------------------------------------------------

def transmission(v: np.ndarray, energy: float, g: Grid) -> np.ndarray:
    """t = IFFT(FFT(exp(i sigma V)) A) (Multislice.swift:83-103)."""
    t = np.exp(1j * (interaction_parameter(energy) * v))
    return np.fft.ifft2(np.fft.fft2(t) * antialias_aperture(g))


def propagator(g: Grid, energy: float, dz: float, tilt=(0.0, 0.0)) -> np.ndarray:
    """P = exp(-i pi lambda dz k^2) A, times the tilt phase (Multislice.swift:108-130)."""
    lam = wavelength(energy)
    kx, ky = g.kx()[:, None], g.ky()[None, :]
    k2 = kx * kx + ky * ky
    x = -k2 * math.pi * dz * lam
    p = (np.cos(x) + 1j * np.sin(x)) * antialias_aperture(g)
    if tilt[0] != 0 or tilt[1] != 0:
        t = -2 * math.pi * dz * (kx * math.tan(tilt[0] / 1e3) + ky * math.tan(tilt[1] / 1e3))
        p = p * (np.cos(t) + 1j * np.sin(t))
    return p


def exit_planes(kind, n: int):
    """ExitPlanes.planes (Multislice.swift:13-40): 'last', ('every', m) or ('after', [..])."""
    if kind == "last":
        return [n - 1]
    if kind[0] == "every":
        m = kind[1]
        if m >= n:
            return [n - 1]
        p = list(range(m - 1, n, m))
        if p[-1] != n - 1:
            p.append(n - 1)
        return [-1] + p
    lst = list(kind[1])
    return lst if lst and lst[-1] == n - 1 else lst + [n - 1]


def multislice(psi: np.ndarray, transmissions, thicknesses, energy: float, g: Grid, planes=None, tilt=(0.0, 0.0)):
    """Per slice: psi <- IFFT(FFT(psi t) P) (Multislice.swift:132-157). Returns the waves at `planes`."""
    n = len(thicknesses)
    planes = [n - 1] if planes is None else planes
    out = [psi.copy()] if planes and planes[0] == -1 else []
    wanted = set(planes)
    props = {}
    for j, dz in enumerate(thicknesses):
        if dz not in props:
            props[dz] = propagator(g, energy, dz, tilt)
        psi = np.fft.ifft2(np.fft.fft2(psi * transmissions[j]) * props[dz])
        if j in wanted:
            out.append(psi)
    return out


def plane_wave(g: Grid) -> np.ndarray:
    return np.ones((g.nx, g.ny), dtype=np.complex128)


# ---------------------------------------------------------------------------------------------------------------------
# Probe (Sources/SimulatoProbe/Probe.swift:25-156, Aberrations.swift:39-59)
# ---------------------------------------------------------------------------------------------------------------------
ABERRATION_SYMBOLS = ("C10", "C12", "phi12", "C21", "phi21", "C23", "phi23", "C30", "C32", "phi32", "C34", "phi34",
                      "C41", "phi41", "C43", "phi43", "C45", "phi45", "C50", "C52", "phi52", "C54", "phi54", "C56",
                      "phi56")


def chi(alpha, phi, ab: dict, lam: float):
    """(2 pi / lambda) sum_n alpha^(n+1)/(n+1) sum_m C_nm cos(m (phi - phi_nm)) (Aberrations.swift:39-59)."""
    g = lambda k: float(ab.get(k, 0.0))  # noqa: E731
    x = np.zeros_like(alpha)
    if g("C10") or g("C12") or g("phi12"):
        x = x + 1 / 2 * alpha ** 2 * (g("C10") + g("C12") * np.cos(2 * (phi - g("phi12"))))
    if g("C21") or g("phi21") or g("C23") or g("phi23"):
        x = x + 1 / 3 * alpha ** 3 * (g("C21") * np.cos(phi - g("phi21")) + g("C23") * np.cos(3 * (phi - g("phi23"))))
    if g("C30") or g("C32") or g("phi32") or g("C34") or g("phi34"):
        x = x + 1 / 4 * alpha ** 4 * (g("C30") + g("C32") * np.cos(2 * (phi - g("phi32")))
                                      + g("C34") * np.cos(4 * (phi - g("phi34"))))
    if g("C41") or g("phi41") or g("C43") or g("phi43") or g("C45") or g("phi45"):
        x = x + 1 / 5 * alpha ** 5 * (g("C41") * np.cos(phi - g("phi41")) + g("C43") * np.cos(3 * (phi - g("phi43")))
                                      + g("C45") * np.cos(5 * (phi - g("phi45"))))
    if g("C50") or g("C52") or g("phi52") or g("C54") or g("phi54") or g("C56") or g("phi56"):
        x = x + 1 / 6 * alpha ** 6 * (g("C50") + g("C52") * np.cos(2 * (phi - g("phi52")))
                                      + g("C54") * np.cos(4 * (phi - g("phi54"))) + g("C56") * np.cos(6 * (phi - g("phi56"))))
    return x * (2 * math.pi / lam)


def aperture_values(g: Grid, lam: float, semiangle_mrad: float, soft: bool = True) -> np.ndarray:
    """abTEM's soft aperture with a one-pixel edge (Probe.swift:25-48)."""
    if math.isinf(semiangle_mrad):
        return np.ones((g.nx, g.ny))
    kx, ky = g.kx()[:, None], g.ky()[None, :]
    cutoff = semiangle_mrad * 1e-3
    rs = g.reciprocal_sampling
    dax = rs[0] * 1e3 * lam * 1e-3
    day = rs[1] * 1e3 * lam * 1e-3
    alpha = np.sqrt(kx * kx + ky * ky) * lam
    if not soft:
        return (alpha <= cutoff).astype(np.float64)
    phi = np.arctan2(ky + 0 * kx, kx + 0 * ky)
    a = np.cos(phi) * dax
    b = np.sin(phi) * day
    d = np.sqrt(a * a + b * b)
    d[0, 0] = 1.0
    out = np.clip((cutoff - alpha) / d + 0.5, 0.0, 1.0)
    out[0, 0] = 1.0
    return out


def _ab(ab: dict, k: str) -> float:
    return float(ab.get(k, 0.0))


def dchi_dalpha(alpha, phi, ab: dict, lam: float):
    """Aberrations.dChiDAlpha (ContrastTransferFunction.swift:12-21): abTEM's d chi / d alpha."""
    g = lambda k: _ab(ab, k)  # noqa: E731
    p, a = phi, alpha
    t1 = (g("C12") * np.cos(2 * (p - g("phi12"))) + g("C10")) * a
    t2 = (g("C23") * np.cos(3 * (p - g("phi23"))) + g("C21") * np.cos(1 * (p - g("phi21")))) * a ** 2
    t3 = (g("C34") * np.cos(4 * (p - g("phi34"))) + g("C32") * np.cos(2 * (p - g("phi32"))) + g("C30")) * a ** 3
    t4 = (g("C45") * np.cos(5 * (p - g("phi45"))) + g("C43") * np.cos(3 * (p - g("phi43")))
          + g("C41") * np.cos(1 * (p - g("phi41")))) * a ** 4
    t5 = (g("C56") * np.cos(6 * (p - g("phi56"))) + g("C54") * np.cos(4 * (p - g("phi54")))
          + g("C52") * np.cos(2 * (p - g("phi52"))) + g("C50")) * a ** 5
    return 2 * math.pi / lam * (t1 + t2 + t3 + t4 + t5)


def dchi_dphi(alpha, phi, ab: dict, lam: float):
    """Aberrations.dChiDPhi (ContrastTransferFunction.swift:24-34): abTEM's azimuthal term."""
    g = lambda k: _ab(ab, k)  # noqa: E731
    p, a = phi, alpha
    t1 = 1 / 2.0 * (2.0 * g("C12") * np.sin(2.0 * (p - g("phi12")))) * a
    t2 = 1 / 3.0 * (3.0 * g("C23") * np.sin(3.0 * (p - g("phi23"))) + 1.0 * g("C21") * np.sin(1.0 * (p - g("phi21")))) * a ** 2
    t3 = 1 / 4.0 * (4.0 * g("C34") * np.sin(4.0 * (p - g("phi34"))) + 2.0 * g("C32") * np.sin(2.0 * (p - g("phi32")))) * a ** 3
    t4 = 1 / 5.0 * (5.0 * g("C45") * np.sin(5.0 * (p - g("phi45"))) + 3.0 * g("C43") * np.sin(3.0 * (p - g("phi43")))
                    + 1.0 * g("C41") * np.sin(1.0 * (p - g("phi41")))) * a ** 4
    t5 = (1 / 6.0) * (6.0 * g("C56") * np.sin(6.0 * (p - g("phi56"))) + 4.0 * g("C54") * np.sin(4.0 * (p - g("phi54")))
                      + 2.0 * g("C52") * np.sin(2.0 * (p - g("phi52")))) * a ** 5
    return -2 * math.pi / lam * (t1 + t2 + t3 + t4 + t5)


def temporal_envelope(alpha, lam: float, focal_spread: float):
    """exp(-((pi/2 / lambda) Delta alpha^2)^2) (ContrastTransferFunction.swift:68-72)."""
    x = 0.5 * math.pi / lam * focal_spread * alpha * alpha
    return np.exp(-(x * x))


def spatial_envelope(alpha, phi, lam: float, ab: dict, angular_spread: float):
    """exp(-sign(beta) (beta/2)^2 ((d chi/d alpha)^2 + (d chi/d phi)^2)), beta in mrad (:75-82)."""
    b = angular_spread / 1e3
    dk = dchi_dalpha(alpha, phi, ab, lam)
    dp = dchi_dphi(alpha, phi, ab, lam)
    sign = 1.0 if b > 0 else (-1.0 if b < 0 else 0.0)
    return np.exp(-sign * (b / 2) * (b / 2) * (dk * dk + dp * dp))


def ctf_kernel(g: "Grid", energy: float, ab: dict, cutoff_mrad: float = math.inf, soft: bool = True,
               focal_spread: float = 0.0, angular_spread: float = 0.0) -> np.ndarray:
    """ContrastTransferFunction.kernel (:85-115): exp(-i chi) x E_s (beta != 0) x E_t (Delta != 0) x aperture (finite
    cutoff), FFT order."""
    lam = wavelength(energy)
    kx, ky = g.kx()[:, None], g.ky()[None, :]
    alpha = np.sqrt(kx * kx + ky * ky) * lam
    phi = np.arctan2(ky + 0 * kx, kx + 0 * ky)
    h = np.exp(-1j * chi(alpha, phi, ab, lam))
    if angular_spread != 0:
        h = h * spatial_envelope(alpha, phi, lam, ab, angular_spread)
    if focal_spread != 0:
        h = h * temporal_envelope(alpha, lam, focal_spread)
    if math.isfinite(cutoff_mrad):
        h = h * aperture_values(g, lam, cutoff_mrad, soft)
    return h


def apply_ctf(psi: np.ndarray, kernel: np.ndarray) -> np.ndarray:
    """Waves.applying (ContrastTransferFunction.swift:146-161): IFFT(FFT(psi) H)."""
    return np.fft.ifft2(np.fft.fft2(psi) * kernel)


def scherzer_defocus(cs: float, energy: float, factor: float = 1.5) -> float:
    """sign(Cs) sqrt(factor |Cs| lambda) (:118-124)."""
    s = 1.0 if cs > 0 else (-1.0 if cs < 0 else 0.0)
    return s * math.sqrt(factor * abs(cs) * wavelength(energy))


def point_resolution(cs: float, energy: float, divisor: float = 6.0) -> float:
    """(lambda^3 |Cs| / divisor)^(1/4) (:127-131)."""
    return math.pow(math.pow(wavelength(energy), 3) * abs(cs) / divisor, 1.0 / 4)


def nyquist_sampling(semiangle: float, energy: float, oversampling: float = 4.0) -> float:
    """1 / (oversampling alpha_c / lambda 1e-3) (:134-142)."""
    return 1 / (oversampling * semiangle / wavelength(energy) * 1e-3)


@dataclass
class ProbeSpec:
    energy: float
    semiangle: float
    aberrations: dict = field(default_factory=dict)
    soft: bool = True
    tilt: tuple = (0.0, 0.0)


def centred_spectrum(p: ProbeSpec, g: Grid) -> np.ndarray:
    """Psi0 = aperture exp(-i chi) / ||.|| (Probe.swift:113-136)."""
    lam = wavelength(p.energy)
    kx, ky = g.kx()[:, None], g.ky()[None, :]
    alpha = np.sqrt(kx * kx + ky * ky) * lam
    phi = np.arctan2(ky + 0 * kx, kx + 0 * ky)
    c = chi(alpha, phi, p.aberrations, lam)
    s = aperture_values(g, lam, p.semiangle, p.soft) * (np.cos(-c) + 1j * np.sin(-c))
    return s / math.sqrt(float((np.abs(s) ** 2).sum()))


def shift_ramps(g: Grid, position):
    """r_x[ix] = exp(-2 pi i p_x[ix] u_x), likewise r_y (Probe.swift:140-156)."""
    ux, uy = position[0] / g.sampling[0], position[1] / g.sampling[1]
    sx = -2 * math.pi * fftfreq(g.nx, 1.0) * ux
    sy = -2 * math.pi * fftfreq(g.ny, 1.0) * uy
    return np.cos(sx) + 1j * np.sin(sx), np.cos(sy) + 1j * np.sin(sy)


def build_probe(p: ProbeSpec, g: Grid, position) -> np.ndarray:
    """Probe.build(at:) (Probe.swift:72-109): shift * aperture * exp(-i chi), normalised, then IFFT."""
    lam = wavelength(p.energy)
    kx, ky = g.kx()[:, None], g.ky()[None, :]
    ap = aperture_values(g, lam, p.semiangle, p.soft)
    rx, ry = shift_ramps(g, position)
    shift = rx[:, None] * ry[None, :]
    alpha = np.sqrt(kx * kx + ky * ky) * lam
    phi = np.arctan2(ky + 0 * kx, kx + 0 * ky)
    c = chi(alpha, phi, p.aberrations, lam)
    psi = shift * ap * (np.cos(-c) + 1j * np.sin(-c))
    psi = psi / math.sqrt(float((np.abs(psi) ** 2).sum()))
    return np.fft.ifft2(psi)


def grid_scan_positions(start, end, nx, ny, endpoint=False) -> np.ndarray:
    """GridScan.positions (GridScan.swift:52-66): x-major, NumPy linspace."""
    def linspace(a, b, n):
        div = n - 1 if endpoint else n
        if div <= 0:
            return np.array([a])
        step = (b - a) / div
        out = np.arange(n) * step + a
        if endpoint and n > 1:
            out[-1] = b
        return out
    xs, ys = linspace(start[0], end[0], nx), linspace(start[1], end[1], ny)
    return np.array([(x, y) for x in xs for y in ys])


# ---------------------------------------------------------------------------------------------------------------------
# Patterns and detectors (Sources/SimulatoCore/Waves.swift:62-96, Sources/SimulatoDetector/Detectors.swift)
# ---------------------------------------------------------------------------------------------------------------------

def diffraction_pattern(psi: np.ndarray, g: Grid, plane_wave_norm: bool) -> np.ndarray:
    """Waves.diffractionPattern(.cutoff) (Waves.swift:62-86)."""
    a = psi / float(g.nx * g.ny) if plane_wave_norm else psi
    f = np.abs(np.fft.fft2(a)) ** 2
    mx, my = cutoff_pattern_size(g)
    return crop_shift(f, mx, my)


def diffraction_intensity(psi: np.ndarray, plane_wave_norm: bool = False) -> np.ndarray:
    """DiffractionIntensity(waves) (Detectors.swift:28-36): |FFT2(psi)|^2, psi / N first for a plane wave."""
    n = psi.shape[0] * psi.shape[1]
    a = psi / float(n) if plane_wave_norm else psi
    return np.abs(np.fft.fft2(a)) ** 2


def angular_sampling(g: Grid, energy: float):
    """Detectors.swift:39-41: reciprocal sampling * lambda * 1e3 [mrad/px]."""
    lam = wavelength(energy)
    rs = g.reciprocal_sampling
    return rs[0] * lam * 1e3, rs[1] * lam * 1e3


def angles(m: int, d: float) -> np.ndarray:
    """fftfreq(m, 1 / d / m) (Detectors.swift:44)."""
    return fftfreq(m, 1.0 / d / m)


def cutoff_angles(g: Grid, energy: float):
    c = cutoff_gpts_same(g)
    a = angular_sampling(g, energy)
    return (c[0] // 2) * a[0], (c[1] // 2) * a[1]


def annular_outer(g: Grid, energy: float, outer):
    """AnnularDetector.outerAngle (Detectors.swift:108-117)."""
    if outer is None:
        c = cutoff_angles(g, energy)
        return math.floor(min(c))
    a = angular_sampling(g, energy)
    maximum = min((g.nx // 2) * a[0], (g.ny // 2) * a[1])
    if outer > maximum and abs(outer - maximum) > 1e-5 + 1e-5 * abs(outer):
        raise ValueError(f"outer {outer} mrad exceeds the maximum simulated angle {maximum} mrad")
    return outer


def annular_mask(g: Grid, energy: float, inner: float, outer) -> np.ndarray:
    o = annular_outer(g, energy, outer)
    a = angular_sampling(g, energy)
    ax, ay = angles(g.nx, a[0])[:, None], angles(g.ny, a[1])[None, :]
    a2 = ax * ax + ay * ay
    return (a2 >= inner * inner) & (a2 < o * o)


def annular_detect(p: np.ndarray, g: Grid, energy: float, inner: float, outer) -> float:
    """Sum of P over inner^2 <= alpha^2 < outer^2 (Detectors.swift:119-135)."""
    return float(p[annular_mask(g, energy, inner, outer)].sum())


def pixelated_size(g: Grid, mode: str):
    """PixelatedDetector.size (Detectors.swift:146-160)."""
    if mode == "full":
        return g.nx, g.ny
    c = cutoff_gpts_same(g)
    if mode == "cutoff":
        return c

    def v(m, n):
        k = int(math.floor(_round_decimals(m / math.sqrt(2.0), 7)))
        if k % 2 != n % 2:
            k += 1
        return k
    return v(c[0], g.nx), v(c[1], g.ny)


def pixelated_detect(p: np.ndarray, g: Grid, mode: str) -> np.ndarray:
    mx, my = pixelated_size(g, mode)
    return crop_shift(p, mx, my)


def com_detect(p: np.ndarray, g: Grid, energy: float, mode: str = "valid", units: str = "inverse") -> np.ndarray:
    """CenterOfMassDetector.detect (Detectors.swift:190-206): sum P alpha over the pixelated region, not / sum P."""
    mx, my = pixelated_size(g, mode)
    pat = crop_shift(p, mx, my)
    a = angular_sampling(g, energy)
    per = 1.0 if units == "mrad" else 1.0 / (wavelength(energy) * 1e3)
    ax = (np.arange(mx) - mx // 2) * a[0] * per
    ay = (np.arange(my) - my // 2) * a[1] * per
    return np.array([float((pat * ax[:, None]).sum()), float((pat * ay[None, :]).sum())])


def segmented_bins(g: Grid, energy: float, nr: int, nphi: int, inner: float, outer: float, rotation: float):
    """The bin of every pixel of the full grid (-1: none) for SegmentedDetector (Detectors.swift:232-263)."""
    a = angular_sampling(g, energy)

    def m(n, d):
        k = int(2 * math.ceil(outer / d)) + 1
        if k % 2 != n % 2:
            k += 1
        return min(k, n)
    mx, my = m(g.nx, a[0]), m(g.ny, a[1])
    sx, sy = crop_indices(g.nx, mx), crop_indices(g.ny, my)
    ax, ay = angles(mx, a[0]), angles(my, a[1])
    bins = -np.ones((g.nx, g.ny), dtype=np.int64)
    two_pi = 2 * math.pi
    for cx in range(mx):
        for cy in range(my):
            alpha = math.sqrt(ax[cx] * ax[cx] + ay[cy] * ay[cy])
            if not (alpha >= inner and alpha < outer):
                continue
            phi = math.fmod(math.atan2(ay[cy], ax[cx]) - rotation, two_pi)
            if phi < 0:
                phi += two_pi
            r = int(math.floor(nr * (alpha - inner) / (outer - inner)))
            if r >= nr:
                continue
            f = math.floor(nphi * (phi / two_pi))
            az = int(min(max(f, 0), nphi - 1))
            bins[sx[cx], sy[cy]] = az + r * nphi
    return bins


def segmented_detect(p: np.ndarray, g: Grid, energy: float, nr, nphi, inner, outer, rotation) -> np.ndarray:
    bins = segmented_bins(g, energy, nr, nphi, inner, outer, rotation)
    out = np.zeros(nr * nphi)
    sel = bins >= 0
    np.add.at(out, bins[sel], p[sel])
    return out


def binned_weights(n: int, samp: float, nb: int, outer: float) -> np.ndarray:
    """[nb, n] overlap weights along one axis: bin k covers [-outer + k w, -outer + (k+1) w), w = 2 outer / nb; pixel i
    covers [alpha_i - samp/2, alpha_i + samp/2) with alpha = angles(n, samp); weight = overlap / samp. No reference
    counterpart: the reference's PixelatedDetector has no numeric-angle mode (Detectors.swift:140-168), so this rule
    (area-weighted rebinning, intensity inside the window conserved) is this project's own and unpinned."""
    al = angles(n, samp)
    w = 2.0 * outer / nb
    lo = -outer + np.arange(nb) * w
    ov = np.minimum(lo[:, None] + w, al[None, :] + 0.5 * samp) - np.maximum(lo[:, None], al[None, :] - 0.5 * samp)
    return np.where(ov > 0, ov / samp, 0.0)


def binned_detect(p: np.ndarray, g: Grid, energy: float, nbx: int, nby: int, outer: float) -> np.ndarray:
    """The pattern on a uniform nbx x nby grid over [-outer, outer) mrad per axis (bin 0 at -outer), by area-weighted
    rebinning of the k-space pixels (binned_weights)."""
    a = angular_sampling(g, energy)
    wx = binned_weights(g.nx, a[0], nbx, outer)
    wy = binned_weights(g.ny, a[1], nby, outer)
    return wx @ p @ wy.T


@dataclass
class DetectorSpec:
    """kind: 'annular' (inner, outer|None), 'pixelated' (mode), 'com' (mode, units), 'segmented' (nr, nphi, inner,
    outer, rotation), 'binned' (nbx, nby, outer)."""
    kind: str
    params: dict

    def detect(self, p, g, energy):
        k, q = self.kind, self.params
        if k == "annular":
            return np.array([annular_detect(p, g, energy, q.get("inner", 0.0), q.get("outer"))])
        if k == "pixelated":
            return pixelated_detect(p, g, q.get("mode", "valid")).ravel()
        if k == "com":
            return com_detect(p, g, energy, q.get("mode", "valid"), q.get("units", "inverse"))
        if k == "segmented":
            return segmented_detect(p, g, energy, q["nr"], q["nphi"], q["inner"], q["outer"], q.get("rotation", 0.0))
        if k == "binned":
            return binned_detect(p, g, energy, q["nbx"], q["nby"], q["outer"]).ravel()
        raise ValueError(k)


def stem_scan(probe: ProbeSpec, potentials, positions, detectors, thicknesses_list=None):
    """STEM.cpuScan (STEM.swift:95-150): every configuration, every position, each detector on |FFT2(exit)|^2,
    summed then divided by the number of configurations. `potentials` are lists of V slices with their Grid and
    thicknesses: [(grid, [V...], [dz...])]."""
    sums = None
    for (g, vs, dzs) in potentials:
        ts = [transmission(v, probe.energy, g) for v in vs]
        for q, pos in enumerate(positions):
            psi0 = build_probe(probe, g, pos)
            ex = multislice(psi0, ts, dzs, probe.energy, g, tilt=probe.tilt)[-1]
            p = diffraction_intensity(ex, False)
            vals = [d.detect(p, g, probe.energy) for d in detectors]
            if sums is None:
                sums = [np.zeros((len(positions), len(v))) for v in vals]
            for d, v in enumerate(vals):
                sums[d][q] += v
    return [s / len(potentials) for s in sums]


# ---------------------------------------------------------------------------------------------------------------------
# Waves detector (Sources/SimulatoDetector/WavesDetector.swift:35-216, Sources/SimulatoCore/WavesResample.swift:16-55)
# ---------------------------------------------------------------------------------------------------------------------

def resample_map(n: int, m: int):
    """Waves.resampleMap (WavesResample.swift:46-54): (source, destination) of every frequency kept going from n to m
    points: the lowest m (crop, crop_indices order) or all n (zero-pad, positive frequencies first)."""
    if m <= n:
        if m == 1:
            return [(0, 0)]
        return [(int(src), dst) for dst, src in enumerate(crop_indices(n, m))]
    if n == 1:
        return [(0, 0)]
    positive = n // 2 if n % 2 == 0 else n // 2 + 1
    return [(i, i if i < positive else m - n + i) for i in range(n)]


def resample_wave(psi: np.ndarray, rows: int, columns: int) -> np.ndarray:
    """Waves.resampled (WavesResample.swift:16-43): FFT, keep the mapped frequencies on the rows x columns grid, inverse
    FFT, times rows columns / (nx ny) so that the values keep their amplitude."""
    nx, ny = psi.shape
    f = np.fft.fft2(psi)
    out = np.zeros((rows, columns), dtype=np.complex128)
    mx, my = resample_map(nx, rows), resample_map(ny, columns)
    sx, dx = [a for a, _ in mx], [b for _, b in mx]
    sy, dy = [a for a, _ in my], [b for _, b in my]
    out[np.ix_(dx, dy)] = f[np.ix_(sx, sy)]
    return np.fft.ifft2(out) * (rows * columns / (nx * ny))


def waves_scan(probe: "ProbeSpec", g: Grid, vs, thicknesses, positions, gpts=None) -> np.ndarray:
    """STEM.scan with a WavesDetector (WavesDetector.swift:115-126, collect :191-216): the exit wave at every position
    through one potential, resampled to gpts = (rows, columns) when given; [position][row][column]."""
    ts = [transmission(v, probe.energy, g) for v in vs]
    out = []
    for pos in positions:
        ex = multislice(build_probe(probe, g, pos), ts, thicknesses, probe.energy, g, tilt=probe.tilt)[-1]
        out.append(ex if gpts is None else resample_wave(ex, gpts[0], gpts[1]))
    return np.array(out)


# ---------------------------------------------------------------------------------------------------------------------
# Frozen phonons (Sources/SimulatoMultislice/FrozenPhonons.swift:14-156)
# ---------------------------------------------------------------------------------------------------------------------
_M64 = (1 << 64) - 1


def _splitmix_finalise(z: int) -> int:
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M64
    return z ^ (z >> 31)


class GaussianGenerator:
    """SplitMix64 -> xoshiro256** -> Box-Muller, both outputs used (FrozenPhonons.swift:14-58)."""

    def __init__(self, seed: int):
        x = seed & _M64
        s = []
        for _ in range(4):
            x = (x + 0x9E3779B97F4A7C15) & _M64
            s.append(_splitmix_finalise(x))
        self.s = s
        self.spare = None

    def next_u64(self) -> int:
        s = self.s

        def rotl(v, k):
            return ((v << k) | (v >> (64 - k))) & _M64
        result = (rotl((s[1] * 5) & _M64, 7) * 9) & _M64
        t = (s[1] << 17) & _M64
        s[2] ^= s[0]
        s[3] ^= s[1]
        s[1] ^= s[2]
        s[0] ^= s[3]
        s[2] ^= t
        s[3] = rotl(s[3], 45)
        return result

    def next_normal(self) -> float:
        if self.spare is not None:
            z, self.spare = self.spare, None
            return z
        u1 = ((self.next_u64() >> 11) + 1) * 2.0 ** -53
        u2 = (self.next_u64() >> 11) * 2.0 ** -53
        r = math.sqrt(-2 * math.log(u1))
        theta = 2 * math.pi * u2
        self.spare = r * math.sin(theta)
        return r * math.cos(theta)


def configuration_seed(seed: int, c: int) -> int:
    """mix(mix(seed) + c) (FrozenPhonons.swift:122-130)."""
    def mix(v):
        return _splitmix_finalise((v + 0x9E3779B97F4A7C15) & _M64)
    return mix((mix(seed) + c) & _M64)


def frozen_displacements(numbers, sigmas: dict, configurations: int, seed: int, directions="xyz"):
    """FrozenPhonons.init(sigmas:configurations:seed:) (FrozenPhonons.swift:99-117)."""
    out = []
    for c in range(configurations):
        g = GaussianGenerator(configuration_seed(seed, c))
        d = np.zeros((len(numbers), 3))
        for a, z in enumerate(numbers):
            r = (g.next_normal(), g.next_normal(), g.next_normal())
            s = sigmas.get(int(z), 0.0)
            for ax, name in enumerate("xyz"):
                d[a, ax] = s * r[ax] if name in directions else 0.0
        out.append(d)
    return out


# ---------------------------------------------------------------------------------------------------------------------
# Comparisons (Tests/SimulatoKitTestSupport/Comparison.swift:8-30) and the rel-L2 gate
# ---------------------------------------------------------------------------------------------------------------------

def rel_max(a, b) -> float:
    a, b = np.asarray(a), np.asarray(b)
    m = float(np.max(np.abs(b))) if b.size else 0.0
    d = float(np.max(np.abs(a - b))) if b.size else 0.0
    return d / m if m > 0 else d


def rel_l2(a, b) -> float:
    a, b = np.asarray(a, dtype=np.complex128), np.asarray(b, dtype=np.complex128)
    nb = float(np.linalg.norm(b.ravel()))
    d = float(np.linalg.norm((a - b).ravel()))
    return d / nb if nb > 0 else d


# ---------------------------------------------------------------------------------------------------------------------
# Structures of the workloads
# ---------------------------------------------------------------------------------------------------------------------

def srtio3_cell(a0: float = 3.905) -> Structure:
    """Sr at 0, Ti at the body centre, O at the face centres (the pins' `srtio3`, pins.py:266-270)."""
    frac = np.array([(0, 0, 0), (0.5, 0.5, 0.5), (0.5, 0.5, 0), (0.5, 0, 0.5), (0, 0.5, 0.5)], dtype=np.float64)
    return Structure((a0, a0, a0), np.array([38, 22, 8, 8, 8]), frac * a0)


def al_fcc_cell(a0: float = 4.05) -> Structure:
    frac = np.array([(0, 0, 0), (0, 0.5, 0.5), (0.5, 0, 0.5), (0.5, 0.5, 0)], dtype=np.float64)
    return Structure((a0, a0, a0), np.array([13, 13, 13, 13]), frac * a0)


def silicon_cell(a0: float = 5.431) -> Structure:
    """Diamond-cubic Si: fcc + (1/4, 1/4, 1/4) basis."""
    fcc = np.array([(0, 0, 0), (0, 0.5, 0.5), (0.5, 0, 0.5), (0.5, 0.5, 0)], dtype=np.float64)
    frac = np.concatenate([fcc, fcc + 0.25])
    return Structure((a0, a0, a0), np.full(8, 14), frac * a0)


# ---------------------------------------------------------------------------------------------------------------------
# Finite projection (no reference implementation: SimulatoKit lists `Potential(projection="finite")` as not ported,
# docs/parity.md:58,251). Parity is anchored on identities: the thick-slab limit equals the infinite projection
# (pins.py:423-446's analytic form), slices add, and the radial profile integrates to the k = 0 value.
# ---------------------------------------------------------------------------------------------------------------------

def lobato_potential_3d(z: int, r):
    """V(r) = sum_i A_i (2 / (B_i r) + 1) exp(-B_i r), the real-space Lobato potential whose projection is the
    infinite projection of LobatoParameterization.swift:51-69 (its 2-D transform is f(k^2))."""
    A, B = scaled_parameters(z)
    r = np.asarray(r, dtype=np.float64)
    return sum(A[i] * (2.0 / (B[i] * r) + 1.0) * np.exp(-B[i] * r) for i in range(5))


def infinite_profile(z: int, rho):
    """Analytic infinite projection 2 sum_i [2 A_i / B_i K0(B_i rho) + A_i rho K1(B_i rho)] (pins.py:432)."""
    from scipy.special import kn
    A, B = scaled_parameters(z)
    rho = np.asarray(rho, dtype=np.float64)
    return 2 * sum(2 * A[i] / B[i] * kn(0, rho * B[i]) + A[i] * rho * kn(1, rho * B[i]) for i in range(5))


def finite_profile(z: int, rho: float, zl: float, zu: float, n: int = 48) -> float:
    """int_{zl}^{zu} V(sqrt(rho^2 + z^2)) dz with z = rho sinh(u): the integrand sum_i A_i (2/B_i + rho cosh u)
    exp(-B_i rho cosh u) is smooth in u; n-point Gauss-Legendre on each side of u = 0."""
    if zu <= zl:
        return 0.0
    A, B = scaled_parameters(z)
    x, w = np.polynomial.legendre.leggauss(n)
    ul, uu = math.asinh(zl / rho), math.asinh(zu / rho)
    parts = [(ul, 0.0), (0.0, uu)] if ul < 0.0 < uu else [(ul, uu)]
    total = 0.0
    for a, b in parts:
        u = 0.5 * (b - a) * x + 0.5 * (b + a)
        c = np.cosh(u)
        f = sum(A[i] * (2.0 / B[i] + rho * c) * np.exp(-B[i] * rho * c) for i in range(5))
        total += 0.5 * (b - a) * float(np.dot(w, f))
    return total


def finite_profile_quad(z: int, rho: float, zl: float, zu: float) -> float:
    """The same integral by adaptive quadrature in z (the independent judge)."""
    from scipy import integrate
    f = lambda t: float(lobato_potential_3d(z, math.sqrt(rho * rho + t * t)))  # noqa: E731
    pts = [0.0] if zl < 0.0 < zu else None
    return integrate.quad(f, zl, zu, epsabs=0.0, epsrel=1e-13, limit=400, points=pts)[0]


def finite_cutoff(z: int, tol: float = 1e-3) -> float:
    """The radius where V(r) falls to `tol` [V], bounded to [1, 6] A (the truncation of an atom's potential)."""
    lo, hi = 0.05, 6.0
    if lobato_potential_3d(z, hi) > tol:
        return hi
    for _ in range(100):
        mid = 0.5 * (lo + hi)
        if lobato_potential_3d(z, mid) > tol:
            lo = mid
        else:
            hi = mid
    return max(1.0, hi)


def finite_potential_slices(numbers, positions, box, nx, ny, thicknesses, n_gl: int = 48):
    """Real-space finite-projection potential of every slice: for each atom and slice, the integral of V over the
    part of the slice within z_a +- R_c, at every pixel within R_c of the atom (periodic in x, y; not in z), with
    rho clamped below to min(dx, dy) / 2. Small cases only (pure Python loops)."""
    dx, dy = box[0] / nx, box[1] / ny
    rmin = 0.5 * min(dx, dy)
    edges = np.concatenate([[0.0], np.cumsum(thicknesses)])
    out = np.zeros((len(thicknesses), nx, ny))
    xs = np.arange(nx) * dx
    ys = np.arange(ny) * dy
    for zn, (px, py, pz) in zip(numbers, positions):
        rc = finite_cutoff(int(zn))
        ddx = (xs - px + box[0] / 2) % box[0] - box[0] / 2
        ddy = (ys - py + box[1] / 2) % box[1] - box[1] / 2
        rho = np.sqrt(ddx[:, None] ** 2 + ddy[None, :] ** 2)
        mask = rho <= rc
        for j in range(len(thicknesses)):
            zl = max(edges[j] - pz, -rc)
            zu = min(edges[j + 1] - pz, rc)
            if zu <= zl:
                continue
            vals = np.zeros_like(rho)
            for idx in zip(*np.nonzero(mask)):
                vals[idx] = finite_profile(int(zn), max(rho[idx], rmin), zl, zu, n_gl)
            out[j] += vals
    return out


# ---------------------------------------------------------------------------------------------------------------------
# The surrogate network's float64 restatement (checks the device's forward and backward passes)
# ---------------------------------------------------------------------------------------------------------------------

def surrogate_features(rho, z):
    """((log rho + 1.5) / 2, asinh(z / rho) / 4): the radius and one slab edge in the u variable of finite_profile,
    scaled to order one."""
    rho = np.asarray(rho, dtype=np.float64)
    return np.stack([(np.log(rho) + 1.5) / 2.0, np.arcsinh(np.asarray(z) / rho) / 4.0], axis=-1)


def _silu(x):
    return x / (1.0 + np.exp(-x))


def _silu_grad(x):
    s = 1.0 / (1.0 + np.exp(-x))
    return s * (1.0 + x * (1.0 - s))


def surrogate_C(params: dict, elem_index, feats):
    """The cumulative profile network: [emb(Z) (16), 2 features] -> 64 -> 64 -> 64 -> 1, SiLU."""
    x0 = np.concatenate([params["emb"][elem_index], feats], axis=1)
    a1 = x0 @ params["W1"].T + params["b1"]
    h1 = _silu(a1)
    a2 = h1 @ params["W2"].T + params["b2"]
    h2 = _silu(a2)
    a3 = h2 @ params["W3"].T + params["b3"]
    h3 = _silu(a3)
    y = h3 @ params["W4"].T + params["b4"]
    return y[:, 0], (x0, a1, h1, a2, h2, a3, h3)


def _surrogate_backward(params, elem_index, cache, dy):
    x0, a1, h1, a2, h2, a3, h3 = cache
    dy = dy[:, None]
    g = {"W4": dy.T @ h3, "b4": dy.sum(0)}
    d3 = (dy @ params["W4"]) * _silu_grad(a3)
    g["W3"], g["b3"] = d3.T @ h2, d3.sum(0)
    d2 = (d3 @ params["W3"]) * _silu_grad(a2)
    g["W2"], g["b2"] = d2.T @ h1, d2.sum(0)
    d1 = (d2 @ params["W2"]) * _silu_grad(a1)
    g["W1"], g["b1"] = d1.T @ x0, d1.sum(0)
    dx0 = d1 @ params["W1"]
    emb = np.zeros_like(params["emb"])
    np.add.at(emb, elem_index, dx0[:, :params["emb"].shape[1]])
    g["emb"] = emb
    return g


def surrogate_gradients(params: dict, elem_index, rho, zl, zu, fraction):
    """F_hat = C(rho, zu) - C(rho, zl); mean-squared error against `fraction`; gradients of every parameter."""
    cu, cache_u = surrogate_C(params, elem_index, surrogate_features(rho, zu))
    cl, cache_l = surrogate_C(params, elem_index, surrogate_features(rho, zl))
    e = (cu - cl) - np.asarray(fraction)
    n = len(e)
    gu = _surrogate_backward(params, elem_index, cache_u, (2.0 / n) * e)
    gl = _surrogate_backward(params, elem_index, cache_l, -(2.0 / n) * e)
    return float(np.mean(e ** 2)), {k: gu[k] + gl[k] for k in gu}


def surrogate_unpack(flat) -> dict:
    """The device's parameter layout: emb[103][16] | W1[64][18] b1 | W2[64][64] b2 | W3[64][64] b3 | W4[64] b4."""
    f = np.asarray(flat, dtype=np.float64)
    o = 0
    out = {}
    for name, shape in (("emb", (103, 16)), ("W1", (64, 18)), ("b1", (64,)), ("W2", (64, 64)), ("b2", (64,)),
                        ("W3", (64, 64)), ("b3", (64,)), ("W4", (1, 64)), ("b4", (1,))):
        n = int(np.prod(shape))
        out[name] = f[o:o + n].reshape(shape)
        o += n
    assert o == f.size
    return out


def surrogate_pack(d: dict) -> np.ndarray:
    return np.concatenate([np.asarray(d[k], dtype=np.float64).ravel()
                           for k in ("emb", "W1", "b1", "W2", "b2", "W3", "b3", "W4", "b4")])



# ---------------------------------------------------------------------------------------------------------------------
# Scan post-processing (Sources/SimulatoDetector/ScanOperations.swift:12-167, IntegratedCenterOfMass.swift:11-41,
# Sources/SimulatoCore/ImageOperations.swift:39-48, 140-176)
# ---------------------------------------------------------------------------------------------------------------------

def gaussian_kernel(sigma_px: float) -> np.ndarray:
    """scipy's gaussian_filter1d weights (ScanOperations.swift:43-50): exp(-x^2 / 2 s^2) for |x| <= floor(4 s + 1/2),
    divided by their sum taken in order."""
    radius = int(4.0 * sigma_px + 0.5)
    w = [math.exp(-0.5 * float(x * x) / (sigma_px * sigma_px)) for x in range(-radius, radius + 1)]
    total = 0.0
    for v in w:
        total += v
    return np.array([v / total for v in w])


def _filter_axis(data: np.ndarray, axis: int, sigma_px: float) -> np.ndarray:
    """One periodic pass (ScanOperations.swift:52-72): out[k] = sum_j w[j] in[(k + j - r) mod L], summed in j order."""
    if not sigma_px > 0:
        return data
    w = gaussian_kernel(sigma_px)
    r = len(w) // 2
    L = data.shape[axis]
    src = np.moveaxis(data, axis, 0)
    out = np.zeros_like(src)
    for k in range(L):
        acc = np.zeros(src.shape[1:])
        for j, wj in enumerate(w):
            acc = acc + wj * src[(k + j - r) % L]
        out[k] = acc
    return np.moveaxis(out, 0, axis)


def gaussian_source_size(values: np.ndarray, scan_shape, sigma_x: float, sigma_y: float, sampling_x: float,
                         sampling_y: float) -> np.ndarray:
    """ScanMeasurement.gaussianSourceSize (ScanOperations.swift:19-36): the values [nx][ny][...] filtered along the
    second scan axis with sigma_y / sampling_y pixels, then the first with sigma_x / sampling_x, both periodic."""
    for v in (sigma_x, sigma_y):
        if not (math.isfinite(v) and v >= 0):
            raise ValueError("the source size must be finite and non-negative")
    for v in (sampling_x, sampling_y):
        if not (math.isfinite(v) and v > 0):
            raise ValueError("the scan sampling must be finite and positive")
    if len(scan_shape) != 2:
        raise ValueError("the source size filters a two-axis scan")
    nx, ny = scan_shape
    d = np.asarray(values, dtype=np.float64).reshape(nx, ny, -1)
    d = _filter_axis(d, 1, sigma_y / sampling_y)
    d = _filter_axis(d, 0, sigma_x / sampling_x)
    return d.reshape(np.shape(values))


def integrate_gradient(gx: np.ndarray, gy: np.ndarray, sampling_x: float, sampling_y: float) -> np.ndarray:
    """integrateGradient (ImageOperations.swift:140-167), abTEM's _integrate_gradient_2d: T^ = (kx g^x + ky g^y) /
    (2 pi i |k|^2), |k|^2 = 1e-12 at zero frequency, the real part of the inverse transform less its minimum."""
    for v in (sampling_x, sampling_y):
        if not (math.isfinite(v) and v > 0):
            raise ValueError("invalid sampling")
    gx, gy = np.asarray(gx, dtype=np.float64), np.asarray(gy, dtype=np.float64)
    nx, ny = gx.shape
    fx, fy = np.fft.fft2(gx.astype(np.complex128)), np.fft.fft2(gy.astype(np.complex128))
    kx, ky = fftfreq(nx, sampling_x)[:, None], fftfreq(ny, sampling_y)[None, :]
    k = kx * kx + ky * ky
    k = np.where(k == 0, 1e-12, k)
    a = fx.real * kx + fy.real * ky
    b = fx.imag * kx + fy.imag * ky
    c = 2 * math.pi * k
    t = np.fft.ifft2(b / c - 1j * (a / c)).real
    return t - t.min()


def integrated_center_of_mass(values: np.ndarray, scan_shape, sampling_x: float, sampling_y: float) -> np.ndarray:
    """ScanMeasurement.integratedCenterOfMass (IntegratedCenterOfMass.swift:36-40): the (x, y) pairs of a
    centre-of-mass measurement as two images over the scan, integrated."""
    if len(scan_shape) != 2:
        raise ValueError("a centre-of-mass image needs a two-axis scan")
    v = np.asarray(values, dtype=np.float64).reshape(scan_shape[0], scan_shape[1], 2)
    return integrate_gradient(v[..., 0], v[..., 1], sampling_x, sampling_y)


def _uniform(rng: GaussianGenerator) -> float:
    """PoissonSampler.uniform (ScanOperations.swift:133-135): the top 53 bits over 2^53."""
    return (rng.next_u64() >> 11) * (1.0 / 9007199254740992.0)


def poisson_draw(lam: float, rng: GaussianGenerator) -> int:
    """PoissonSampler.draw (ScanOperations.swift:137-166): Knuth's product below a mean of 10, Hoermann's PTRS
    (transformed rejection with squeeze) above."""
    if lam <= 0:
        return 0
    if lam < 10:
        limit = math.exp(-lam)
        product, k = _uniform(rng), 0
        while product > limit:
            product *= _uniform(rng)
            k += 1
        return k
    slam, loglam = math.sqrt(lam), math.log(lam)
    b = 0.931 + 2.53 * slam
    a = -0.059 + 0.02483 * b
    invalpha = 1.1239 + 1.1328 / (b - 3.4)
    vr = 0.9277 - 3.6224 / (b - 2)
    while True:
        u = _uniform(rng) - 0.5
        v = _uniform(rng)
        us = 0.5 - abs(u)
        if us <= 0:
            continue
        kd = math.floor((2 * a / us + b) * u + lam + 0.43)
        if not (math.isfinite(kd) and abs(kd) < 9e18):
            continue
        k = int(kd)
        if us >= 0.07 and v <= vr:
            return k
        if k < 0 or (us < 0.013 and v > us):
            continue
        if math.log(v) + math.log(invalpha) - math.log(a / (us * us) + b) <= -lam + k * loglam - math.lgamma(k + 1.0):
            return k


def poisson_noise_sequential(values, dose: float, seed: int, samples: int = 1) -> np.ndarray:
    """ScanMeasurement.poissonNoise (ScanOperations.swift:80-117): max(value dose, 0) drawn in order from ONE generator
    stream over every value and sample -- the reference's own bits. Shape (samples, values). Finite values only."""
    if not (math.isfinite(dose) and dose >= 0):
        raise ValueError("the dose must be finite and non-negative")
    rng = GaussianGenerator(seed)
    means = [max(float(v) * dose, 0.0) for v in np.asarray(values, dtype=np.float64).ravel()]
    return np.array([[float(poisson_draw(m, rng)) for m in means] for _ in range(samples)])


def poisson_value_seed(seed: int, index: int) -> int:
    """The seed of value `index` (sample s of value i: index s * count + i) in the device's per-value streams: the
    same mix as a frozen-phonon configuration's seed, mix(mix(seed) + index)."""
    return configuration_seed(seed, index)


def poisson_noise_streams(values, dose: float, seed: int, samples: int = 1) -> np.ndarray:
    """The device's Poisson noise: max(value dose, 0) drawn by PoissonSampler.draw from a generator of its own per value
    and sample, seeded by poisson_value_seed. The same seed gives the same noise on every run and any split of the
    work; the draws are not the reference's sequential stream. Shape (samples, values). Finite values only."""
    if not (math.isfinite(dose) and dose >= 0):
        raise ValueError("the dose must be finite and non-negative")
    v = np.asarray(values, dtype=np.float64).ravel()
    n = v.size
    out = np.zeros((samples, n))
    for s in range(samples):
        for i in range(n):
            m = max(float(v[i]) * dose, 0.0)
            out[s, i] = float(poisson_draw(m, GaussianGenerator(poisson_value_seed(seed, s * n + i)))) if m > 0 else 0.0
    return out


# ---------------------------------------------------------------------------------------------------------------------
# Potential tiling, projection and crystal slicing (Sources/SimulatoMultislice/ProjectedPotential.swift:64-105,
# Slicing.swift:43-69)
# ---------------------------------------------------------------------------------------------------------------------

def project_slices(values: np.ndarray) -> np.ndarray:
    """ProjectedPotential.project: the slices [S][nx][ny] summed in order from 0."""
    v = np.asarray(values, dtype=np.float64)
    out = np.zeros(v.shape[1:])
    for s in range(v.shape[0]):
        out = out + v[s]
    return out


def tile_slices(values: np.ndarray, rx: int, ry: int, rz: int = 1) -> np.ndarray:
    """ProjectedPotential.tiled: every slice tiled rx x ry in the plane, then the stack repeated rz times."""
    v = np.asarray(values, dtype=np.float64)
    return np.tile(v, (rz, rx, ry))


def crystal_slice_thicknesses(z, depth: float, tolerance: float = 0.2):
    """Slicing.crystalSliceThicknesses: the z of every atom with 0 and the depth, binned by floor(z / tolerance); the
    differences between the occupied bins' centres (b + 1/2) tolerance. Raises ValueError where the reference throws."""
    if not (math.isfinite(tolerance) and tolerance > 0):
        raise ValueError("invalid tolerance")
    bins = set()
    for v in list(np.asarray(z, dtype=np.float64)) + [0.0, depth]:
        q = float(v) / tolerance
        if not (math.isfinite(q) and abs(math.floor(q)) <= 2.0 ** 53):
            raise ValueError("invalid tolerance")
        bins.add(math.floor(q))
    centres = [(b + 0.5) * tolerance for b in sorted(bins)]
    t = [c1 - c0 for c0, c1 in zip(centres, centres[1:])]
    total = 0.0
    for x in t:
        total += x
    if not t or abs(total - depth) > 1e-8 + 1e-5 * abs(depth):
        raise ValueError("the thicknesses do not sum to the depth")
    return t
