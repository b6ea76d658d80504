"""Potentials and the multislice entry points of the CUDA backend (Sources/SimulatoMultislice/).

`Multislice.run` / `Multislice.runBatch` keep the reference's signatures (Multislice.swift:52-80,
MetalMultislice.swift:52-83); the only backend is `Backend.cuda`, which calls libsimulato_cuda and has no CPU fallback."""

from __future__ import annotations

import ctypes as C
import math
from enum import Enum

import numpy as np

from . import _lib as L
from .core import AtomicStructure, ElectronBeam, Grid, Waves, _refuse
from .engine import Engine, ExecutionOptions, PotentialHandle


class Backend(Enum):
    """The compute backend (Multislice.swift:43-46 gains `.cuda`)."""
    cuda = "cuda"


class LobatoParameterization:
    """Lobato & Van Dyck (2014), pi exact or abTEM's float32 pi (LobatoParameterization.swift:11-24)."""
    EXACT = "exact"
    ABTEM_FLOAT32 = "abTEMFloat32"

    def __init__(self, pi_constant: str = "exact"):
        if pi_constant not in (self.EXACT, self.ABTEM_FLOAT32):
            _refuse(f"unknown pi constant {pi_constant!r}")
        self.pi_constant = pi_constant

    @staticmethod
    def supports(z: int) -> bool:
        return 1 <= int(z) <= 103

    @property
    def code(self) -> int:
        return L.PI_ABTEM_FLOAT32 if self.pi_constant == self.ABTEM_FLOAT32 else L.PI_EXACT


class Slicing:
    """Slices along z (Sources/SimulatoMultislice/Slicing.swift)."""
    maximum_slice_count = 1_000_000

    @staticmethod
    def thicknesses(depth: float, requested: float, maximum_count: int = 1_000_000):
        if not (math.isfinite(requested) and requested > 0):
            _refuse(f"invalid slice thickness {requested}")
        n = math.ceil(depth / requested)
        if not (1 <= n <= min(maximum_count, 1 << 53)):
            _refuse(f"invalid slice thickness {requested}")
        return [depth / n] * int(n)

    @staticmethod
    def validated(lst, depth: float, maximum_count: int = 1_000_000):
        lst = [float(s) for s in lst]
        if not lst or len(lst) > maximum_count:
            _refuse("invalid slice thickness list")
        for s in lst:
            if not (math.isfinite(s) and s > 0):
                _refuse(f"invalid slice thickness {s}")
        total = sum(lst)
        if abs(total - depth) > 1e-8 + 1e-5 * abs(depth):
            _refuse(f"slice thicknesses sum to {total}, not the depth {depth}")
        return lst

    @staticmethod
    def crystalSliceThicknesses(structure: AtomicStructure, tolerance: float = 0.2):
        """Slice thicknesses that follow the crystal planes (Slicing.swift:43-69, abTEM crystal_slice_thicknesses):
        the z of every atom (as given) with 0 and the depth added, binned by floor(z / tolerance); the thicknesses are
        the differences between the occupied bins' centres (b + 1/2) tolerance, in increasing z. Refused: a tolerance
        that is not finite and positive (or z / tolerance past 2^53), and thicknesses that do not sum to the depth."""
        if not (math.isfinite(tolerance) and tolerance > 0):
            _refuse(f"invalid slice thickness {tolerance}")
        depth = float(structure.box[2])
        bins = set()
        for z in list(np.asarray(structure.positions, dtype=np.float64)[:, 2]) + [0.0, depth]:
            b = math.floor(float(z) / tolerance) if math.isfinite(float(z) / tolerance) else math.inf
            if not (math.isfinite(b) and abs(b) <= 2.0 ** 53):
                _refuse(f"invalid slice thickness {tolerance}")
            bins.add(int(b))
        centres = [(b + 0.5) * tolerance for b in sorted(bins)]
        thicknesses = [c1 - c0 for c0, c1 in zip(centres, centres[1:])]
        total = 0.0
        for t in thicknesses:
            total += t
        if not thicknesses or abs(total - depth) > 1e-8 + 1e-5 * abs(depth):
            _refuse(f"slice thicknesses sum to {total}, not the depth {depth}")
        return thicknesses

    @staticmethod
    def wrapped(s: AtomicStructure) -> np.ndarray:
        """Fractional mod 1 (ASE's wrap(eps=0)), z -> 0 within 1e-10 of the top face (Slicing.swift:71-84)."""
        p = s.positions.copy()
        for d in range(3):
            f = np.fmod(p[:, d] / s.box[d], 1.0)
            f = np.where(f < 0, f + 1.0, f)
            f = np.where(f == 1.0, 0.0, f)
            p[:, d] = f * s.box[d]
        p[p[:, 2] > s.box[2] - 1e-10, 2] = 0.0
        return p

    @staticmethod
    def slice_indices(z: np.ndarray, thicknesses) -> np.ndarray:
        """e_{j-1} <= z < e_j, e_j = sum_{i<=j} s_i - 1e-12; past the last edge: the last slice (Slicing.swift:88-104)."""
        edges = np.cumsum(np.array(thicknesses, dtype=np.float64))
        acc = 0.0
        for i, t in enumerate(thicknesses):  # the running sum in order, as the reference adds them
            acc += t
            edges[i] = acc
        edges = edges - 1e-12
        return np.minimum(np.searchsorted(edges, z, side="right"), len(thicknesses) - 1).astype(np.int32)


class Surrogate:
    """The learned finite-projection profile: an MLP trained on the device on samples the float64 quadrature labels
    (no counterpart in SimulatoKit, whose finite projection is not ported, docs/parity.md:58,251)."""

    def __init__(self, elements, n_samples: int = 1_000_000, steps: int = 6000, batch: int = 4096,
                 learning_rate: float = 2e-3, seed: int = 1, max_thickness: float = 4.0, rho_min: float = 0.01,
                 engine: Engine | None = None):
        self.engine = engine or Engine.require()
        z = np.ascontiguousarray(sorted(set(int(e) for e in elements)), dtype=np.int32)
        out = C.c_void_p()
        L.check(self.engine.lib.simk_surrogate_train(self.engine.handle, len(z), L.iptr(z), int(n_samples),
                                                     int(steps), int(batch), float(learning_rate), int(seed),
                                                     float(max_thickness), float(rho_min), C.byref(out)))
        self.handle = out
        self.elements = [int(v) for v in z]
        lib = self.engine.lib
        self._finalizer = __import__("weakref").finalize(self, lambda: lib.simk_surrogate_destroy(out))

    @property
    def info(self) -> dict:
        v = np.zeros(8)
        L.check(self.engine.lib.simk_surrogate_info(self.handle, L.dptr(v)))
        keys = ["train_loss", "val_max_rel", "val_rms_rel", "y_mean", "y_std", "steps", "samples", "max_thickness"]
        return dict(zip(keys, v.tolist()))

    def evaluate(self, z, rho, zl, zu) -> np.ndarray:
        z = np.ascontiguousarray(np.broadcast_to(z, np.shape(rho)), dtype=np.int32).ravel()
        r, l, u = (np.ascontiguousarray(np.broadcast_to(a, np.shape(rho)), dtype=np.float64).ravel()
                   for a in (rho, zl, zu))
        out = np.empty(len(r))
        L.check(self.engine.lib.simk_surrogate_evaluate(self.engine.handle, self.handle, len(r), L.iptr(z), L.dptr(r),
                                                        L.dptr(l), L.dptr(u), L.dptr(out)))
        return out

    def parameters(self, set_to: np.ndarray | None = None, mean_std=None):
        """The float32 parameters (and the target's mean and spread); with set_to, replace them."""
        ms = np.zeros(2)
        if set_to is not None:
            arr = np.ascontiguousarray(set_to, dtype=np.float32)
            ms = np.ascontiguousarray(mean_std, dtype=np.float64) if mean_std is not None else None
            L.check(self.engine.lib.simk_surrogate_parameters(
                self.engine.handle, self.handle, None, arr.ctypes.data_as(C.POINTER(C.c_float)),
                L.dptr(ms) if ms is not None else None))
            return None
        out = np.empty(L.SURROGATE_PARAMS, dtype=np.float32)
        L.check(self.engine.lib.simk_surrogate_parameters(self.engine.handle, self.handle,
                                                          out.ctypes.data_as(C.POINTER(C.c_float)), None, L.dptr(ms)))
        return out, (float(ms[0]), float(ms[1]))

    def gradients(self, z, rho, zl, zu, target):
        z = np.ascontiguousarray(z, dtype=np.int32)
        r, l, u, t = (np.ascontiguousarray(a, dtype=np.float64) for a in (rho, zl, zu, target))
        g = np.empty(L.SURROGATE_PARAMS, dtype=np.float32)
        loss = C.c_double(0)
        L.check(self.engine.lib.simk_surrogate_gradients(self.engine.handle, self.handle, len(z), L.iptr(z), L.dptr(r),
                                                         L.dptr(l), L.dptr(u), L.dptr(t),
                                                         g.ctypes.data_as(C.POINTER(C.c_float)), C.byref(loss)))
        return float(loss.value), g


def finite_profile(z, rho, zl, zu, engine: Engine | None = None) -> np.ndarray:
    """P(rho; zl, zu) = int_zl^zu V(sqrt(rho^2 + z^2)) dz by the device's float64 quadrature."""
    e = engine or Engine.require()
    z = np.ascontiguousarray(np.broadcast_to(z, np.shape(rho)), dtype=np.int32).ravel()
    r, l, u = (np.ascontiguousarray(np.broadcast_to(a, np.shape(rho)), dtype=np.float64).ravel() for a in (rho, zl, zu))
    out = np.empty(len(r))
    L.check(e.lib.simk_finite_profile(e.handle, len(r), L.iptr(z), L.dptr(r), L.dptr(l), L.dptr(u), L.dptr(out)))
    return out


class Potential:
    """A structure sliced on a grid, built on the device when first used (Potential.swift:12-92).

    projection: "infinite" (the reference's Lobato projection, the default) or "finite" (real-space integration of
    each atom over the slices it reaches; with `surrogate`, the learned profile where trained, judged against the
    quadrature with `error_bound`)."""

    def __init__(self, structure: AtomicStructure, nx: int = None, ny: int = None, slice_thickness: float = None,
                 slice_thicknesses=None, parameterization: LobatoParameterization | None = None, sampling=None,
                 maximum_slice_count: int = 1_000_000, projection: str = "infinite",
                 surrogate: Surrogate | None = None, error_bound: float = 1e-2):
        if sampling is not None:
            sx, sy = (sampling, sampling) if np.isscalar(sampling) else sampling
            g = Grid.from_sampling(structure.box[0], structure.box[1], sx, sy)
            nx, ny = g.nx, g.ny
        self.grid = Grid(int(nx), int(ny), structure.box[0], structure.box[1])
        if slice_thicknesses is None:
            t = Slicing.thicknesses(structure.box[2], slice_thickness, maximum_slice_count)
        else:
            t = slice_thicknesses
        self.slice_thicknesses = Slicing.validated(t, structure.box[2], maximum_slice_count)
        self.parameterization = parameterization or LobatoParameterization()
        for z in structure.numbers:
            if not LobatoParameterization.supports(z):
                _refuse(f"unsupported element Z = {int(z)}")
        self.numbers = structure.numbers.astype(np.int32)
        self.positions = Slicing.wrapped(structure)
        self.slice_of_atom = Slicing.slice_indices(self.positions[:, 2], self.slice_thicknesses)
        if projection not in ("infinite", "finite"):
            _refuse(f"unknown projection {projection!r}")
        self.projection = projection
        self.surrogate = surrogate
        self.error_bound = float(error_bound)
        self.used_surrogate = None
        self.judged_max_rel = None
        self._handles = {}

    @property
    def slice_count(self) -> int:
        return len(self.slice_thicknesses)

    @property
    def thickness(self) -> float:
        return float(sum(self.slice_thicknesses))

    def handle(self, engine: Engine) -> PotentialHandle:
        h = self._handles.get(id(engine))
        if h is None:
            out = C.c_void_p()
            dz = np.ascontiguousarray(self.slice_thicknesses, dtype=np.float64)
            xyz = np.ascontiguousarray(self.positions, dtype=np.float64)
            z = np.ascontiguousarray(self.numbers, dtype=np.int32)
            s = np.ascontiguousarray(self.slice_of_atom, dtype=np.int32)
            g = self.grid.c()
            if self.projection == "finite":
                used, judged = C.c_int32(0), C.c_double(0)
                L.check(engine.lib.simk_potential_from_atoms_finite(
                    engine.handle, C.byref(g), len(dz), L.dptr(dz), len(z), L.iptr(z), L.dptr(xyz),
                    self.surrogate.handle if self.surrogate else None, self.error_bound, C.byref(used),
                    C.byref(judged), C.byref(out)))
                self.used_surrogate, self.judged_max_rel = bool(used.value), float(judged.value)
            else:
                L.check(engine.lib.simk_potential_from_atoms(engine.handle, C.byref(g), len(dz), L.dptr(dz),
                                                             self.parameterization.code, len(z), L.iptr(z),
                                                             L.dptr(xyz), L.iptr(s), C.byref(out)))
            h = PotentialHandle(engine, out)
            self._handles[id(engine)] = h
        return h

    def build(self, engine: Engine | None = None) -> "ProjectedPotential":
        """V of every slice as the device builds it (float64), as a ProjectedPotential."""
        e = engine or Engine.require()
        v = self.handle(e).read_slices(self.slice_count, self.grid.nx, self.grid.ny)
        return ProjectedPotential(self.grid, v, self.slice_thicknesses)

    def project(self, engine: Engine | None = None):
        """Potential.project: the sum of the slices as an image (equal to build().project())."""
        return _project(self, engine)

    def tiled(self, repetitionsX: int, repetitionsY: int, repetitionsZ: int = 1) -> "TiledPotential":
        """The built potential tiled on the device (ProjectedPotential.tiled, ProjectedPotential.swift:76-105)."""
        return TiledPotential(self, repetitionsX, repetitionsY, repetitionsZ)


def _project(p, engine):
    """The sum of a potential's slices in slice order, on the device (ProjectedPotential.swift:64-73), as a RealField."""
    from .detector import RealField
    e = engine or Engine.require()
    out = np.empty(p.grid.nx * p.grid.ny)
    L.check(e.lib.simk_potential_project(e.handle, p.handle(e).handle, L.dptr(out)))
    return RealField(p.grid.nx, p.grid.ny, out, p.grid.extent_x / p.grid.nx, p.grid.extent_y / p.grid.ny)


def _check_repetitions(slices: int, nx: int, ny: int, rx, ry, rz):
    """ProjectedPotential.tiled's refusals (ProjectedPotential.swift:82-92), all before any allocation: a count below
    1 on any axis, more than 1,000,000 slices, a tiled slice of more than 2^28 values, more than 2^31 values in all."""
    for r in (rx, ry, rz):
        if isinstance(r, bool) or not isinstance(r, (int, np.integer)):
            _refuse(f"repetitions must be integers, got ({rx}, {ry}, {rz})")
    rx, ry, rz = int(rx), int(ry), int(rz)
    per_slice = nx * rx * ny * ry
    if (min(rx, ry, rz) < 1 or slices * rz > Slicing.maximum_slice_count or per_slice > 1 << 28
            or per_slice * slices * rz > 1 << 31):
        _refuse(f"repetitions must be at least 1 along both axes and give at most 2^28 values, got ({rx}, {ry})")
    return rx, ry, rz


class TiledPotential:
    """A potential's slices tiled repetitionsX x repetitionsY times in the plane and the stack repeated repetitionsZ
    times (ProjectedPotential.tiled, ProjectedPotential.swift:76-105; abTEM PotentialArray.tile): extent multiplied,
    sampling kept. Built on the device from the source's device potential (simk_potential_tile) on first use, so a
    periodic crystal costs one cell's build and a copy. Usable wherever a potential is."""

    def __init__(self, source, repetitionsX: int, repetitionsY: int, repetitionsZ: int = 1):
        g = source.grid
        self.repetitions = _check_repetitions(source.slice_count, g.nx, g.ny, repetitionsX, repetitionsY,
                                              repetitionsZ)
        rx, ry, rz = self.repetitions
        self.source = source
        self.grid = Grid(g.nx * rx, g.ny * ry, g.extent_x * rx, g.extent_y * ry)
        self.slice_thicknesses = list(source.slice_thicknesses) * rz
        self.slice_of_atom = []
        self._handles = {}

    @property
    def slice_count(self) -> int:
        return len(self.slice_thicknesses)

    @property
    def thickness(self) -> float:
        return float(sum(self.slice_thicknesses))

    def handle(self, engine: Engine) -> PotentialHandle:
        h = self._handles.get(id(engine))
        if h is None:
            out = C.c_void_p()
            rx, ry, rz = self.repetitions
            L.check(engine.lib.simk_potential_tile(engine.handle, self.source.handle(engine).handle, rx, ry, rz,
                                                   C.byref(out)))
            h = PotentialHandle(engine, out)
            self._handles[id(engine)] = h
        return h

    def build(self, engine: Engine | None = None) -> "ProjectedPotential":
        e = engine or Engine.require()
        v = self.handle(e).read_slices(self.slice_count, self.grid.nx, self.grid.ny)
        return ProjectedPotential(self.grid, v, self.slice_thicknesses)

    def project(self, engine: Engine | None = None):
        return _project(self, engine)

    def tiled(self, repetitionsX: int, repetitionsY: int, repetitionsZ: int = 1) -> "TiledPotential":
        return TiledPotential(self, repetitionsX, repetitionsY, repetitionsZ)


class ProjectedPotential:
    """Slices of V [V A] on a grid (ProjectedPotential.swift:24-106)."""

    def __init__(self, grid: Grid, values: np.ndarray, thicknesses):
        values = np.ascontiguousarray(values, dtype=np.float64)
        if values.shape != (len(thicknesses), grid.nx, grid.ny):
            _refuse("every slice must match the grid")
        self.grid = grid
        self.values = values
        self.slice_thicknesses = [float(t) for t in thicknesses]
        self._handles = {}

    @property
    def slice_count(self) -> int:
        return len(self.slice_thicknesses)

    def handle(self, engine: Engine) -> PotentialHandle:
        h = self._handles.get(id(engine))
        if h is None:
            out = C.c_void_p()
            dz = np.ascontiguousarray(self.slice_thicknesses, dtype=np.float64)
            g = self.grid.c()
            L.check(engine.lib.simk_potential_from_values(engine.handle, C.byref(g), len(dz), L.dptr(dz),
                                                          L.dptr(self.values), C.byref(out)))
            h = PotentialHandle(engine, out)
            self._handles[id(engine)] = h
        return h

    @property
    def thickness(self) -> float:
        return float(sum(self.slice_thicknesses))

    def project(self, engine: Engine | None = None):
        """ProjectedPotential.project (ProjectedPotential.swift:64-73): the slices summed in order, on the device; a
        potential without slices projects to zeros."""
        if self.slice_count == 0:
            from .detector import RealField
            g = self.grid
            return RealField(g.nx, g.ny, np.zeros(g.nx * g.ny), g.extent_x / g.nx, g.extent_y / g.ny)
        return _project(self, engine)

    def tiled(self, repetitionsX: int, repetitionsY: int, repetitionsZ: int = 1):
        """ProjectedPotential.tiled (ProjectedPotential.swift:76-105) on the device. A potential without slices tiles
        to one without slices on the tiled grid (after the same refusals)."""
        if self.slice_count == 0:
            rx, ry, rz = _check_repetitions(0, self.grid.nx, self.grid.ny, repetitionsX, repetitionsY, repetitionsZ)
            g = self.grid
            return ProjectedPotential(Grid(g.nx * rx, g.ny * ry, g.extent_x * rx, g.extent_y * ry),
                                      np.zeros((0, g.nx * rx, g.ny * ry)), [])
        return TiledPotential(self, repetitionsX, repetitionsY, repetitionsZ)


class ExitPlanes:
    """Which slices' exit waves to return (Multislice.swift:13-40)."""

    def __init__(self, kind: str = "last", value=None):
        self.kind, self.value = kind, value

    @staticmethod
    def last():
        return ExitPlanes("last")

    @staticmethod
    def every(m: int):
        return ExitPlanes("every", m)

    @staticmethod
    def after_slices(lst):
        return ExitPlanes("after", list(lst))

    def planes(self, n: int):
        if self.kind == "last":
            return [n - 1]
        if self.kind == "every":
            m = self.value
            if m < 1:
                _refuse(f"every({m}): the step must be at least 1")
            if m >= n:
                return [n - 1]
            p = list(range(m - 1, n, m))
            if p[-1] != n - 1:
                p.append(n - 1)
            return [-1] + p
        lst = self.value
        if lst != sorted(lst) or len(set(lst)) != len(lst) or not all(-1 <= v < n for v in lst):
            _refuse(f"afterSlices must be ascending, distinct, within -1 ..< {n}")
        return lst if lst and lst[-1] == n - 1 else lst + [n - 1]


def _split(field: np.ndarray):
    a = np.asarray(field, dtype=np.complex128)
    return np.ascontiguousarray(a.real), np.ascontiguousarray(a.imag)


class Multislice:
    """Multislice.run / runBatch / transmissionFunctions on the CUDA backend."""

    @staticmethod
    def run(incident: Waves, through, exit_planes: ExitPlanes | None = None, backend: Backend = Backend.cuda,
            options: ExecutionOptions | None = None, engine: Engine | None = None):
        """The waves at the requested exit planes, in plane order (Multislice.swift:52-80)."""
        if not incident.grid.matches(through.grid):
            _refuse("grid mismatch")
        e = engine or Engine.require()
        e.apply(options)
        planes = (exit_planes or ExitPlanes.last()).planes(through.slice_count)
        out = [incident] if planes and planes[0] == -1 else []
        dev_planes = np.ascontiguousarray([p for p in planes if p >= 0], dtype=np.int32)
        nx, ny = incident.grid.nx, incident.grid.ny
        re, im = _split(incident.field)
        ore = np.empty((len(dev_planes), nx, ny))
        oim = np.empty_like(ore)
        h = through.handle(e)
        L.check(e.lib.simk_run(e.handle, h.handle, incident.beam.energy, float(incident.tilt[0]),
                               float(incident.tilt[1]), L.dptr(re), L.dptr(im), len(dev_planes), L.iptr(dev_planes),
                               L.dptr(ore), L.dptr(oim)))
        for q in range(len(dev_planes)):
            out.append(Waves(ore[q] + 1j * oim[q], incident.grid, incident.beam, incident.normalization,
                             incident.tilt))
        return out

    @staticmethod
    def runBatch(incidents, through, backend: Backend = Backend.cuda, options: ExecutionOptions | None = None,
                 engine: Engine | None = None):
        """The exit waves of a batch through one potential (MetalMultislice.swift:52-83); the waves must share their
        beam and tilt (MetalMultislice.swift:86-92)."""
        if not incidents:
            return []
        first = incidents[0]
        for w in incidents:
            if not w.grid.matches(through.grid):
                _refuse("grid mismatch")
            if tuple(w.tilt) != tuple(first.tilt):
                _refuse("the waves of one batch must share one tilt; run each tilt separately")
            if w.beam != first.beam:
                _refuse("the waves of one batch must share one beam")
        e = engine or Engine.require()
        e.apply(options)
        stack = np.stack([w.field for w in incidents])
        re, im = _split(stack)
        ore, oim = np.empty_like(re), np.empty_like(im)
        h = through.handle(e)
        L.check(e.lib.simk_run_batch(e.handle, h.handle, first.beam.energy, float(first.tilt[0]), float(first.tilt[1]),
                                     len(incidents), L.dptr(re), L.dptr(im), L.dptr(ore), L.dptr(oim)))
        return [Waves(ore[k] + 1j * oim[k], w.grid, w.beam, w.normalization, w.tilt) for k, w in enumerate(incidents)]

    run_batch = runBatch

    @staticmethod
    def transmissionFunctions(potential, beam: ElectronBeam, engine: Engine | None = None):
        """The bandlimited t of each slice as stored on the device (Multislice.swift:83-103)."""
        e = engine or Engine.require()
        h = potential.handle(e)
        return [h.read_transmission(beam.energy, j, potential.grid.nx, potential.grid.ny)
                for j in range(potential.slice_count)]


# ---- frozen phonons (Sources/SimulatoMultislice/FrozenPhonons.swift) -------------------------------------------------
_M64 = (1 << 64) - 1


def _finalise(z: int) -> int:
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M64
    return z ^ (z >> 31)


class GaussianGenerator:
    """SplitMix64 seeds xoshiro256**; Box-Muller, both outputs used (FrozenPhonons.swift:14-58)."""

    def __init__(self, seed: int):
        x = int(seed) & _M64
        self._s = []
        for _ in range(4):
            x = (x + 0x9E3779B97F4A7C15) & _M64
            self._s.append(_finalise(x))
        self._spare = None

    def next_uint64(self) -> int:
        s = self._s
        rotl = lambda v, k: ((v << k) | (v >> (64 - k))) & _M64  # noqa: E731
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
        if self._spare is not None:
            z, self._spare = self._spare, None
            return z
        u1 = ((self.next_uint64() >> 11) + 1) * 2.0 ** -53
        u2 = (self.next_uint64() >> 11) * 2.0 ** -53
        r = math.sqrt(-2 * math.log(u1))
        theta = 2 * math.pi * u2
        self._spare = r * math.sin(theta)
        return r * math.cos(theta)


class JobTable:
    """Independent multislice jobs, each its own potential, energy and incident wave (a plane wave or a probe at a
    position), run as one table: jobs of one grid shape advance together, one row and one column launch per slice
    step (simk_job_table_run). `run` returns each job's exit-wave intensity |psi|^2 (nx x ny) and its completion time
    on the device [ms from the start of the call]. With ExecutionOptions(form="plain") the jobs run one after another
    through the plain path: the sequential baseline."""

    def __init__(self):
        self.jobs = []

    def add_plane_wave(self, potential: "Potential", energy: float):
        self.jobs.append((potential, float(energy), None, None))
        return self

    def add_probe(self, potential: "Potential", probe, position):
        self.jobs.append((potential, float(probe.beam.energy), probe, (float(position[0]), float(position[1]))))
        return self

    def run(self, options: ExecutionOptions | None = None, engine: Engine | None = None):
        e = engine or Engine.require()
        e.apply(options)
        n = len(self.jobs)
        outs = [np.zeros((p.grid.nx, p.grid.ny)) for p, _, _, _ in self.jobs]
        arr = (L.Job_t * max(n, 1))()
        for i, (p, energy, probe, pos) in enumerate(self.jobs):
            h = p.handle(e).handle
            arr[i].potential = h.value if isinstance(h, C.c_void_p) else h
            arr[i].energy = energy
            if probe is not None:
                arr[i].incident = L.JOB_PROBE
                arr[i].probe = probe.c()
                arr[i].x, arr[i].y = pos
            else:
                arr[i].incident = L.JOB_PLANE_WAVE
            arr[i].intensity = L.dptr(outs[i])
        done = np.zeros(max(n, 1))
        L.check(e.lib.simk_job_table_run(e.handle, n, arr, L.dptr(done)))
        return outs, done[:n]


class FrozenPhonons:
    """A frozen-phonon ensemble of one structure (FrozenPhonons.swift:61-156)."""

    def __init__(self, structure: AtomicStructure, displacements=None, sigmas: dict | None = None,
                 configurations: int = 1, seed: int = 0, directions: str = "xyz"):
        self.structure = structure
        if displacements is None:
            if configurations < 1:
                _refuse("configurations must be at least 1")
            sig = {int(k): float(v) for k, v in (sigmas or {}).items()}
            for z in set(int(z) for z in structure.numbers):
                if z not in sig:
                    _refuse(f"sigma must be given for every element; Z = {z} has none")
            for z, s in sig.items():
                if not (math.isfinite(s) and s >= 0):
                    _refuse(f"sigma of Z = {z} must be finite and non-negative")
            displacements = []
            for c in range(configurations):
                g = GaussianGenerator(self.configuration_seed(seed, c))
                d = np.zeros((len(structure.numbers), 3))
                for a, z in enumerate(structure.numbers):
                    r = (g.next_normal(), g.next_normal(), g.next_normal())
                    s = sig.get(int(z), 0.0)
                    for ax, name in enumerate("xyz"):
                        d[a, ax] = s * r[ax] if name in directions else 0.0
                displacements.append(d)
        if not displacements:
            _refuse("no configuration")
        for c, d in enumerate(displacements):
            d = np.asarray(d, dtype=np.float64)
            if d.shape != (len(structure.numbers), 3):
                _refuse(f"configuration {c} has {len(d)} displacements for {len(structure.numbers)} atoms")
            if not np.isfinite(d).all():
                _refuse(f"configuration {c} has a non-finite displacement")
        self.displacements = [np.asarray(d, dtype=np.float64) for d in displacements]

    @staticmethod
    def configuration_seed(seed: int, c: int) -> int:
        mix = lambda v: _finalise((v + 0x9E3779B97F4A7C15) & _M64)  # noqa: E731
        return mix((mix(int(seed) & _M64) + c) & _M64)

    @property
    def count(self) -> int:
        return len(self.displacements)

    def configuration(self, c: int) -> AtomicStructure:
        s = self.structure
        return AtomicStructure(s.box, s.numbers, s.positions + self.displacements[c])

    def lazy_potentials(self, nx: int, ny: int, slice_thickness: float,
                        parameterization: LobatoParameterization | None = None):
        return [Potential(self.configuration(c), nx, ny, slice_thickness=slice_thickness,
                          parameterization=parameterization) for c in range(self.count)]

    lazyPotentials = lazy_potentials
