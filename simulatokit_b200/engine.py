"""The CUDA engine: one library context per device (the MetalEngine.require analogue,
Sources/SimulatoMultislice/MetalEngine.swift:63-77), its options, and the potential handles on it."""

from __future__ import annotations

import ctypes as C
import threading
import weakref

import numpy as np

from . import _lib as L


class ExecutionOptions:
    """How the CUDA backend executes (ExecutionOptions, Sources/SimulatoMultislice/ExecutionOptions.swift:21-49).

    form: "plain" (one operation per launch), "fused" (batched fused passes, the default) or "bf16x3" (fused with
    tensor-core DFT stages). batch: waves per batch (0 = from batch_bytes). batch_bytes: bytes of waves one batch
    may hold (default 1 GiB). graphs: capture each batch's slice loop in a CUDA graph. col_tile: columns per CTA of
    the fused column pass (0 = automatic). tma: the TMA-pipelined persistent column pass where available. autotune:
    time the column tile, TMA passes and batch size on the first fused scan of a grid and use the fastest where the
    settings above are automatic. tcgen05: the bf16x3 form's DFT stages on the fifth-generation tensor cores
    (tcgen05.mma, tensor-memory accumulators) at grid sides 256 and 512: 2 (default) six stacked products a stage,
    1 twelve products of N = 32, 0 / False the warp-level mma.sync stages.
    epilogue_detect: sum the channel detectors inside the last column pass (TMA passes) instead of separate kernels.
    composite: at grid sides 3 or 5 times a power of two (384, 640, 768, 1536) the fused passes transform each line as
    register-resident power-of-two transforms of its decimated sub-lines; False keeps the shared-memory Stockham
    engine. paired: at grid sides 512, 1024 and 256 the fused column pass takes tiles of 8 or 16 columns, one thread
    per pair of adjacent columns (64- and 128-byte row segments in HBM), where col_tile is 0 or that width; False
    keeps one column a thread."""

    FORMS = {"plain": L.FORM_PLAIN, "fused": L.FORM_FUSED, "bf16x3": L.FORM_BF16X3}

    def __init__(self, form: str = "fused", batch: int = 0, batch_bytes: int = 1 << 30, graphs: bool = True,
                 col_tile: int = 0, tma: bool = True, autotune: bool = False, tcgen05: int = 2,
                 epilogue_detect: bool = True, composite: bool = True, paired: bool = True):
        if form not in self.FORMS:
            raise L.InvalidArgument(L.SIMK_ERR_INVALID, f"unknown form {form!r}")
        self.form = form
        self.batch = max(0, int(batch))
        self.batch_bytes = max(1, int(batch_bytes))
        self.graphs = bool(graphs)
        self.col_tile = int(col_tile)
        self.tma = bool(tma)
        self.autotune = bool(autotune)
        self.tcgen05 = int(tcgen05)  # 2: six stacked products a stage, 1 / True: twelve of N = 32, 0: mma.sync
        self.epilogue_detect = bool(epilogue_detect)
        self.composite = bool(composite)
        self.paired = bool(paired)

    @staticmethod
    def standard() -> "ExecutionOptions":
        return ExecutionOptions()


class Engine:
    """A library context on one device; calls are serialised by the library's own mutex."""

    _instances: dict = {}
    _lock = threading.Lock()

    def __init__(self, device: int = 0):
        self.lib = L.lib()
        n = C.c_int32(0)
        L.check(self.lib.simk_cuda_available(C.byref(n)))
        h = C.c_void_p()
        L.check(self.lib.simk_context_create(device, C.byref(h)))
        self.handle = h
        self.device = device
        self._finalizer = weakref.finalize(self, Engine._destroy, self.lib, h)

    @staticmethod
    def _destroy(lib, h):
        lib.simk_context_destroy(h)

    @classmethod
    def require(cls, device: int = 0) -> "Engine":
        with cls._lock:
            e = cls._instances.get(device)
            if e is None:
                e = Engine(device)
                cls._instances[device] = e
            return e

    def apply(self, options: ExecutionOptions | None):
        o = options or ExecutionOptions.standard()
        L.check(self.lib.simk_context_set_option(self.handle, L.OPT_FORM, ExecutionOptions.FORMS[o.form]))
        L.check(self.lib.simk_context_set_option(self.handle, L.OPT_BATCH, o.batch))
        L.check(self.lib.simk_context_set_option(self.handle, L.OPT_BATCH_BYTES, o.batch_bytes))
        L.check(self.lib.simk_context_set_option(self.handle, L.OPT_GRAPHS, 1 if o.graphs else 0))
        L.check(self.lib.simk_context_set_option(self.handle, L.OPT_COL_TILE, o.col_tile))
        L.check(self.lib.simk_context_set_option(self.handle, L.OPT_TMA, 1 if o.tma else 0))
        L.check(self.lib.simk_context_set_option(self.handle, L.OPT_AUTOTUNE, 1 if o.autotune else 0))
        L.check(self.lib.simk_context_set_option(self.handle, L.OPT_TCGEN05, int(o.tcgen05)))
        L.check(self.lib.simk_context_set_option(self.handle, L.OPT_EPILOGUE_DETECT, 1 if o.epilogue_detect else 0))
        L.check(self.lib.simk_context_set_option(self.handle, L.OPT_COMPOSITE, 1 if o.composite else 0))
        L.check(self.lib.simk_context_set_option(self.handle, L.OPT_PAIRED, 1 if o.paired else 0))

    def set_stream(self, stream_ptr: int | None):
        L.check(self.lib.simk_context_set_stream(self.handle, C.c_void_p(stream_ptr or 0)))

    def synchronize(self):
        L.check(self.lib.simk_context_synchronize(self.handle))

    def launch_count(self, reset: bool = False) -> int:
        v = C.c_int64(0)
        L.check(self.lib.simk_context_launch_count(self.handle, C.byref(v), 1 if reset else 0))
        return int(v.value)

    def tuned(self) -> dict:
        """The last autotuning's choice (-1 before any): column tile, TMA passes, batch, and the line-FFT engine where
        the grid offers one (the composite option of the fused form, the tcgen05 option of bf16x3; -1: none)."""
        out = {}
        for k, opt in (("col_tile", L.OPT_TUNED_COL_TILE), ("tma", L.OPT_TUNED_TMA), ("batch", L.OPT_TUNED_BATCH),
                       ("engine", L.OPT_TUNED_ENGINE)):
            v = C.c_int64(0)
            L.check(self.lib.simk_context_get_option(self.handle, opt, C.byref(v)))
            out[k] = int(v.value)
        return out

    def last_table(self) -> dict:
        """The last fused job table: host launch calls for its slice steps (1 when captured as one CUDA graph), the
        kernels inside them and the grid shapes they covered."""
        out = {}
        for k, opt in (("launches", L.OPT_TABLE_LAUNCHES), ("kernels", L.OPT_TABLE_KERNELS),
                       ("shapes", L.OPT_TABLE_SHAPES)):
            v = C.c_int64(0)
            L.check(self.lib.simk_context_get_option(self.handle, opt, C.byref(v)))
            out[k] = int(v.value)
        return out

    def graphs_cached(self) -> int:
        """Slice loops the context holds as instantiated CUDA graphs."""
        v = C.c_int64(0)
        L.check(self.lib.simk_context_get_option(self.handle, L.OPT_GRAPHS_CACHED, C.byref(v)))
        return int(v.value)

    def set_timing(self, on: bool):
        L.check(self.lib.simk_context_set_option(self.handle, L.OPT_TIMING, 1 if on else 0))

    def kernel_time(self, name: str, reset: bool = False):
        """(total ms, launches, algorithmic bytes) of hot-path kernel `name` while timing was on."""
        ms, n, b = C.c_double(0), C.c_int64(0), C.c_double(0)
        L.check(self.lib.simk_context_kernel_time(self.handle, name.encode(), C.byref(ms), C.byref(n), C.byref(b),
                                                  1 if reset else 0))
        return ms.value, int(n.value), b.value

    def fft2(self, field: np.ndarray, inverse: bool = False, precision: int = 32) -> np.ndarray:
        """The device FFT of one or more nx x ny fields (FFT2D, Sources/SimulatoCore/FFT2D.swift:169-265)."""
        a = np.asarray(field, dtype=np.complex128)
        shape = a.shape
        if a.ndim == 2:
            a = a[None]
        count, nx, ny = a.shape
        re, im = np.ascontiguousarray(a.real), np.ascontiguousarray(a.imag)
        ore, oim = np.empty_like(re), np.empty_like(im)
        L.check(self.lib.simk_fft2(self.handle, nx, ny, count, 1 if inverse else 0, precision, L.dptr(re), L.dptr(im),
                                   L.dptr(ore), L.dptr(oim)))
        return (ore + 1j * oim).reshape(shape)


class PotentialHandle:
    """A potential built on the device (`simk_potential`), owned by the Python object that made it."""

    def __init__(self, engine: Engine, handle):
        self.engine = engine
        self.handle = handle
        self._finalizer = weakref.finalize(self, PotentialHandle._destroy, engine.lib, handle)

    @staticmethod
    def _destroy(lib, h):
        lib.simk_potential_destroy(h)

    def read_slices(self, n_slices: int, nx: int, ny: int) -> np.ndarray:
        out = np.empty((n_slices, nx, ny))
        L.check(self.engine.lib.simk_potential_read_slices(self.engine.handle, self.handle, L.dptr(out)))
        return out

    def read_transmission(self, energy: float, j: int, nx: int, ny: int) -> np.ndarray:
        re, im = np.empty((nx, ny)), np.empty((nx, ny))
        L.check(self.engine.lib.simk_potential_read_transmission(self.engine.handle, self.handle, energy, j,
                                                                  L.dptr(re), L.dptr(im)))
        return re + 1j * im
