"""The no-allocation entry point, simk_probe_spectrum_noalloc, against the regular simk_probe_spectrum.

Some callers cannot let this library allocate device memory: a host framework that owns every device byte through
its own allocator (PyTorch's caching allocator, an XLA custom call) needs the library to write into buffers it
handed over. This entry point keeps its scratch in a fixed device array instead of allocating. Here the caller's
output buffer comes from torch, the call goes through the C ABI, and two calls in a row (different grids and probes,
so the second reuses the scratch the first left behind) must each match the regular entry point's float64 spectrum
within complex64 rounding (1e-6 of the largest value). This file sorts last so a run that stops at the first failure
has already run every other test; it also passes alone in a fresh process.
"""

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

sk = pytest.importorskip("simulatokit_b200")
torch = pytest.importorskip("torch")

from simulatokit_b200 import _lib as L  # noqa: E402


def _noalloc(grid, probe):
    lib = L.lib()
    out = torch.empty(grid.nx * grid.ny, dtype=torch.complex64, device="cuda")
    g, p = grid.c(), probe.c()
    stream = torch.cuda.current_stream()
    L.check(lib.simk_probe_spectrum_noalloc(C.byref(g), C.byref(p), C.c_void_p(out.data_ptr()),
                                            C.c_void_p(stream.cuda_stream)))
    stream.synchronize()
    return out.cpu().numpy().reshape(grid.nx, grid.ny).astype(np.complex128)


def _rel_max(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def test_noalloc_spectrum_matches_the_regular_entry_point_twice():
    torch.cuda.set_device(0)
    engine = sk.Engine.require(0)
    cases = [
        (sk.Grid(256, 256, 16.2, 16.2), dict(energy=200e3, semiangle=20.0, ab=sk.Aberrations())),
        (sk.Grid(120, 160, 11.715, 15.62),
         dict(energy=300e3, semiangle=25.0, ab=sk.Aberrations(C10=-50.0, C30=1.0e4, C12=20.0, phi12=0.3))),
    ]
    for grid, c in cases:
        probe = sk.Probe(sk.ElectronBeam(c["energy"]), grid, sk.Aperture(c["semiangle"]), c["ab"])
        ref = probe.centred_spectrum(engine)
        got = _noalloc(grid, probe)
        assert _rel_max(got, ref) <= 1e-6


def test_noalloc_refuses_grids_beyond_its_scratch():
    grid = sk.Grid(4096, 2048, 100.0, 50.0)
    probe = sk.Probe(sk.ElectronBeam(200e3), grid, sk.Aperture(20.0))
    g, p = grid.c(), probe.c()
    st = L.lib().simk_probe_spectrum_noalloc(C.byref(g), C.byref(p), C.c_void_p(1), C.c_void_p(0))
    assert st == L.SIMK_ERR_INVALID
    assert b"exceeds" in L.lib().simk_last_error()
