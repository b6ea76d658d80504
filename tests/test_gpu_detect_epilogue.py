"""Detection inside the last column pass (the fused form's epilogue) against detection from the stored k-space waves.

With the TMA passes on, the fused form sums the channel detectors (annular, centre of mass, segmented) from the last
column pass's finished tile in shared memory and writes no k-space wave unless a pixelated or binned detector reads it
(Sources/SimulatoDetector/Detectors.swift:119-263, STEM.swift:137-144). With the epilogue switched off, the same waves
go through the separate detection kernels: the per-pixel products are the same float32 values and only the float64
summation order differs, so the images agree to 1e-12 relative L2; each path is bit-deterministic. Without the TMA
passes the transforms themselves round differently (float32), within 1e-6.
"""

import numpy as np
import pytest

from oracle import simk_oracle as O

pytestmark = pytest.mark.gpu

sk = pytest.importorskip("simulatokit_b200")


@pytest.fixture(scope="module")
def engine():
    return sk.Engine.require()


def _scan(engine, tma, n=256, col_tile=4, dets=None, form="fused", epilogue=True):
    s = O.srtio3_cell().repeated(4, 4, 4)
    pot = sk.Potential(sk.AtomicStructure(s.box, s.numbers, s.positions), n, n, slice_thickness=1.9525)
    probe = sk.Probe(sk.ElectronBeam(200e3), pot.grid, sk.Aperture(20.0))
    scan = sk.GridScan((3.905, 3.905), (2 * 3.905, 2 * 3.905), 5, 4)
    dets = dets or [sk.AnnularDetector(0, 20), sk.AnnularDetector(50, 120), sk.SegmentedDetector(2, 4, 0, 20, 0.3),
                    sk.CenterOfMassDetector("cutoff", "mrad")]
    opts = sk.ExecutionOptions(form=form, tma=tma, col_tile=col_tile, epilogue_detect=epilogue)
    return [m.values.copy() for m in sk.STEM.scan(probe, [pot], scan, dets, options=opts, engine=engine)]


def _compare(a, b, bound, what):
    for d, (x, y) in enumerate(zip(a, b)):
        e = O.rel_l2(x, y)
        bad = np.nonzero(np.abs(x - y) > max(bound, 1e-12) * np.abs(y).max())[0]
        assert e <= bound, f"{what}: detector {d} rel-L2 {e:.2e}, positions {bad[:10]}"


@pytest.mark.parametrize("col_tile", [2, 4, 8])
def test_epilogue_detection_equals_separate_kernels(engine, col_tile):
    a = _scan(engine, True, col_tile=col_tile)
    b = _scan(engine, True, col_tile=col_tile, epilogue=False)
    _compare(a, b, 1e-12, "epilogue vs separate kernels")
    _compare(a, _scan(engine, False, col_tile=col_tile), 1e-6, "TMA passes vs the others")
    again = _scan(engine, True, col_tile=col_tile)
    for x, y in zip(a, again):
        assert np.array_equal(x, y)


def test_epilogue_with_pixel_outputs_stores_the_waves(engine):
    """A pixelated detector beside the channel detectors: the pass also stores the k-space waves it reads."""
    dets = [sk.AnnularDetector(50, 120), sk.PixelatedDetector("cutoff"), sk.AnnularDetector(0, 20)]
    _compare(_scan(engine, True, dets=dets), _scan(engine, True, dets=dets, epilogue=False), 1e-12, "with pixels")


@pytest.mark.parametrize("form", ["fused", "bf16x3"])
def test_epilogue_mixed_radix_and_tensor_core_engines(engine, form):
    """The shared-memory engine's TMA passes (384 = 3 x 2^7) and the bf16x3 form's tensor-core passes (512) with the
    detection epilogue."""
    n = 384 if form == "fused" else 512
    a = _scan(engine, True, n=n, form=form)
    _compare(a, _scan(engine, True, n=n, form=form, epilogue=False), 1e-12, f"{form} {n}")
    if form == "fused":
        _compare(a, _scan(engine, False, n=n), 1e-6, "TMA passes vs the runtime-plan kernels")
