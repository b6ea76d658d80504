"""Detection inside the last column pass (the fused form's epilogue) against detection from the stored k-space waves.

With the TMA passes on, the fused form sums the channel detectors (annular, centre of mass, segmented) from the last
column pass's finished tile in shared memory and writes no k-space wave unless a pixelated or binned detector reads it
(Sources/SimulatoDetector/Detectors.swift:119-263, STEM.swift:137-144). With them off, the same waves go through the
separate detection kernels. The per-pixel products are the same float32 values; only the float64 summation order
differs, so the images agree to 1e-12 relative L2, and each path is bit-deterministic.
"""

import numpy as np
import pytest

from oracle import simk_oracle as O

pytestmark = pytest.mark.gpu

sk = pytest.importorskip("simulatokit_b200")


@pytest.fixture(scope="module")
def engine():
    return sk.Engine.require()


def _scan(engine, tma, n=256, col_tile=4, dets=None, form="fused"):
    s = O.srtio3_cell().repeated(4, 4, 4)
    pot = sk.Potential(sk.AtomicStructure(s.box, s.numbers, s.positions), n, n, slice_thickness=1.9525)
    probe = sk.Probe(sk.ElectronBeam(200e3), pot.grid, sk.Aperture(20.0))
    scan = sk.GridScan((3.905, 3.905), (2 * 3.905, 2 * 3.905), 5, 4)
    dets = dets or [sk.AnnularDetector(0, 20), sk.AnnularDetector(50, 120), sk.SegmentedDetector(2, 4, 0, 20, 0.3),
                    sk.CenterOfMassDetector("cutoff", "mrad")]
    opts = sk.ExecutionOptions(form=form, tma=tma, col_tile=col_tile)
    return [m.values.copy() for m in sk.STEM.scan(probe, [pot], scan, dets, options=opts, engine=engine)]


@pytest.mark.parametrize("col_tile", [2, 4, 8])
def test_epilogue_detection_equals_separate_kernels(engine, col_tile):
    a = _scan(engine, True, col_tile=col_tile)
    b = _scan(engine, False, col_tile=col_tile)
    for x, y in zip(a, b):
        assert O.rel_l2(x, y) <= 1e-12
    again = _scan(engine, True, col_tile=col_tile)
    for x, y in zip(a, again):
        assert np.array_equal(x, y)


def test_epilogue_with_pixel_outputs_stores_the_waves(engine):
    """A pixelated detector beside the channel detectors: the pass also stores the k-space waves it reads."""
    dets = [sk.AnnularDetector(50, 120), sk.PixelatedDetector("cutoff"), sk.AnnularDetector(0, 20)]
    a = _scan(engine, True, dets=dets)
    b = _scan(engine, False, dets=dets)
    for x, y in zip(a, b):
        assert O.rel_l2(x, y) <= 1e-12


def test_epilogue_mixed_radix_engine(engine):
    """The shared-memory engine's TMA passes (384 = 3 x 2^7) with the detection epilogue."""
    a = _scan(engine, True, n=384)
    b = _scan(engine, False, n=384)
    for x, y in zip(a, b):
        assert O.rel_l2(x, y) <= 1e-6  # different transform engines: float32 rounding of the waves differs
