"""The fused float32 form's power-of-two engine at every grid side it serves and every column tile width, against the
float64 oracle: a plane wave's exit wave (the column pass's transform-multiply-transform mode) and a 2 x 2 STEM scan
(which ends in the propagator-only mode that leaves k-space for the detectors). Both store their tiles from shared
memory with TMA, so every side, tile width and mode goes through that path. Bounds as the form's other tests: 1e-5
rel-L2 for waves, 1e-4 for detector values."""

import functools

import numpy as np
import pytest

from oracle import simk_oracle as O

pytestmark = pytest.mark.gpu

sk = pytest.importorskip("simulatokit_b200")


@pytest.fixture(scope="module")
def engine():
    return sk.Engine.require()


@functools.lru_cache(maxsize=None)
def _case(n):
    """SrTiO3 cells at 64 points a cell (0.122 A sampling), two slices of 1.9525 A; the oracle's exit wave and the
    2 x 2 scan's detector values, computed once per side."""
    reps = max(1, n // 64)
    s = O.srtio3_cell().repeated(reps, reps, 1)
    op = O.Potential.from_structure(s, n, n, slice_thickness=1.9525)
    vs = op.build()
    ts = [O.transmission(v, 200e3, op.grid) for v in vs]
    wave = O.multislice(O.plane_wave(op.grid), ts, op.thicknesses, 200e3, op.grid)[-1]
    scan = sk.GridScan((0.0, 0.0), (3.905, 3.905), 2, 2)
    det = O.stem_scan(O.ProbeSpec(200e3, 20.0), [(op.grid, vs, op.thicknesses)], scan.positions,
                      [O.DetectorSpec("annular", {"inner": 0, "outer": 20}),
                       O.DetectorSpec("annular", {"inner": 40, "outer": 80})])
    return s, wave, det


def _potential(n):
    s, _, _ = _case(n)
    return sk.Potential(sk.AtomicStructure(s.box, s.numbers, s.positions), n, n, slice_thickness=1.9525)


@pytest.mark.parametrize("n", [128, 256, 1024, 2048])
@pytest.mark.parametrize("tile", [2, 4, 8])
def test_exit_wave(engine, n, tile):
    _, ref, _ = _case(n)
    pot = _potential(n)
    ex = sk.Multislice.run(sk.Waves.plane_wave(sk.ElectronBeam(200e3), pot.grid), pot,
                           options=sk.ExecutionOptions(form="fused", col_tile=tile), engine=engine)[-1]
    assert O.rel_l2(ex.field, ref) <= 1e-5


@pytest.mark.parametrize("n", [128, 256, 1024, 2048])
@pytest.mark.parametrize("tile", [2, 4, 8])
def test_small_scan(engine, n, tile):
    _, _, ores = _case(n)
    pot = _potential(n)
    probe = sk.Probe(sk.ElectronBeam(200e3), pot.grid, sk.Aperture(20.0))
    scan = sk.GridScan((0.0, 0.0), (3.905, 3.905), 2, 2)
    res = sk.STEM.scan(probe, [pot], scan, [sk.AnnularDetector(0, 20), sk.AnnularDetector(40, 80)],
                       options=sk.ExecutionOptions(form="fused", col_tile=tile), engine=engine)
    for m, r in zip(res, ores):
        assert O.rel_l2(m.values, np.asarray(r).ravel()) <= 1e-4
