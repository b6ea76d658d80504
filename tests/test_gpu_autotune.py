"""Autotuning (SIMK_OPT_AUTOTUNE): the tuned column tile, TMA choice and batch are valid, are kept per grid, and give
the same detector values as the same settings chosen by hand (the transform of a column does not depend on them)."""

import numpy as np
import pytest

from oracle import simk_oracle as O

pytestmark = pytest.mark.gpu

sk = pytest.importorskip("simulatokit_b200")


@pytest.fixture(scope="module")
def engine():
    return sk.Engine.require()


@pytest.mark.parametrize("n", [256, 768])
def test_autotune_choice_and_results(engine, n):
    s = O.srtio3_cell().repeated(2, 2, 3)
    pot = sk.Potential(sk.AtomicStructure(s.box, s.numbers, s.positions), n, n, slice_thickness=1.9525)
    probe = sk.Probe(sk.ElectronBeam(200e3), pot.grid, sk.Aperture(20.0))
    scan = sk.GridScan((0.0, 0.0), (3.905, 3.905), 6, 6)
    dets = [sk.AnnularDetector(0, 20), sk.AnnularDetector(50, 120)]
    tuned_res = sk.STEM.scan(probe, [pot], scan, dets, options=sk.ExecutionOptions(autotune=True), engine=engine)
    t = engine.tuned()
    print(n, t)
    assert t["col_tile"] in (2, 4, 8) and t["tma"] in (0, 1) and 1 <= t["batch"] <= 1024
    by_hand = sk.STEM.scan(probe, [pot], scan, dets,
                           options=sk.ExecutionOptions(col_tile=t["col_tile"], tma=bool(t["tma"]), batch=t["batch"]),
                           engine=engine)
    for a, b in zip(tuned_res, by_hand):
        assert np.array_equal(a.values, b.values)
    default = sk.STEM.scan(probe, [pot], scan, dets, engine=engine)
    for a, b in zip(tuned_res, default):
        assert O.rel_l2(a.values, b.values) <= 1e-6
    # kept per grid: a second tuned scan does not retune (the same choice comes back)
    sk.STEM.scan(probe, [pot], scan, dets, options=sk.ExecutionOptions(autotune=True), engine=engine)
    assert engine.tuned() == t
