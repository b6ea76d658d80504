"""Autotuning (SIMK_OPT_AUTOTUNE): the tuned column tile, TMA choice, batch and line-FFT engine are valid, are kept per
grid, and give the same detector values as the same settings chosen by hand (the transform of a column does not
depend on the tile or the batch)."""

import numpy as np
import pytest

from oracle import simk_oracle as O

pytestmark = pytest.mark.gpu

sk = pytest.importorskip("simulatokit_b200")


@pytest.fixture(scope="module")
def engine():
    return sk.Engine.require()


@pytest.mark.parametrize("form,n", [("fused", 256), ("fused", 768), ("bf16x3", 256)])
def test_autotune_choice_and_results(engine, form, n):
    s = O.srtio3_cell().repeated(2, 2, 3)
    pot = sk.Potential(sk.AtomicStructure(s.box, s.numbers, s.positions), n, n, slice_thickness=1.9525)
    probe = sk.Probe(sk.ElectronBeam(200e3), pot.grid, sk.Aperture(20.0))
    scan = sk.GridScan((0.0, 0.0), (3.905, 3.905), 6, 6)
    dets = [sk.AnnularDetector(0, 20), sk.AnnularDetector(50, 120)]
    tuned_res = sk.STEM.scan(probe, [pot], scan, dets, options=sk.ExecutionOptions(form=form, autotune=True),
                             engine=engine)
    t = engine.tuned()
    print(form, n, t)
    assert t["col_tile"] in ((2, 4, 8, 16) if (form, n) == ("fused", 256) else (2, 4, 8))
    assert t["tma"] in (0, 1) and 1 <= t["batch"] <= 1024
    # the engine: composite or shared-memory at 768 (fused), a tcgen05 product order or mma.sync at 256 (bf16x3)
    assert t["engine"] in ((0, 1) if (form, n) == ("fused", 768) else (0, 1, 2) if form == "bf16x3" else (-1,))
    kw = {}
    if t["engine"] >= 0:
        kw = {"composite": bool(t["engine"])} if form == "fused" else {"tcgen05": t["engine"]}
    by_hand = sk.STEM.scan(probe, [pot], scan, dets,
                           options=sk.ExecutionOptions(form=form, col_tile=t["col_tile"], tma=bool(t["tma"]),
                                                       batch=t["batch"], **kw),
                           engine=engine)
    for a, b in zip(tuned_res, by_hand):
        assert np.array_equal(a.values, b.values)
    default = sk.STEM.scan(probe, [pot], scan, dets, options=sk.ExecutionOptions(form=form), engine=engine)
    for a, b in zip(tuned_res, default):
        assert O.rel_l2(a.values, b.values) <= (1e-6 if form == "fused" else 2e-5)
    # kept per grid: a second tuned scan does not retune (the same choice comes back)
    sk.STEM.scan(probe, [pot], scan, dets, options=sk.ExecutionOptions(form=form, autotune=True), engine=engine)
    assert engine.tuned() == t
