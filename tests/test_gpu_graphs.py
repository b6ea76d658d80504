"""The fused forms' slice loop replayed from CUDA graphs (SIMK_OPT_GRAPHS): bit-identical to eager launches.

A scan is run in batches of 4 positions so that the loop of one batch shape is seen many times: the first batch runs
eagerly, the second is captured, the rest are replayed. Graph replays must give the same detector values bit for bit,
count the same kernel launches, and follow a change of potential (frozen-phonon configurations) or of form.
"""

import numpy as np
import pytest

from oracle import simk_oracle as O

pytestmark = pytest.mark.gpu

sk = pytest.importorskip("simulatokit_b200")


@pytest.fixture(scope="module")
def engine():
    return sk.Engine.require()


def _setup(n=256, configs=1):
    s = O.srtio3_cell().repeated(2, 2, 6)
    st = sk.AtomicStructure(s.box, s.numbers, s.positions)
    if configs == 1:
        pots = [sk.Potential(st, n, n, slice_thickness=1.9525)]
    else:
        fp = sk.FrozenPhonons(st, sigmas={38: 0.08, 22: 0.08, 8: 0.08}, configurations=configs, seed=3)
        pots = [sk.Potential(fp.configuration(c), n, n, slice_thickness=1.9525) for c in range(fp.count)]
    probe = sk.Probe(sk.ElectronBeam(200e3), pots[0].grid, sk.Aperture(20.0))
    scan = sk.GridScan((0.0, 0.0), (3.905, 3.905), 6, 6)
    dets = [sk.AnnularDetector(0, 20), sk.AnnularDetector(50, 120), sk.SegmentedDetector(2, 4, 0, 20)]
    return probe, pots, scan, dets


@pytest.mark.parametrize("form", ["fused", "bf16x3"])
def test_graph_replay_is_bit_identical(engine, form):
    probe, pots, scan, dets = _setup()
    eager = sk.STEM.scan(probe, pots, scan, dets, options=sk.ExecutionOptions(form=form, batch=4, graphs=False),
                         engine=engine)
    assert engine.graphs_cached() == 0
    engine.launch_count(reset=True)
    sk.STEM.scan(probe, pots, scan, dets, options=sk.ExecutionOptions(form=form, batch=4, graphs=False),
                 engine=engine)
    n_eager = engine.launch_count(reset=True)
    graphed = sk.STEM.scan(probe, pots, scan, dets, options=sk.ExecutionOptions(form=form, batch=4, graphs=True),
                           engine=engine)
    n_graph = engine.launch_count(reset=True)
    assert engine.graphs_cached() >= 1
    assert n_graph == n_eager
    for a, b in zip(eager, graphed):
        assert np.array_equal(a.values, b.values)
    # replayed again, all batches from the cache
    again = sk.STEM.scan(probe, pots, scan, dets, options=sk.ExecutionOptions(form=form, batch=4, graphs=True),
                         engine=engine)
    for a, b in zip(eager, again):
        assert np.array_equal(a.values, b.values)


def test_graphs_follow_the_potential(engine):
    probe, pots, scan, dets = _setup(configs=3)
    eager = sk.STEM.scan(probe, pots, scan, dets, options=sk.ExecutionOptions(batch=4, graphs=False), engine=engine)
    graphed = sk.STEM.scan(probe, pots, scan, dets, options=sk.ExecutionOptions(batch=4, graphs=True), engine=engine)
    assert engine.graphs_cached() >= 3  # one slice loop per configuration's transmissions
    for a, b in zip(eager, graphed):
        assert np.array_equal(a.values, b.values)
