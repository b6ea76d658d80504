"""The waves detector on the device against the reference's abTEM pins (Detector/WavesDetectorTests.swift): the exit
waves of a 3 x 2 scan through Al 1 x 1 x 2 on 48 x 48 (4 slices, 200 keV, 20 mrad), on the simulation grid and
Fourier-resampled to 33 x 40, 81 x 96, 30 x 71, 64 x 25 and 10 x 11 (crop and zero-pad, odd and even). Bound: the
reference's registered bound for a float32 device wave (MetalAccuracy.registered.wave, ExecutionOptions.swift:55-94):
max |dpsi| / max |psi| <= 1e-4, complex."""

import numpy as np
import pytest

import golden_io as G
from oracle import simk_oracle as O

pytestmark = pytest.mark.gpu

sk = pytest.importorskip("simulatokit_b200")


@pytest.fixture(scope="module")
def engine():
    return sk.Engine.require()


def _setup():
    w = G.pins()["waves"]
    st = sk.AtomicStructure(tuple(w["box"]), [a[0] for a in w["atoms"]], [a[1] for a in w["atoms"]])
    n = w["gpts"]
    pot = sk.Potential(st, n, n, slice_thickness=w["sliceThickness"],
                       parameterization=sk.LobatoParameterization("abTEMFloat32"))
    probe = sk.Probe(sk.ElectronBeam(w["energy"]), pot.grid, sk.Aperture(w["semiangle"]))
    scan = sk.GridScan(tuple(w["scan"]["start"]), tuple(w["scan"]["end"]), *w["scan"]["gpts"])
    return w, st, pot, probe, scan


@pytest.mark.parametrize("form", ["plain", "fused"])
@pytest.mark.parametrize("run", range(6))
def test_waves_match_pins(engine, run, form):
    w, _, pot, probe, scan = _setup()
    entry = w["runs"][run]
    det = sk.WavesDetector(*entry["gpts"]) if entry["gpts"] else sk.WavesDetector()
    out = sk.STEM.scan(probe, [pot], scan, det, options=sk.ExecutionOptions(form=form), engine=engine)
    ref = G.array("waves", entry["name"])
    got = out.array()
    assert list(got.shape) == entry["shape"]
    e = float(np.max(np.abs(got - ref)) / np.max(np.abs(ref)))
    print(f"{form} {entry['name']}: max |dpsi| / max |psi| {e:.2e}, rel-L2 {O.rel_l2(got, ref):.2e}")
    assert e <= 1e-4
    assert out[2, 1].field.shape == tuple(entry["shape"][2:])


def test_waves_of_frozen_phonons(engine):
    """One ScanWaves per configuration (complex waves are not averaged), each equal to that configuration's own scan."""
    w, st, pot, probe, scan = _setup()
    fp = sk.FrozenPhonons(st, sigmas={13: 0.1}, configurations=3, seed=2)
    det = sk.WavesDetector(33, 40)
    per = sk.STEM.scanFrozenPhonons(probe, fp, 48, 48, w["sliceThickness"], scan, det, engine=engine)
    assert len(per) == 3
    for c, sw in enumerate(per):
        one = sk.STEM.scan(probe, [sk.Potential(fp.configuration(c), 48, 48, slice_thickness=w["sliceThickness"])],
                           scan, det, engine=engine)
        assert np.array_equal(sw.values, one.values)
    assert not np.array_equal(per[0].values, per[1].values)


def test_waves_refusals(engine):
    w, _, pot, probe, scan = _setup()
    with pytest.raises(sk.InvalidArgument, match="need"):
        sk.STEM.scan(probe, [pot], scan, sk.WavesDetector(), engine=engine, memory_limit=1000)
