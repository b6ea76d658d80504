"""4D-STEM with frozen phonons, the workload's shape at reduced size, against the float64 oracle.

Diamond-cubic Si (a = 5.431 A) tiled 6 x 6 x 2 on a 768 x 768 grid (radix-3 plans; 8 slices of 1.35775 A), 300 keV,
25 mrad, C10 = -50 A, two frozen-phonon configurations with sigma = 0.075 A from the kit's generator, 2 x 2 probe
positions; a pixelated detector on a 128 x 128 grid up to 60 mrad (binned, this library's numeric-angle rule) and a
centre-of-mass detector. Bounds: <= 1e-4 relative L2 per detector image for every form.
"""

import pytest

from oracle import simk_oracle as O

pytestmark = pytest.mark.gpu

sk = pytest.importorskip("simulatokit_b200")


@pytest.fixture(scope="module")
def engine():
    return sk.Engine.require()


@pytest.fixture(scope="module")
def case():
    s = O.silicon_cell().repeated(6, 6, 2)
    st = sk.AtomicStructure(s.box, s.numbers, s.positions)
    fp = sk.FrozenPhonons(st, sigmas={14: 0.075}, configurations=2, seed=1)
    structs = [fp.configuration(c) for c in range(fp.count)]
    pots = [sk.Potential(x, 768, 768, slice_thickness=1.35775) for x in structs]
    assert pots[0].slice_count == 8
    probe = sk.Probe(sk.ElectronBeam(300e3), pots[0].grid, sk.Aperture(25.0), sk.Aberrations(C10=-50.0))
    scan = sk.GridScan((2 * 5.431, 2 * 5.431), (3 * 5.431, 3 * 5.431), 2, 2)
    dets = [sk.BinnedPixelatedDetector(60.0, (128, 128)), sk.CenterOfMassDetector("valid", "mrad")]
    opots = []
    for x in structs:
        op = O.Potential.from_structure(O.Structure(x.box, x.numbers, x.positions), 768, 768, slice_thickness=1.35775)
        opots.append((op.grid, op.build(), op.thicknesses))
    ores = O.stem_scan(O.ProbeSpec(300e3, 25.0, {"C10": -50.0}), opots, scan.positions,
                       [O.DetectorSpec("binned", {"nbx": 128, "nby": 128, "outer": 60.0}),
                        O.DetectorSpec("com", {"mode": "valid", "units": "mrad"})])
    return probe, pots, scan, dets, ores


def test_binned_shape(engine, case):
    probe, pots, scan, dets, _ = case
    assert sk.detector_shape(dets[0], probe.grid, 300e3) == [128, 128]
    with pytest.raises(sk.InvalidArgument, match="largest simulated angle"):  # a window beyond the grid's angles
        sk.STEM.scan(probe, pots[:1], scan, [sk.BinnedPixelatedDetector(1e4)], engine=engine)


@pytest.mark.parametrize("form", ["plain", "fused", "bf16x3"])
def test_4dstem_frozen_phonons_768(engine, case, form):
    probe, pots, scan, dets, ores = case
    res = sk.STEM.scan(probe, pots, scan, dets, options=sk.ExecutionOptions(form=form), engine=engine)
    e_bin = O.rel_l2(res[0].values, ores[0].ravel())
    e_com = O.rel_l2(res[1].values, ores[1].ravel())
    print(f"{form}: binned 128x128 rel-L2 {e_bin:.2e}, COM rel-L2 {e_com:.2e}")
    assert res[0].array().shape == (2, 2, 128, 128)
    assert e_bin <= 1e-4 and e_com <= 1e-4
