"""The bf16x3 form against the float64 oracle.

The form runs the fused TMA passes with each line FFT's radix-16 stages as tensor-core products of split-BF16 operands
with float32 accumulation (radix 2/3/4/8 first stage and twiddles in float32): on the fifth-generation tensor cores
(tcgen05.mma, data in three BF16 terms) at grid sides 256 and 512, and with warp-level mma.sync (data in two terms)
at 768, 1024 and 2048 or when the tcgen05 option is off. Its bound is the one stated for this form: <= 1e-4 relative
L2 against the float64 oracle on every detector image, and on the exit wave; the measured errors are printed.
"""

import numpy as np
import pytest

from oracle import simk_oracle as O

pytestmark = pytest.mark.gpu

sk = pytest.importorskip("simulatokit_b200")


@pytest.fixture(scope="module")
def engine():
    return sk.Engine.require()


def _opts(form="bf16x3", tcgen05=2):
    return sk.ExecutionOptions(form=form, tcgen05=tcgen05)


@pytest.mark.parametrize("tcgen05", [2, 1, 0])
def test_hrtem_srtio3_exit_wave(engine, tcgen05):
    """SrTiO3 4x4x5, 256^2, 10 slices of 1.9525 A, 200 keV plane wave, on the tcgen05 engine (six stacked or twelve
    products a stage) and on the mma.sync engine."""
    s = O.srtio3_cell().repeated(4, 4, 5)
    op = O.Potential.from_structure(s, 256, 256, slice_thickness=1.9525)
    og = op.grid
    ts = [O.transmission(v, 200e3, og) for v in op.build()]
    ref = O.multislice(O.plane_wave(og), ts, op.thicknesses, 200e3, og)[-1]
    pot = sk.Potential(sk.AtomicStructure(s.box, s.numbers, s.positions), 256, 256, slice_thickness=1.9525)
    ex = sk.Multislice.run(sk.Waves.plane_wave(sk.ElectronBeam(200e3), pot.grid), pot, options=_opts(tcgen05=tcgen05),
                           engine=engine)[-1]
    e_wave = O.rel_l2(ex.field, ref)
    e_int = O.rel_l2(np.abs(ex.field) ** 2, np.abs(ref) ** 2)
    name = {1: "tcgen05", 2: "tcgen05 stacked", 0: "mma.sync"}[tcgen05]
    print(f"bf16x3 ({name}) HRTEM 256^2 x 10 slices: exit wave rel-L2 {e_wave:.2e}, intensity {e_int:.2e}")
    assert e_wave <= 1e-4 and e_int <= 1e-4
    if tcgen05:  # three-term data split: float32-like accuracy
        assert e_wave <= 1e-5


def _scan_vs_oracle(engine, cells, n, positions_per_side, dets_sk, dets_o, slice_thickness=3.905):
    s = O.srtio3_cell().repeated(*cells)
    st = sk.AtomicStructure(s.box, s.numbers, s.positions)
    pot = sk.Potential(st, n, n, slice_thickness=slice_thickness)
    probe = sk.Probe(sk.ElectronBeam(200e3), pot.grid, sk.Aperture(20.0))
    c0 = (cells[0] // 2) * 3.905
    scan = sk.GridScan((c0, c0), (c0 + 3.905, c0 + 3.905), positions_per_side, positions_per_side)
    op = O.Potential.from_structure(s, n, n, slice_thickness=slice_thickness)
    ores = O.stem_scan(O.ProbeSpec(200e3, 20.0), [(op.grid, op.build(), op.thicknesses)], scan.positions, dets_o)
    out = {}
    for form in ("bf16x3", "fused"):
        res = sk.STEM.scan(probe, [pot], scan, dets_sk, options=_opts(form), engine=engine)
        out[form] = [O.rel_l2(m.values, r.ravel()) for m, r in zip(res, ores)]
    return out


def test_small_stem_scan_256(engine):
    """The STEM workload's shape at 256^2: SrTiO3 2x2x20, 20 slices of 3.905 A, 20 mrad, BF 0-20 and HAADF 50-120."""
    errs = _scan_vs_oracle(engine, (2, 2, 20), 256, 6,
                           [sk.AnnularDetector(0, 20), sk.AnnularDetector(50, 120)],
                           [O.DetectorSpec("annular", {"inner": 0, "outer": 20}),
                            O.DetectorSpec("annular", {"inner": 50, "outer": 120})])
    print("rel-L2 vs float64 oracle (BF, HAADF):", errs)
    assert max(errs["bf16x3"]) <= 1e-4
    assert max(errs["fused"]) <= 1e-4


def test_stacked_products_equal_the_twelve(engine):
    """The six stacked products (N = 96, 64, 32) sum the same terms as the twelve of N = 32: a 512^2 scan agrees to
    float32 rounding. (With hi x hi first in a stacked accumulator block, the small terms added to it inside the
    tensor core lost low bits and the two differed by 1.7e-5; it now has a block of its own.)"""
    s = O.srtio3_cell().repeated(4, 4, 6)
    pot = sk.Potential(sk.AtomicStructure(s.box, s.numbers, s.positions), 512, 512, slice_thickness=1.9525)
    probe = sk.Probe(sk.ElectronBeam(200e3), pot.grid, sk.Aperture(20.0))
    scan = sk.GridScan((3.905, 3.905), (2 * 3.905, 2 * 3.905), 4, 4)
    dets = [sk.AnnularDetector(0, 20), sk.AnnularDetector(50, 120)]
    a = sk.STEM.scan(probe, [pot], scan, dets, options=_opts(tcgen05=1), engine=engine)
    b = sk.STEM.scan(probe, [pot], scan, dets, options=_opts(tcgen05=2), engine=engine)
    for x, y in zip(a, b):
        assert O.rel_l2(x.values, y.values) <= 1e-5


def test_stem_scan_512_full_cell(engine):
    """The STEM HAADF+BF workload itself (SrTiO3 8x8x20, 512^2, 20 slices, BF 0-20, HAADF 50-200) on a 4x4 scan."""
    errs = _scan_vs_oracle(engine, (8, 8, 20), 512, 4,
                           [sk.AnnularDetector(0, 20), sk.AnnularDetector(50, 200)],
                           [O.DetectorSpec("annular", {"inner": 0, "outer": 20}),
                            O.DetectorSpec("annular", {"inner": 50, "outer": 200})])
    print("512^2 rel-L2 vs float64 oracle (BF, HAADF):", errs)
    assert max(errs["bf16x3"]) <= 1e-4
    assert max(errs["fused"]) <= 1e-4


def test_probe_exit_wave_768(engine):
    """A 768^2 grid (radix-3 first stage): silicon 2x2x2, 25 mrad probe at 300 keV with C10 = -50 A, 8 slices."""
    s = O.silicon_cell().repeated(2, 2, 2)
    op = O.Potential.from_structure(s, 768, 768, slice_thickness=1.35775)
    og = op.grid
    spec = O.ProbeSpec(300e3, 25.0, {"C10": -50.0})
    pos = (s.box[0] / 2, s.box[1] / 2)
    psi0 = O.build_probe(spec, og, pos)
    ts = [O.transmission(v, 300e3, og) for v in op.build()]
    ref = O.multislice(psi0, ts, op.thicknesses, 300e3, og)[-1]
    pot = sk.Potential(sk.AtomicStructure(s.box, s.numbers, s.positions), 768, 768, slice_thickness=1.35775)
    probe = sk.Probe(sk.ElectronBeam(300e3), pot.grid, sk.Aperture(25.0), sk.Aberrations(C10=-50.0))
    inc = probe.build(pos, engine)
    ex = sk.Multislice.run(inc, pot, options=_opts(), engine=engine)[-1]
    e = O.rel_l2(ex.field, ref)
    ei = O.rel_l2(np.abs(np.fft.fft2(ex.field)) ** 2, np.abs(np.fft.fft2(ref)) ** 2)
    print(f"bf16x3 768^2 probe x {len(op.thicknesses)} slices: exit wave rel-L2 {e:.2e}, pattern {ei:.2e}")
    assert e <= 1e-4 and ei <= 1e-4


def test_scan_deterministic_and_batch_independent(engine):
    s = O.srtio3_cell().repeated(2, 2, 4)
    st = sk.AtomicStructure(s.box, s.numbers, s.positions)
    pot = sk.Potential(st, 256, 256, slice_thickness=1.9525)
    probe = sk.Probe(sk.ElectronBeam(200e3), pot.grid, sk.Aperture(20.0))
    scan = sk.GridScan((0.0, 0.0), (3.905, 3.905), 5, 5)
    dets = [sk.AnnularDetector(50, 120), sk.SegmentedDetector(2, 4, 0, 20)]
    a = sk.STEM.scan(probe, [pot], scan, dets, options=sk.ExecutionOptions(form="bf16x3"), engine=engine)
    b = sk.STEM.scan(probe, [pot], scan, dets, options=sk.ExecutionOptions(form="bf16x3"), engine=engine)
    c = sk.STEM.scan(probe, [pot], scan, dets, options=sk.ExecutionOptions(form="bf16x3", batch=3), engine=engine)
    for x, y, z in zip(a, b, c):
        assert np.array_equal(x.values, y.values)
        assert np.array_equal(x.values, z.values)


@pytest.mark.parametrize("n", [128, 500])
def test_refuses_grids_it_does_not_cover(engine, n):
    s = O.srtio3_cell().repeated(2, 2, 1)
    pot = sk.Potential(sk.AtomicStructure(s.box, s.numbers, s.positions), n, n, slice_thickness=1.9525)
    with pytest.raises(sk.InvalidArgument, match="bf16x3"):
        sk.Multislice.run(sk.Waves.plane_wave(sk.ElectronBeam(200e3), pot.grid), pot, options=_opts(), engine=engine)
