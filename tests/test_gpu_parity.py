"""CUDA path against the float64 oracle and the reference's golden vectors, through the C ABI.

Tolerances (the reference's MetalAccuracy registry, Sources/SimulatoMultislice/ExecutionOptions.swift:55-94, and the
stricter gates of the workloads): exit waves <= 1e-5 relative L2 (float32 path, plane-wave HRTEM), detector images
<= 1e-4 relative L2 and <= 2e-4 x max(image max, 1e-5 x incident) max-abs; float64 device results (potential,
float64 FFT) at the reference's own float64 bounds.
"""

import numpy as np
import pytest

import golden_io as G
from oracle import simk_oracle as O

pytestmark = pytest.mark.gpu

sk = pytest.importorskip("simulatokit_b200")


@pytest.fixture(scope="module")
def engine():
    return sk.Engine.require()


FORMS = ["plain", "fused"]


def _rng_field(shape, seed=0):
    r = np.random.default_rng(seed)
    return r.standard_normal(shape) + 1j * r.standard_normal(shape)


# ---- the transform (SimulatoCoreTests.swift:21-179) ------------------------------------------------------------------
@pytest.mark.parametrize("nx,ny", [(2, 3), (7, 11), (13, 100), (97, 6), (45, 49), (127, 20), (8, 8), (100, 90),
                                   (1000, 3), (250, 506), (500, 21), (97, 11), (496, 127), (121, 169), (512, 512),
                                   (768, 768), (90, 75), (640, 384), (1009, 4)])
def test_fft2_any_length(engine, nx, ny):
    x = _rng_field((2, nx, ny), seed=nx * 1000 + ny)
    ref = np.fft.fft2(x)
    f64 = engine.fft2(x, precision=64)
    assert np.max(np.abs(f64 - ref)) <= 1e-12 * np.max(np.abs(ref))
    f32 = engine.fft2(x, precision=32)
    assert O.rel_l2(f32, ref) <= 2e-6
    back = engine.fft2(ref, inverse=True, precision=64)
    assert np.max(np.abs(back - x)) <= 1e-12 * np.max(np.abs(x))


# ---- potential and transmission (PotentialPinsTests.swift) ---------------------------------------------------------
def _pot_from_case(c, pi="abTEMFloat32"):
    s = sk.AtomicStructure(tuple(c["box"]), np.array(c["numbers"], dtype=int),
                           np.array(c["positions"], dtype=np.float64).reshape(-1, 3))
    return sk.Potential(s, c["gpts"][0], c["gpts"][1], slice_thicknesses=c["slice_thickness"],
                        parameterization=sk.LobatoParameterization(pi))


@pytest.mark.parametrize("name", ["A1", "A2", "D1"])
def test_device_potential_matches_pins(engine, name):
    c = G.case("slice-1", name)
    pot = _pot_from_case(c)
    assert list(pot.slice_of_atom) == c["slice_of_atom"]
    v = pot.build(engine).values
    for j in range(c["V_stored_slices"]):
        assert O.rel_max(v[j], G.array("slice-1", f"{name}.V.{j}")) <= 1e-11
    for j in range(len(c["slice_thickness"])):
        assert abs(np.max(np.abs(v[j])) - c["V_max_abs"][j]) <= 1e-10 * max(c["V_max_abs"][j], 1)


@pytest.mark.parametrize("name", ["A1", "D1"])
def test_device_transmission_matches_pins(engine, name):
    c = G.case("slice-1", name)
    pot = _pot_from_case(c)
    t = sk.Multislice.transmissionFunctions(pot, sk.ElectronBeam(c["energy"]), engine)[0]
    ref = G.array("slice-1", f"{name}.t.0")
    assert O.rel_max(t, ref) <= 1e-6  # complex64 storage of a float64 result


# ---- multislice (MultislicePinsTests.swift) ------------------------------------------------------------------------
@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("name,beam", [("A1", "plane"), ("D1", "plane"), ("D1", "probe")])
def test_exit_waves_match_pins(engine, name, beam, form):
    c = G.case("slice-1", name)
    b = c["beams"][beam]
    pot = _pot_from_case(c)
    grid = pot.grid
    ebeam = sk.ElectronBeam(c["energy"])
    if beam == "plane":
        inc = sk.Waves.plane_wave(ebeam, grid)
    else:
        probe = sk.Probe(ebeam, grid, sk.Aperture(b["cutoff_mrad"]))
        inc = probe.build(b["position"], engine)
        assert O.rel_max(inc.field, G.array("slice-1", f"{name}/{beam}.incident")) <= 2e-6
    ex = sk.Multislice.run(inc, pot, options=sk.ExecutionOptions(form=form), engine=engine)[-1]
    ref = G.array("slice-1", f"{name}/{beam}.exit.0")
    assert O.rel_l2(ex.field, ref) <= 1e-5
    assert O.rel_max(ex.field, ref) <= 1e-4


def test_probe_builder_aberrated(engine):
    c = G.case("slice-1", "B2")
    b = c["beams"]["probe"]
    grid = sk.Grid(c["gpts"][0], c["gpts"][1], c["box"][0], c["box"][1])
    ab = sk.Aberrations(**b["aberrations"])
    probe = sk.Probe(sk.ElectronBeam(c["energy"]), grid, sk.Aperture(b["cutoff_mrad"]), ab)
    got = probe.build(b["position"], engine).field
    assert O.rel_max(got, G.array("slice-1", "B2/probe.incident")) <= 2e-6
    # the device spectrum in float64 (Probe.centredSpectrum)
    og = O.Grid(grid.nx, grid.ny, grid.extent_x, grid.extent_y)
    spec = O.centred_spectrum(O.ProbeSpec(c["energy"], b["cutoff_mrad"], b["aberrations"]), og)
    assert O.rel_max(probe.centred_spectrum(engine), spec) <= 1e-12


def test_config1_hrtem_srtio3(engine):
    """SrTiO3 4x4x5 (400 atoms), 256^2, 10 slices of 1.9525 A, 200 keV plane wave: exit wave <= 1e-5 rel L2 (FP32)."""
    s = O.srtio3_cell().repeated(4, 4, 5)
    op = O.Potential.from_structure(s, 256, 256, slice_thickness=1.9525)
    og = op.grid
    ts = [O.transmission(v, 200e3, og) for v in op.build()]
    ref = O.multislice(O.plane_wave(og), ts, op.thicknesses, 200e3, og)[-1]
    pot = sk.Potential(sk.AtomicStructure(s.box, s.numbers, s.positions), 256, 256, slice_thickness=1.9525)
    for form in FORMS:
        ex = sk.Multislice.run(sk.Waves.plane_wave(sk.ElectronBeam(200e3), pot.grid), pot,
                               options=sk.ExecutionOptions(form=form), engine=engine)[-1]
        assert O.rel_l2(ex.field, ref) <= 1e-5, form
        assert O.rel_l2(np.abs(ex.field) ** 2, np.abs(ref) ** 2) <= 1e-5, form


def test_exit_planes_and_batch(engine):
    c = G.case("slice-1", "D1")
    pot = _pot_from_case(c)
    grid, ebeam = pot.grid, sk.ElectronBeam(c["energy"])
    inc = sk.Waves.plane_wave(ebeam, grid)
    outs = sk.Multislice.run(inc, pot, sk.ExitPlanes.every(3), engine=engine)
    assert len(outs) == 1 + len(sk.ExitPlanes.every(3).planes(10)) - 1
    probe = sk.Probe(ebeam, grid, sk.Aperture(25.0))
    incs = probe.build_many([(5.3, 7.9), (1.0, 2.0), (9.0, 3.5)], engine)
    batch = sk.Multislice.runBatch(incs, pot, engine=engine)
    for w, b in zip(incs, batch):
        single = sk.Multislice.run(w, pot, engine=engine)[-1]
        assert np.array_equal(single.field, b.field)  # a batch equals sequential runs, bit for bit


def _scan_case(name):
    s2 = G.pins()["slice-2"]
    c = s2["cases"][name]
    base = sk.AtomicStructure(tuple(c["box"]), np.array(c["numbers"], dtype=int),
                              np.array(c["positions"], dtype=np.float64).reshape(-1, 3))
    pots = []
    for k in range(c["num_configs"]):
        d = G.array("slice-2", f"{name}.displacement.{k}")
        s = sk.AtomicStructure(base.box, base.numbers, base.positions + d if len(d) else base.positions)
        pots.append(sk.Potential(s, c["gpts"][0], c["gpts"][1], slice_thickness=c["slice_thickness_requested"],
                                 parameterization=sk.LobatoParameterization("abTEMFloat32")))
    return s2, c, pots


def _detectors(meta):
    out = []
    for name, kind, p in meta:
        if kind == "annular":
            out.append((name, sk.AnnularDetector(p["inner"], p["outer"])))
        elif kind == "pixelated":
            out.append((name, sk.PixelatedDetector(p["max_angle"])))
        else:
            out.append((name, sk.SegmentedDetector(p["nbins_radial"], p["nbins_azimuthal"], p["inner"], p["outer"],
                                                   p["rotation"])))
    return out


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("name", ["S1", "S2", "S3"])
def test_stem_detectors_match_pins(engine, name, form):
    s2, c, pots = _scan_case(name)
    dets = _detectors(s2["detectors"])
    grid = pots[0].grid
    probe = sk.Probe(sk.ElectronBeam(c["energy"]), grid, sk.Aperture(c["cutoff_mrad"]))
    scan = sk.GridScan(tuple(c["scan"]["start"]), tuple(c["scan"]["end"]), *c["scan"]["gpts"])
    res = sk.STEM.scan(probe, pots, scan, [d for _, d in dets], options=sk.ExecutionOptions(form=form), engine=engine)
    sg = tuple(c["scan"]["gpts"])
    for (dname, d), m in zip(dets, res):
        meta = c["detectors"][dname]
        bound = 2e-4 * max(meta["scale"], 1e-5)
        if isinstance(d, sk.PixelatedDetector):
            arr = m.array()
            for q in meta["stored_positions"]:
                ref = G.array("slice-2", f"{name}.{dname}.position.{q[0]}.{q[1]}")
                assert np.max(np.abs(arr[q[0], q[1]] - ref)) <= bound, dname
                assert O.rel_l2(arr[q[0], q[1]], ref) <= 1e-4, dname
            assert np.max(np.abs(arr.reshape(sg + (-1,)).sum(-1) - np.array(meta["sums"]))) <= bound
        else:
            key = f"{name}.{dname}.float64" if isinstance(d, sk.SegmentedDetector) else f"{name}.{dname}"
            ref = G.array("slice-2", key)
            got = m.array().reshape(ref.shape)
            assert np.max(np.abs(got - ref)) <= bound, dname
            if np.max(np.abs(ref)) > 1e-3 * meta["scale"]:
                assert O.rel_l2(got, ref) <= 1e-4, dname


def test_com_detector_matches_pins(engine):
    meta = G.pins()["slice-4-scan"]
    box = meta["box"]
    s = O.al_fcc_cell()
    st = sk.AtomicStructure(s.box, s.numbers, s.positions).repeated(1, 1, 2)
    assert np.allclose(st.box, box)
    n = meta["gpts"]
    pot = sk.Potential(st, n, n, slice_thickness=meta["sliceThickness"],
                       parameterization=sk.LobatoParameterization("abTEMFloat32"))
    probe = sk.Probe(sk.ElectronBeam(meta["energy"]), pot.grid, sk.Aperture(meta["semiangle"]))
    scan = sk.GridScan(tuple(meta["scan"]["start"]), tuple(meta["scan"]["end"]), *meta["scan"]["gpts"])
    res = sk.STEM.scan(probe, [pot], scan, [sk.CenterOfMassDetector("cutoff", "mrad"),
                                            sk.CenterOfMassDetector("cutoff", "inverse"),
                                            sk.PixelatedDetector("cutoff")], engine=engine)
    dp = G.array("slice-4-scan", "dp")
    assert np.max(np.abs(res[2].array() - dp)) <= 2e-4 * np.max(dp)
    for m, key in zip(res[:2], ["com_mrad", "com_inv"]):
        ref = G.array("slice-4-scan", key)
        got = m.array()
        refv = np.stack([ref.real, ref.imag], axis=-1)
        assert np.max(np.abs(got - refv)) <= 2e-4 * np.max(np.abs(refv)), key


def test_scan_deterministic(engine):
    s2, c, pots = _scan_case("S2")
    grid = pots[0].grid
    probe = sk.Probe(sk.ElectronBeam(c["energy"]), grid, sk.Aperture(c["cutoff_mrad"]))
    scan = sk.GridScan((0.0, 0.0), (4.05, 4.05), 4, 4)
    dets = [sk.AnnularDetector(50, 120), sk.SegmentedDetector(2, 4, 0, 20)]
    a = sk.STEM.scan(probe, pots, scan, dets, engine=engine)
    b = sk.STEM.scan(probe, pots, scan, dets, engine=engine)
    for x, y in zip(a, b):
        assert np.array_equal(x.values, y.values)


def test_forms_agree_on_a_small_c2_scan(engine):
    """C2 shape at reduced size: SrTiO3, 20 slices of 3.905 A, 20 mrad probe, BF 0-20 and HAADF 50-200 mrad."""
    s = O.srtio3_cell().repeated(2, 2, 20)
    st = sk.AtomicStructure(s.box, s.numbers, s.positions)
    pot = sk.Potential(st, 128, 128, slice_thickness=3.905)
    probe = sk.Probe(sk.ElectronBeam(200e3), pot.grid, sk.Aperture(20.0))
    scan = sk.GridScan((3.905, 3.905), (2 * 3.905, 2 * 3.905), 6, 6)
    dets = [sk.AnnularDetector(0, 20), sk.AnnularDetector(50, 120)]
    # oracle
    op = O.Potential.from_structure(s, 128, 128, slice_thickness=3.905)
    ores = O.stem_scan(O.ProbeSpec(200e3, 20.0), [(op.grid, op.build(), op.thicknesses)], scan.positions,
                       [O.DetectorSpec("annular", {"inner": 0, "outer": 20}),
                        O.DetectorSpec("annular", {"inner": 50, "outer": 120})])
    for form in FORMS:
        res = sk.STEM.scan(probe, [pot], scan, dets, options=sk.ExecutionOptions(form=form), engine=engine)
        for m, r in zip(res, ores):
            assert O.rel_l2(m.values, r.ravel()) <= 1e-4, form


def test_refusals(engine):
    c = G.case("slice-1", "A1")
    pot = _pot_from_case(c)
    probe = sk.Probe(sk.ElectronBeam(200e3), pot.grid, sk.Aperture(20.0))
    scan = sk.GridScan((0.0, 0.0), (1.0, 1.0), 2, 2)
    with pytest.raises(sk.InvalidArgument):  # beyond the maximum simulated angle (Detectors.swift:108-117)
        sk.STEM.scan(probe, [pot], scan, [sk.AnnularDetector(0, 5000.0)], engine=engine)
    other = sk.Grid(64, 64, 10.0, 10.0)
    with pytest.raises(sk.InvalidArgument):
        sk.Multislice.run(sk.Waves.plane_wave(sk.ElectronBeam(200e3), other), pot, engine=engine)


@pytest.mark.parametrize("composite", [True, False])
@pytest.mark.parametrize("nx,ny", [(384, 384), (640, 384), (768, 768), (1536, 1536)])
def test_fused_mixed_radix_lengths(engine, nx, ny, composite):
    """The fused form's TMA passes at grid sides that are not powers of two, on the composite register engine (each line
    as 3 or 5 register-resident power-of-two transforms of its decimated sub-lines) and on the float32 shared-memory
    engine (radix 8/4/2 then 3 or 5): exit wave of a plane wave through SrTiO3 2x2x2 (4 slices) <= 1e-5 relative L2."""
    s = O.srtio3_cell().repeated(2, 2, 2)
    op = O.Potential.from_structure(s, nx, ny, slice_thickness=1.9525)
    og = op.grid
    ts = [O.transmission(v, 200e3, og) for v in op.build()]
    ref = O.multislice(O.plane_wave(og), ts, op.thicknesses, 200e3, og)[-1]
    pot = sk.Potential(sk.AtomicStructure(s.box, s.numbers, s.positions), nx, ny, slice_thickness=1.9525)
    ex = sk.Multislice.run(sk.Waves.plane_wave(sk.ElectronBeam(200e3), pot.grid), pot,
                           options=sk.ExecutionOptions(form="fused", composite=composite), engine=engine)[-1]
    assert O.rel_l2(ex.field, ref) <= 1e-5


@pytest.mark.parametrize("n,col_tile", [(768, 4), (768, 2), (384, 8), (640, 4)])
def test_composite_engine_scan(engine, n, col_tile):
    """A probe scan at a side 3 or 5 times a power of two on the composite register engine: the probes' row passes,
    the slices' row and column passes and the last column pass with the detectors in its epilogue (annular, centre of
    mass) against the float64 oracle (annular <= 1e-4, centre of mass <= 1e-3 relative L2) and against the
    shared-memory engine (annular <= 5e-6, centre of mass <= 1e-4)."""
    s = O.srtio3_cell().repeated(2, 2, 2)
    st = sk.AtomicStructure(s.box, s.numbers, s.positions)
    pot = sk.Potential(st, n, n, slice_thickness=1.9525)
    probe = sk.Probe(sk.ElectronBeam(200e3), pot.grid, sk.Aperture(20.0))
    scan = sk.GridScan((1.0, 1.0), (4.0, 4.0), 3, 3)
    dets = [sk.AnnularDetector(0, 20), sk.AnnularDetector(40, 120), sk.CenterOfMassDetector("cutoff", "mrad")]
    out = {}
    for composite in (True, False):
        opts = sk.ExecutionOptions(form="fused", composite=composite, col_tile=col_tile)
        out[composite] = sk.STEM.scan(probe, [pot], scan, dets, options=opts, engine=engine)
    op = O.Potential.from_structure(s, n, n, slice_thickness=1.9525)
    ores = O.stem_scan(O.ProbeSpec(200e3, 20.0), [(op.grid, op.build(), op.thicknesses)], scan.positions,
                       [O.DetectorSpec("annular", {"inner": 0, "outer": 20}),
                        O.DetectorSpec("annular", {"inner": 40, "outer": 120}),
                        O.DetectorSpec("com", {"mode": "cutoff", "units": "mrad"})])
    for (a, b, r), (to, te) in zip(zip(out[True], out[False], ores), [(1e-4, 5e-6), (1e-4, 5e-6), (1e-3, 1e-4)]):
        e_o, e_e = O.rel_l2(a.values, r.ravel()), O.rel_l2(a.values, b.values)
        print(f"{n}^2 tile {col_tile}: composite vs float64 {e_o:.2e}, vs shared-memory engine {e_e:.2e}")
        assert e_o <= to and e_e <= te


@pytest.mark.parametrize("n", [512, 256, 1024])
def test_column_pairs(engine, n):
    """The column pass on column pairs (8-column tiles at 512 and 1024, 16 at 256, one thread per pair of adjacent
    columns: the slices' passes, the probes' generation from their spectrum and the last pass with the detector epilogue
    or the k-space store) against the one-column-a-thread pass and the float64 oracle: a plane-wave exit wave (<= 1e-5 against
    float64; the two passes run the same butterflies and twiddles per column, but the compiler's fused multiply-adds
    may differ, so they agree to float32 rounding, <= 1e-6) and a probe scan with annular, centre-of-mass and
    pixelated detectors (<= 1e-4 / 1e-3 against float64, <= 1e-6 between the passes)."""
    s = O.srtio3_cell().repeated(2, 2, 2)
    st = sk.AtomicStructure(s.box, s.numbers, s.positions)
    op = O.Potential.from_structure(s, n, n, slice_thickness=1.9525)
    og = op.grid
    ts = [O.transmission(v, 200e3, og) for v in op.build()]
    ref = O.multislice(O.plane_wave(og), ts, op.thicknesses, 200e3, og)[-1]
    pot = sk.Potential(st, n, n, slice_thickness=1.9525)
    waves = {}
    for paired in (True, False):
        opts = sk.ExecutionOptions(form="fused", paired=paired)
        waves[paired] = sk.Multislice.run(sk.Waves.plane_wave(sk.ElectronBeam(200e3), pot.grid), pot, options=opts,
                                          engine=engine)[-1].field
    e_ref, e_pair = O.rel_l2(waves[True], ref), O.rel_l2(waves[True], waves[False])
    print(f"{n}^2 exit wave: pairs vs float64 {e_ref:.2e}, vs single columns {e_pair:.2e}, "
          f"identical {np.array_equal(waves[True], waves[False])}")
    assert e_ref <= 1e-5 and e_pair <= 1e-6
    probe = sk.Probe(sk.ElectronBeam(200e3), pot.grid, sk.Aperture(20.0))
    scan = sk.GridScan((1.0, 1.0), (4.0, 4.0), 3, 3)
    dets = [sk.AnnularDetector(0, 20), sk.AnnularDetector(50, 120), sk.CenterOfMassDetector("cutoff", "mrad")]
    pix = [sk.PixelatedDetector("cutoff")]
    out = {}
    for paired in (True, False):
        opts = sk.ExecutionOptions(form="fused", paired=paired)
        out[paired] = (sk.STEM.scan(probe, [pot], scan, dets, options=opts, engine=engine),
                       sk.STEM.scan(probe, [pot], scan, dets + pix, options=opts, engine=engine))
    ores = O.stem_scan(O.ProbeSpec(200e3, 20.0), [(og, op.build(), op.thicknesses)], scan.positions,
                       [O.DetectorSpec("annular", {"inner": 0, "outer": 20}),
                        O.DetectorSpec("annular", {"inner": 50, "outer": 120}),
                        O.DetectorSpec("com", {"mode": "cutoff", "units": "mrad"})])
    for k in range(2):  # channel detectors in the epilogue; with a pixelated detector, from the stored k-space waves
        for a, b, r, to in zip(out[True][k], out[False][k], ores, (1e-4, 1e-4, 1e-3)):
            e_o, e_e = O.rel_l2(a.values, np.asarray(r).ravel()), O.rel_l2(a.values, b.values)
            print(f"{n}^2 scan {k}: pairs vs float64 {e_o:.2e}, vs single columns {e_e:.2e}")
            assert e_o <= to and e_e <= 1e-6
    e_pix = O.rel_l2(out[True][1][-1].values, out[False][1][-1].values)
    print(f"{n}^2 pixelated: pairs vs single columns {e_pix:.2e}")
    assert e_pix <= 1e-6
