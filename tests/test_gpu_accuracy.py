"""Every form against float64 at the configurations the reference checks its float32 device path on.

- The STEM HAADF+BF workload itself (SrTiO3 8x8x20, 512^2, 20 slices of 3.905 A, 200 keV, 20 mrad, BF 0-20 and HAADF
  50-200 mrad) at 16 positions over the central unit cell, plain, fused and bf16x3 against the C++ float64 restatement
  of STEM.cpuScan: <= 1e-4 relative L2 on each detector image.
- The reference's float32-against-float64 check of every exit plane (Tests/SimulatoKitParityTests/Multislice/
  MetalTests.swift:30-47, bounds MetalAccuracy.registered, Sources/SimulatoMultislice/ExecutionOptions.swift:55-94):
  exit wave 1e-4, intensity 2e-4, diffraction pattern 2e-4 (each x the reference array's maximum) and total intensity
  sum |psi|^2 within 1.5e-6 per slice, on the pinned cases A1, A2, B1, B2, C1 and D1 with their exit planes, and on the
  Al 8x8x50 crystal at 512^2 with 100 slices (plane wave and a 25 mrad probe at 30 A defocus, every 25 slices).
- Any grid size and beam tilt (GridSamplingAndTiltTests.swift, fixtures slice-4): the 90 x 75 grid with tilted and
  untilted plane waves and probes, against the reference's abTEM exit waves at the registered float32 wave bound.

The measured errors are printed (pytest -s).
"""

import numpy as np
import pytest

import golden_io as G
from oracle import simk_oracle as O

pytestmark = pytest.mark.gpu

sk = pytest.importorskip("simulatokit_b200")

# MetalAccuracy.registered (ExecutionOptions.swift:55-94)
WAVE, INTENSITY, PATTERN, TOTAL_PER_SLICE = 1e-4, 2e-4, 2e-4, 1.5e-6
TC_SIDES = (256, 512, 768, 1024, 2048)


@pytest.fixture(scope="module")
def engine():
    return sk.Engine.require()


def _forms(grid):
    forms = ["plain", "fused"]
    if grid.nx in TC_SIDES and grid.ny in TC_SIDES:
        forms.append("bf16x3")
    return forms


# ---- the STEM HAADF+BF workload at its full size ----------------------------------------------------------------------
@pytest.fixture(scope="module")
def c2_reference():
    from oracle import simk_cpu as K
    s = O.srtio3_cell().repeated(8, 8, 20)
    thicknesses = O.slice_thicknesses(s.box[2], 3.905)
    assert len(thicknesses) == 20
    inputs = K.ScanInputs.from_structure(O.ProbeSpec(200e3, 20.0), s, 512, 512, thicknesses, [(0, 20), (50, 200)])
    scan = sk.GridScan((4 * 3.905, 4 * 3.905), (5 * 3.905, 5 * 3.905), 4, 4)
    return s, scan, inputs.scan(scan.positions, threads=8)


@pytest.mark.parametrize("form", ["plain", "fused", "bf16x3"])
def test_stem_workload_full_size(engine, c2_reference, form):
    s, scan, ref = c2_reference
    pot = sk.Potential(sk.AtomicStructure(s.box, s.numbers, s.positions), 512, 512, slice_thickness=3.905)
    probe = sk.Probe(sk.ElectronBeam(200e3), pot.grid, sk.Aperture(20.0))
    res = sk.STEM.scan(probe, [pot], scan, [sk.AnnularDetector(0, 20), sk.AnnularDetector(50, 200)],
                       options=sk.ExecutionOptions(form=form), engine=engine)
    errs = [O.rel_l2(m.values, ref[:, d]) for d, m in enumerate(res)]
    print(f"STEM workload 512^2 x 20 slices, 16 positions, {form}: BF {errs[0]:.2e}, HAADF {errs[1]:.2e}")
    assert max(errs) <= 1e-4


# ---- every exit plane against float64 (MetalTests.swift) ---------------------------------------------------------------
def _compare_planes(engine, form, incident, pot, ts, thicknesses, planes, plane_wave, label):
    """The device run at `planes` against the float64 oracle on the same incident wave and transmissions; returns the
    worst (wave, intensity, pattern, total per slice)."""
    g = O.Grid(pot.grid.nx, pot.grid.ny, pot.grid.extent_x, pot.grid.extent_y)
    energy = incident.beam.energy
    ref = O.multislice(incident.field, ts, thicknesses, energy, g, planes=list(planes), tilt=tuple(incident.tilt))
    got = sk.Multislice.run(incident, pot, sk.ExitPlanes.after_slices(list(planes)),
                            options=sk.ExecutionOptions(form=form), engine=engine)
    assert len(got) == len(ref) == len(planes)
    worst = [0.0, 0.0, 0.0, 0.0]
    for a, b, plane in zip(got, ref, planes):
        w = O.rel_max(a.field, b)
        i = O.rel_max(np.abs(a.field) ** 2, np.abs(b) ** 2)
        p = O.rel_max(O.diffraction_pattern(a.field, g, plane_wave), O.diffraction_pattern(b, g, plane_wave))
        tb = float(np.sum(np.abs(b) ** 2))
        t = abs(float(np.sum(np.abs(a.field) ** 2)) - tb) / tb
        assert w <= WAVE, f"{label} {form} plane {plane}: exit wave {w:.2e}"
        assert i <= INTENSITY, f"{label} {form} plane {plane}: intensity {i:.2e}"
        assert p <= PATTERN, f"{label} {form} plane {plane}: pattern {p:.2e}"
        assert t <= TOTAL_PER_SLICE * (plane + 1), f"{label} {form} plane {plane}: total intensity {t:.2e}"
        worst = [max(worst[0], w), max(worst[1], i), max(worst[2], p),
                 max(worst[3], t / (plane + 1) if plane >= 0 else 0.0)]
    print(f"{label} {form}: wave {worst[0]:.2e}, intensity {worst[1]:.2e}, pattern {worst[2]:.2e}, "
          f"total per slice {worst[3]:.2e}")
    return worst


PINNED = [("A1", "plane"), ("A2", "plane"), ("B1", "plane"), ("B2", "probe"), ("C1", "plane"), ("C1", "probe"),
          ("D1", "plane"), ("D1", "probe")]


@pytest.mark.parametrize("name,beam", PINNED)
def test_every_exit_plane_of_the_pinned_cases(engine, name, beam):
    c = G.case("slice-1", name)
    b = c["beams"][beam]
    s = sk.AtomicStructure(tuple(c["box"]), np.array(c["numbers"], dtype=int),
                           np.array(c["positions"], dtype=np.float64).reshape(-1, 3))
    pot = sk.Potential(s, c["gpts"][0], c["gpts"][1], slice_thicknesses=c["slice_thickness"],
                       parameterization=sk.LobatoParameterization("exact"))
    ebeam = sk.ElectronBeam(c["energy"])
    if beam == "plane":
        inc = sk.Waves.plane_wave(ebeam, pot.grid)
    else:
        probe = sk.Probe(ebeam, pot.grid, sk.Aperture(b["cutoff_mrad"]), sk.Aberrations(**b.get("aberrations", {})))
        inc = probe.build(b["position"], engine)
    g = O.Grid(pot.grid.nx, pot.grid.ny, pot.grid.extent_x, pot.grid.extent_y)
    # the device's float64 potential (pinned at 1e-11 by test_gpu_parity) is the input of both sides, as the reference
    # gives one ProjectedPotential to both backends
    vs = pot.build(engine).values
    ts = [O.transmission(v, c["energy"], g) for v in vs]
    for form in _forms(pot.grid):
        _compare_planes(engine, form, inc, pot, ts, c["slice_thickness"], c["exit_planes"], beam == "plane",
                        f"{name}/{beam}")


@pytest.fixture(scope="module")
def al_512(engine):
    s = O.al_fcc_cell()
    st = sk.AtomicStructure(s.box, s.numbers, s.positions).repeated(8, 8, 50)
    pot = sk.Potential(st, 512, 512, slice_thickness=2.025)
    assert pot.slice_count == 100
    g = O.Grid(512, 512, pot.grid.extent_x, pot.grid.extent_y)
    ts = [O.transmission(v, 300e3, g) for v in pot.build(engine).values]
    return pot, ts


@pytest.mark.parametrize("form", ["plain", "fused", "bf16x3"])
@pytest.mark.parametrize("beam", ["plane", "probe"])
def test_every_exit_plane_512_squared_100_slices(engine, al_512, form, beam):
    """MetalTests.swift:58-76: Al 8x8x50 at 512^2, 100 slices of 2.025 A, 300 keV, every 25 slices."""
    pot, ts = al_512
    ebeam = sk.ElectronBeam(300e3)
    if beam == "plane":
        inc = sk.Waves.plane_wave(ebeam, pot.grid)
    else:
        probe = sk.Probe(ebeam, pot.grid, sk.Aperture(25.0), sk.Aberrations(C10=-30.0))  # defocus 30 A = -C10
        inc = probe.build((15.3, 16.9), engine)
    planes = sk.ExitPlanes.every(25).planes(100)
    _compare_planes(engine, form, inc, pot, ts, [2.025] * 100, planes, beam == "plane", f"Al 512^2 {beam}")


# ---- any grid size and beam tilt (GridSamplingAndTiltTests.swift) ------------------------------------------------------
@pytest.fixture(scope="module")
def slice4():
    meta = G.pins()["slice-4"]
    nums = np.array([a[0] for a in meta["atoms"]], dtype=int)
    pos = np.array([a[1] for a in meta["atoms"]], dtype=np.float64)
    s = sk.AtomicStructure(tuple(meta["box"]), nums, pos)
    nx, ny = meta["gpts"]
    pot = sk.Potential(s, nx, ny, slice_thickness=meta["sliceThickness"],
                       parameterization=sk.LobatoParameterization("abTEMFloat32"))
    return meta, pot


def _slice4_incident(engine, meta, pot, run):
    beam = sk.ElectronBeam(meta["energy"])
    tilt = tuple(meta["runs"][run]["tilt"])
    if run.startswith("plane"):
        return sk.Waves.plane_wave(beam, pot.grid, tilt=tilt)
    probe = sk.Probe(beam, pot.grid, sk.Aperture(20.0), tilt=tilt)
    return probe.build(tuple(meta["probePosition"]), engine)


@pytest.mark.parametrize("form", ["plain", "fused"])
@pytest.mark.parametrize("run", ["plane0", "planeT", "probe0", "probeT"])
def test_odd_grid_and_tilt_match_abtem(engine, slice4, run, form):
    """exitWavesOnAnOddGridMatchAbTEM / metalMatchesCPUOnAnOddGridWithTilt: 90 x 75 (mixed radix on x, Bluestein-free
    odd length on y), 6 slices of 2.025 A at 200 keV; the device exit wave against abTEM's at the float32 wave bound."""
    meta, pot = slice4
    assert (pot.grid.nx, pot.grid.ny) == (90, 75)
    inc = _slice4_incident(engine, meta, pot, run)
    ex = sk.Multislice.run(inc, pot, options=sk.ExecutionOptions(form=form), engine=engine)[-1]
    assert tuple(ex.tilt) == tuple(meta["runs"][run]["tilt"])
    e = O.rel_max(ex.field, G.array("slice-4", run))
    print(f"slice-4 {run} {form}: rel max {e:.2e}")
    assert e <= WAVE


def test_tilt_moves_the_exit_wave(engine, slice4):
    """tiltChangesTheExitWave: a 1.5 mrad tilt moves the device's exit wave by more than 1e-3 of its maximum."""
    meta, pot = slice4
    a = sk.Multislice.run(_slice4_incident(engine, meta, pot, "planeT"), pot, engine=engine)[-1].field
    b = sk.Multislice.run(_slice4_incident(engine, meta, pot, "plane0"), pot, engine=engine)[-1].field
    assert O.rel_max(a, b) > 1e-3


@pytest.mark.parametrize("form", ["plain", "fused"])
def test_tilted_scan_matches_float64(engine, slice4, form):
    """A STEM scan with a tilted probe (the tilt enters every slice's propagator) against the float64 oracle."""
    meta, pot = slice4
    g = O.Grid(pot.grid.nx, pot.grid.ny, pot.grid.extent_x, pot.grid.extent_y)
    tilt = (2.0, 1.0)
    probe = sk.Probe(sk.ElectronBeam(meta["energy"]), pot.grid, sk.Aperture(20.0), tilt=tilt)
    scan = sk.GridScan((0.0, 0.0), (4.05, 4.05), 3, 3)
    dets = [sk.AnnularDetector(0, 20), sk.AnnularDetector(40, 100)]
    res = sk.STEM.scan(probe, [pot], scan, dets, options=sk.ExecutionOptions(form=form), engine=engine)
    vs = pot.build(engine).values
    ores = O.stem_scan(O.ProbeSpec(meta["energy"], 20.0, tilt=tilt), [(g, vs, pot.slice_thicknesses)], scan.positions,
                       [O.DetectorSpec("annular", {"inner": 0, "outer": 20}),
                        O.DetectorSpec("annular", {"inner": 40, "outer": 100})])
    for m, r in zip(res, ores):
        assert O.rel_l2(m.values, np.asarray(r).ravel()) <= 1e-4
