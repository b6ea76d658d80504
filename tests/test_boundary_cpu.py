"""CPU-only checks of the boundary and the host logic: the C ABI library loads and exports every symbol the header
declares, host-only entry points answer without a device, and the Python mirror of the reference's host types (slicing,
exit planes, scan positions, frozen-phonon generator, detector shapes) agrees with the oracle."""

import ctypes as C
import os
import re

import numpy as np
import pytest

import golden_io as G
from oracle import simk_oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "simulato_cuda.h")


def _header_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(simk_\w+)\(", text, flags=re.M)))


@pytest.fixture(scope="module")
def lib():
    from simulatokit_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        from simulatokit_b200 import build
        build.build()
    return _lib.lib()


def test_library_exports_every_header_symbol(lib):
    syms = _header_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(lib, s), s
    from simulatokit_b200 import _lib
    assert sorted(_lib.EXPORTED) == syms


def test_no_device_is_reported_cleanly_or_a_device_is_found(lib):
    n = C.c_int32(-1)
    st = lib.simk_cuda_available(C.byref(n))
    assert st in (0, 3)
    if st == 3:
        assert n.value == 0
        assert b"device" in lib.simk_last_error()


def test_detector_shapes_host_only(lib):
    import simulatokit_b200 as sk
    g = sk.Grid(128, 128, 8.1, 8.1)
    og = O.Grid(128, 128, 8.1, 8.1)
    assert sk.detector_shape(sk.AnnularDetector(0, 20), g, 200e3) == []
    for mode in ("cutoff", "valid", "full"):
        assert sk.detector_shape(sk.PixelatedDetector(mode), g, 200e3) == list(O.pixelated_size(og, mode))
    assert sk.detector_shape(sk.CenterOfMassDetector(), g, 200e3) == [2]
    assert sk.detector_shape(sk.SegmentedDetector(2, 4, 0, 20), g, 200e3) == [2, 4]
    assert O.pixelated_size(og, "cutoff") == (86, 86) and O.pixelated_size(og, "valid") == (60, 60)


def test_slicing_and_wrapping_match_the_oracle():
    import simulatokit_b200 as sk
    for name in ("A1", "A2", "D1", "B1"):
        c = G.case("slice-1", name)
        s = sk.AtomicStructure(tuple(c["box"]), np.array(c["numbers"], dtype=int),
                               np.array(c["positions"], dtype=np.float64).reshape(-1, 3))
        p = sk.Potential(s, c["gpts"][0], c["gpts"][1], slice_thickness=c["slice_thickness_requested"])
        assert p.slice_thicknesses == c["slice_thickness"]
        assert list(p.slice_of_atom) == c["slice_of_atom"]


def test_exit_planes():
    import simulatokit_b200 as sk
    assert sk.ExitPlanes.last().planes(10) == [9]
    assert sk.ExitPlanes.every(2).planes(20) == G.case("slice-1", "B1")["exit_planes"]
    assert sk.ExitPlanes.every(1).planes(10) == G.case("slice-1", "C1")["exit_planes"]
    assert sk.ExitPlanes.after_slices([-1, 3]).planes(10) == [-1, 3, 9]
    with pytest.raises(sk.InvalidArgument):
        sk.ExitPlanes.after_slices([3, 1]).planes(10)
    with pytest.raises(sk.InvalidArgument):
        sk.ExitPlanes.every(0).planes(10)


def test_grid_scan_positions():
    import simulatokit_b200 as sk
    c = G.pins()["slice-2"]["cases"]["S1"]
    scan = sk.GridScan(tuple(c["scan"]["start"]), tuple(c["scan"]["end"]), *c["scan"]["gpts"])
    assert np.array_equal(scan.positions.reshape(6, 6, 2), G.array("slice-2", "S1.scan_positions"))


def test_frozen_phonon_generator_matches_the_oracle():
    import simulatokit_b200 as sk
    s = O.silicon_cell().repeated(2, 2, 2)
    st = sk.AtomicStructure(s.box, s.numbers, s.positions)
    fp = sk.FrozenPhonons(st, sigmas={14: 0.075}, configurations=3, seed=1)
    ref = O.frozen_displacements(s.numbers, {14: 0.075}, 3, 1)
    for a, b in zip(fp.displacements, ref):
        assert np.array_equal(a, b)


def test_host_refusals():
    import simulatokit_b200 as sk
    with pytest.raises(sk.InvalidArgument):
        sk.Grid(1, 8, 1.0, 1.0)
    with pytest.raises(sk.InvalidArgument):
        sk.ElectronBeam(-1.0)
    with pytest.raises(sk.InvalidArgument):
        sk.AnnularDetector(5.0, 2.0)
    with pytest.raises(sk.InvalidArgument):
        sk.SegmentedDetector(0, 4, 0, 20)
    with pytest.raises(sk.InvalidArgument):
        sk.GridScan((0.0, 0.0), (0.0, 0.0), 2, 2)
    s = sk.AtomicStructure((4.0, 4.0, 4.0), [200], [[0, 0, 0]])
    with pytest.raises(sk.InvalidArgument):
        sk.Potential(s, 16, 16, slice_thickness=1.0)
    with pytest.raises(sk.InvalidArgument):
        sk.Potential(sk.AtomicStructure((4.0, 4.0, 4.0), [6], [[0, 0, 0]]), 16, 16, slice_thicknesses=[1.0, 1.0])


def test_beam_matches_pins():
    import simulatokit_b200 as sk
    for row in G.pins()["slice-1"]["beam"]:
        b = sk.ElectronBeam(row["energy"])
        assert b.wavelength == row["wavelength"]
        assert abs(b.interaction_parameter - row["sigma"]) <= 1e-15 * row["sigma"]


def test_waves_detector_refusals_on_the_host():
    """WavesDetector(rows:columns:) and STEM.scan's waves refusals (WavesDetector.swift:41-48, 115-131) need no device."""
    import simulatokit_b200 as sk
    from oracle import simk_oracle as O
    with pytest.raises(sk.InvalidArgument):
        sk.WavesDetector(1, 8)
    with pytest.raises(sk.InvalidArgument):
        sk.WavesDetector(8, None)
    s = O.al_fcc_cell()
    st = sk.AtomicStructure(s.box, s.numbers, s.positions)
    pots = [sk.Potential(st, 48, 48, slice_thickness=2.025) for _ in range(2)]
    probe = sk.Probe(sk.ElectronBeam(200e3), pots[0].grid, sk.Aperture(20.0))
    scan = sk.GridScan((0.0, 0.0), (4.05, 4.05), 3, 2)
    with pytest.raises(sk.InvalidArgument, match="one potential, got 2"):
        sk.STEM.scan(probe, pots, scan, sk.WavesDetector())
    with pytest.raises(sk.InvalidArgument, match="one potential, got 0"):
        sk.STEM.scan(probe, [], scan, sk.WavesDetector())


def test_ctf_closed_forms_on_the_host():
    """Scherzer defocus, point resolution and Nyquist sampling (ContrastTransferFunction.swift:118-142) against the
    reference's pins at 1e-15, and its textbook values (CTFTests.closedFormsEqualAbTEMAndTheTextbook)."""
    import simulatokit_b200 as sk
    CTF = sk.ContrastTransferFunction
    s3 = G.pins()["slice-3"]
    for row in s3["closed_forms"]:
        assert abs(CTF.scherzer_defocus(row["Cs"], row["energy"]) - row["scherzer"]) <= 1e-15 * abs(row["scherzer"])
        assert abs(CTF.point_resolution(row["Cs"], row["energy"]) - row["point_resolution"]) <= \
            1e-15 * row["point_resolution"]
    for row in s3["nyquist"]:
        assert abs(CTF.nyquist_sampling(row["semiangle"], row["energy"]) - row["sampling"]) <= 1e-15 * row["sampling"]
    assert abs(CTF.scherzer_defocus(1.2e7, 200e3) - 671.9) < 0.05
    assert abs(CTF.point_resolution(1.2e7, 200e3) - 2.370) < 0.0005
    assert abs(CTF.nyquist_sampling(20, 200e3) - 0.3135) < 0.00005
    with pytest.raises(sk.InvalidArgument):
        CTF(focal_spread=-1.0)
