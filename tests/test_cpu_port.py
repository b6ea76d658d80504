"""The C++ float64 restatement of the reference's CPU scan path (oracle/cpu/simk_cpu.cpp), which the benchmark times as
the CPU baseline: its FFT path selection against the reference's pinned lengths and cost rule
(Tests/SimulatoCoreTests/SimulatoCoreTests.swift:57-81), its transforms against NumPy's, and its scan against the NumPy
oracle. CPU only."""

import math

import numpy as np
import pytest

from oracle import simk_cpu as K
from oracle import simk_oracle as O


def test_lengths_pick_their_fft_path():
    # SimulatoCoreTests.lengthsPickTheirFFTPath: vDSP's lengths, the mixed-radix ones and the Bluestein ones
    assert K.fft_path(256) == "direct" and K.fft_path(480) == "direct"
    for n in [2, 3, 6, 7, 11, 13, 45, 47, 49, 90, 100, 250, 496, 500, 506, 1000, 1001]:
        assert K.fft_path(n) == "mixedRadix", n
    for n in [97, 106, 127, 509, 514, 1009]:
        assert K.fft_path(n) == "bluestein", n


def test_mixed_radix_cost_rule_is_pocketffts():
    # SimulatoCoreTests.mixedRadixCostRuleIsPocketffts
    assert K.factorization(506) == [2, 11, 23]
    assert K.factorization(1000) == [2, 4, 5, 5, 5]
    assert K.factorization(1) is None
    assert abs(K.cost_guess(506) - (2 + 1.1 * 11 + 1.1 * 23) * 506) < 1e-9
    assert K.cost_guess(1024) == 20 * 1024
    assert K.fft_path(47) != "bluestein"      # below 50
    assert K.fft_path(1001) != "bluestein"    # 13 <= sqrt(1001)


@pytest.mark.parametrize("nx,ny", [(1, 1), (2, 3), (8, 8), (12, 20), (15, 21), (45, 49), (67, 64), (77, 52),
                                   (97, 106), (128, 96), (250, 6), (509, 4), (1536, 16), (131, 257)])
def test_fft2_matches_numpy(nx, ny):
    rng = np.random.default_rng(nx * 1000 + ny)
    a = rng.standard_normal((2, nx, ny)) + 1j * rng.standard_normal((2, nx, ny))
    f, r = K.fft2(a), np.fft.fft2(a)
    assert np.abs(f - r).max() <= 1e-13 * np.abs(r).max()
    b, rb = K.fft2(a, inverse=True), np.fft.ifft2(a)
    assert np.abs(b - rb).max() <= 1e-13 * np.abs(rb).max()
    # the round trip returns the input (SimulatoCoreTests' forward / inverse bound is 1e-7)
    assert np.abs(K.fft2(f, inverse=True) - a).max() <= 1e-12 * np.abs(a).max()


def _case(nx, ny, thicknesses=None):
    s = O.srtio3_cell().repeated(2, 2, 2)
    if thicknesses is None:
        op = O.Potential.from_structure(s, nx, ny, slice_thickness=1.9525)
    else:
        op = O.Potential.from_structure(s, nx, ny, thicknesses=thicknesses)
    return op


@pytest.mark.parametrize("nx,ny,thicknesses", [(64, 48, None), (45, 53, [1.9525, 1.9525, 3.905, 0.5, 1.3025])])
def test_scan_matches_numpy_oracle(nx, ny, thicknesses):
    op = _case(nx, ny, thicknesses)
    g = op.grid
    spec = O.ProbeSpec(200e3, 20.0)
    vs = op.build()
    pos = O.grid_scan_positions((0.0, 0.0), (3.905, 3.905), 3, 3)
    dets = [(0.0, 20.0), (30.0, 60.0)]
    ores = O.stem_scan(spec, [(g, vs, op.thicknesses)], pos,
                       [O.DetectorSpec("annular", {"inner": a, "outer": b}) for a, b in dets])
    ts = [O.transmission(v, 200e3, g) for v in vs]
    si = K.ScanInputs(spec, g, ts, op.thicknesses, K.annular_masks(g, 200e3, dets))
    one = si.scan(pos, threads=1)
    for d in range(len(dets)):
        r = np.asarray(ores[d]).ravel()
        assert np.abs(one[:, d] - r).max() <= 1e-12 * np.abs(r).max()
    # positions over threads are bit-equal to the sequential run (runCPUParallel's property)
    assert np.array_equal(si.scan(pos, threads=3), one)
    assert np.array_equal(si.scan(pos[4:5], threads=1)[0], one[4])


def test_scan_refuses_bad_arguments():
    op = _case(16, 16)
    g = op.grid
    spec = O.ProbeSpec(200e3, 20.0)
    ts = [O.transmission(v, 200e3, g) for v in op.build()]
    si = K.ScanInputs(spec, g, ts, op.thicknesses, K.annular_masks(g, 200e3, [(0.0, 10.0)]))
    assert si.scan(np.zeros((0, 2))).shape == (0, 1)
    with pytest.raises(ValueError):
        K.fft2(np.zeros((0, 4), dtype=complex))


# ---- the per-potential set-up in C++ --------------------------------------------------------------------------------

def test_setup_stages_match_numpy():
    s = O.srtio3_cell().repeated(2, 2, 2)
    for pi in ("exact", "abtem"):
        op = O.Potential.from_structure(s, 64, 48, slice_thickness=1.9525, pi_choice=pi)
        assert O.rel_max(K.potential(s, 64, 48, op.thicknesses, pi), np.array(op.build())) <= 1e-13
    g = op.grid
    v = op.build()[0]
    assert O.rel_max(K.transmission(v, 200e3, g), O.transmission(v, 200e3, g)) <= 1e-13
    for tilt in ((0.0, 0.0), (3.0, -2.0)):
        assert O.rel_max(K.propagator(g, 200e3, 1.9525, tilt), O.propagator(g, 200e3, 1.9525, tilt)) <= 1e-13
    for ab, soft, semi in [({}, True, 20.0), ({}, False, 20.0), ({}, True, math.inf),
                           ({"C10": -50.0, "C30": 1e4, "C12": 20.0, "phi12": 0.3, "C23": 100.0, "phi23": 0.5,
                             "C50": 1e6}, True, 25.0)]:
        p = O.ProbeSpec(200e3, semi, ab, soft)
        assert O.rel_max(K.probe_spectrum(p, g), O.centred_spectrum(p, g)) <= 1e-13
    assert np.array_equal(K.annular_mask(g, 200e3, 30.0, 60.0), O.annular_mask(g, 200e3, 30.0, 60.0).astype(float))
    gen = O.GaussianGenerator(7)
    assert np.array_equal(K.normals(7, 9), np.array([gen.next_normal() for _ in range(9)]))


@pytest.mark.parametrize("name", ["A1", "D1"])
def test_cpp_potential_is_pinned_to_the_reference(name):
    # the reference's abTEM fixtures at its own bound (PotentialPinsTests.swift: 1e-11 with abTEM's float32 pi)
    import golden_io as G
    c = G.case("slice-1", name)
    s = O.Structure(tuple(c["box"]), np.array(c["numbers"], dtype=int),
                    np.array(c["positions"], dtype=np.float64).reshape(-1, 3))
    v = K.potential(s, c["gpts"][0], c["gpts"][1], c["slice_thickness"], "abtem")
    for j in range(c["V_stored_slices"]):
        assert O.rel_max(v[j], G.array("slice-1", f"{name}.V.{j}")) <= 1e-11


def test_a_scan_built_in_cpp_matches_the_oracle():
    s = O.srtio3_cell().repeated(2, 2, 2)
    op = O.Potential.from_structure(s, 64, 48, slice_thickness=1.9525)
    spec = O.ProbeSpec(200e3, 20.0, {"C10": -30.0})
    dets = [(0.0, 20.0), (30.0, 60.0)]
    pos = O.grid_scan_positions((0.0, 0.0), (3.905, 3.905), 3, 3)
    ores = O.stem_scan(spec, [(op.grid, op.build(), op.thicknesses)], pos,
                       [O.DetectorSpec("annular", {"inner": a, "outer": b}) for a, b in dets])
    got = K.ScanInputs.from_structure(spec, s, 64, 48, op.thicknesses, dets).scan(pos, threads=2)
    for d in range(len(dets)):
        r = np.asarray(ores[d]).ravel()
        assert np.abs(got[:, d] - r).max() <= 1e-12 * np.abs(r).max()
