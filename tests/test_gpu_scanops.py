"""Scan post-processing on the device through the C ABI: the Gaussian source size bit-equal to the oracle (and so to
the reference's float64 loop) and within the reference's 1e-7 of scipy's fixtures; Poisson noise bit-equal to the
oracle's restatement of the per-value streams, with the reference's own statistical, seeding and clipping checks; the
integrated gradient and iCOM against abTEM's fixtures at assert_allclose's rtol 1e-7 (atol 1e-12 of the largest
value), and iCOM of the device's own centre-of-mass scan kept on the device
(Tests/SimulatoKitParityTests/Detector/ScanPatternsAndNoiseTests.swift, IcomPinsTests.swift)."""

import ctypes as C
import math

import numpy as np
import pytest

import golden_io as G
from oracle import simk_oracle as O

pytestmark = pytest.mark.gpu

sk = pytest.importorskip("simulatokit_b200")
torch = pytest.importorskip("torch")

from simulatokit_b200 import _lib as L  # noqa: E402


@pytest.fixture(scope="module")
def engine():
    return sk.Engine.require()


def allclose_excess(a, b, rtol=1e-7):
    a, b = np.ravel(a), np.ravel(b)
    atol = 1e-12 * np.abs(b).max()
    return float((np.abs(a - b) - (atol + rtol * np.abs(b))).max())


# ---- Gaussian source size ------------------------------------------------------------------------------------------

def _dp():
    p = G.pins()["slice-4-scan"]
    dp = G.array("slice-4-scan", "dp")
    return p, sk.ScanMeasurement([6, 5], [42, 42], dp.reshape(-1).copy()), dp


def test_gaussian_source_size_is_the_reference_loop(engine):
    p, m, dp = _dp()
    s, sg = p["scanSampling"], p["sigma"]
    a = m.gaussianSourceSize(sigmaX=sg[0], sigmaY=sg[1], samplingX=s[0], samplingY=s[1], engine=engine)
    want = O.gaussian_source_size(dp, [6, 5], sg[0], sg[1], s[0], s[1])
    assert np.array_equal(a.values.reshape(want.shape), want)
    assert O.rel_max(a.values, G.array("slice-4-scan", "dp_gauss").ravel()) <= 1e-7
    b = m.gaussianSourceSize(p["sigmaBig"], samplingX=s[0], samplingY=s[1], engine=engine)
    assert np.array_equal(b.values.reshape(dp.shape),
                          O.gaussian_source_size(dp, [6, 5], p["sigmaBig"], p["sigmaBig"], s[0], s[1]))
    assert O.rel_max(b.values, G.array("slice-4-scan", "dp_gauss_big").ravel()) <= 1e-7
    zero = m.gaussianSourceSize(0.0, samplingX=s[0], samplingY=s[1], engine=engine)
    assert np.array_equal(zero.values, m.values)
    assert abs(a.values.sum() - dp.sum()) <= 1e-9 * dp.sum()
    # one axis only, and a scan image without a value axis
    y_only = m.gaussianSourceSize(sigmaX=0.0, sigmaY=sg[1], samplingX=s[0], samplingY=s[1], engine=engine)
    assert np.array_equal(y_only.values.reshape(dp.shape), O.gaussian_source_size(dp, [6, 5], 0.0, sg[1], s[0], s[1]))
    img = sk.ScanMeasurement([13, 7], [], np.random.default_rng(3).random(91))
    g = img.gaussianSourceSize(1.3, samplingX=0.4, samplingY=0.3, engine=engine)
    assert np.array_equal(g.values, O.gaussian_source_size(img.values, [13, 7], 1.3, 1.3, 0.4, 0.3))


@pytest.mark.parametrize("nx,ny,v,sigma", [(300, 4, 40, 3.0), (4, 270, 33, 30.0), (70, 9, 31, 1.0)])
def test_gaussian_source_size_long_axes_and_ragged_columns(engine, nx, ny, v, sigma):
    # axes longer than the staged whole (windows of outputs plus the radius), column counts off a multiple of 32,
    # and a value axis too short for the staged form
    vals = np.random.default_rng(nx * ny + v).random(nx * ny * v)
    m = sk.ScanMeasurement([nx, ny], [v], vals)
    got = m.gaussianSourceSize(sigma, samplingX=0.25, samplingY=0.25, engine=engine)
    want = O.gaussian_source_size(vals, [nx, ny], sigma, sigma, 0.25, 0.25)
    assert np.array_equal(got.values, want)


def test_gaussian_source_size_device_form_in_place(engine):
    p, m, dp = _dp()
    s, sg = p["scanSampling"], p["sigma"]
    d = torch.tensor(dp.reshape(-1), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    L.check(engine.lib.simk_gaussian_source_size_device(engine.handle, 6, 5, 42 * 42, sg[0], sg[1], s[0], s[1],
                                                        C.c_void_p(d.data_ptr()), C.c_void_p(d.data_ptr())))
    want = O.gaussian_source_size(dp, [6, 5], sg[0], sg[1], s[0], s[1])
    assert np.array_equal(d.cpu().numpy(), want.reshape(-1))
    st = engine.lib.simk_gaussian_source_size_device(engine.handle, 6, 5, 42 * 42, -1.0, 0.0, 1.0, 1.0,
                                                     C.c_void_p(d.data_ptr()), C.c_void_p(d.data_ptr()))
    assert st == L.SIMK_ERR_INVALID


# ---- Poisson noise -------------------------------------------------------------------------------------------------

def test_poisson_noise_is_the_oracles_per_value_streams(engine):
    rng = np.random.default_rng(9)
    # means across Knuth (< 10) and PTRS (>= 10), zeros and negatives
    v = np.concatenate([rng.random(150) * 3.0, 3.0 + rng.random(150) * 400.0, [0.0, -2.0, 10.0 / 3.0]])
    m = sk.ScanMeasurement([len(v), 1], [], v)
    draws = m.poissonNoise(3.0, samples=2, seed=123, engine=engine)
    want = O.poisson_noise_streams(v, 3.0, 123, samples=2)
    for s in range(2):
        assert np.array_equal(draws[s].values, want[s])
    single = m.poissonNoise(3.0, seed=123, engine=engine)
    assert np.array_equal(single.values, want[0])


def test_poisson_noise_in_the_reference_order_is_the_references_stream(engine):
    """stream="reference": one GaussianGenerator over every sample and value in order (ScanOperations.swift:80-117),
    bit-equal to the oracle's restatement of that loop, so a seed gives the reference's own draws; the samples
    continue one stream, so sample 0 is the single draw of the same seed."""
    rng = np.random.default_rng(10)
    v = np.concatenate([rng.random(120) * 3.0, 3.0 + rng.random(120) * 400.0, [0.0, -2.0, 10.0 / 3.0, 1e4]])
    m = sk.ScanMeasurement([len(v), 1], [], v)
    draws = m.poissonNoise(3.0, samples=3, seed=2024, stream="reference", engine=engine)
    want = O.poisson_noise_sequential(v, 3.0, 2024, samples=3)
    for s in range(3):
        assert np.array_equal(draws[s].values, want[s])
    single = m.poissonNoise(3.0, seed=2024, stream="reference", engine=engine)
    assert np.array_equal(single.values, want[0])
    # the default per-value streams are untouched by the option (it is reset after the call)
    assert np.array_equal(m.poissonNoise(3.0, seed=123, engine=engine).values, O.poisson_noise_streams(v, 3.0, 123)[0])
    with pytest.raises(sk.InvalidArgument):
        m.poissonNoise(3.0, seed=1, stream="other", engine=engine)


@pytest.mark.parametrize("mean", [0.5, 4.0, 9.9, 10.0, 37.0, 800.0])
def test_poisson_noise_has_the_poisson_mean_and_variance(engine, mean):
    n = 20000
    m = sk.ScanMeasurement([n, 1], [], np.full(n, mean / 3.0))
    noisy = m.poissonNoise(3.0, seed=11, engine=engine).values
    mu = noisy.mean()
    var = ((noisy - mu) ** 2).sum() / (n - 1)
    assert abs(mu - mean) <= 5 * math.sqrt(mean / n)
    assert abs(var - mean) <= 6 * mean * math.sqrt(2.0 / n) + 0.02 * mean
    assert np.all((noisy >= 0) & (noisy == np.round(noisy)))


def test_poisson_noise_is_seeded_clipped_and_refuses_bad_doses(engine):
    m = sk.ScanMeasurement([2, 2], [], np.array([1.0, -3.0, 0.0, 5.0]))
    a = m.poissonNoise(2.0, seed=7, engine=engine)
    b = m.poissonNoise(2.0, seed=7, engine=engine)
    big = sk.ScanMeasurement([40, 40], [], np.full(1600, 5.0))
    assert np.array_equal(a.values, b.values)
    assert not np.array_equal(big.poissonNoise(2.0, seed=7, engine=engine).values,
                              big.poissonNoise(2.0, seed=8, engine=engine).values)
    assert a.values[1] == 0 and a.values[2] == 0
    assert np.array_equal(m.poissonNoise(0.0, seed=1, engine=engine).values, np.zeros(4))
    per_area = m.poissonNoise(dosePerArea=1.0, samplingX=0.5, samplingY=4.0, seed=7, engine=engine)
    assert np.array_equal(per_area.values, a.values)
    for bad in (-1.0, math.nan, math.inf):
        st = engine.lib.simk_poisson_noise(engine.handle, 4, L.dptr(m.values), bad, 1, 1, L.dptr(np.zeros(4)))
        assert st == L.SIMK_ERR_INVALID
    nan_values = np.array([1.0, math.nan])
    st = engine.lib.simk_poisson_noise(engine.handle, 2, L.dptr(nan_values), 1.0, 1, 1, L.dptr(np.zeros(2)))
    assert st == L.SIMK_ERR_INVALID


# ---- integrated gradient and iCOM ----------------------------------------------------------------------------------

@pytest.mark.parametrize("label", ["even", "odd", "mixed", "tiny", "rand", "randOdd"])
def test_integrated_gradient_matches_abtem(engine, label):
    c = next(c for c in G.pins()["icom"]["gradients"] if c["label"] == label)
    g = G.array("icom", f"grad_{label}_g")
    nx, ny = c["shape"]
    sx, sy = c["sampling"]
    out = sk.RealField.integratingGradient(sk.RealField(nx, ny, g.real.reshape(-1).copy(), sx, sy),
                                           sk.RealField(nx, ny, g.imag.reshape(-1).copy(), sx, sy), engine=engine)
    assert allclose_excess(out.values, G.array("icom", f"grad_{label}_out")) <= 0
    assert O.rel_max(out.values, O.integrate_gradient(g.real, g.imag, sx, sy).ravel()) <= 1e-13
    if label in ("even", "odd", "mixed"):
        t = G.array("icom", f"grad_{label}_T")
        assert O.rel_max(out.values, (t - t.min()).ravel()) <= 1e-9


def test_icom_of_abtems_centre_of_mass(engine):
    sc = G.pins()["icom"]["scan"]
    (sx, sy), (nx, ny) = sc["sampling"], sc["scanGpts"]
    for tag in ("inv", "mrad"):
        com = G.array("icom", f"scan_com_{tag}")
        m = sk.ScanMeasurement([nx, ny], [2], np.stack([com.real, com.imag], axis=-1).reshape(-1))
        icom = m.integratedCenterOfMass(sx, sy, engine=engine)
        assert (icom.nx, icom.ny) == (nx, ny)
        assert allclose_excess(icom.values, G.array("icom", f"scan_icom_{tag}")) <= 0


def test_icom_of_the_devices_own_scan_stays_on_the_device(engine):
    """IcomPins.scan: Al, 64^2, 2.025 A slices, 200 keV, 20 mrad, 12 x 10 positions; the centre of mass by
    simk_scan_device into device buffers, integrated there (interleaved pairs, stride 2)."""
    sc = G.pins()["icom"]["scan"]
    nums = np.array([a[0] for a in sc["atoms"]], dtype=int)
    pos = np.array([a[1] for a in sc["atoms"]], dtype=np.float64)
    st = sk.AtomicStructure(tuple(sc["box"]), nums, pos)
    n = sc["gpts"]
    pot = sk.Potential(st, n, n, slice_thickness=sc["sliceThickness"])
    probe = sk.Probe(sk.ElectronBeam(sc["energy"]), pot.grid, sk.Aperture(sc["semiangle"]))
    gx, gy = sc["scanGpts"]
    scan = sk.GridScan(tuple(sc["start"]), tuple(sc["end"]), gx, gy)
    (sx, sy) = sc["sampling"]
    dets = [sk.CenterOfMassDetector("cutoff", "inverse"), sk.CenterOfMassDetector("cutoff", "mrad")]
    h = pot.handle(engine)
    positions = torch.tensor(np.asarray(scan.positions), dtype=torch.float64, device="cuda")
    outs = [torch.zeros(gx * gy * 2, dtype=torch.float64, device="cuda") for _ in dets]
    icoms = [torch.zeros(gx * gy, dtype=torch.float64, device="cuda") for _ in dets]
    torch.cuda.synchronize()
    harr = (C.c_void_p * 1)(h.handle)
    darr = (L.Detector_t * 2)(*[d.c() for d in dets])
    oarr = (C.c_void_p * 2)(*[o.data_ptr() for o in outs])
    pc = probe.c()
    L.check(engine.lib.simk_scan_device(engine.handle, C.byref(pc), 1, harr, gx * gy, C.c_void_p(positions.data_ptr()),
                                        2, darr, oarr))
    for o, ic in zip(outs, icoms):
        L.check(engine.lib.simk_integrate_gradient_device(engine.handle, gx, gy, sx, sy, C.c_void_p(o.data_ptr()),
                                                          C.c_void_p(o.data_ptr() + 8), 2, C.c_void_p(ic.data_ptr())))
    engine.synchronize()
    for tag, o, ic in zip(("inv", "mrad"), outs, icoms):
        want = G.array("icom", f"scan_icom_{tag}").ravel()
        got = ic.cpu().numpy()
        # the float32 centre of mass (2e-4 of its largest value against the pins), carried through the integration
        assert O.rel_max(got, want) <= 2e-4, tag
        # the device integration of the device's own centre of mass equals the host form's
        m = sk.ScanMeasurement([gx, gy], [2], o.cpu().numpy())
        assert O.rel_max(got, m.integratedCenterOfMass(sx, sy, engine=engine).values) <= 1e-14, tag


def test_sizes_past_the_limits_are_refused_before_any_work(engine):
    small = np.zeros(4)
    st = engine.lib.simk_gaussian_source_size(engine.handle, 1 << 15, 1 << 15, 1 << 20, 1.0, 1.0, 1.0, 1.0,
                                              L.dptr(small), L.dptr(small))
    assert st == L.SIMK_ERR_INVALID
    st = engine.lib.simk_poisson_noise(engine.handle, 1 << 40, L.dptr(small), 1.0, 2, 1, L.dptr(small))
    assert st == L.SIMK_ERR_INVALID
    st = engine.lib.simk_integrate_gradient(engine.handle, 1 << 15, 1 << 15, 1.0, 1.0, L.dptr(small), L.dptr(small),
                                            1, L.dptr(small))
    assert st == L.SIMK_ERR_INVALID
