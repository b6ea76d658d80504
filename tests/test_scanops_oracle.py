"""Scan post-processing in the oracle against the reference's pins, and the host-side refusals of the package's
methods (which raise before any device work). Mirrors Tests/SimulatoKitParityTests/Detector/ScanPatternsAndNoiseTests.swift
(Gaussian source size 1e-7 of scipy via abTEM; the Poisson sampler's mean and variance) and
Tests/SimulatoKitParityTests/Detector/IcomPinsTests.swift (integrate_gradient and iCOM at assert_allclose's rtol 1e-7,
atol 1e-12 of the largest value). CPU only."""

import math

import numpy as np
import pytest

import golden_io as G
from oracle import simk_oracle as O


def allclose_excess(a, b, rtol=1e-7):
    """assert_allclose(a, b, rtol, atol = 1e-12 max|b|): the worst excess over the bound; <= 0 passes."""
    a, b = np.ravel(a), np.ravel(b)
    atol = 1e-12 * np.abs(b).max()
    return float((np.abs(a - b) - (atol + rtol * np.abs(b))).max())


def _scan4():
    p = G.pins()["slice-4-scan"]
    return p, G.array("slice-4-scan", "dp")


def test_gaussian_source_size_matches_scipy_via_abtem():
    p, dp = _scan4()
    s, sg = p["scanSampling"], p["sigma"]
    a = O.gaussian_source_size(dp, [6, 5], sg[0], sg[1], s[0], s[1])
    assert O.rel_max(a, G.array("slice-4-scan", "dp_gauss")) <= 1e-7
    # a sigma larger than the scan wraps around it (2.4 pixels on a 5-point axis)
    b = O.gaussian_source_size(dp, [6, 5], p["sigmaBig"], p["sigmaBig"], s[0], s[1])
    assert O.rel_max(b, G.array("slice-4-scan", "dp_gauss_big")) <= 1e-7
    # no source size leaves the scan alone, and the total is conserved
    assert np.array_equal(O.gaussian_source_size(dp, [6, 5], 0.0, 0.0, s[0], s[1]), dp)
    assert abs(a.sum() - dp.sum()) <= 1e-9 * dp.sum()
    with pytest.raises(ValueError):
        O.gaussian_source_size(dp, [6, 5], -1.0, 1.0, 1.0, 1.0)


def test_gaussian_kernel_is_scipys():
    # radius floor(4 s + 1/2), normalised, symmetric
    for s in (0.3, 1.0, 1.19, 2.4, 7.5):
        w = O.gaussian_kernel(s)
        assert len(w) == 2 * int(4 * s + 0.5) + 1
        assert abs(w.sum() - 1.0) <= 1e-15
        assert np.array_equal(w, w[::-1])


def _gradient(label):
    c = next(c for c in G.pins()["icom"]["gradients"] if c["label"] == label)
    g = G.array("icom", f"grad_{label}_g")
    return c, g.real, g.imag


@pytest.mark.parametrize("label", ["even", "odd", "mixed", "tiny", "rand", "randOdd"])
def test_integrated_gradient_matches_abtem(label):
    c, gx, gy = _gradient(label)
    out = O.integrate_gradient(gx, gy, c["sampling"][0], c["sampling"][1])
    assert allclose_excess(out, G.array("icom", f"grad_{label}_out")) <= 0


@pytest.mark.parametrize("label", ["even", "odd", "mixed"])
def test_planted_potentials_are_recovered(label):
    c, gx, gy = _gradient(label)
    t = G.array("icom", f"grad_{label}_T")
    want = t - t.min()
    assert O.rel_max(O.integrate_gradient(gx, gy, c["sampling"][0], c["sampling"][1]), want) <= 1e-9


def test_scan_icom_of_abtems_centre_of_mass():
    sc = G.pins()["icom"]["scan"]
    s, n = sc["sampling"], sc["scanGpts"]
    for tag in ("inv", "mrad"):
        com = G.array("icom", f"scan_com_{tag}")
        values = np.stack([com.real, com.imag], axis=-1).reshape(-1)
        icom = O.integrated_center_of_mass(values, n, s[0], s[1])
        assert allclose_excess(icom, G.array("icom", f"scan_icom_{tag}")) <= 0
    assert allclose_excess(G.array("icom", "scan_icom_chain"), G.array("icom", "scan_icom_inv")) <= 0


@pytest.mark.parametrize("mean", [0.5, 4.0, 9.9, 10.0, 37.0, 800.0])
def test_sequential_poisson_sampler_has_the_poisson_mean_and_variance(mean):
    # ScanPatternsAndNoiseTests.poissonNoiseHasThePoissonMeanAndVariance on the reference's own stream
    n = 20000
    noisy = O.poisson_noise_sequential(np.full(n, mean / 3.0), 3.0, 11)[0]
    mu = noisy.mean()
    var = ((noisy - mu) ** 2).sum() / (n - 1)
    assert abs(mu - mean) <= 5 * math.sqrt(mean / n)
    assert abs(var - mean) <= 6 * mean * math.sqrt(2.0 / n) + 0.02 * mean
    assert np.all((noisy >= 0) & (noisy == np.round(noisy)))


def test_poisson_streams_are_seeded_and_clipped():
    v = np.array([1.0, -3.0, 0.0, 5.0])
    a = O.poisson_noise_streams(v, 2.0, 7)
    assert np.array_equal(a, O.poisson_noise_streams(v, 2.0, 7))
    assert a[0, 1] == 0 and a[0, 2] == 0
    assert np.array_equal(O.poisson_noise_streams(v, 0.0, 1), np.zeros((1, 4)))
    # sample 0 of several is the single draw; other samples differ
    many = O.poisson_noise_streams(np.full(50, 3.0), 1.0, 5, samples=3)
    assert np.array_equal(many[0], O.poisson_noise_streams(np.full(50, 3.0), 1.0, 5)[0])
    assert not np.array_equal(many[0], many[1])
    assert O.poisson_value_seed(5, 0) == O.configuration_seed(5, 0)


def test_package_refuses_before_any_device_work():
    import simulatokit_b200 as sk
    m = sk.ScanMeasurement([2, 2], [], np.array([1.0, -3.0, 0.0, 5.0]))
    for kw in ({"sigma": -1.0, "samplingX": 1.0, "samplingY": 1.0},
               {"sigma": math.nan, "samplingX": 1.0, "samplingY": 1.0},
               {"sigma": 1.0, "samplingX": 0.0, "samplingY": 1.0},
               {"samplingX": 1.0, "samplingY": 1.0}):
        with pytest.raises(sk.InvalidArgument):
            m.gaussianSourceSize(**kw)
    line = sk.ScanMeasurement([4], [], np.ones(4))
    with pytest.raises(sk.InvalidArgument):
        line.gaussianSourceSize(sigma=1.0, samplingX=1.0, samplingY=1.0)
    for bad in (-1.0, math.nan, math.inf):
        with pytest.raises(sk.InvalidArgument):
            m.poissonNoise(bad, seed=1)
    with pytest.raises(sk.InvalidArgument):
        m.poissonNoise(1.0, samples=0)
    with pytest.raises(sk.InvalidArgument):
        m.poissonNoise(dosePerArea=1.0, samplingX=0.0, samplingY=1.0)
    with pytest.raises(sk.InvalidArgument):
        m.integratedCenterOfMass(1.0, 1.0)          # one value per position
    com = sk.ScanMeasurement([1, 4], [2], np.ones(8))
    with pytest.raises(sk.InvalidArgument):
        com.integratedCenterOfMass(1.0, 1.0)        # an axis shorter than 2
    a = sk.RealField(3, 3, np.zeros(9), 1.0, 1.0)
    with pytest.raises(sk.InvalidArgument):
        sk.RealField.integratingGradient(a, sk.RealField(3, 3, np.zeros(9), 1.0, 2.0))
