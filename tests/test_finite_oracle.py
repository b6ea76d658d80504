"""The finite-projection oracle and the surrogate network's float64 restatement, on the CPU.

No reference implementation exists (SimulatoKit lists the finite projection as not ported, docs/parity.md:58,251):
the anchors are the identities of the construction: Gauss-Legendre in u against adaptive quadrature in z, the thick
slab against the analytic infinite projection of pins.py:432 (which the reference's far-field truth pins), additivity
over split slices, and the network's analytic gradients against finite differences."""

import math

import numpy as np
import pytest

from oracle import simk_oracle as O

CASES = [(0.01, -0.5, 0.5), (0.05, -3.0, -2.0), (0.2, 0.2, 1.2), (1.0, -1.0, 3.0), (3.0, -0.5, 0.5), (0.3, -4, 4)]


@pytest.mark.parametrize("z", [6, 8, 14, 38, 79])
def test_gauss_legendre_matches_adaptive_quadrature(z):
    for rho, zl, zu in CASES:
        a, b = O.finite_profile(z, rho, zl, zu), O.finite_profile_quad(z, rho, zl, zu)
        assert abs(a - b) <= 1e-11 * abs(b), (z, rho, zl, zu)


@pytest.mark.parametrize("z", [6, 13, 79])
def test_thick_slab_is_the_infinite_projection(z):
    for rho in (0.02, 0.1, 0.5, 1.0, 2.0):
        fin = O.finite_profile(z, rho, -25.0, 25.0)
        inf = float(O.infinite_profile(z, rho))
        assert abs(fin - inf) <= 1e-9 * inf


def test_slices_add():
    for z in (8, 79):
        for rho in (0.03, 0.4, 2.5):
            whole = O.finite_profile(z, rho, -1.3, 2.2)
            parts = O.finite_profile(z, rho, -1.3, 0.4) + O.finite_profile(z, rho, 0.4, 2.2)
            assert abs(whole - parts) <= 1e-13 * whole


def test_real_space_splat_integrates_to_the_slab_profile():
    """A single atom in a 12 A slab of many slices: summing the slices gives the thick-slab profile at every pixel."""
    box = (8.0, 8.0, 12.0)
    slices = O.finite_potential_slices([14], [(4.0, 4.0, 6.0)], box, 32, 32, [2.0] * 6, n_gl=32)
    total = slices.sum(0)
    rc = O.finite_cutoff(14)
    for ix, iy in ((16, 16), (16, 20), (22, 16), (10, 13)):
        rho = max(math.hypot(ix * 0.25 - 4.0, iy * 0.25 - 4.0), 0.125)
        ref = O.finite_profile(14, rho, -rc, rc) if rho <= rc else 0.0
        assert abs(total[ix, iy] - ref) <= 1e-9 * max(ref, 1.0)


def test_surrogate_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    params = {"emb": rng.normal(0, 0.1, (103, 16)), "W1": rng.normal(0, 0.2, (64, 18)), "b1": rng.normal(0, 0.1, 64),
              "W2": rng.normal(0, 0.12, (64, 64)), "b2": rng.normal(0, 0.1, 64), "W3": rng.normal(0, 0.12, (64, 64)),
              "b3": rng.normal(0, 0.1, 64), "W4": rng.normal(0, 0.12, (1, 64)), "b4": rng.normal(0, 0.1, 1)}
    z = np.array([6, 8, 14, 79, 6, 79])
    rho = np.array([0.05, 0.3, 1.2, 2.0, 0.02, 0.7])
    zl = np.array([-1, 0.1, -2, -0.5, -3, 1.0])
    zu = np.array([1, 0.9, -1, 2.5, -2.5, 3.0])
    target = rng.uniform(0, 1, len(z))
    loss, g = O.surrogate_gradients(params, z - 1, rho, zl, zu, target)
    flat = O.surrogate_pack(params)
    gflat = O.surrogate_pack(g)
    h = 1e-6
    checked = 0
    for idx in rng.choice(flat.size, 80, replace=False).tolist() + [flat.size - 1]:
        if idx < 1648 and gflat[idx] == 0:
            continue  # an embedding row of an element not in the batch
        fp, fm = flat.copy(), flat.copy()
        fp[idx] += h
        fm[idx] -= h
        lp = O.surrogate_gradients(O.surrogate_unpack(fp), z - 1, rho, zl, zu, target)[0]
        lm = O.surrogate_gradients(O.surrogate_unpack(fm), z - 1, rho, zl, zu, target)[0]
        fd = (lp - lm) / (2 * h)
        assert abs(fd - gflat[idx]) <= 1e-6 * max(1.0, abs(fd)), idx
        checked += 1
    assert checked > 40
    # the bias of the output layer cancels in C(zu) - C(zl): its gradient is zero
    assert gflat[-1] == 0.0
