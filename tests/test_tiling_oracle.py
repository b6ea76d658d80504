"""Potential projection, tiling and crystal-plane slicing: the oracle against the numbers abTEM 1.0.10 gave the
reference's tests (held inline there: Tests/SimulatoMultisliceTests/PotentialProjectTileTests.swift:32-67 and
CrystalSliceThicknessTests.swift:24-55, rtol 1e-7), the package's host-side crystal slicing against the same, and the
package's refusals, which come before any device work. CPU only."""

import math

import numpy as np
import pytest

from oracle import simk_oracle as O

# abTEM's planted PotentialArray: 3 slices on 4 x 5, values k^1.3 (k the flat index over all slices), thicknesses
# 1, 1.5, 0.5 A, extent 2 x 2.5 A (PotentialProjectTileTests.swift:17-24)
PLANTED_PROJECT = [170.0992068579204, 178.26246245022838, 186.96329271595343, 195.98402939465967, 205.25906320258483,
                   214.75256861125797, 224.4411280205199, 234.30787148190774, 244.33987262942208, 254.52679454798368,
                   264.8601082341936, 275.3326063892693, 285.9380832382715, 296.6711140312202, 307.5268975939282,
                   318.50114048503565, 329.5899695928622, 340.7898647593841, 352.0976058713826, 363.510230635932]
# (repetitions, (slices, nx, ny), extent, weighted, sum, projected weighted) (PotentialProjectTileTests.swift:42-46)
TILE_CASES = [((2, 3, 1), (3, 8, 15), (4.0, 7.5), 7810729.876804397, 31462.523464463502, 2021200.3158708385),
              ((2, 1, 2), (6, 8, 5), (4.0, 2.5), 3002294.8578713303, 20975.015642975668, 457231.794640888),
              ((1, 1, 3), (9, 4, 5), (2.0, 2.5), 1611947.7293367172, 15731.261732231753, 185611.2286583485)]
# CrystalSliceThicknessTests.swift:26-40
CRYSTAL_CASES = [([0.0, 0.6, 1.0, 2.05, 3.99], 4.0, 0.2, [0.4, 0.6000000000000001, 1.0, 1.8000000000000003,
                                                          0.20000000000000018]),
                 ([0.0, 0.6, 1.0, 2.05, 3.99], 4.0, 0.5, [0.5, 0.5, 1.0, 1.5, 0.5]),
                 ([0.3, 0.6, 1.8, 3.0, 4.2, 5.4], 6.0, 0.2, [0.20000000000000004, 0.19999999999999996,
                                                             1.4000000000000001, 1.2, 1.1999999999999997,
                                                             1.2000000000000002, 0.6000000000000005])]


def planted():
    return np.array([[float(s * 20 + k) ** 1.3 for k in range(20)] for s in range(3)]).reshape(3, 4, 5)


def weighted(v):
    v = np.ravel(v)
    return float(sum(float(x) * (i + 1) for i, x in enumerate(v)))


def close(a, b):
    return abs(a - b) <= 1e-7 * abs(b)


def test_project_sums_the_slices():
    p = O.project_slices(planted())
    assert all(close(a, b) for a, b in zip(p.ravel(), PLANTED_PROJECT))


@pytest.mark.parametrize("reps,shape,extent,w,total,pw", TILE_CASES)
def test_tiled_matches_abtem(reps, shape, extent, w, total, pw):
    t = O.tile_slices(planted(), *reps)
    assert t.shape == shape
    assert close(weighted(t), w) and close(float(t.sum()), total)
    assert close(weighted(O.project_slices(t)), pw)


@pytest.mark.parametrize("z,depth,tol,want", CRYSTAL_CASES)
def test_crystal_slices_match_abtem(z, depth, tol, want):
    import simulatokit_b200 as sk
    got = O.crystal_slice_thicknesses(z, depth, tol)
    assert len(got) == len(want) and all(close(a, b) for a, b in zip(got, want))
    st = sk.AtomicStructure((4.0, 4.0, depth), np.full(len(z), 6), np.array([[1.0, 2.0, v] for v in z]))
    pkg = sk.Slicing.crystalSliceThicknesses(st, tolerance=tol)
    assert pkg == got


def test_crystal_slices_of_aluminium():
    import simulatokit_b200 as sk
    s = O.al_fcc_cell()
    st = sk.AtomicStructure(s.box, s.numbers, s.positions)
    t = sk.Slicing.crystalSliceThicknesses(st, tolerance=0.45)
    assert len(t) == 2 and close(t[0], 1.7999999999999998) and close(t[1], 2.2500000000000004)
    assert sk.Potential(st, 16, 16, slice_thicknesses=t).slice_count == 2


def test_crystal_slices_refuse_what_abtem_refuses():
    import simulatokit_b200 as sk

    def planted_structure(z, depth):
        return sk.AtomicStructure((4.0, 4.0, depth), np.full(len(z), 6), np.array([[1.0, 2.0, v] for v in z]))
    s = O.al_fcc_cell()
    al = sk.AtomicStructure(s.box, s.numbers, s.positions)
    for st, tol in [(planted_structure([0.3, 0.6, 1.8, 3.0, 4.2, 5.4], 6.0), 0.7), (al, 0.2),
                    (planted_structure([-0.3, 1.0], 4.0), 0.2), (planted_structure([0.05], 0.1), 0.2)]:
        with pytest.raises(sk.InvalidArgument):
            sk.Slicing.crystalSliceThicknesses(st, tolerance=tol)
        with pytest.raises(ValueError):
            O.crystal_slice_thicknesses(st.positions[:, 2], st.box[2], tol)
    four = planted_structure([0.0, 1.0], 4.0)
    for t in (0.0, -0.2, math.nan, math.inf, 1e-300):
        with pytest.raises(sk.InvalidArgument):
            sk.Slicing.crystalSliceThicknesses(four, tolerance=t)


def test_tiling_refuses_bad_repetitions_before_any_device_work():
    import simulatokit_b200 as sk
    g = sk.Grid(4, 5, 2.0, 2.5)
    p = sk.ProjectedPotential(g, planted(), [1.0, 1.5, 0.5])
    big = (1 << 63) - 1
    for x, y, z in [(0, 1, 1), (1, 0, 1), (1, 1, 0), (-1, 2, 2), (1 << 20, 1 << 20, 1), (1, 1, 400_000),
                    (1_000, 1_000, 200), (1, 1, big), (big // 2, 1, 1)]:
        with pytest.raises(sk.InvalidArgument):
            p.tiled(x, y, z)
    empty = sk.ProjectedPotential(g, np.zeros((0, 4, 5)), [])
    with pytest.raises(sk.InvalidArgument):
        empty.tiled(big // 2, 1)
    e = empty.tiled(2, 2, 3)
    assert e.slice_count == 0 and (e.grid.nx, e.grid.ny) == (8, 10)
    t = p.tiled(2, 3)
    assert (t.grid.nx, t.grid.ny, t.grid.extent_x, t.grid.extent_y) == (8, 15, 4.0, 7.5)
    assert t.slice_thicknesses == [1.0, 1.5, 0.5] and t.thickness == 3.0
    assert p.tiled(1, 1, 3).slice_thicknesses == [1.0, 1.5, 0.5] * 3
