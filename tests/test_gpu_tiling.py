"""Potential projection and tiling on the device through the C ABI: copies and in-order sums bit-equal to the oracle,
the reference's abTEM numbers (PotentialProjectTileTests.swift:32-96, rtol 1e-7), and a periodic crystal built as one
tiled unit cell against the same crystal built atom by atom: the potentials agree to FFT rounding and so do the exit
waves through them."""

import numpy as np
import pytest

from oracle import simk_oracle as O
from test_tiling_oracle import PLANTED_PROJECT, TILE_CASES, close, planted, weighted

pytestmark = pytest.mark.gpu

sk = pytest.importorskip("simulatokit_b200")


@pytest.fixture(scope="module")
def engine():
    return sk.Engine.require()


def _planted():
    return sk.ProjectedPotential(sk.Grid(4, 5, 2.0, 2.5), planted(), [1.0, 1.5, 0.5])


def test_project_on_the_device(engine):
    p = _planted().project(engine)
    assert (p.nx, p.ny, p.samplingX, p.samplingY) == (4, 5, 0.5, 0.5)
    assert np.array_equal(p.values, O.project_slices(planted()).ravel())
    assert all(close(a, b) for a, b in zip(p.values, PLANTED_PROJECT))


@pytest.mark.parametrize("reps,shape,extent,w,total,pw", TILE_CASES)
def test_tiled_on_the_device_matches_abtem(engine, reps, shape, extent, w, total, pw):
    t = _planted().tiled(*reps)
    assert (t.slice_count, t.grid.nx, t.grid.ny) == shape
    assert (t.grid.extent_x, t.grid.extent_y) == extent
    built = t.build(engine)
    assert np.array_equal(built.values, O.tile_slices(planted(), *reps))
    assert close(weighted(built.values), w) and close(float(built.values.sum()), total)
    assert close(weighted(t.project(engine).values), pw)
    # tiling a tiled potential composes
    assert np.array_equal(t.tiled(1, 2).build(engine).values, O.tile_slices(built.values, 1, 2))


def test_tiling_once_is_the_identity(engine):
    p = _planted()
    assert np.array_equal(p.tiled(1, 1).build(engine).values, p.values)


def test_aluminium_projection_matches_abtem(engine):
    s = O.al_fcc_cell()
    st = sk.AtomicStructure(s.box, s.numbers, s.positions).repeated(1, 1, 2)
    pot = sk.Potential(st, 16, 16, slice_thickness=2.025, parameterization=sk.LobatoParameterization("abTEMFloat32"))
    p = pot.project(engine)
    assert pot.slice_count == 4
    assert np.array_equal(p.values, pot.build(engine).project(engine).values), "the lazy projection is the built one"
    assert close(float(p.values.sum()), 35209.17454763371)
    assert close(float(p.values.max()), 907.726975700707)
    assert close(weighted(p.values), 4215022.430595551)


def test_a_tiled_unit_cell_is_the_crystal(engine):
    """SrTiO3: one cell on 64^2 with one 3.905 A slice, tiled 4 x 4 x 5, against the 4 x 4 x 5 crystal (1,600 atoms on
    256^2, five 3.905 A slices); then a 200 keV plane wave through both."""
    cell = O.srtio3_cell()
    unit = sk.Potential(sk.AtomicStructure(cell.box, cell.numbers, cell.positions), 64, 64, slice_thickness=3.905)
    tiled = unit.tiled(4, 4, 5)
    crystal = cell.repeated(4, 4, 5)
    direct = sk.Potential(sk.AtomicStructure(crystal.box, crystal.numbers, crystal.positions), 256, 256,
                          slice_thickness=3.905)
    assert tiled.grid.matches(direct.grid) and tiled.slice_count == direct.slice_count == 5
    vt, vd = tiled.build(engine).values, direct.build(engine).values
    assert O.rel_max(vt, vd) <= 1e-10
    beam = sk.ElectronBeam(200e3)
    wt = sk.Multislice.run(sk.Waves.plane_wave(beam, tiled.grid), tiled, engine=engine)[-1]
    wd = sk.Multislice.run(sk.Waves.plane_wave(beam, direct.grid), direct, engine=engine)[-1]
    assert O.rel_l2(wt.field, wd.field) <= 1e-6
