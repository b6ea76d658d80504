"""Job tables (simk_job_table_run): independent jobs with their own grid, potential, energy, slice count and incident
wave in one call, against the float64 oracle job by job, for the fused form (jobs of one grid shape advance together)
and the plain form (one job after another)."""

import numpy as np
import pytest

from oracle import simk_oracle as O

pytestmark = pytest.mark.gpu

sk = pytest.importorskip("simulatokit_b200")


@pytest.fixture(scope="module")
def engine():
    return sk.Engine.require()


# (cell, repeats, grid, slice thickness, energy, probe (semiangle, C10) or None)
JOBS = [
    ("srtio3", (2, 2, 2), (256, 256), 1.9525, 200e3, None),
    ("silicon", (2, 2, 1), (384, 384), 1.35775, 300e3, (25.0, -50.0)),
    ("srtio3", (2, 2, 4), (256, 256), 1.9525, 80e3, (20.0, 0.0)),
    ("al", (3, 3, 1), (640, 640), 1.0125, 120e3, None),
    ("srtio3", (3, 3, 1), (500, 500), 1.9525, 150e3, None),
    ("silicon", (2, 2, 2), (384, 384), 1.35775, 250e3, None),
]


def _cell(name):
    return {"srtio3": O.srtio3_cell, "silicon": O.silicon_cell, "al": O.al_fcc_cell}[name]()


def _build(jobs):
    t = sk.JobTable()
    refs = []
    for name, rep, (nx, ny), dz, energy, probe in jobs:
        s = _cell(name).repeated(*rep)
        pot = sk.Potential(sk.AtomicStructure(s.box, s.numbers, s.positions), nx, ny, slice_thickness=dz)
        op = O.Potential.from_structure(s, nx, ny, slice_thickness=dz)
        og = op.grid
        ts = [O.transmission(v, energy, og) for v in op.build()]
        if probe is None:
            t.add_plane_wave(pot, energy)
            psi0 = O.plane_wave(og)
        else:
            pr = sk.Probe(sk.ElectronBeam(energy), pot.grid, sk.Aperture(probe[0]), sk.Aberrations(C10=probe[1]))
            pos = (s.box[0] / 2, s.box[1] / 2)
            t.add_probe(pot, pr, pos)
            psi0 = O.build_probe(O.ProbeSpec(energy, probe[0], {"C10": probe[1]}), og, pos)
        ex = O.multislice(psi0, ts, op.thicknesses, energy, og)[-1]
        refs.append((np.abs(ex) ** 2, len(op.thicknesses)))
    return t, refs


@pytest.fixture(scope="module")
def table():
    return _build(JOBS)


@pytest.mark.parametrize("form", ["fused", "plain"])
def test_job_table_matches_oracle(engine, table, form):
    t, refs = table
    outs, done = t.run(options=sk.ExecutionOptions(form=form), engine=engine)
    for k, (out, (ref, _)) in enumerate(zip(outs, refs)):
        e = O.rel_l2(out, ref)
        print(f"{form} job {k} {JOBS[k][2]}: intensity rel-L2 {e:.2e}, done at {done[k]:.2f} ms")
        assert e <= 1e-5, (k, e)
    assert np.all(done > 0)
    if form == "fused":
        # within a grid shape, a job with more slices does not finish before one with fewer
        for a in range(len(JOBS)):
            for b in range(len(JOBS)):
                if JOBS[a][2] == JOBS[b][2] and refs[a][1] > refs[b][1]:
                    assert done[a] >= done[b]


def test_job_table_is_one_launch_over_four_shapes(engine, table):
    """With CUDA graphs on, the fused table's whole schedule (four grid shapes: 256, 384, 500, 640; every slice step,
    the finishing row passes and the intensities) runs as one graph launch, and gives the same intensities bit for bit
    as the same schedule launched kernel by kernel, with completion times in the same order."""
    t, refs = table
    outs_g, done_g = t.run(options=sk.ExecutionOptions(form="fused", graphs=True), engine=engine)
    lt = engine.last_table()
    print("one-launch table:", lt)
    assert lt["launches"] == 1 and lt["shapes"] == 4 and lt["kernels"] >= 4
    outs_e, done_e = t.run(options=sk.ExecutionOptions(form="fused", graphs=False), engine=engine)
    le = engine.last_table()
    assert le["launches"] == le["kernels"] == lt["kernels"] and le["shapes"] == 4
    for a, b in zip(outs_g, outs_e):
        assert np.array_equal(a, b)
    assert np.all(done_g > 0)
    for a in range(len(JOBS)):
        for b in range(len(JOBS)):
            if JOBS[a][2] == JOBS[b][2] and refs[a][1] > refs[b][1]:
                assert done_g[a] >= done_g[b]


def test_job_table_refusals(engine):
    s = O.srtio3_cell().repeated(2, 2, 1)
    pot = sk.Potential(sk.AtomicStructure(s.box, s.numbers, s.positions), 256, 256, slice_thickness=1.9525)
    t = sk.JobTable().add_plane_wave(pot, 200e3).add_plane_wave(pot, 300e3)
    with pytest.raises(sk.InvalidArgument, match="different energies"):
        t.run(engine=engine)
    outs, done = sk.JobTable().run(engine=engine)
    assert outs == [] and len(done) == 0


def test_job_table_column_pairs_512(engine):
    """Jobs of one 512 x 512 shape with different energies, slice counts and incident waves: each wave reads its own
    propagator tile in the column pairs' P buffer. Intensities against the float64 oracle (<= 1e-5 relative L2) and
    against the one-column-a-thread passes (<= 1e-6)."""
    jobs = [("srtio3", (2, 2, 2), (512, 512), 1.9525, 200e3, None),
            ("srtio3", (2, 2, 3), (512, 512), 1.9525, 120e3, (20.0, 0.0)),
            ("silicon", (2, 2, 1), (512, 512), 1.35775, 300e3, (25.0, -50.0))]
    t, refs = _build(jobs)
    outs = {}
    for paired in (True, False):
        outs[paired], done = t.run(options=sk.ExecutionOptions(form="fused", paired=paired), engine=engine)
        assert np.all(done > 0)
    for k, (a, b, (ref, _)) in enumerate(zip(outs[True], outs[False], refs)):
        e_o, e_p = O.rel_l2(a, ref), O.rel_l2(a, b)
        print(f"512 job {k}: pairs vs float64 {e_o:.2e}, vs single columns {e_p:.2e}")
        assert e_o <= 1e-5 and e_p <= 1e-6, (k, e_o, e_p)
