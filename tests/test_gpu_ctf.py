"""The contrast transfer function on the device against the reference's abTEM pins (Probe/CTFTests.swift): the float64
kernels H1-H3, K1, K2 at the reference's 1e-12; the HRTEM images of the SrTiO3 3x3x5 exit wave (120^2, 300 keV)
through H1-H3, with the float32 application on the oracle's float64 exit wave (isolating the CTF step) and end to
end from the device's own exit wave (at the reference's registered float32 bound for intensities, 2e-4 max-relative,
MetalAccuracy, ExecutionOptions.swift:55-94)."""

import math

import numpy as np
import pytest

import golden_io as G
from oracle import simk_oracle as O

pytestmark = pytest.mark.gpu

sk = pytest.importorskip("simulatokit_b200")


@pytest.fixture(scope="module")
def engine():
    return sk.Engine.require()


def _ctf(cid):
    c = G.pins()["slice-3"]["cases"][cid]
    ab = sk.Aberrations(**c["aberrations"])
    cutoff = c["cutoff_mrad"] if c["cutoff_mrad"] is not None else math.inf
    ctf = sk.ContrastTransferFunction(ab, cutoff, c["soft"], c["focal_spread"], c["angular_spread"])
    return c, ctf, sk.Grid(c["gpts"][0], c["gpts"][1], c["extent"][0], c["extent"][1])


@pytest.mark.parametrize("cid", ["H1", "H2", "H3", "K1", "K2"])
def test_ctf_kernels(engine, cid):
    c, ctf, grid = _ctf(cid)
    h = ctf.kernel(grid, c["energy"], engine)
    assert O.rel_max(h, G.array("slice-3", f"{cid}.kernel")) <= 1e-12


def test_hrtem_images(engine):
    s = O.srtio3_cell().repeated(3, 3, 5)
    op = O.Potential.from_structure(s, 120, 120, slice_thickness=1.9525, pi_choice="abtem")
    ts = [O.transmission(v, 300e3, op.grid) for v in op.build()]
    ex64 = O.multislice(O.plane_wave(op.grid), ts, op.thicknesses, 300e3, op.grid)[-1]
    pot = sk.Potential(sk.AtomicStructure(s.box, s.numbers, s.positions), 120, 120, slice_thickness=1.9525,
                       parameterization=sk.LobatoParameterization("abTEMFloat32"))
    ex32 = sk.Multislice.run(sk.Waves.plane_wave(sk.ElectronBeam(300e3), pot.grid), pot, engine=engine)[-1]
    beam = sk.ElectronBeam(300e3)
    w64 = sk.Waves(ex64, pot.grid, beam)
    for cid in ("H1", "H2", "H3"):
        _, ctf, _ = _ctf(cid)
        ref = G.array("slice-3", f"{cid}.image")
        _, img_a = ctf.apply(w64, engine)  # the float32 CTF step alone
        _, img_b = ctf.apply(ex32, engine)  # the device end to end
        ea, eb = O.rel_max(img_a, ref), O.rel_max(img_b, ref)
        print(f"{cid}: CTF step {ea:.2e}, end to end {eb:.2e} max-relative")
        assert ea <= 1e-5 and eb <= 2e-4


def test_ctf_batch_and_identity(engine):
    s = O.srtio3_cell().repeated(2, 2, 2)
    pot = sk.Potential(sk.AtomicStructure(s.box, s.numbers, s.positions), 96, 96, slice_thickness=1.9525)
    beam = sk.ElectronBeam(200e3)
    rng = np.random.default_rng(4)
    ws = [sk.Waves(rng.standard_normal((96, 96)) + 1j * rng.standard_normal((96, 96)), pot.grid, beam) for _ in range(3)]
    out, imgs = sk.ContrastTransferFunction().apply(ws, engine)  # no aberrations, envelopes or aperture: identity
    for w, o, im in zip(ws, out, imgs):
        assert O.rel_max(o.field, w.field) <= 1e-6
        assert np.allclose(im, np.abs(o.field) ** 2)
    one, _ = sk.ContrastTransferFunction(sk.Aberrations(C10=-50.0), 20.0).apply(ws[1], engine)
    many, _ = sk.ContrastTransferFunction(sk.Aberrations(C10=-50.0), 20.0).apply(ws, engine)
    assert np.array_equal(one.field, many[1].field)
