"""The standalone deck runner on the GPU against the oracle: a deck shaped
like the reference's Example3 (98 MeV electrons, phase dumps, drifts,
quadrupoles, ideal-RF cavities, 150-type dipoles, a slice-output control
whose table is checked), written with impz_b200.deck, run by run_deck (FP64)
and by the oracle over the same lattice_segments.  fort.24-30 rms columns
within 1e-8, z exact, the phase dump holds every particle."""
import os

import numpy as np
import pytest

from conftest import load_impz, load_oracle

pytestmark = pytest.mark.gpu

impz = load_impz()
orc = load_oracle()
from impz_b200 import beams, deck  # noqa: E402

RMS_COLS = [6, 7, 8, 9, 11, 12, 13, 14, 15, 17, 18, 19, 20, 21, 23]


def example_like_deck(workdir, n=4000):
    pts, ref = beams.gaussian_bunch(n, seed=beams.SEED0 + 41, mass=beams.ELECTRON_MASS_EV,
                                    charge=-1.0, ekin=98.169272e6, current=0.13, freq=1.3e9,
                                    sig_x=0.5e-3, sig_y=0.5e-3, sig_xp=0.05e-3, sig_yp=0.05e-3,
                                    sig_phase_deg=1.0, sig_e=50e3)
    d = deck.Deck(np=n, nx=16, ny=16, nz=32, xrad=1.0, yrad=1.0, perdlen=7.64,
                  nptlist=[n], currlist=[0.13], qmcclist=[float(pts[0, 6])], bcurr=0.13,
                  bkenergy=98.169272e6, bmass=beams.ELECTRON_MASS_EV, bcharge=-1.0,
                  bfreq=1.3e9, phsini=0.0)
    z24 = lambda *v: list(v) + [0.0] * (24 - len(v))  # noqa: E731
    d.elements = [
        deck.Element(0.0, 0, 201, -8, z24(101.0)),
        deck.Element(0.0, 0, 1001, -2, z24(1.0)),
        deck.Element(0.5, 4, 1, 0, z24(1.0)),
        deck.Element(0.1, 4, 1, 1, z24(10.0, 0.0, 1.0)),
        deck.Element(0.3, 4, 1, 0, z24(1.0)),
        deck.Element(0.1, 4, 1, 1, z24(-10.0, 0.0, 1.0)),
        deck.Element(1.037743, 4, 1, 103, z24(0.1090744783e8, 1.3e9, -17.43982832, -1.01, 1.0)),
        deck.Element(0.124410139621, 6, 1, 4, z24(0.0221138265963, 0.0, 150, 0.03, 0.0,
                                                   0.0221138265963, 0.0, 0.0, 0.40)),
        deck.Element(0.5, 4, 1, 0, z24(1.0)),
        deck.Element(0.124410139621, 6, 1, 4, z24(-0.0221138265963, 0.0, 150, 0.03,
                                                   -0.0221138265963, 0.0, 0.0, 0.0, 0.40)),
        deck.Element(0.0, 0, 1002, -2, z24(1.0)),
        deck.Element(0.4, 4, 1, 0, z24(1.0)),
        deck.Element(0.0, 0, 0, -99, z24()),
    ]
    deck.write_deck(os.path.join(workdir, "ImpactZ.in"), d)
    deck.write_particles(os.path.join(workdir, "particle.in"), pts)
    return d


def test_deck_runner_matches_the_oracle(tmp_path):
    wd = str(tmp_path)
    d = example_like_deck(wd)
    out = deck.run_deck(wd)
    assert out["skipped"] == []
    # the slice table of the -8 at the start: the initial bunch's
    pts = deck.read_particles(os.path.join(wd, "particle.in"))
    nslice, ax, bx, ay, by = deck.slice_params(d.elements[0])
    want = deck.slice_output(pts, pts.shape[0], nslice, d.bcurr / d.bfreq, d.bmass, ax, bx, ay,
                             by, -d.refptcl()[5], beams.scxl(d.bfreq))
    got = np.loadtxt(os.path.join(wd, "fort.201"))
    assert got.shape == want.shape == (101, 11)
    fin = np.isfinite(want)
    assert np.array_equal(fin, np.isfinite(got))
    # the table sums over the downloaded bunch, whose particle order the
    # upload changed (sorted by cell): sums agree to rounding
    np.testing.assert_allclose(got[fin], want[fin], rtol=1e-10, atol=0)
    # the oracle over the same segments
    ref, z, rows_o = d.refptcl(), 0.0, []
    for kind, item in deck.lattice_segments(d, wd, {-8}):
        if kind == "run":
            seg, pts, beam = orc.run(item, pts, d.bcurr, d.bmass, d.bcharge, d.bfreq, ref,
                                     (d.nx, d.ny, d.nz), z)
            ref, z = np.array(beam.refptcl[:]), beam.z
            rows_o += list(seg[1:] if rows_o else seg)
    rows_o = np.array(rows_o)
    rows_g = out["rows"]
    assert rows_g.shape == rows_o.shape
    np.testing.assert_allclose(rows_g[:, 0], rows_o[:, 0], rtol=0, atol=0)
    for c in RMS_COLS:
        scale = np.max(np.abs(rows_o[:, c])) + 1e-300
        assert np.max(np.abs(rows_g[:, c] - rows_o[:, c])) / scale <= 1e-8, c
    # files: the diagnostics and both phase dumps
    f24 = deck.read_diag(wd, "fort.24")
    np.testing.assert_array_equal(f24, np.c_[rows_g[:, 0], rows_g[:, 6:12]])
    for name in ("fort.1001", "fort.1002"):
        dump = np.loadtxt(os.path.join(wd, name))
        assert dump.shape == (d.np, 9)


def test_checkpoint_and_restart(tmp_path):
    """A -7 checkpoint after the quadrupoles; the deck run again with its
    restart flag from that file reproduces the rest of the full run
    (records after the checkpoint within 1e-10: the restart re-sorts the
    particles, so moment sums differ at rounding level)."""
    import shutil

    wd = str(tmp_path / "full")
    os.makedirs(wd)
    d = example_like_deck(wd)
    z24 = lambda *v: list(v) + [0.0] * (24 - len(v))  # noqa: E731
    cav = next(i for i, e in enumerate(d.elements) if e.type == 103)
    d.elements.insert(cav, deck.Element(0.0, 0, 2001, -7, z24()))
    deck.write_deck(os.path.join(wd, "ImpactZ.in"), d)
    full = deck.run_deck(wd, skip={-8})
    ck = deck.read_checkpoint(os.path.join(wd, "fort.2001"))
    assert ck["pts"].shape[0] == 4000 and ck["inb"] == cav + 1
    rd = str(tmp_path / "restart")
    os.makedirs(rd)
    shutil.copy(os.path.join(wd, "fort.2001"), rd)
    d.restart = 1
    deck.write_deck(os.path.join(rd, "ImpactZ.in"), d)
    rest = deck.run_deck(rd, skip={-8})
    rows_f, rows_r = full["rows"], rest["rows"]
    k0 = int(np.argmin(np.abs(rows_f[:, 0] - ck["z"])))
    tail = rows_f[k0:]
    assert tail.shape == rows_r.shape
    np.testing.assert_allclose(rows_r[:, 0], tail[:, 0], rtol=0, atol=0)
    for c in RMS_COLS:
        scale = np.max(np.abs(tail[:, c])) + 1e-300
        assert np.max(np.abs(rows_r[:, c] - tail[:, c])) / scale <= 1e-10, c


def test_lorentz_dtl_deck_matches_the_oracle(tmp_path):
    """A deck shaped like the reference's Example1: Flagmap=2 (the Lorentz
    integrator) over DTL cells whose rfdataN.in hold Fourier coefficients
    (read3_Data), a quadrupole and a drift, with space charge, then a -25
    switch to the map integrator for a last drift and quadrupole; run_deck
    on the GPU against the oracle over the same segments."""
    from test_lorentz import rf_cell
    wd = str(tmp_path)
    n, mass, freq, cur = 4000, beams.PROTON_MASS_EV, 324e6, 0.03
    pts, _ = beams.gaussian_bunch(n, seed=beams.SEED0 + 89, mass=mass, charge=1.0,
                                  ekin=3.35e6, current=cur, freq=freq)
    d = deck.Deck(np=n, flagmap=2, nx=32, ny=32, nz=64, xrad=0.02, yrad=0.02, perdlen=0.1,
                  nptlist=[n], currlist=[cur], qmcclist=[float(pts[0, 6])], bcurr=cur,
                  bkenergy=3.35e6, bmass=mass, bcharge=1.0, bfreq=freq, phsini=0.0)
    z24 = lambda *v: list(v) + [0.0] * (24 - len(v))  # noqa: E731
    coef, _ = rf_cell()
    for fid, scale in ((852, 1.0), (868, 0.9)):
        np.savetxt(os.path.join(wd, "rfdata%d.in" % fid), coef * scale)
    cell = lambda fid, th: deck.Element(  # noqa: E731
        0.08, 12, 20, 101, z24(2.5e6, freq, th, fid, 0.0065, 0.02, 68.0, 0.02, -67.0))
    d.elements = [
        cell(852, 222.0), cell(868, 218.0), cell(852, 214.0),
        deck.Element(0.045, 4, 20, 1, z24(-19.15, 0.0, 0.009)),
        deck.Element(0.09, 6, 20, 0, z24(0.009)),
        deck.Element(0.0, 0, 1, -25, z24()),
        deck.Element(0.05, 4, 1, 0, z24(0.009)),
        deck.Element(0.045, 4, 1, 1, z24(18.9, 0.0, 0.011)),
        deck.Element(0.0, 0, 0, -99, z24()),
    ]
    deck.write_deck(os.path.join(wd, "ImpactZ.in"), d)
    deck.write_particles(os.path.join(wd, "particle.in"), pts)
    out = deck.run_deck(wd)
    ref, z, rows_o, fm = d.refptcl(), 0.0, [], d.flagmap
    for kind, item in deck.lattice_segments(d, wd):
        if kind == "run":
            seg, pts, beam = orc.run(item, pts, d.bcurr, d.bmass, d.bcharge, d.bfreq, ref,
                                     (d.nx, d.ny, d.nz), z, flagmap=fm)
            ref, z = np.array(beam.refptcl[:]), beam.z
            rows_o += list(seg[1:] if rows_o else seg)
        elif kind == "integrator":
            fm = item
    assert fm == 1
    rows_o = np.array(rows_o)
    rows_g = out["rows"]
    assert rows_g.shape == rows_o.shape == (1 + 3 * 12 + 4 + 6 + 4 + 4, 45)
    np.testing.assert_allclose(rows_g[:, 0], rows_o[:, 0], rtol=0, atol=0)
    assert rows_o[-1, 2] > rows_o[0, 2]  # the cells accelerate (fort.18 gamma)
    for c in RMS_COLS:
        scale = np.max(np.abs(rows_o[:, c])) + 1e-300
        assert np.max(np.abs(rows_g[:, c] - rows_o[:, c])) / scale <= 1e-8, c


def test_two_charge_state_deck_writes_fort32(tmp_path):
    """A deck of two charge states (Nchrg = 2; particle.in rows 7 and 8 per
    particle) under the Lorentz integrator through DTL cells with space
    charge and a narrow aperture: run_deck's rows against the oracle's, and
    fort.32 (z and the count of each charge state, Output.f90:352) equal to
    the oracle's chgupdate counts (the deck's nptlist at the first record)."""
    from test_lorentz import rf_cell
    wd = str(tmp_path)
    npt, qs, cur, freq = [2500, 1500], (33.0, 34.0), [0.004, 0.003], 80.5e6
    pts, _, mass, qmc = beams.charge_state_bunch(npt, qs, cur, seed=beams.SEED0 + 119,
                                                 freq=freq)
    n = sum(npt)
    d = deck.Deck(np=n, flagmap=2, nx=16, ny=16, nz=32, xrad=0.02, yrad=0.02, perdlen=0.1,
                  nchrg=2, nptlist=npt, currlist=cur, qmcclist=list(qmc), bcurr=sum(cur),
                  bkenergy=0.5e6 * 238, bmass=mass, bcharge=qs[0], bfreq=freq, phsini=0.0)
    z24 = lambda *v: list(v) + [0.0] * (24 - len(v))  # noqa: E731
    coef, _ = rf_cell()
    np.savetxt(os.path.join(wd, "rfdata852.in"), coef)
    cell = lambda th: deck.Element(  # noqa: E731
        0.08, 12, 20, 101, z24(2.5e6, freq, th, 852, 0.0035, 0.02, 68.0, 0.02, -67.0))
    d.elements = [cell(222.0), cell(218.0), deck.Element(0.09, 6, 20, 0, z24(0.0035)),
                  deck.Element(0.0, 0, 0, -99, z24())]
    deck.write_deck(os.path.join(wd, "ImpactZ.in"), d)
    deck.write_particles(os.path.join(wd, "particle.in"), pts)
    out = deck.run_deck(wd)
    ref, z, rows_o, cs_o = d.refptcl(), 0.0, [], []
    npl = np.array(npt, dtype=np.int32)
    p = pts
    for kind, item in deck.lattice_segments(d, wd):
        if kind == "run":
            nrec = 1 + sum(e.nseg for e in item)
            cs = np.zeros((nrec, 2), dtype=np.int32)
            seg, p, beam = orc.run(item, p, d.bcurr, d.bmass, d.bcharge, d.bfreq, ref,
                                   (d.nx, d.ny, d.nz), z, flagmap=2,
                                   charge_states=(qmc, npl, cs))
            ref, z = np.array(beam.refptcl[:]), beam.z
            rows_o += list(seg[1:] if rows_o else seg)
            cs_o += list(cs[1:] if cs_o else cs)
    rows_o, cs_o = np.array(rows_o), np.array(cs_o)
    rows_g = out["rows"]
    assert rows_g.shape == rows_o.shape
    assert rows_o[-1, 32] < n  # the aperture lost particles
    np.testing.assert_allclose(rows_g[:, 0], rows_o[:, 0], rtol=0, atol=0)
    for c in RMS_COLS:
        scale = np.max(np.abs(rows_o[:, c])) + 1e-300
        assert np.max(np.abs(rows_g[:, c] - rows_o[:, c])) / scale <= 1e-8, c
    np.testing.assert_array_equal(out["charge_states"], cs_o)
    f32 = np.loadtxt(os.path.join(wd, "fort.32"))
    np.testing.assert_array_equal(f32[:, 0], rows_g[:, 0])
    np.testing.assert_array_equal(f32[:, 1:], cs_o)
