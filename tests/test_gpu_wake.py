"""GPU parity of the read-in wakefield (type -41 elements) through the C ABI
against the oracle.  The GPU path sums the line density in int64 fixed point
(2^-40 of a particle), convolves directly and adds the per-plane field in
the field kernel; the oracle sums in FP64 in particle order, so the two
agree to the fixed-point resolution, far inside the run tolerances:
  * FP64 form: rms columns of every record within 1e-8 of the oracle
  * FP32-convolution form: rms sizes within 1e-5
and the wake's own effect on the bunch is checked to be far above them."""
import os

import numpy as np
import pytest

from conftest import load_impz, load_oracle
from test_wake import synthetic_table

pytestmark = pytest.mark.gpu

impz = load_impz()
orc = load_oracle()
from impz_b200 import beams, deck  # noqa: E402

RMS_COLS = [6, 7, 8, 9, 11, 12, 13, 14, 15, 17, 18, 19, 20, 21, 23]
CURRENT = 1.3


def electron_cfg(n=20_000):
    pts, ref = beams.gaussian_bunch(n, seed=beams.SEED0 + 51, mass=beams.ELECTRON_MASS_EV,
                                    charge=-1.0, ekin=98.169272e6, current=CURRENT, freq=1.3e9,
                                    sig_x=0.5e-3, sig_y=0.5e-3, sig_xp=0.05e-3, sig_yp=0.05e-3,
                                    sig_phase_deg=1.0, sig_e=50e3)
    lat = [impz.elem(0, 0.5, 8, 1, [1.0]), impz.elem(1, 0.1, 4, 1, [10.0, 0.0, 1.0]),
           impz.elem(0, 0.5, 8, 1, [1.0]), impz.elem(1, 0.1, 4, 1, [-10.0, 0.0, 1.0])]
    return dict(pts=pts, refptcl=ref, current=CURRENT, mass=beams.ELECTRON_MASS_EV, charge=-1.0,
                freq=1.3e9, grid=(16, 16, 32), lattice=lat)


def oracle_rows(cfg, wake):
    try:
        if wake is not None:
            orc.wake_set(*wake)
        rows, p, beam = orc.run(cfg["lattice"], cfg["pts"], cfg["current"], cfg["mass"],
                                cfg["charge"], cfg["freq"], cfg["refptcl"], cfg["grid"])
    finally:
        orc.wake_off()
    return rows


def gpu_rows(b, cfg, rows_o):
    recs, zs = b.run(cfg["lattice"])
    assert recs.shape[0] == rows_o.shape[0]
    np.testing.assert_allclose(zs, rows_o[:, 0], rtol=0, atol=0)
    refs = b.run_reference()
    return np.array([impz.diag_row(zs[i], recs[i], refs[i], cfg["mass"], cfg["freq"])
                     for i in range(len(recs))])


def worst(rows_g, rows_o, cols):
    w = 0.0
    for c in cols:
        scale = np.max(np.abs(rows_o[:, c])) + 1e-300
        w = max(w, float(np.max(np.abs(rows_g[:, c] - rows_o[:, c])) / scale))
    return w


@pytest.mark.parametrize("form,transverse,cols,tol", [
    (impz.FORM_FP64, False, RMS_COLS, 1e-8),
    (impz.FORM_FP64, True, RMS_COLS, 1e-8),
    (impz.FORM_FP32CONV, False, [7, 9, 11, 13, 15, 17, 19, 21, 23], 1e-5)])
def test_wake_run_matches_the_oracle(form, transverse, cols, tol):
    cfg = electron_cfg()
    wake = (synthetic_table(), 1.0, transverse)
    rows_o = oracle_rows(cfg, wake)
    rows_nowake = oracle_rows(cfg, None)
    # the wake moves the moments far beyond the tolerance
    assert worst(rows_nowake, rows_o, [21, 23]) > 1e3 * tol
    b = impz.Bunch(cfg["pts"], cfg["current"], cfg["mass"], cfg["charge"], cfg["freq"],
                   cfg["refptcl"], cfg["grid"], form=form, track_ids=False)
    try:
        b.wake(*wake)
        rows_g = gpu_rows(b, cfg, rows_o)
        assert worst(rows_g, rows_o, cols) <= tol
        # off again: the cached step graphs are rebuilt without the wake
        b.wake_off()
        b.upload(cfg["pts"], cfg["current"], cfg["refptcl"])
        rows_g = gpu_rows(b, cfg, rows_nowake)
        assert worst(rows_g, rows_nowake, cols) <= tol
    finally:
        b.close()


def test_wake_launches_are_counted():
    cfg = electron_cfg(n=4096)
    cfg["lattice"] = [impz.elem(0, 0.5, 4, 1, [1.0])]
    b = impz.Bunch(cfg["pts"], cfg["current"], cfg["mass"], cfg["charge"], cfg["freq"],
                   cfg["refptcl"], cfg["grid"], form=impz.FORM_FP64, track_ids=False)
    try:
        b.run(cfg["lattice"])
        b.upload(cfg["pts"], cfg["current"], cfg["refptcl"])
        n0 = impz.kernel_launches()
        b.run(cfg["lattice"])
        plain = impz.kernel_launches() - n0
        b.wake(synthetic_table(), 1.0, False)
        b.upload(cfg["pts"], cfg["current"], cfg["refptcl"])
        n0 = impz.kernel_launches()
        b.run(cfg["lattice"])
        assert impz.kernel_launches() - n0 == plain + 2 * 4  # two wake kernels per step
    finally:
        b.close()


def test_deck_runner_with_wake_controls_matches_the_oracle(tmp_path):
    """An Example3-shaped deck with -41 controls around its cavity (wake on
    with the table of rfdata41.in, off again after the first bend) and a
    -52 laser heater before it, through run_deck (FP64) and through the
    oracle over the same segments."""
    from test_gpu_deck import example_like_deck

    wd = str(tmp_path)
    d = example_like_deck(wd)
    z24 = lambda *v: list(v) + [0.0] * (24 - len(v))  # noqa: E731
    cav = next(i for i, e in enumerate(d.elements) if e.type == 103)
    d.elements.insert(cav, deck.Element(0.0, 0, 1, -41, z24(1.0, 41, 1.0)))
    bend = next(i for i, e in enumerate(d.elements) if e.type == 4)
    d.elements.insert(bend + 1, deck.Element(0.0, 0, 1, -41, z24(1.0, 41, -1.0)))
    # laser heater: 1 mm laser spot, 1030 nm, 200 keV amplitude
    d.elements.insert(cav, deck.Element(0.0, 0, 1, -52, z24(1.0e-3, 1.03e-6, 2.0e5)))
    deck.write_deck(os.path.join(wd, "ImpactZ.in"), d)
    np.savetxt(os.path.join(wd, "rfdata41.in"), synthetic_table())
    out = deck.run_deck(wd, skip={-8})
    pts = deck.read_particles(os.path.join(wd, "particle.in"))
    ref, z, rows_o, nwake, nlaser = d.refptcl(), 0.0, [], 0, 0
    try:
        for kind, item in deck.lattice_segments(d, wd, {-8}):
            if kind == "run":
                seg, pts, beam = orc.run(item, pts, d.bcurr, d.bmass, d.bcharge, d.bfreq, ref,
                                         (d.nx, d.ny, d.nz), z)
                ref, z = np.array(beam.refptcl[:]), beam.z
                rows_o += list(seg[1:] if rows_o else seg)
            elif kind == "wake":
                nwake += 1
                if item["on"]:
                    orc.wake_set(item["table"], item["scale"], item["transverse"])
                else:
                    orc.wake_off()
            elif kind == "laser":
                nlaser += 1
                pts = np.ascontiguousarray(pts)
                orc.lib().orc_laser_heater(orc.dp(pts), pts.shape[0], pts.shape[0],
                                           item["rsig"], item["wavelength"], item["ez"],
                                           d.bmass)
    finally:
        orc.wake_off()
    assert nwake == 2 and nlaser == 1
    rows_o = np.array(rows_o)
    rows_g = out["rows"]
    assert rows_g.shape == rows_o.shape
    np.testing.assert_allclose(rows_g[:, 0], rows_o[:, 0], rtol=0, atol=0)
    assert worst(rows_g, rows_o, RMS_COLS) <= 1e-8


def structure(wake, length=0.3, nseg=6):
    """A 1.3 GHz structure as an ideal-RF gap (type 105, v4 < 0) with, when
    `wake`, the analytic wake of Param(13..15): iris radius 11.6 mm, gap
    29 mm, period 35 mm (AccSimulator.f90:865-875)."""
    v = [2.0e6, 1.3e9, 0.0, -1.0, 1.0] + [0.0] * 19
    if wake:
        v[11], v[12], v[13] = 0.0116, 0.029, 0.035
    return impz.elem(105, length, nseg, 1, v)


@pytest.mark.parametrize("form,cols,tol", [
    (impz.FORM_FP64, RMS_COLS, 1e-8),
    (impz.FORM_FP32CONV, [7, 9, 11, 13, 15, 17, 19, 21, 23], 1e-5)])
def test_analytic_structure_wake_matches_the_oracle(form, cols, tol):
    """A drift, a 105 structure with its analytic wake (longitudinal and
    transverse), a drift: the wake acts only inside the structure."""
    cfg = electron_cfg()
    cfg["lattice"] = [impz.elem(0, 0.3, 6, 1, [1.0]), structure(True),
                      impz.elem(0, 0.3, 6, 1, [1.0])]
    rows_o = oracle_rows(cfg, None)
    plain = dict(cfg, lattice=[cfg["lattice"][0], structure(False), cfg["lattice"][2]])
    rows_plain = oracle_rows(plain, None)
    assert worst(rows_plain, rows_o, [21, 23]) > 1e3 * tol
    b = impz.Bunch(cfg["pts"], cfg["current"], cfg["mass"], cfg["charge"], cfg["freq"],
                   cfg["refptcl"], cfg["grid"], form=form, track_ids=False)
    try:
        rows_g = gpu_rows(b, cfg, rows_o)
    finally:
        b.close()
    assert worst(rows_g, rows_o, cols) <= tol


def test_read_in_wake_switched_off_by_a_structure_without_wake():
    """With a read-in wake on, a 105 structure whose Param(15) is 0 sets
    flagwake = 0, and the read-in wake stays off after it, into the next
    run, until the next -41 (AccSimulator.f90:865-875): GPU = oracle over
    two runs, and != the wake kept on."""
    cfg = electron_cfg()
    drift = impz.elem(0, 0.3, 6, 1, [1.0])
    lat = [drift, structure(False), drift]
    wake = (synthetic_table(), 1.0, False)
    try:
        orc.wake_set(*wake)
        r1, p1, beam1 = orc.run(lat, cfg["pts"], cfg["current"], cfg["mass"], cfg["charge"],
                                cfg["freq"], cfg["refptcl"], cfg["grid"])
        r2, _, _ = orc.run([drift], p1, cfg["current"], cfg["mass"], cfg["charge"], cfg["freq"],
                           np.array(beam1.refptcl[:]), cfg["grid"], beam1.z, beam1)
        orc.wake_set(*wake)
        rk, _, _ = orc.run([drift, drift, drift], cfg["pts"], cfg["current"], cfg["mass"],
                           cfg["charge"], cfg["freq"], cfg["refptcl"], cfg["grid"])
    finally:
        orc.wake_off()
    b = impz.Bunch(cfg["pts"], cfg["current"], cfg["mass"], cfg["charge"], cfg["freq"],
                   cfg["refptcl"], cfg["grid"], form=impz.FORM_FP64, track_ids=False)
    try:
        b.wake(*wake)
        g1 = gpu_rows(b, dict(cfg, lattice=lat), r1)
        g2 = gpu_rows(b, dict(cfg, lattice=[drift]), r2)
    finally:
        b.close()
    assert worst(g1, r1, RMS_COLS) <= 1e-8
    assert worst(g2, r2, RMS_COLS) <= 1e-8
    assert worst(rk[: r1.shape[0]], r1, [21, 23]) > 1e-5


def test_laser_heater_kick_matches_the_oracle():
    """impz_laser_heater (AccSimulator.f90:982-1006) on the device = the
    oracle's kick on the same particles, per particle (sin/exp to 1e-12 of
    the kick's scale), and it moves pt by far more than that."""
    cfg = electron_cfg(n=20_000)
    b = impz.Bunch(cfg["pts"], cfg["current"], cfg["mass"], cfg["charge"], cfg["freq"],
                   cfg["refptcl"], cfg["grid"], form=impz.FORM_FP64, track_ids=True)
    try:
        b.laser_heater(1.0e-3, 1.03e-6, 2.0e5)
        got = b.download()
    finally:
        b.close()
    orc.physconst(cfg["freq"])
    want = np.ascontiguousarray(cfg["pts"]).copy()
    orc.lib().orc_laser_heater(orc.dp(want), want.shape[0], want.shape[0], 1.0e-3, 1.03e-6,
                               2.0e5, cfg["mass"])
    got = got[np.argsort(got[:, 8])]
    want = want[np.argsort(want[:, 8])]
    kick = np.abs(want[:, 5] - cfg["pts"][np.argsort(cfg["pts"][:, 8])][:, 5]).max()
    assert kick > 1e-3 * np.abs(want[:, 5]).max()
    np.testing.assert_array_equal(got[:, :5], want[:, :5])
    assert np.abs(got[:, 5] - want[:, 5]).max() <= 1e-12 * kick
