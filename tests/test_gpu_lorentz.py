"""GPU parity of the Lorentz integrator (Flagmap=2: drift2 half steps
around the kick2/scatter2 Lorentz kick, BeamBunch.f90:467-509, 2187-3071)
through the C ABI against the oracle, on the proton FODO lattice with
space charge: rms columns of every record within 1e-8 (FP64) and 1e-5
(FP32 form), z exact; the run differs from the map integrator's by far more
than that.  A lattice of the other elements kick2 carries (Enge-fringe
quadrupole, ramped solenoid, constant focusing) is held to the same bounds,
with the reference particle exact."""
import numpy as np
import pytest

from conftest import load_impz, load_oracle

pytestmark = pytest.mark.gpu

impz = load_impz()
orc = load_oracle()
from impz_b200 import beams  # noqa: E402

RMS_COLS = [6, 7, 8, 9, 11, 12, 13, 14, 15, 17, 18, 19, 20, 21, 23]


def worst(rows_g, rows_o, cols):
    w = 0.0
    for c in cols:
        scale = np.max(np.abs(rows_o[:, c])) + 1e-300
        w = max(w, float(np.max(np.abs(rows_g[:, c] - rows_o[:, c])) / scale))
    return w


@pytest.mark.parametrize("form,cols,tol", [
    (impz.FORM_FP64, RMS_COLS, 1e-8),
    (impz.FORM_FP32CONV, [7, 9, 11, 13, 15, 17, 19, 21, 23], 1e-5)])
def test_lorentz_fodo_matches_the_oracle(form, cols, tol):
    cfg = beams.fodo_1e5(n=20_000, seed=beams.SEED0 + 72)
    lat = beams.fodo(2)
    run_o = lambda fm: orc.run(lat, cfg["pts"], cfg["current"], cfg["mass"],  # noqa: E731
                               cfg["charge"], cfg["freq"], cfg["refptcl"], cfg["grid"],
                               flagmap=fm)[0]
    rows_o, rows_map = run_o(2), run_o(1)
    assert worst(rows_map, rows_o, [7, 13]) > 1e3 * tol
    b = impz.Bunch(cfg["pts"], cfg["current"], cfg["mass"], cfg["charge"], cfg["freq"],
                   cfg["refptcl"], cfg["grid"], form=form, track_ids=False)
    try:
        b.set_integrator(2)
        recs, zs = b.run(lat)
        refs = b.run_reference()
        # a bend is outside this integrator
        with pytest.raises(impz.ImpzError):
            b.run([impz.elem(4, 0.2, 4, 1, [0.05, 0.0, 150.0, 0.01])])
    finally:
        b.close()
    assert recs.shape[0] == rows_o.shape[0]
    np.testing.assert_allclose(zs, rows_o[:, 0], rtol=0, atol=0)
    rows_g = np.array([impz.diag_row(zs[i], recs[i], refs[i], cfg["mass"], cfg["freq"])
                       for i in range(len(recs))])
    assert worst(rows_g, rows_o, cols) <= tol


def test_lorentz_without_current_matches_the_oracle():
    """Zero current: the element's field alone (scatter20), FP64: rms
    columns within 1e-10 of the oracle."""
    cfg = beams.fodo_1e5(n=20_000, seed=beams.SEED0 + 74)
    lat = beams.fodo(1)
    rows_o = orc.run(lat, cfg["pts"], 0.0, cfg["mass"], cfg["charge"], cfg["freq"],
                     cfg["refptcl"], cfg["grid"], flagmap=2)[0]
    b = impz.Bunch(cfg["pts"], 0.0, cfg["mass"], cfg["charge"], cfg["freq"], cfg["refptcl"],
                   cfg["grid"], form=impz.FORM_FP64, track_ids=False)
    try:
        b.set_integrator(2)
        recs, zs = b.run(lat)
        refs = b.run_reference()
    finally:
        b.close()
    np.testing.assert_allclose(zs, rows_o[:, 0], rtol=0, atol=0)
    rows_g = np.array([impz.diag_row(zs[i], recs[i], refs[i], cfg["mass"], cfg["freq"])
                       for i in range(len(recs))])
    assert worst(rows_g, rows_o, RMS_COLS) <= 1e-10


def element_lattice():
    """Drift, Enge-fringe quadrupole, ramped solenoid, constant focusing with
    Ez (which moves gamma0) and a hard-edge quadrupole under kick2."""
    return [impz.elem(0, 0.1, 4, 1, [1.0]),
            impz.elem(1, 0.2, 8, 1, [20.0, 0.1, 0.01]),
            impz.elem(3, 0.3, 8, 1, [0.5, 0.0, 0.03]),
            impz.elem(2, 0.2, 4, 1, [6e9, 9e9, 1e-3, 1.0]),
            impz.elem(1, 0.1, 4, 1, [-20.0, 0.0, 1.0])]


@pytest.mark.parametrize("current,form,cols,tol", [
    (0.030, impz.FORM_FP64, RMS_COLS, 1e-8),
    (0.030, impz.FORM_FP32CONV, [7, 9, 11, 13, 15, 17, 19, 21, 23], 1e-5),
    (0.0, impz.FORM_FP64, RMS_COLS, 1e-10)])
def test_lorentz_element_fields_match_the_oracle(current, form, cols, tol):
    """The element fields of getfld_Quadrupole (Enge fringe), getfld_Sol
    (ramps and body) and getfld_ConstFoc, and gamma0's change by Ez0, on the
    GPU as in the oracle; the reference particle of every record equal."""
    cfg = beams.fodo_1e5(n=20_000, seed=beams.SEED0 + 79)
    lat = element_lattice()
    rows_o, _, beam = orc.run(lat, cfg["pts"], current, cfg["mass"], cfg["charge"], cfg["freq"],
                              cfg["refptcl"], cfg["grid"], flagmap=2)
    b = impz.Bunch(cfg["pts"], current, cfg["mass"], cfg["charge"], cfg["freq"],
                   cfg["refptcl"], cfg["grid"], form=form, track_ids=False)
    try:
        b.set_integrator(2)
        recs, zs = b.run(lat)
        refs = b.run_reference()
    finally:
        b.close()
    np.testing.assert_allclose(zs, rows_o[:, 0], rtol=0, atol=0)
    np.testing.assert_array_equal(refs[-1], np.array(beam.refptcl[:]))
    assert refs[-1][5] != cfg["refptcl"][5]  # Ez0 of the constant focusing
    rows_g = np.array([impz.diag_row(zs[i], recs[i], refs[i], cfg["mass"], cfg["freq"])
                       for i in range(len(recs))])
    assert worst(rows_g, rows_o, cols) <= tol


@pytest.mark.parametrize("form,cols,tol", [
    (impz.FORM_FP64, RMS_COLS, 1e-8),
    (impz.FORM_FP32CONV, [7, 9, 11, 13, 15, 17, 19, 21, 23], 1e-5)])
def test_lorentz_read_in_wake_matches_the_oracle(form, cols, tol):
    """kick2wake/scatter2wake (BeamBunch.f90:5048-5938): under the Lorentz
    integrator the wake kernel leaves the node fields alone and hands the
    raw per-plane wake to the push, which interpolates it at each particle
    and adds it after the space-charge scaling."""
    from test_wake import synthetic_table
    cur = 1.3
    pts, ref = beams.gaussian_bunch(20_000, seed=beams.SEED0 + 82, mass=beams.ELECTRON_MASS_EV,
                                    charge=-1.0, ekin=98.169272e6, current=cur, freq=1.3e9,
                                    sig_x=0.5e-3, sig_y=0.5e-3, sig_xp=0.05e-3,
                                    sig_yp=0.05e-3, sig_phase_deg=1.0, sig_e=50e3)
    scxl = 2.99792458e8 / (2 * np.pi * 1.3e9)
    pts = pts.copy()
    pts[:, 0] += 0.5e-3 / scxl
    pts[:, 2] += 0.3e-3 / scxl
    lat = [impz.elem(0, 0.5, 8, 1, [1.0]), impz.elem(1, 0.1, 4, 1, [10.0, 0.0, 1.0]),
           impz.elem(0, 0.5, 8, 1, [1.0])]
    table = synthetic_table()
    mass, freq, grid = beams.ELECTRON_MASS_EV, 1.3e9, (16, 16, 32)

    def oracle(wake):
        try:
            if wake:
                orc.wake_set(table, 1.0, True)
            return orc.run(lat, pts, cur, mass, -1.0, freq, ref, grid, flagmap=2)[0]
        finally:
            orc.wake_off()

    rows_o, rows_nowake = oracle(True), oracle(False)
    assert worst(rows_nowake, rows_o, [20, 21]) > 1e3 * tol
    b = impz.Bunch(pts, cur, mass, -1.0, freq, ref, grid, form=form, track_ids=False)
    try:
        b.set_integrator(2)
        b.wake(table, 1.0, True)
        recs, zs = b.run(lat)
        refs = b.run_reference()
    finally:
        b.close()
    np.testing.assert_allclose(zs, rows_o[:, 0], rtol=0, atol=0)
    rows_g = np.array([impz.diag_row(zs[i], recs[i], refs[i], mass, freq)
                       for i in range(len(recs))])
    assert worst(rows_g, rows_o, cols) <= tol


@pytest.mark.parametrize("current,form,cols,tol", [
    (0.010, impz.FORM_FP64, RMS_COLS, 1e-8),
    (0.010, impz.FORM_FP32CONV, [7, 9, 11, 13, 15, 17, 19, 21, 23], 1e-5),
    (0.0, impz.FORM_FP64, RMS_COLS, 1e-10)])
def test_lorentz_rf_cavities_match_the_oracle(current, form, cols, tol):
    """A DTL cell (with its drift-tube quadrupoles), a drift and a CCL cell
    over read3_Data Fourier coefficients under kick2 (getfldpts_DTL,
    getfldpts_CCL): the cos/sin of each particle's RF phase on the GPU,
    the reference particle's energy gain exact."""
    from test_lorentz import rf_cell
    coef, _ = rf_cell()
    mass, freq = beams.PROTON_MASS_EV, 324e6
    pts, ref = beams.gaussian_bunch(20_000, seed=beams.SEED0 + 84, mass=mass, charge=1.0,
                                    ekin=3.35e6, current=current, freq=freq)
    lat = [impz.elem(101, 0.08, 16, 20, [2.5e6, freq, 222.0, 1.0, 0.0065, 0.02, 68.0, 0.02,
                                         -67.0], rf=coef),
           impz.elem(0, 0.05, 4, 1, [0.0065]),
           impz.elem(103, 0.08, 16, 20, [2.5e6, freq, 30.0, 1.0, 0.0065], rf=coef)]
    grid = (32, 32, 64)
    rows_o, _, beam = orc.run(lat, pts, current, mass, 1.0, freq, ref, grid, flagmap=2)
    b = impz.Bunch(pts, current, mass, 1.0, freq, ref, grid, form=form, track_ids=False)
    try:
        b.set_integrator(2)
        recs, zs = b.run(lat)
        refs = b.run_reference()
    finally:
        b.close()
    np.testing.assert_allclose(zs, rows_o[:, 0], rtol=0, atol=0)
    np.testing.assert_array_equal(refs[-1], np.array(beam.refptcl[:]))
    assert -refs[-1][5] + ref[5] > 1e-4  # the cells accelerate
    rows_g = np.array([impz.diag_row(zs[i], recs[i], refs[i], mass, freq)
                       for i in range(len(recs))])
    assert worst(rows_g, rows_o, cols) <= tol


@pytest.mark.parametrize("current,form,cols,tol", [
    (0.010, impz.FORM_FP64, RMS_COLS, 1e-8),
    (0.0, impz.FORM_FP64, RMS_COLS, 1e-10)])
def test_lorentz_solrf_and_tws_match_the_oracle(current, form, cols, tol):
    """A SolRF (105: the cavity's series and the solenoid's Bz profile
    scaled by Param(12)) and a TWS (106: two waves, the second 90 degrees
    on over the middle) under kick2 (getfld_SolRF, getfld_TWS)."""
    from test_abi import tws_coefficients
    from test_lorentz import solrf_two_series
    mass, freq = beams.PROTON_MASS_EV, 402.5e6
    pts, ref = beams.gaussian_bunch(20_000, seed=beams.SEED0 + 86, mass=mass, charge=1.0,
                                    ekin=2.5e6, current=current, freq=freq)
    lat = [impz.elem(105, 0.2, 16, 20, [1e6, freq, 60.0, 1.0, 1.0, 0, 0, 0, 0, 0, 0.5],
                     rf=solrf_two_series()),
           impz.elem(0, 0.05, 4, 1, [1.0]),
           impz.elem(106, 0.2, 16, 20, [1e6, freq, 60.0, 1.0, 1.0, 0, 0, 0, 0, 0, 90.0],
                     rf=tws_coefficients())]
    grid = (32, 32, 64)
    rows_o, _, beam = orc.run(lat, pts, current, mass, 1.0, freq, ref, grid, flagmap=2)
    b = impz.Bunch(pts, current, mass, 1.0, freq, ref, grid, form=form, track_ids=False)
    try:
        b.set_integrator(2)
        recs, zs = b.run(lat)
        refs = b.run_reference()
    finally:
        b.close()
    np.testing.assert_allclose(zs, rows_o[:, 0], rtol=0, atol=0)
    np.testing.assert_array_equal(refs[-1], np.array(beam.refptcl[:]))
    rows_g = np.array([impz.diag_row(zs[i], recs[i], refs[i], mass, freq)
                       for i in range(len(recs))])
    assert worst(rows_g, rows_o, cols) <= tol


@pytest.mark.parametrize("form,cols,tol", [
    (impz.FORM_FP64, RMS_COLS, 1e-8),
    (impz.FORM_FP32CONV, [7, 9, 11, 13, 15, 17, 19, 21, 23], 1e-5)])
def test_lorentz_multipoles_match_the_oracle(form, cols, tol):
    """Sextupole, octupole and decapole (getfld_Multipole, MAD notation)
    between drifts and a quadrupole, with space charge, under kick2."""
    cfg = beams.fodo_1e5(n=20_000, seed=beams.SEED0 + 88)
    lat = [impz.elem(0, 0.1, 4, 1, [1.0]),
           impz.elem(5, 0.05, 4, 1, [2, 3.0e3, 0.0, 1.0]),
           impz.elem(1, 0.1, 4, 1, [20.0, 0.0, 1.0]),
           impz.elem(5, 0.05, 4, 1, [3, 2.0e6, 0.0, 1.0]),
           impz.elem(5, 0.05, 4, 1, [4, 1.0e9, 0.0, 1.0]),
           impz.elem(0, 0.1, 4, 1, [1.0])]
    rows_o, _, beam = orc.run(lat, cfg["pts"], cfg["current"], cfg["mass"], cfg["charge"],
                              cfg["freq"], cfg["refptcl"], cfg["grid"], flagmap=2)
    b = impz.Bunch(cfg["pts"], cfg["current"], cfg["mass"], cfg["charge"], cfg["freq"],
                   cfg["refptcl"], cfg["grid"], form=form, track_ids=False)
    try:
        b.set_integrator(2)
        recs, zs = b.run(lat)
        refs = b.run_reference()
    finally:
        b.close()
    np.testing.assert_allclose(zs, rows_o[:, 0], rtol=0, atol=0)
    rows_g = np.array([impz.diag_row(zs[i], recs[i], refs[i], cfg["mass"], cfg["freq"])
                       for i in range(len(recs))])
    assert worst(rows_g, rows_o, cols) <= tol


@pytest.mark.parametrize("current", [0.030, 0.0])
def test_per_step_lorentz_calls_reproduce_the_runner(current):
    """The Fortran driver's Flagmap=2 step (AccSimulator.f90:1109-1116,
    1122-1405, 1446-1469) through the per-step calls: drift2, conv1st /
    deposit / Poisson, kick2 in the element at z, drift2; against impz_run
    with the Lorentz integrator over the same FODO: every particle (by id)
    and the reference particle agree to rounding."""
    cfg = beams.fodo_1e5(n=20_000, seed=beams.SEED0 + 90)
    lat = beams.fodo(1, nseg=3)
    args = (cfg["pts"], current, cfg["mass"], cfg["charge"], cfg["freq"], cfg["refptcl"],
            cfg["grid"])
    b1 = impz.Bunch(*args, form=impz.FORM_FP64, track_ids=True)
    b2 = impz.Bunch(*args, form=impz.FORM_FP64, track_ids=True)
    try:
        b1.set_integrator(2)
        b1.run(lat)
        p1, i1 = b1.download(), b1.info()
        z = 0.0
        for e in lat:
            zedge, tau = z, e.length / e.nseg
            rad = e.val[0] if e.type == 0 else e.val[2]
            for _ in range(e.nseg):
                z = b2.drift2(z, tau)
                if current > 0:
                    b2.sc_prepare(rad, rad)
                    b2.deposit(want_rho=False, want_counts=False)
                    b2.poisson(want_phi=False)
                b2.kick2(e, zedge, z, tau)
                z = b2.drift2(z, tau)
        p2, i2 = b2.download(), b2.info()
        if current == 0.0:  # without a solve, a bunch with current is refused
            b3 = impz.Bunch(cfg["pts"], 0.03, cfg["mass"], cfg["charge"], cfg["freq"],
                            cfg["refptcl"], cfg["grid"], form=impz.FORM_FP64)
            try:
                with pytest.raises(impz.ImpzError):
                    b3.kick2(lat[1], 0.1, 0.15, 0.025)
            finally:
                b3.close()
    finally:
        b1.close()
        b2.close()
    assert p1.shape == p2.shape
    p1 = p1[np.argsort(p1[:, 8])]
    p2 = p2[np.argsort(p2[:, 8])]
    np.testing.assert_allclose(p2[:, :6], p1[:, :6], rtol=1e-12, atol=1e-300)
    np.testing.assert_allclose(i2["refptcl"], i1["refptcl"], rtol=1e-15, atol=0)
    assert abs(z - i1["z"]) < 1e-12 and abs(i2["z"] - i1["z"]) < 1e-12


def test_batched_runs_keep_each_bunchs_integrator():
    """impz_run_batch over a bunch under the map integrator and one under
    the Lorentz integrator: each bunch's records equal its own run alone, to
    the rounding of the moment sums (1e-12 of each record column's largest
    magnitude: the particles' order within a cell, and so the order of the
    sums, follows the sort's atomics)."""
    cfg = beams.fodo_1e5(n=20_000, seed=beams.SEED0 + 91)
    lat = beams.fodo(1)
    args = (cfg["pts"], cfg["current"], cfg["mass"], cfg["charge"], cfg["freq"],
            cfg["refptcl"], cfg["grid"])
    solo = {}
    for fm in (1, 2):
        b = impz.Bunch(*args, form=impz.FORM_FP64, track_ids=False)
        try:
            b.set_integrator(fm)
            solo[fm] = b.run(lat)[0]
        finally:
            b.close()
    assert np.max(np.abs(solo[1] - solo[2])) > 0
    b1 = impz.Bunch(*args, form=impz.FORM_FP64, track_ids=False)
    b2 = impz.Bunch(*args, form=impz.FORM_FP64, track_ids=False)
    try:
        b2.set_integrator(2)
        out = impz.run_batch([b1, b2], [lat, lat])
    finally:
        b1.close()
        b2.close()
    for got, want in ((out[0][0], solo[1]), (out[1][0], solo[2])):
        assert got.shape == want.shape
        scale = np.max(np.abs(want), axis=0) + 1e-300
        assert np.max(np.abs(got - want) / scale) <= 1e-12


@pytest.mark.parametrize("current,form,cols,tol", [
    (0.010, impz.FORM_FP64, RMS_COLS, 1e-8),
    (0.010, impz.FORM_FP32CONV, [7, 9, 11, 13, 15, 17, 19, 21, 23], 1e-5),
    (0.0, impz.FORM_FP64, RMS_COLS, 1e-10)])
def test_lorentz_emfld_maps_match_the_oracle(current, form, cols, tol):
    """EMfld 110 elements over read4_Data x-y-z maps (scatter2 with
    FlagDisc 1, FlagCart 2): an RF map whose complex fields vary in x, y and
    z (the plane at each kick quadratic in z, each particle's field
    quadratic in x and y, times escale e^{i(ww t + theta0)}) and a static
    quadrupole map: GPU = oracle, the reference particle exact."""
    from test_lorentz import emfld, emfld_grid, quad_map
    cfg = beams.fodo_1e5(n=20_000, seed=beams.SEED0 + 94)
    length = 0.2

    def rf(x, y, z):
        k = np.pi / length
        ez = 1.0e7 * np.sin(k * z) * (1 + 0.1j) * (1 - 200.0 * (x * x + y * y))
        ex = -1.0e8 * x * np.cos(k * z) * (1 - 0.3j)
        ey = -1.0e8 * y * np.cos(k * z) * (1 - 0.3j)
        bx = 0.02 * y * np.sin(k * z) * 1j
        by = -0.02 * x * np.sin(k * z) * 1j
        return ex, ey, ez, bx, by, 0.001 * np.cos(k * z) + 0 * x
    lat = [impz.elem(0, 0.05, 2, 1, [1.0]),
           emfld(length, 8, emfld_grid(rf, length, nz=20), 1.2, 402.5e6, 20.0),
           impz.elem(0, 0.05, 2, 1, [1.0]),
           emfld(0.1, 4, emfld_grid(quad_map(15.0), 0.1))]
    rows_o, _, beam = orc.run(lat, cfg["pts"], current, cfg["mass"], cfg["charge"], cfg["freq"],
                              cfg["refptcl"], cfg["grid"], flagmap=2)
    b = impz.Bunch(cfg["pts"], current, cfg["mass"], cfg["charge"], cfg["freq"],
                   cfg["refptcl"], cfg["grid"], form=form, track_ids=False)
    try:
        b.set_integrator(2)
        recs, zs = b.run(lat)
        refs = b.run_reference()
    finally:
        b.close()
    np.testing.assert_allclose(zs, rows_o[:, 0], rtol=0, atol=0)
    np.testing.assert_array_equal(refs[-1], np.array(beam.refptcl[:]))
    assert abs(-refs[-1][5] + cfg["refptcl"][5]) > 1e-6  # the RF map changes the energy
    rows_g = np.array([impz.diag_row(zs[i], recs[i], refs[i], cfg["mass"], cfg["freq"])
                       for i in range(len(recs))])
    assert worst(rows_g, rows_o, cols) <= tol
