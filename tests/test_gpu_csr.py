"""GPU parity of the CSR wake of bends through the C ABI against the oracle:
a 250 MeV electron bunch through a small chicane whose dipoles have file ID
300 (CSR inside the bends) or 600 (also the transient CSR downstream of each
bend, AccSimulator.f90:1035-1051, 1131-1138).  The GPU evaluates the same
integrated Green functions (Field.f90:1003-1303), one thread per plane, on
the fixed-point line density; the CSR field amplifies rounding (it differences
neighbouring IGF values), so the FP64 form is held to 1e-7 on the rms
columns, the FP32 form to 1e-5 on the rms sizes, and CSR's own effect on the
bunch is checked to be far larger.  A lattice split into two runs keeps the
bend bookkeeping between them."""
import numpy as np
import pytest

from conftest import load_impz, load_oracle

pytestmark = pytest.mark.gpu

impz = load_impz()
orc = load_oracle()
from impz_b200 import beams  # noqa: E402

RMS_COLS = [6, 7, 8, 9, 11, 12, 13, 14, 15, 17, 18, 19, 20, 21, 23]


def chicane_cfg(fid, n=20_000):
    pts, ref = beams.flat_top_bunch(n, seed=beams.SEED0 + 31, current=10.0)
    lat = beams.chicane(ldrift_in=0.5, drift_steps_in=8, file_id=fid)
    lat.append(impz.elem(0, 0.3, 4, 1, [1.0]))
    return dict(pts=pts, refptcl=ref, current=10.0, mass=beams.ELECTRON_MASS_EV, charge=-1.0,
                freq=1.3e9, grid=(16, 16, 64), lattice=lat)


def rows_of(b, cfg, lat, zs_want):
    recs, zs = b.run(lat)
    np.testing.assert_allclose(zs, zs_want, rtol=0, atol=0)
    refs = b.run_reference()
    return np.array([impz.diag_row(zs[i], recs[i], refs[i], cfg["mass"], cfg["freq"])
                     for i in range(len(recs))])


def worst(rows_g, rows_o, cols):
    w = 0.0
    for c in cols:
        scale = np.max(np.abs(rows_o[:, c])) + 1e-300
        w = max(w, float(np.max(np.abs(rows_g[:, c] - rows_o[:, c])) / scale))
    return w


def oracle(cfg, lat, state=None, pts=None, ref=None, z=0.0):
    return orc.run(lat, cfg["pts"] if pts is None else pts, cfg["current"], cfg["mass"],
                   cfg["charge"], cfg["freq"], cfg["refptcl"] if ref is None else ref,
                   cfg["grid"], z, state)


@pytest.mark.parametrize("fid,form,cols,tol", [
    (300.0, impz.FORM_FP64, RMS_COLS, 1e-7),
    (600.0, impz.FORM_FP64, RMS_COLS, 1e-7),
    (600.0, impz.FORM_FP32CONV, [7, 9, 11, 13, 15, 17, 19, 21, 23], 1e-5)])
def test_csr_chicane_matches_the_oracle(fid, form, cols, tol):
    cfg = chicane_cfg(fid)
    rows_o, _, _ = oracle(cfg, cfg["lattice"])
    rows_plain, _, _ = oracle(cfg, beams.chicane(ldrift_in=0.5, drift_steps_in=8) +
                              [impz.elem(0, 0.3, 4, 1, [1.0])])
    assert worst(rows_plain, rows_o, [21, 23]) > 1e3 * tol  # CSR's own effect
    b = impz.Bunch(cfg["pts"], cfg["current"], cfg["mass"], cfg["charge"], cfg["freq"],
                   cfg["refptcl"], cfg["grid"], form=form, track_ids=False)
    try:
        rows_g = rows_of(b, cfg, cfg["lattice"], rows_o[:, 0])
    finally:
        b.close()
    assert worst(rows_g, rows_o, cols) <= tol


def test_csr_state_carries_across_runs():
    """The chicane's bends in one run and the drift after it in a second:
    the downstream transient still acts, as in one run."""
    cfg = chicane_cfg(600.0)
    lat = cfg["lattice"]
    r1, p1, beam1 = oracle(cfg, lat[:-1])
    r2, _, _ = oracle(cfg, lat[-1:], state=beam1, pts=p1, ref=np.array(beam1.refptcl[:]),
                      z=beam1.z)
    rows_o = np.r_[r1, r2[1:]]
    b = impz.Bunch(cfg["pts"], cfg["current"], cfg["mass"], cfg["charge"], cfg["freq"],
                   cfg["refptcl"], cfg["grid"], form=impz.FORM_FP64, track_ids=False)
    try:
        g1 = rows_of(b, cfg, lat[:-1], r1[:, 0])
        g2 = rows_of(b, cfg, lat[-1:], r2[:, 0])
    finally:
        b.close()
    rows_g = np.r_[g1, g2[1:]]
    assert worst(rows_g, rows_o, RMS_COLS) <= 1e-7
    # without the carried state the last drift would have no CSR
    r2n, _, _ = oracle(cfg, lat[-1:], pts=p1, ref=np.array(beam1.refptcl[:]), z=beam1.z)
    assert worst(r2n[1:], r2[1:], [21, 23]) > 1e-4


def test_csr_transient_under_the_lorentz_integrator():
    """The chicane's bends under the map integrator, then (as after a -25
    switch) the drift behind it under kick2: the downstream transient CSR
    acts through kick2wake (BeamBunch.f90:5048-5938), the raw wake added per
    particle, on the GPU as in the oracle."""
    cfg = chicane_cfg(600.0)
    lat = cfg["lattice"]
    r1, p1, beam1 = oracle(cfg, lat[:-1])
    ref1 = np.array(beam1.refptcl[:])

    def second(state):
        return orc.run(lat[-1:], p1, cfg["current"], cfg["mass"], cfg["charge"], cfg["freq"],
                       ref1, cfg["grid"], beam1.z, state, flagmap=2)[0]

    r2, r2_plain = second(beam1), second(None)
    assert worst(r2_plain[1:], r2[1:], [21, 23]) > 1e-4  # the transient acts
    rows_o = np.r_[r1, r2[1:]]
    b = impz.Bunch(cfg["pts"], cfg["current"], cfg["mass"], cfg["charge"], cfg["freq"],
                   cfg["refptcl"], cfg["grid"], form=impz.FORM_FP64, track_ids=False)
    try:
        g1 = rows_of(b, cfg, lat[:-1], r1[:, 0])
        b.set_integrator(2)
        g2 = rows_of(b, cfg, lat[-1:], r2[:, 0])
    finally:
        b.close()
    assert worst(np.r_[g1, g2[1:]], rows_o, RMS_COLS) <= 1e-7
