"""GPU parity of the Lorentz integrator (Flagmap=2: drift2 half steps
around the kick2/scatter2 Lorentz kick, BeamBunch.f90:467-509, 2187-3071)
through the C ABI against the oracle, on the proton FODO lattice with
space charge: rms columns of every record within 1e-8 (FP64) and 1e-5
(FP32 form), z exact; the run differs from the map integrator's by far more
than that."""
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
