"""The C-ABI library loads and exports every entry point of include/impz_b200.h;
its host-only entry points (RK6 maps, diagnostic formulas, step counting)
agree bit for bit with the oracle.  No GPU needed."""
import ctypes

import numpy as np
import pytest

from conftest import load_impz, load_oracle

impz = load_impz()
orc = load_oracle()
from impz_b200 import beams  # noqa: E402


def test_library_exports_every_declared_symbol():
    L = impz.lib()
    declared = impz.declared_symbols()
    assert len(declared) >= 20
    missing = [s for s in declared if not hasattr(L, s)]
    assert not missing, missing


def test_error_strings_and_version():
    assert "sm_100a" in impz.lib().impz_version().decode()
    for code in range(0, -10, -1):
        assert impz.error_string(code) != "unknown error"


def test_create_rejects_bad_arguments_without_device():
    pts, ref = beams.gaussian_bunch(64)
    h = ctypes.c_void_p()
    r = pts.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    rf = ref.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    L = impz.lib()
    # non-power-of-two grid: refused before any device call
    assert L.impz_bunch_create(r, 64, 0.03, 938e6, 1.0, 402.5e6, rf, 30, 32, 64, 0, 0,
                               ctypes.byref(h)) == impz.ERR_UNSUPPORTED
    assert L.impz_bunch_create(r, 0, 0.03, 938e6, 1.0, 402.5e6, rf, 32, 32, 64, 0, 0,
                               ctypes.byref(h)) == impz.ERR_ARG


@pytest.mark.parametrize("mapstp", [1, 3])
def test_quad_linear_map_matches_oracle_bitwise(mapstp):
    freq, mass, charge = 402.5e6, beams.PROTON_MASS_EV, 1.0
    ref = beams.refptcl_for(2.5e6, mass)
    e = impz.elem(1, 0.1, 4, mapstp, [20.0, 0.0, 1.0])
    xm_p, ref_p = impz.maplinear(e, 0.0, 0.3, 0.0125, ref, charge, mass, freq)
    orc.physconst(freq)
    xm_o = np.zeros(36)
    ref_o = ref.copy()
    orc.lib().orc_maplinear_quad(0.3, 0.0125, orc.dp(xm_o), orc.dp(ref_o), 20.0, mapstp, charge,
                                 mass)
    np.testing.assert_array_equal(xm_p, xm_o.reshape(6, 6, order="F"))
    np.testing.assert_array_equal(ref_p, ref_o)


def test_ccl_linear_map_matches_oracle_bitwise():
    freq, mass, charge = 402.5e6, beams.PROTON_MASS_EV, 1.0
    ref = beams.refptcl_for(2.5e6, mass)
    zt = np.linspace(0.0, 0.2, 41)
    ez = 1e6 * np.sin(np.pi * zt / 0.2)
    ezp = 1e6 * np.pi / 0.2 * np.cos(np.pi * zt / 0.2)
    ezpp = -1e6 * (np.pi / 0.2) ** 2 * np.sin(np.pi * zt / 0.2)
    e = impz.elem(103, 0.2, 4, 5, [1.0, 402.5e6, -30.0, 1.0, 0.01], rf=(zt, ez, ezp, ezpp))
    xm_p, ref_p = impz.maplinear(e, 0.0, 0.05, 0.025, ref, charge, mass, freq)
    orc.physconst(freq)
    xm_o = np.zeros(36)
    ref_o = ref.copy()
    cols = [np.ascontiguousarray(c) for c in (zt, ez, ezp, ezpp)]
    orc.lib().orc_maplinear_ccl(0.05, 0.025, orc.dp(xm_o), orc.dp(ref_o), 0.0, 1.0, 402.5e6,
                                -30.0, 5, charge, mass, len(zt), *[orc.dp(c) for c in cols])
    np.testing.assert_array_equal(xm_p, xm_o.reshape(6, 6, order="F"))
    np.testing.assert_array_equal(ref_p, ref_o)


def test_diag_row_matches_oracle_bitwise():
    freq, mass = 402.5e6, beams.PROTON_MASS_EV
    pts, ref = beams.gaussian_bunch(5000, seed=3)
    orc.physconst(freq)
    raw = np.zeros(orc.RAW_LEN)
    orc.lib().orc_moment_sums(orc.dp(np.ascontiguousarray(pts)), pts.shape[0], orc.dp(raw))
    row_o = np.zeros(orc.DIAG_LEN)
    orc.lib().orc_diag_row(0.7, orc.dp(raw), pts.shape[0], pts.shape[0], orc.dp(ref), mass,
                           orc.dp(row_o))
    rec = np.zeros(impz.MOMREC)
    rec[:44] = raw
    rec[44] = rec[45] = pts.shape[0]
    row_p = impz.diag_row(0.7, rec, ref, mass, freq)
    np.testing.assert_array_equal(row_p, row_o)


def test_count_steps():
    assert impz.count_steps(beams.fodo(10)) == 160
    assert impz.count_steps(beams.fodo(25, nseg=10)) == 1000


def test_footprint_is_exact_arena_plus_tables():
    mib2 = 2 << 20
    grid = (64, 64, 128)
    f0 = impz.footprint(4_000_000, grid)
    # particles (two parity sets of six FP64 columns) dominate; granule-rounded
    assert f0 % mib2 == 0
    assert f0 >= 4_000_000 * 96 + 64 * 64 * 128 * 16
    assert impz.footprint(4_000_000, grid, track_ids=True) >= f0 + 4_000_000 * 16
    # the FP32 form holds smaller spectra than the FP64 form
    assert impz.footprint(4_000_000, grid, form=impz.FORM_FP64) > f0
    # a run's tables add to the bunch alone
    assert impz.footprint(4_000_000, grid, nsteps=1000) > f0
    assert impz.lib().impz_bunch_footprint(0, 64, 64, 128, 1, 0, 0) == -1
    assert impz.lib().impz_bunch_footprint(10, 64, 64, 128, 1, 0, -1) == -1


@pytest.mark.parametrize("etype", [101, 102, 104])
def test_dtl_ccdtl_sc_linear_maps_match_oracle_bitwise(etype):
    """CCDTL and SC use CCL's map; DTL adds its drift-tube quadrupoles
    (getBgradfld_DTL: 5 cm at +8 T/m, 4 cm at -6 T/m at the ends)."""
    freq, mass, charge = 402.5e6, beams.PROTON_MASS_EV, 1.0
    ref = beams.refptcl_for(2.5e6, mass)
    zt = np.linspace(0.0, 0.2, 41)
    ez = 1e6 * np.sin(np.pi * zt / 0.2)
    ezp = 1e6 * np.pi / 0.2 * np.cos(np.pi * zt / 0.2)
    ezpp = -1e6 * (np.pi / 0.2) ** 2 * np.sin(np.pi * zt / 0.2)
    vals = [1.0, 402.5e6, -30.0, 1.0, 0.01, 0.05, 8.0, 0.04, -6.0]
    e = impz.elem(etype, 0.2, 4, 5, vals, rf=(zt, ez, ezp, ezpp))
    cols = [np.ascontiguousarray(c) for c in (zt, ez, ezp, ezpp)]
    orc.physconst(freq)
    for t in (0.01, 0.08, 0.17):  # in the first quadrupole, between, in the second
        xm_p, ref_p = impz.maplinear(e, 0.0, t, 0.025, ref, charge, mass, freq)
        xm_o, ref_o = np.zeros(36), ref.copy()
        args = (t, 0.025, orc.dp(xm_o), orc.dp(ref_o), 0.0, 1.0, 402.5e6, -30.0, 5, charge,
                mass, len(zt), *[orc.dp(c) for c in cols])
        if etype == 101:
            orc.lib().orc_maplinear_dtl(*args, 0.2, 0.05, 8.0, 0.04, -6.0)
        else:
            orc.lib().orc_maplinear_ccl(*args)
        np.testing.assert_array_equal(xm_p, xm_o.reshape(6, 6, order="F"))
        np.testing.assert_array_equal(ref_p, ref_o)
    if etype == 101:  # the quadrupole shows in the transverse blocks
        xm_d, _ = impz.maplinear(e, 0.0, 0.01, 0.025, ref, charge, mass, freq)
        xm_c, _ = impz.maplinear(impz.elem(103, 0.2, 4, 5, vals, rf=(zt, ez, ezp, ezpp)), 0.0,
                                 0.01, 0.025, ref, charge, mass, freq)
        assert abs(xm_d[1, 0] - xm_c[1, 0]) > 1e-3 * abs(xm_c[1, 0]) + 1e-9
        assert abs(xm_d[3, 2] - xm_c[3, 2]) > 1e-3 * abs(xm_c[3, 2]) + 1e-9


def solrf_coefficients(length=0.2):
    """read3_Data's layout: count, start, end, period, then the constant,
    cosine and sine terms of a cavity-like Ez."""
    terms = [0.4, 0.8, 0.0, -0.3, 0.05, 0.1, 0.02]
    return np.array([len(terms), 0.0, length, length] + terms)


def test_solrf_linear_map_matches_oracle_bitwise():
    """maplinear_SolRF (SolRF.f90:126-353): the Fourier on-axis field and a
    0.2 T solenoid whose rotation couples x and y."""
    freq, mass, charge = 402.5e6, beams.PROTON_MASS_EV, 1.0
    ref = beams.refptcl_for(2.5e6, mass)
    coef = solrf_coefficients()
    vals = [1e6, 402.5e6, -30.0, 1.0, 0.01, 0, 0, 0, 0, 0, 0.2]
    e = impz.elem(105, 0.2, 4, 5, vals, rf=coef)
    orc.physconst(freq)
    for t in (0.0, 0.07, 0.175):
        xm_p, ref_p = impz.maplinear(e, 0.0, t, 0.025, ref, charge, mass, freq)
        xm_o, ref_o = np.zeros(36), ref.copy()
        orc.lib().orc_maplinear_solrf(t, 0.025, orc.dp(xm_o), orc.dp(ref_o), 0.0, 1e6, 402.5e6,
                                      -30.0, 5, charge, mass, 0.2, 0.2, len(coef), orc.dp(coef))
        np.testing.assert_array_equal(xm_p, xm_o.reshape(6, 6, order="F"))
        np.testing.assert_array_equal(ref_p, ref_o)
    assert abs(xm_p[0, 2]) > 1e-6 and abs(xm_p[2, 0]) > 1e-6  # the solenoid couples x, y
    assert abs(ref_p[5] - ref[5]) > 1e-7  # and the gap changes the energy


def tws_coefficients(length=0.2):
    """Two series (read3_Data's layout for TWS): a standing wave over the
    element and a second one over its middle."""
    s1 = [0.3, 0.9, 0.1, -0.2, 0.05]
    s2 = [0.2, 0.5, -0.4, 0.1, 0.0, 0.02, 0.03]
    return np.array([len(s1), 0.0, length, length] + s1 +
                    [len(s2), 0.05, 0.15, 0.1] + s2)


def test_tws_linear_map_matches_oracle_bitwise():
    """maplinear_TWS (TWS.f90:129-466): two standing waves, the second 90
    degrees later and only over the middle of the element."""
    freq, mass, charge = 402.5e6, beams.PROTON_MASS_EV, 1.0
    ref = beams.refptcl_for(2.5e6, mass)
    coef = tws_coefficients()
    vals = [1e6, 402.5e6, -30.0, 1.0, 0.01, 0, 0, 0, 0, 0, 90.0]
    e = impz.elem(106, 0.2, 4, 5, vals, rf=coef)
    orc.physconst(freq)
    outs = []
    for t in (0.0, 0.06, 0.175):
        xm_p, ref_p = impz.maplinear(e, 0.0, t, 0.025, ref, charge, mass, freq)
        xm_o, ref_o = np.zeros(36), ref.copy()
        orc.lib().orc_maplinear_tws(t, 0.025, orc.dp(xm_o), orc.dp(ref_o), 0.0, 1e6, 402.5e6,
                                    -30.0, 5, charge, mass, 0.2, 90.0, len(coef), orc.dp(coef))
        np.testing.assert_array_equal(xm_p, xm_o.reshape(6, 6, order="F"))
        np.testing.assert_array_equal(ref_p, ref_o)
        outs.append(xm_p)
    # the second wave acts in the middle: a zero second series changes it there
    c0 = coef.copy()
    c0[14:] = 0.0
    xm_1, _ = impz.maplinear(impz.elem(106, 0.2, 4, 5, vals, rf=c0), 0.0, 0.06, 0.025, ref,
                             charge, mass, freq)
    assert abs(xm_1[1, 0] - outs[1][1, 0]) > 1e-6 * abs(outs[1][1, 0])


def quad_profile(length=0.1, g=20.0, n=51):
    """A gradient profile with soft edges (Enge-like tanh), z from 0."""
    z = np.linspace(0.0, length, n)
    prof = g * 0.25 * (1 + np.tanh((z - 0.015) / 0.005)) * (1 + np.tanh((length - 0.015 - z) /
                                                                          0.005))
    return z, prof, np.zeros(n), np.zeros(n)


def test_fringe_field_quadrupole_map_matches_oracle_bitwise():
    """maplinear_Quadrupole with a gradient profile (file ID v2 > 1e-5,
    getfldfrg_Quadrupole): host = oracle bitwise, and the soft edges make
    it weaker than the hard-edge quadrupole of the peak gradient."""
    freq, mass, charge = 402.5e6, beams.PROTON_MASS_EV, 1.0
    ref = beams.refptcl_for(2.5e6, mass)
    z, g, z0, z1 = quad_profile()
    e = impz.elem(1, 0.1, 4, 5, [20.0, 7.0, 1.0], rf=(z, g, z0, z1))
    orc.physconst(freq)
    for t in (0.0, 0.0125, 0.05):
        xm_p, ref_p = impz.maplinear(e, 0.0, t, 0.0125, ref, charge, mass, freq)
        xm_o, ref_o = np.zeros(36), ref.copy()
        orc.lib().orc_maplinear_quad_fringe(t, 0.0125, orc.dp(xm_o), orc.dp(ref_o), 0.0, 5,
                                            charge, mass, len(z), orc.dp(np.ascontiguousarray(z)),
                                            orc.dp(np.ascontiguousarray(g)))
        np.testing.assert_array_equal(xm_p, xm_o.reshape(6, 6, order="F"))
        np.testing.assert_array_equal(ref_p, ref_o)
    hard, _ = impz.maplinear(impz.elem(1, 0.1, 4, 5, [20.0, 0.0, 1.0]), 0.0, 0.0, 0.0125, ref,
                             charge, mass, freq)
    soft, _ = impz.maplinear(e, 0.0, 0.0, 0.0125, ref, charge, mass, freq)
    assert abs(soft[1, 0]) < abs(hard[1, 0])


def test_solenoid_map_matches_oracle_bitwise():
    """maplinear_Sol (Sol.f90:120-316): a 0.5 T solenoid rotates x into y."""
    freq, mass, charge = 402.5e6, beams.PROTON_MASS_EV, 1.0
    ref = beams.refptcl_for(2.5e6, mass)
    e = impz.elem(3, 0.2, 4, 5, [0.5, 0.0, 1.0, 0.0])
    orc.physconst(freq)
    xm_p, ref_p = impz.maplinear(e, 0.0, 0.05, 0.025, ref, charge, mass, freq)
    xm_o, ref_o = np.zeros(36), ref.copy()
    orc.lib().orc_maplinear_sol(0.05, 0.025, orc.dp(xm_o), orc.dp(ref_o), 0.5, 5, charge, mass)
    np.testing.assert_array_equal(xm_p, xm_o.reshape(6, 6, order="F"))
    np.testing.assert_array_equal(ref_p, ref_o)
    assert abs(xm_p[0, 2]) > 1e-6 and abs(xm_p[2, 0]) > 1e-6


def test_constant_focusing_map_matches_oracle_bitwise():
    """maplinear_ConstFoc (ConstFoc.f90): kx0^2, ky0^2, kz0^2."""
    freq, mass, charge = 402.5e6, beams.PROTON_MASS_EV, 1.0
    ref = beams.refptcl_for(2.5e6, mass)
    k2 = np.array([30.0, 20.0, 5.0])
    e = impz.elem(2, 0.2, 4, 5, list(k2) + [1.0])
    orc.physconst(freq)
    xm_p, ref_p = impz.maplinear(e, 0.0, 0.05, 0.025, ref, charge, mass, freq)
    xm_o, ref_o = np.zeros(36), ref.copy()
    orc.lib().orc_maplinear_constfoc(0.05, 0.025, orc.dp(xm_o), orc.dp(ref_o), orc.dp(k2), 5)
    np.testing.assert_array_equal(xm_p, xm_o.reshape(6, 6, order="F"))
    np.testing.assert_array_equal(ref_p, ref_o)
    assert xm_p[1, 0] < 0 and xm_p[3, 2] < 0 and xm_p[5, 4] < 0  # focusing in all three
