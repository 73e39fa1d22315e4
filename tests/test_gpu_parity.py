"""GPU parity: the CUDA path, called through the C ABI, against the CPU oracle.

Tolerances (plain FP64 form):
  * grid geometry, cell indices, per-cell counts: bit-exact
  * charge density, potential, fields: relative L2 <= 1e-12
  * particle coordinates after one kick and half map: max relative error
    <= 1e-11 of each column's rms (the potential differs at rounding level)
  * rms sizes, emittances, centroids after a full lattice: rel <= 1e-8
FP32-convolution form: rms moments within 1e-5 relative of the FP64 oracle.
"""
import ctypes

import numpy as np
import pytest

from conftest import load_impz, load_oracle

pytestmark = pytest.mark.gpu

impz = load_impz()
orc = load_oracle()
from impz_b200 import beams  # noqa: E402


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def oracle_step(pts, cfg, e_first, tau, piperad):
    """One space-charge step of the reference sequence on the oracle:
    drift1 half map -> conv1st -> update_CompDom -> deposit -> openBC3D ->
    cvbkforth1st -> kick1 (AccSimulator.f90:1109-1426)."""
    P = orc.physconst(cfg["freq"])
    L = orc.lib()
    p = np.ascontiguousarray(pts, dtype=np.float64).copy()
    n = p.shape[0]
    ref = np.array(cfg["refptcl"], dtype=np.float64)
    L.orc_drift_exact(orc.dp(p), n, orc.dp(ref), tau / 2)
    cur = ctypes.c_double(cfg["current"])
    npt = ctypes.c_int(n)
    ptrange = np.zeros(6)
    nl = L.orc_conv1st(orc.dp(p), n, ctypes.byref(cur), ctypes.byref(npt), orc.dp(ref),
                       piperad, piperad, orc.dp(ptrange))
    mesh = np.array(cfg["grid"], dtype=np.int32)
    rng, msize = np.zeros(6), np.zeros(3)
    L.orc_update_compdom(orc.dp(ptrange), mesh.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                         orc.dp(rng), orc.dp(msize))
    G = int(np.prod(cfg["grid"]))
    rho = np.zeros(G)
    counts = np.zeros(G, dtype=np.int32)
    cells = np.zeros(nl, dtype=np.int64)
    L.orc_deposit(orc.dp(p), nl, mesh.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), orc.dp(rng),
                  orc.dp(msize), orc.dp(rho), counts.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                  cells.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)))
    phi = rho.copy()
    assert L.orc_poisson_open(int(mesh[0]), int(mesh[1]), int(mesh[2]), msize[0], msize[1],
                              msize[2], orc.dp(phi)) == 0
    L.orc_cvbkforth1st(orc.dp(p), nl, orc.dp(ref))
    eg = np.zeros(3 * G)
    L.orc_kick1(orc.dp(p), nl, orc.dp(phi), mesh.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                orc.dp(rng), orc.dp(msize), -ref[5], cur.value, tau, cfg["mass"], cfg["charge"],
                orc.dp(eg))
    L.orc_drift_exact(orc.dp(p), nl, orc.dp(ref), tau / 2)
    return dict(pts=p[:nl], ptrange=ptrange, range=rng, msize=msize, rho=rho, counts=counts,
                phi=phi, eg=eg, nptot=npt.value, current=cur.value, ref=ref)


def gpu_step(pts, cfg, e_first, tau, piperad, form=impz.FORM_FP64):
    b = impz.Bunch(pts, cfg["current"], cfg["mass"], cfg["charge"], cfg["freq"], cfg["refptcl"],
                   cfg["grid"], form=form, track_ids=True)
    z, ih = b.map_half(e_first, 0.0, 0.0, tau / 2, 1, 0)
    nptot, ptrange, rng, msize = b.sc_prepare(piperad, piperad)
    rho, counts = b.deposit()
    phi = b.poisson()
    eg = b.kick(tau, want_e=True)
    z, ih = b.map_half(e_first, 0.0, z, tau / 2, 1, ih)
    out = dict(pts=b.download(), ptrange=ptrange, range=rng, msize=msize, rho=rho, counts=counts,
               phi=phi, eg=eg, nptot=nptot, info=b.info())
    b.close()
    return out


@pytest.fixture(scope="module")
def small():
    cfg = beams.fodo_1e5(n=20_000, seed=beams.SEED0 + 7)
    return cfg


def test_single_step_fp64_parity(small):
    cfg = small
    e = impz.elem(0, 0.1, 4, 1, [1.0])
    tau = 0.1 / 4
    o = oracle_step(cfg["pts"], cfg, e, tau, 1.0)
    g = gpu_step(cfg["pts"], cfg, e, tau, 1.0)
    # geometry and cells bit-exact
    assert g["nptot"] == o["nptot"]
    np.testing.assert_array_equal(g["ptrange"], o["ptrange"])
    np.testing.assert_array_equal(g["range"], o["range"])
    np.testing.assert_array_equal(g["msize"], o["msize"])
    np.testing.assert_array_equal(g["counts"], o["counts"])
    assert rel_l2(g["rho"], o["rho"]) <= 1e-12
    assert rel_l2(g["phi"], o["phi"]) <= 1e-12
    assert rel_l2(g["eg"], o["eg"]) <= 1e-12
    # particles, matched by id
    gp = g["pts"][np.argsort(g["pts"][:, 8])]
    op = o["pts"][np.argsort(o["pts"][:, 8])]
    np.testing.assert_array_equal(gp[:, 8], op[:, 8])
    for c in range(6):
        scale = np.sqrt(np.mean(op[:, c] ** 2))
        err = np.max(np.abs(gp[:, c] - op[:, c])) / scale
        assert err <= 1e-11, (c, err)


def test_charge_conservation_and_counts(small):
    cfg = small
    e = impz.elem(0, 0.1, 4, 1, [1.0])
    g = gpu_step(cfg["pts"], cfg, e, 0.025, 1.0)
    n = cfg["pts"].shape[0]
    w = cfg["pts"][0, 7]
    assert int(g["counts"].sum()) == n
    assert abs(g["rho"].sum() - n * w) <= 1e-12 * n * abs(w)


def test_quad_kmap_and_linear_map_parity(small):
    cfg = small
    n = 4096
    pts = cfg["pts"][:n].copy()
    # gradient quad: RK6 linear map built on the host, applied on the GPU
    eq = impz.elem(1, 0.1, 4, 3, [20.0, 0.0, 1.0])
    P = orc.physconst(cfg["freq"])
    xm_o = np.zeros(36)
    ref_o = np.array(cfg["refptcl"])
    orc.lib().orc_maplinear_quad(0.0, 0.0125, orc.dp(xm_o), orc.dp(ref_o), 20.0, 3,
                                 cfg["charge"], cfg["mass"])
    p_o = pts.copy()
    orc.lib().orc_apply_xm(orc.dp(p_o), n, orc.dp(xm_o))
    b = impz.Bunch(pts, cfg["current"], cfg["mass"], cfg["charge"], cfg["freq"], cfg["refptcl"],
                   (32, 32, 64), track_ids=True)
    b.map_half(eq, 0.0, 0.0, 0.0125, 1, 0)
    p_g = b.download()
    p_g = p_g[np.argsort(p_g[:, 8])]  # the upload ordered the bunch by cell; ids are 1..n
    np.testing.assert_array_equal(p_g[:, :6], p_o[:, :6])
    np.testing.assert_array_equal(b.info()["refptcl"], ref_o)
    b.close()
    # K-map (file ID in (-10,-1e-6)): per-particle cos/cosh, CUDA libm
    ek = impz.elem(1, 0.1, 4, 1, [30.0, -1.0, 1.0])
    p_o = pts.copy()
    ref_o = np.array(cfg["refptcl"])
    orc.lib().orc_transfmapK(0.0125, 30.0, orc.dp(ref_o), orc.dp(p_o), n,
                             cfg["charge"] / cfg["mass"])
    b = impz.Bunch(pts, cfg["current"], cfg["mass"], cfg["charge"], cfg["freq"], cfg["refptcl"],
                   (32, 32, 64), track_ids=True)
    b.map_half(ek, 0.0, 0.0, 0.0125, 1, 0)
    p_g = b.download()
    p_g = p_g[np.argsort(p_g[:, 8])]
    for c in range(6):
        scale = np.sqrt(np.mean(p_o[:, c] ** 2)) + 1e-300
        assert np.max(np.abs(p_g[:, c] - p_o[:, c])) / scale <= 1e-13
    b.close()


def _row_cmp(rows_g, rows_o, cols, tol):
    worst = 0.0
    for c in cols:
        scale = np.max(np.abs(rows_o[:, c])) + 1e-300
        worst = max(worst, float(np.max(np.abs(rows_g[:, c] - rows_o[:, c])) / scale))
    assert worst <= tol, worst
    return worst


RMS_COLS = [6, 7, 8, 9, 11, 12, 13, 14, 15, 17, 18, 19, 20, 21, 23]


def gpu_rows(cfg, form):
    b = impz.Bunch(cfg["pts"], cfg["current"], cfg["mass"], cfg["charge"], cfg["freq"],
                   cfg["refptcl"], cfg["grid"], form=form, track_ids=False)
    recs, zs = b.run(cfg["lattice"])
    # the reference particle of each record follows the same host arithmetic
    rows_g = []
    b.close()
    return recs, zs


def test_full_lattice_fp64_moments():
    cfg = beams.fodo_1e5(n=20_000, seed=beams.SEED0 + 11)
    cfg["lattice"] = beams.fodo(2)  # 32 steps
    rows_o, p_o, beam = orc.run(cfg["lattice"], cfg["pts"], cfg["current"], cfg["mass"],
                                cfg["charge"], cfg["freq"], cfg["refptcl"], cfg["grid"])
    recs, zs = gpu_rows(cfg, impz.FORM_FP64)
    assert recs.shape[0] == rows_o.shape[0]
    np.testing.assert_allclose(zs, rows_o[:, 0], rtol=0, atol=0)
    # rebuild rows with the oracle's reference trajectory (fort.18 columns)
    rows_g = np.array([impz.diag_row(rows_o[i, 0], recs[i], _ref_of(rows_o[i], cfg), cfg["mass"],
                                     cfg["freq"]) for i in range(len(recs))])
    _row_cmp(rows_g, rows_o, RMS_COLS, 1e-8)


def test_full_lattice_fp32conv_moments():
    cfg = beams.fodo_1e5(n=20_000, seed=beams.SEED0 + 11)
    cfg["lattice"] = beams.fodo(2)
    rows_o, p_o, beam = orc.run(cfg["lattice"], cfg["pts"], cfg["current"], cfg["mass"],
                                cfg["charge"], cfg["freq"], cfg["refptcl"], cfg["grid"])
    recs, zs = gpu_rows(cfg, impz.FORM_FP32CONV)
    rows_g = np.array([impz.diag_row(rows_o[i, 0], recs[i], _ref_of(rows_o[i], cfg), cfg["mass"],
                                     cfg["freq"]) for i in range(len(recs))])
    _row_cmp(rows_g, rows_o, [7, 9, 11, 13, 15, 17, 19, 21, 23], 1e-5)


def _ref_of(row, cfg):
    """refptcl from a fort.18 row: refptcl(5) and -gamma."""
    r = np.zeros(6)
    r[4] = row[1]
    r[5] = -row[2]
    return r


def mixed_lattice():
    """Drift, quadrupoles, an ideal RF gap (v4 < 0) and a sector bend: every
    map kind of the runner beyond drifts and block-diagonal maps."""
    rf = impz.elem(101, 0.1, 4, 1, [1.0e6, 402.5e6, -30.0, -1.0, 1.0])
    bend = impz.elem(4, 0.2, 4, 1, [0.05, 0.0, 150.0, 0.01, 0.0, 0.0, 0.0, 0.0, 0.0])
    return (beams.fodo(1) + [rf, impz.elem(0, 0.1, 4, 1, [1.0]), bend,
                             impz.elem(0, 0.1, 4, 1, [1.0])])


def test_mixed_lattice_after_light_run_fp64_moments():
    cfg = beams.fodo_1e5(n=20_000, seed=beams.SEED0 + 12)
    lat = mixed_lattice()
    rows_o, p_o, beam = orc.run(lat, cfg["pts"], cfg["current"], cfg["mass"], cfg["charge"],
                                cfg["freq"], cfg["refptcl"], cfg["grid"])
    b = impz.Bunch(cfg["pts"], cfg["current"], cfg["mass"], cfg["charge"], cfg["freq"],
                   cfg["refptcl"], cfg["grid"], form=impz.FORM_FP64, track_ids=False)
    # a drift/quadrupole run first: its graphs hold the light particle pass,
    # which must not be replayed for the bend and RF steps
    b.run(beams.fodo(1))
    b.upload(cfg["pts"], cfg["current"], cfg["refptcl"])
    recs, zs = b.run(lat)
    b.close()
    assert recs.shape[0] == rows_o.shape[0]
    np.testing.assert_allclose(zs, rows_o[:, 0], rtol=0, atol=0)
    rows_g = np.array([impz.diag_row(rows_o[i, 0], recs[i], _ref_of(rows_o[i], cfg), cfg["mass"],
                                     cfg["freq"]) for i in range(len(recs))])
    _row_cmp(rows_g, rows_o, RMS_COLS, 1e-8)


@pytest.mark.parametrize("grid,form,tol,etol", [((16, 16, 1024), impz.FORM_FP64, 1e-12, 1e-10),
                                                ((16, 16, 2048), impz.FORM_FP32CONV, 1e-5, 1e-4)])
def test_single_step_long_z_grid(grid, form, tol, etol):
    """Long z lines: the z convolution and the Green DCT take fewer lines per
    block (shared memory), down to four; the potential matches the oracle to
    `tol` (FP64: 1e-12; FP32 convolution: 1e-5 relative L2).  The field is a
    centred difference of neighbouring potentials, which on a 1024-cell axis
    differ by ~1e-3 of their value, so it carries the potential's rounding
    amplified ~1e3: `etol` = 100 tol."""
    cfg = beams.fodo_1e5(n=20_000, seed=beams.SEED0 + 13)
    cfg["grid"] = grid
    e = impz.elem(0, 0.1, 4, 1, [1.0])
    o = oracle_step(cfg["pts"], cfg, e, 0.025, 1.0)
    g = gpu_step(cfg["pts"], cfg, e, 0.025, 1.0, form=form)
    if form == impz.FORM_FP64:
        np.testing.assert_array_equal(g["counts"], o["counts"])
    else:  # FP32 form: rounding-level map differences may move a particle's cell
        assert np.abs(g["counts"] - o["counts"]).sum() <= 8
    assert rel_l2(g["phi"], o["phi"]) <= tol
    assert rel_l2(g["eg"], o["eg"]) <= etol


def test_electron_chicane_fp64_moments_and_bunching():
    """250 MeV electrons with a 1 % density modulation at 10 µm through a drift
    and the four sector bends of a chicane (pole faces and the Brown map of
    Dipole.f90), FP64: rms columns of every record within 1e-8 of the oracle.
    The bunching factor of the final bunch equals numpy's on the downloaded
    particles (1e-12)."""
    pts, ref = beams.flat_top_bunch(20_000, seed=beams.SEED0 + 31, current=10.0)
    cfg = dict(pts=pts, refptcl=ref, current=10.0, mass=beams.ELECTRON_MASS_EV, charge=-1.0,
               freq=1.3e9, grid=(16, 16, 64),
               lattice=beams.chicane(ldrift_in=0.5, drift_steps_in=8))
    rows_o, p_o, beam = orc.run(cfg["lattice"], cfg["pts"], cfg["current"], cfg["mass"],
                                cfg["charge"], cfg["freq"], cfg["refptcl"], cfg["grid"])
    b = impz.Bunch(cfg["pts"], cfg["current"], cfg["mass"], cfg["charge"], cfg["freq"],
                   cfg["refptcl"], cfg["grid"], form=impz.FORM_FP64, track_ids=False)
    recs, zs = b.run(cfg["lattice"])
    assert recs.shape[0] == rows_o.shape[0]
    np.testing.assert_allclose(zs, rows_o[:, 0], rtol=0, atol=0)
    rows_g = np.array([impz.diag_row(rows_o[i, 0], recs[i], _ref_of(rows_o[i], cfg), cfg["mass"],
                                     cfg["freq"]) for i in range(len(recs))])
    _row_cmp(rows_g, rows_o, RMS_COLS, 1e-8)
    k = 2 * np.pi / 10e-6
    got = b.bunching(k)
    p = b.download()
    gam0 = -b.info()["refptcl"][5]
    z = -p[:, 4] * np.sqrt(1 - 1 / gam0 ** 2) * beams.scxl(cfg["freq"])
    want = np.mean(np.exp(-1j * k * z))
    b.close()
    assert abs(got - want) <= 1e-12 * max(1.0, abs(want)) + 1e-12


@pytest.mark.parametrize("form", [impz.FORM_FP64, impz.FORM_FP32CONV])
def test_single_step_with_particle_loss(small, form):
    """A pipe of radius 2 mm (1 mm rms beam) loses particles in conv1st: the
    surviving count, the rescaled current, the range (which still includes
    the lost particles), cells and per-cell counts equal the oracle's bit for
    bit; the kicked survivors match by id (FP64: 1e-11; FP32 convolution:
    the fields to 1e-5)."""
    cfg = small
    e = impz.elem(0, 0.1, 4, 1, [1.0])
    rad = 2e-3
    o = oracle_step(cfg["pts"], cfg, e, 0.025, rad)
    g = gpu_step(cfg["pts"], cfg, e, 0.025, rad, form=form)
    n = cfg["pts"].shape[0]
    assert 0 < o["nptot"] < n
    assert g["pts"].shape[0] == g["nptot"] and int(g["counts"].sum()) == g["nptot"]
    if form == impz.FORM_FP64:
        assert g["nptot"] == o["nptot"]
        assert g["info"]["current"] == o["current"]
        np.testing.assert_array_equal(g["ptrange"], o["ptrange"])
        np.testing.assert_array_equal(g["range"], o["range"])
        np.testing.assert_array_equal(g["counts"], o["counts"])
        np.testing.assert_array_equal(np.sort(g["pts"][:, 8]), np.sort(o["pts"][:, 8]))
        assert rel_l2(g["rho"], o["rho"]) <= 1e-12
        assert rel_l2(g["eg"], o["eg"]) <= 1e-12
        gp = g["pts"][np.argsort(g["pts"][:, 8])]
        op = o["pts"][np.argsort(o["pts"][:, 8])]
        for c in range(6):
            scale = np.sqrt(np.mean(op[:, c] ** 2))
            assert np.max(np.abs(gp[:, c] - op[:, c])) / scale <= 1e-11, c
    else:
        # the FP32 form's maps use reciprocal/rsqrt arithmetic: positions agree
        # to rounding, so geometry agrees to 1e-12 and a particle on a pipe or
        # cell boundary may fall on the other side
        assert abs(g["nptot"] - o["nptot"]) <= 2
        np.testing.assert_allclose(g["ptrange"], o["ptrange"], rtol=1e-12, atol=0)
        np.testing.assert_allclose(g["range"], o["range"], rtol=1e-12, atol=0)
        assert np.abs(g["counts"] - o["counts"]).sum() <= 8
        assert rel_l2(g["eg"], o["eg"]) <= 1e-5


def rf_table(length=0.2, amp=1e6, n=41):
    zt = np.linspace(0.0, length, n)
    k = np.pi / length
    return zt, amp * np.sin(k * zt), amp * k * np.cos(k * zt), -amp * k * k * np.sin(k * zt)


def test_rf_linear_maps_lattice_fp64_moments():
    """Drift, then a DTL (101, with its drift-tube quadrupoles), a CCDTL
    (102), a CCL (103) and an SC cavity (104) as linear maps over an
    on-axis table (maplinear_DTL/CCDTL/CCL/SC), a SolRF (105, Fourier field
    and a 0.2 T solenoid) and a TWS (106, two standing waves), after a
    quadrupole with a soft-edged gradient profile, an undulator section
    (a quadrupole with v2 < -10), a 0.5 T solenoid (type 3) and a
    constant-focusing channel (type 2), FP64: rms
    columns of every record within 1e-8 of the oracle, z exact."""
    from test_abi import quad_profile, solrf_coefficients, tws_coefficients

    cfg = beams.fodo_1e5(n=20_000, seed=beams.SEED0 + 14)
    tab = rf_table()
    gap = lambda t, v: impz.elem(t, 0.2, 4, 5, v, rf=tab)  # noqa: E731
    lat = [impz.elem(0, 0.1, 2, 1, [1.0]),
           impz.elem(1, 0.1, 4, 5, [20.0, 7.0, 1.0], rf=quad_profile()),
           impz.elem(1, 0.2, 4, 1, [40.0, -20.0, 1.0]),
           impz.elem(3, 0.2, 4, 5, [0.5, 0.0, 1.0, 0.0]),
           impz.elem(2, 0.2, 4, 5, [30.0, 20.0, 5.0, 1.0]),
           gap(101, [1.0, 402.5e6, -30.0, 1.0, 1.0, 0.05, 15.0, 0.05, -15.0]),
           gap(102, [1.0, 402.5e6, -30.0, 1.0, 1.0]), gap(103, [1.0, 402.5e6, -30.0, 1.0, 1.0]),
           gap(104, [1.0, 402.5e6, -30.0, 1.0, 1.0]),
           impz.elem(105, 0.2, 4, 5, [1e6, 402.5e6, -30.0, 1.0, 1.0, 0, 0, 0, 0, 0, 0.2],
                     rf=solrf_coefficients()),
           impz.elem(106, 0.2, 4, 5, [1e6, 402.5e6, -30.0, 1.0, 1.0, 0, 0, 0, 0, 0, 90.0],
                     rf=tws_coefficients()),
           impz.elem(0, 0.1, 2, 1, [1.0])]
    rows_o, p_o, beam = orc.run(lat, cfg["pts"], cfg["current"], cfg["mass"], cfg["charge"],
                                cfg["freq"], cfg["refptcl"], cfg["grid"])
    b = impz.Bunch(cfg["pts"], cfg["current"], cfg["mass"], cfg["charge"], cfg["freq"],
                   cfg["refptcl"], cfg["grid"], form=impz.FORM_FP64, track_ids=False)
    recs, zs = b.run(lat)
    refs = b.run_reference()
    b.close()
    assert recs.shape[0] == rows_o.shape[0] == 45
    np.testing.assert_allclose(zs, rows_o[:, 0], rtol=0, atol=0)
    np.testing.assert_allclose(refs[:, 4:6], np.c_[rows_o[:, 1], -rows_o[:, 2]], rtol=1e-14,
                               atol=0)
    rows_g = np.array([impz.diag_row(zs[i], recs[i], refs[i], cfg["mass"], cfg["freq"])
                       for i in range(len(recs))])
    _row_cmp(rows_g, rows_o, RMS_COLS, 1e-8)
    assert abs(rows_o[-1, 3] - rows_o[0, 3]) > 1e-5  # the cavities change the energy
