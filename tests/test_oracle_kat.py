"""Known-answer tests that pin the CPU oracle (the reference itself cannot be
built here, and ships no golden outputs): analytic maps, direct convolution,
analytic potentials, charge conservation, Gaussian moments."""
import ctypes
import math

import numpy as np
import pytest

from conftest import load_impz, load_oracle

impz = load_impz()
orc = load_oracle()
from impz_b200 import beams  # noqa: E402

IP = ctypes.POINTER(ctypes.c_int)


def test_fft_convolution_equals_direct_sum():
    rng = np.random.default_rng(1)
    nx, ny, nz = 8, 4, 8
    rho = rng.random(nx * ny * nz)
    phi = rho.copy()
    orc.physconst(402.5e6)
    assert orc.lib().orc_poisson_open(nx, ny, nz, 1e-3, 2e-3, 1.5e-3, orc.dp(phi)) == 0
    ref = np.zeros_like(rho)
    orc.lib().orc_poisson_direct(nx, ny, nz, 1e-3, 2e-3, 1.5e-3, orc.dp(rho), orc.dp(ref))
    assert np.linalg.norm(phi - ref) / np.linalg.norm(ref) < 1e-13


def test_poisson_linearity():
    rng = np.random.default_rng(2)
    n = (8, 8, 16)
    G = int(np.prod(n))
    a, b = rng.random(G), rng.random(G)
    orc.physconst(402.5e6)

    def solve(r):
        p = r.copy()
        orc.lib().orc_poisson_open(*n, 1e-3, 1e-3, 2e-3, orc.dp(p))
        return p

    lhs = solve(2.0 * a - 3.0 * b)
    rhs = 2.0 * solve(a) - 3.0 * solve(b)
    assert np.linalg.norm(lhs - rhs) / np.linalg.norm(rhs) < 1e-13


def test_uniform_sphere_potential():
    # phi = sum rho*G with G the cell average of 1/r: a uniform sphere of total
    # charge Q gives Q/r outside and Q(3R^2-r^2)/(2R^3) inside.
    n, h, R = 32, 1.0, 8.0
    c = (n - 1) / 2.0
    idx = np.arange(n) - c
    X, Y, Z = np.meshgrid(idx, idx, idx, indexing="ij")
    r = np.sqrt(X ** 2 + Y ** 2 + Z ** 2)
    rho = (r <= R).astype(np.float64)
    Q = rho.sum()
    phi = np.asfortranarray(rho).ravel(order="F").copy()
    orc.physconst(402.5e6)
    orc.lib().orc_poisson_open(n, n, n, h, h, h, orc.dp(phi))
    phi = phi.reshape((n, n, n), order="F")
    inside = r < R - 2
    outside = r > R + 2
    an_in = Q * (3 * R ** 2 - r ** 2) / (2 * R ** 3)
    an_out = Q / np.maximum(r, 1e-9)
    assert np.max(np.abs(phi[inside] - an_in[inside]) / an_in[inside]) < 0.03
    assert np.max(np.abs(phi[outside] - an_out[outside]) / an_out[outside]) < 0.03


def test_igf_symmetry_and_far_field():
    n = 8
    orc.physconst(402.5e6)
    g = np.zeros((n + 1) ** 3)
    orc.lib().orc_igf(n, n, n, 1.0, 1.0, 1.0, orc.dp(g))
    g = g.reshape((n + 1,) * 3, order="F")
    # the 8-corner difference cancels catastrophically far out (Field.f90:420-428)
    np.testing.assert_allclose(g, g.transpose(1, 0, 2), rtol=1e-10)
    np.testing.assert_allclose(g, g.transpose(2, 1, 0), rtol=1e-10)
    # far from the source the cell average of 1/r is 1/r to O(h^2/r^2)
    for (i, j, k) in [(8, 0, 0), (6, 6, 0), (5, 5, 5)]:
        r = math.sqrt(i * i + j * j + k * k)
        assert abs(g[i, j, k] - 1 / r) * r < 0.01


def _map_expected(K, L, gb, xl):
    k = math.sqrt(abs(K))
    if K > 0:
        c, s = math.cos(k * L), math.sin(k * L)
        return np.array([[c, s / (k * gb * xl)], [-k * gb * xl * s, c]])
    c, s = math.cosh(k * L), math.sinh(k * L)
    return np.array([[c, s / (k * gb * xl)], [k * gb * xl * s, c]])


def test_quad_rk6_map_matches_analytic():
    freq, mass, charge = 402.5e6, beams.PROTON_MASS_EV, 1.0
    P = orc.physconst(freq)
    ref = beams.refptcl_for(2.5e6, mass)
    gam = -ref[5]
    gb = math.sqrt(gam * gam - 1)
    grad, L = 20.0, 0.05
    brho = gb * mass / P["Clight"] / charge
    K = grad / brho
    xm = np.zeros(36)
    r = ref.copy()
    orc.lib().orc_maplinear_quad(0.0, L, orc.dp(xm), orc.dp(r), grad, 40, charge, mass)
    xm = xm.reshape(6, 6, order="F")
    np.testing.assert_allclose(xm[:2, :2], _map_expected(K, L, gb, P["Scxl"]), rtol=1e-9)
    np.testing.assert_allclose(xm[2:4, 2:4], _map_expected(-K, L, gb, P["Scxl"]), rtol=1e-9)
    # refptcl(5) advances by L/(beta0*Scxl)
    beta0 = gb / gam
    assert abs((r[4] - ref[4]) - L / (beta0 * P["Scxl"])) < 1e-12 * L / (beta0 * P["Scxl"])


def test_kmap_matches_analytic_for_reference_momentum():
    freq, mass = 402.5e6, beams.PROTON_MASS_EV
    P = orc.physconst(freq)
    ref = beams.refptcl_for(2.5e6, mass)
    gam = -ref[5]
    gb = math.sqrt(gam * gam - 1)
    K, L = 30.0, 0.04
    pts = np.zeros((2, 9))
    pts[:, 6] = 1.0 / mass
    pts[0, 0] = 1e-3 / P["Scxl"]
    pts[1, 1] = 1e-3 * gb
    orc.lib().orc_transfmapK(L, K, orc.dp(ref.copy()), orc.dp(pts), 2, 1.0 / mass)
    M = _map_expected(K, L, gb, P["Scxl"])
    np.testing.assert_allclose([pts[0, 0], pts[0, 1]], M @ [1e-3 / P["Scxl"], 0], rtol=1e-12)
    np.testing.assert_allclose([pts[1, 0], pts[1, 1]], M @ [0, 1e-3 * gb], rtol=1e-12)


def test_drift_there_and_back():
    freq = 402.5e6
    orc.physconst(freq)
    pts, ref = beams.gaussian_bunch(1000, seed=5)
    p = pts.copy()
    r = ref.copy()
    orc.lib().orc_drift_exact(orc.dp(p), 1000, orc.dp(r), 0.37)
    orc.lib().orc_drift_exact(orc.dp(p), 1000, orc.dp(r), -0.37)
    for c in range(6):
        s = np.sqrt(np.mean(pts[:, c] ** 2))
        assert np.max(np.abs(p[:, c] - pts[:, c])) <= 1e-12 * s
    assert abs(r[4]) < 1e-9


def test_deposit_conserves_charge_and_counts():
    freq = 402.5e6
    orc.physconst(freq)
    pts, ref = beams.gaussian_bunch(20000, seed=9)
    p = pts.copy()
    n = p.shape[0]
    cur = ctypes.c_double(0.03)
    npt = ctypes.c_int(n)
    pr = np.zeros(6)
    nl = orc.lib().orc_conv1st(orc.dp(p), n, ctypes.byref(cur), ctypes.byref(npt), orc.dp(ref),
                               1.0, 1.0, orc.dp(pr))
    assert nl == n
    mesh = np.array([32, 32, 64], dtype=np.int32)
    rg, ms = np.zeros(6), np.zeros(3)
    orc.lib().orc_update_compdom(orc.dp(pr), mesh.ctypes.data_as(IP), orc.dp(rg), orc.dp(ms))
    # the padded grid spans exactly Meshnum-1 cells of size h
    for k in range(3):
        assert rg[2 * k] < pr[2 * k] and rg[2 * k + 1] > pr[2 * k + 1]
    rho = np.zeros(32 * 32 * 64)
    cnt = np.zeros(32 * 32 * 64, dtype=np.int32)
    orc.lib().orc_deposit(orc.dp(p), nl, mesh.ctypes.data_as(IP), orc.dp(rg), orc.dp(ms),
                          orc.dp(rho), cnt.ctypes.data_as(IP), None)
    w = pts[0, 7]
    assert cnt.sum() == n
    assert abs(rho.sum() - n * w) <= 1e-12 * n * w


def test_gaussian_moments_match_sigma():
    freq, mass = 402.5e6, beams.PROTON_MASS_EV
    P = orc.physconst(freq)
    pts, ref = beams.gaussian_bunch(200_000, seed=11)
    raw = np.zeros(orc.RAW_LEN)
    orc.lib().orc_moment_sums(orc.dp(pts), pts.shape[0], orc.dp(raw))
    row = np.zeros(orc.DIAG_LEN)
    orc.lib().orc_diag_row(0.0, orc.dp(raw), pts.shape[0], pts.shape[0], orc.dp(ref), mass,
                           orc.dp(row))
    # truncation at 4 sigma shrinks sigma by 0.1 %
    assert abs(row[7] - 1e-3) < 0.01e-3       # xrms [m]
    assert abs(row[13] - 1e-3) < 0.01e-3      # yrms [m]
    assert abs(row[9] - 1e-3) < 0.01e-3       # x' rms
    assert abs(row[19] - 5.0) < 0.05          # phase rms [deg]
    assert abs(row[21] - 0.05) < 0.0005       # dE rms [MeV]
    gb = math.sqrt(ref[5] ** 2 - 1)
    assert abs(row[11] - gb * 1e-6) < 0.02 * gb * 1e-6  # normalised emittance [m rad]


def test_full_lattice_runs_and_conserves_particles():
    cfg = beams.fodo_1e5(n=3000)
    cfg["lattice"] = beams.fodo(1)
    rows, p, beam = orc.run(cfg["lattice"], cfg["pts"], cfg["current"], cfg["mass"],
                            cfg["charge"], cfg["freq"], cfg["refptcl"], cfg["grid"])
    assert rows.shape == (17, orc.DIAG_LEN)
    assert np.all(rows[:, 32] == 3000)
    assert np.all(np.isfinite(rows))
    np.testing.assert_allclose(rows[-1, 0], 0.4, rtol=1e-12)
