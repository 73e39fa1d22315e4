"""The Lorentz integrator (Flagmap=2) on the oracle, no GPU needed:
drift2 half steps around kick2/scatter2 (BeamBunch.f90:467-509,
2187-3071).  Through a FODO lattice its second-order splitting of the
quadrupoles' focusing converges to the linear map integrator's result as
the steps shrink."""
import os

import numpy as np
import pytest

from conftest import load_impz, load_oracle, reference_path

impz = load_impz()
orc = load_oracle()
from impz_b200 import beams  # noqa: E402


def test_lorentz_integrator_converges_to_the_map_integrator():
    cfg = beams.fodo_1e5(n=5000, seed=beams.SEED0 + 71)
    gaps = []
    for nseg in (4, 16, 64):
        lat = beams.fodo(1, nseg=nseg)
        run = lambda fm: orc.run(lat, cfg["pts"], cfg["current"], cfg["mass"],  # noqa: E731
                                 cfg["charge"], cfg["freq"], cfg["refptcl"], (16, 16, 32),
                                 flagmap=fm)[0]
        r1, r2 = run(1), run(2)
        np.testing.assert_array_equal(r1[:, 0], r2[:, 0])  # the same steps and z
        gaps.append(max(abs(r2[-1, c] - r1[-1, c]) / abs(r1[-1, c]) for c in (7, 13)))
    # the splitting error falls fast with the step (the space-charge kicks
    # of the two integrators also differ slightly, which leaves a small floor)
    assert gaps[0] > 8 * gaps[1] > 0 and gaps[1] > 2 * gaps[2] and gaps[2] < 1e-3


def test_lorentz_integrator_refuses_elements_outside_it():
    cfg = beams.fodo_1e5(n=500)
    bend = impz.elem(4, 0.2, 4, 1, [0.05, 0.0, 150.0, 0.01])
    try:
        orc.run([bend], cfg["pts"], cfg["current"], cfg["mass"], cfg["charge"], cfg["freq"],
                cfg["refptcl"], (16, 16, 32), flagmap=2)
    except RuntimeError as e:
        assert "-10" in str(e)
    else:
        raise AssertionError("a bend under the Lorentz integrator must be refused")


def test_lorentz_integrator_without_current_converges_too():
    """Zero current: kick2 is scatter20, the quadrupoles' field alone on the
    stored coordinates (BeamBunch.f90:3075-3531)."""
    cfg = beams.fodo_1e5(n=2000, seed=beams.SEED0 + 73)
    gaps = []
    for nseg in (4, 32):
        lat = beams.fodo(1, nseg=nseg)
        run = lambda fm: orc.run(lat, cfg["pts"], 0.0, cfg["mass"], cfg["charge"],  # noqa: E731
                                 cfg["freq"], cfg["refptcl"], (16, 16, 32), flagmap=fm)[0]
        r1, r2 = run(1), run(2)
        gaps.append(max(abs(r2[-1, c] - r1[-1, c]) / abs(r1[-1, c]) for c in (7, 13)))
    assert gaps[0] > 8 * gaps[1] and gaps[1] < 2e-3


def _lz_run(lat, cfg, current=0.0, pts=None):
    return orc.run(lat, cfg["pts"] if pts is None else pts, current, cfg["mass"], cfg["charge"],
                   cfg["freq"], cfg["refptcl"], (16, 16, 32), flagmap=2)


def test_uniform_solenoid_rotates_the_transverse_momentum():
    """A solenoid with no ramp (Param(4) = 0, getfld_Sol's body over the
    whole length) and no current: each kick is a Cayley rotation of
    (px, py) about z, so |p_perp| and pt of every particle stay as they
    were (to rounding) and a particle's momentum turns by nseg Cayley angles 2 atan(q Bz tau / 2pz),
    close to q Bz L / pz."""
    cfg = beams.fodo_1e5(n=2000, seed=beams.SEED0 + 75)
    bz, length, nseg = 0.8, 0.5, 40
    rows, p1, beam = _lz_run([impz.elem(3, length, nseg, 1, [bz, 0.0, 0.0])], cfg)
    p0 = cfg["pts"]
    np.testing.assert_allclose(np.hypot(p1[:, 1], p1[:, 3]), np.hypot(p0[:, 1], p0[:, 3]),
                               rtol=1e-13, atol=1e-300)
    # (1 + a12^2) pt / (1 + a12^2): pt to the last bit or two
    np.testing.assert_allclose(p1[:, 5], p0[:, 5], rtol=1e-15, atol=0)
    gam = -cfg["refptcl"][5]
    pz = np.sqrt((gam - p0[:, 5]) ** 2 - 1.0 - p0[:, 1] ** 2 - p0[:, 3] ** 2)
    # q B / (m c) [1/m] with Pts1(7) = q/m [1/eV]: 2.99792458e8 B q / m
    want = -2.99792458e8 * bz * p0[:, 6] * length / pz
    turned = np.angle((p1[:, 1] + 1j * p1[:, 3]) / (p0[:, 1] + 1j * p0[:, 3]))
    np.testing.assert_allclose(turned, np.angle(np.exp(1j * want)), rtol=0, atol=1e-3)
    # exactly: nseg Cayley rotations by 2 atan(a12), a12 = -tau c Bz q/m / (2 pz)
    cay = nseg * 2 * np.arctan(-(length / nseg) * 2.99792458e8 * bz * p0[:, 6] / (2 * pz))
    np.testing.assert_allclose(turned, np.angle(np.exp(1j * cay)), rtol=0, atol=1e-11)
    np.testing.assert_array_equal(beam.refptcl[5], cfg["refptcl"][5])


def test_enge_quadrupole_approaches_the_hard_edge_one():
    """getfldfrgAna2_Quadrupole's Enge profile with a short fringe (aperture
    2 mm) over a 0.2 m element of effective length 0.1 m focuses like a
    hard-edge 0.1 m quadrupole between two 0.05 m drifts."""
    cfg = beams.fodo_1e5(n=2000, seed=beams.SEED0 + 76)
    g = 20.0
    frg = [impz.elem(1, 0.2, 400, 1, [g, 0.1, 0.002])]
    hard = [impz.elem(0, 0.05, 100, 1, [1.0]), impz.elem(1, 0.1, 200, 1, [g, 0.0, 1.0]),
            impz.elem(0, 0.05, 100, 1, [1.0])]
    drift = [impz.elem(0, 0.2, 400, 1, [1.0])]
    rf, rh, rd = (_lz_run(lat, cfg)[0][-1] for lat in (frg, hard, drift))
    for c in (7, 13):  # rms x, rms y
        assert abs(rf[c] - rh[c]) < 0.02 * abs(rd[c] - rh[c])


def _self_convergence(make, cfg, cols, current=0.0):
    finals = [_lz_run(make(n), cfg, current)[0][-1] for n in (8, 32, 256)]
    err = [max(abs(f[c] - finals[-1][c]) / abs(finals[-1][c]) for c in cols)
           for f in finals[:2]]
    return err


def test_lorentz_element_fields_converge_at_second_order():
    """Quadrupole with Enge fringe, ramped solenoid and constant focusing
    under kick2: the splitting error falls about 16x from 8 to 32 steps."""
    cfg = beams.fodo_1e5(n=1000, seed=beams.SEED0 + 77)
    makers = [
        lambda n: [impz.elem(1, 0.3, n, 1, [15.0, 0.2, 0.02])],
        lambda n: [impz.elem(3, 0.4, n, 1, [0.6, 0.0, 0.05])],
        # getfld_ConstFoc's B = k X / c (its qmcc is a placeholder 1): 20-30 T/m
        lambda n: [impz.elem(2, 0.4, n, 1, [6e9, 9e9, 0.0, 1.0])],
    ]
    for make in makers:
        err = _self_convergence(make, cfg, (7, 8, 13, 14))
        assert err[0] > 8 * err[1] > 0, err


def test_constant_focusing_ez_moves_the_reference_energy():
    """getfld_ConstFoc's Ez = kz t Scxl on axis at the reference time
    changes gamma0 by tau qmcc Ez0 at each kick (kick2_BeamBunch's
    refptcl(6) = -gam); kz = 0 leaves it alone."""
    cfg = beams.fodo_1e5(n=500, seed=beams.SEED0 + 78)
    ref = cfg["refptcl"].copy()
    ref[4] = 2.0  # a nonzero reference time tg
    c2 = dict(cfg, refptcl=ref)
    g0 = -ref[5]
    kz, length, nseg = 1e-3, 0.4, 4
    _, _, beam = _lz_run([impz.elem(2, length, nseg, 1, [40.0, 60.0, kz, 1.0])], c2)
    _, _, beam0 = _lz_run([impz.elem(2, length, nseg, 1, [40.0, 60.0, 0.0, 1.0])], c2)
    assert beam0.refptcl[5] == ref[5]
    # the same recurrence by hand: tg advances by tau/(2 Scxl beta0) per drift2
    scxl = 2.99792458e8 / (2 * np.pi * cfg["freq"])
    qmcc = cfg["charge"] / cfg["mass"]
    tau, tg, gam = length / nseg, ref[4], g0
    for _ in range(nseg):
        tg += 0.5 * tau / (scxl * np.sqrt(1.0 - 1.0 / gam / gam))
        gam = gam + tau * qmcc * (kz * tg * scxl)
        tg += 0.5 * tau / (scxl * np.sqrt(1.0 - 1.0 / gam / gam))
    np.testing.assert_allclose(-beam.refptcl[5], gam, rtol=1e-14)
    assert -beam.refptcl[5] != g0


def test_lorentz_read_in_wake_acts_as_under_the_map_integrator():
    """kick2wake/scatter2wake (BeamBunch.f90:5048-5938) adds the raw
    per-plane wake at the particle, linear in z, after the space-charge
    scaling; kick1wake adds it to the node fields in grid units.  Both give
    a particle tau q/m Ez of energy (and tau q/m Ex / beta of px), so the
    wake's own effect on the bunch (with minus without) is the same under
    both integrators, longitudinal and transverse."""
    from test_wake import synthetic_table
    cur = 1.3
    pts, ref = beams.gaussian_bunch(3000, seed=beams.SEED0 + 81, mass=beams.ELECTRON_MASS_EV,
                                    charge=-1.0, ekin=98.169272e6, current=cur, freq=1.3e9,
                                    sig_x=0.5e-3, sig_y=0.5e-3, sig_xp=0.05e-3,
                                    sig_yp=0.05e-3, sig_phase_deg=1.0, sig_e=50e3)
    scxl = 2.99792458e8 / (2 * np.pi * 1.3e9)
    pts = pts.copy()
    pts[:, 0] += 0.5e-3 / scxl  # offsets drive the dipole (transverse) wake
    pts[:, 2] += 0.3e-3 / scxl
    lat = [impz.elem(0, 1.0, 8, 1, [1.0])]

    def final(fm, wake):
        try:
            if wake:
                orc.wake_set(synthetic_table(), 1.0, True)
            return orc.run(lat, pts, cur, beams.ELECTRON_MASS_EV, -1.0, 1.3e9, ref,
                           (16, 16, 32), flagmap=fm)[0][-1]
        finally:
            orc.wake_off()

    d1 = final(1, True) - final(1, False)
    d2 = final(2, True) - final(2, False)
    assert abs(d1[20]) > 10 * abs(final(1, False)[20])  # the wake dominates <dE>
    for c in (20, 21):  # mean and rms energy
        assert abs(d2[c] - d1[c]) < 1e-3 * abs(d1[c]), (c, d1[c], d2[c])
    for c in (8, 14):  # mean px, py
        assert abs(d1[c]) > 0 and abs(d2[c] - d1[c]) < 1e-3 * abs(d1[c]), (c, d1[c], d2[c])


def rf_cell(length=0.08, harmonics=18):
    """A DTL-like cell's on-axis field as read3_Data's Fourier coefficients
    (Fcoef(1)/2 + sum a_k cos + b_k sin of 2 pi k (z - zmid)/L) and the same
    field sampled as read1_Data's (z, Ez, Ez', Ez'') table from the
    entrance, for the map integrator."""
    k = np.arange(1, harmonics + 1)
    a = 2 * np.exp(-(k / 4.0) ** 2)
    b = 0.01 * (-1.0) ** k / k
    coef = np.empty(1 + 2 * harmonics)
    coef[0], coef[1::2], coef[2::2] = 2.0, a, b
    z = np.linspace(0, length, 4001)
    w = 2 * np.pi * k[None, :] / length
    c, s = np.cos(w * (z[:, None] - length / 2)), np.sin(w * (z[:, None] - length / 2))
    ez = 1.0 + (a * c + b * s).sum(1)
    ezp = (w * (-a * s + b * c)).sum(1)
    ezpp = (w * w * (-a * c - b * s)).sum(1)
    return coef, (z, ez, ezp, ezpp)


@pytest.mark.parametrize("etype", [101, 103])
def test_rf_cavity_under_kick2_gains_the_map_integrators_energy(etype):
    """getfld_DTL / getfld_CCL over Fourier coefficients (DTL.f90:769-958,
    CCL.f90:525-809): gamma0 moves by tau qmcc ez1 cos(w tg + theta0) at
    each kick, so the reference particle's energy gain through a cell
    converges, at second order, to the map integrator's RK6 of the same
    field; the bunch's rms sizes agree to the linear map's own accuracy."""
    coef, table = rf_cell()
    mass, freq = beams.PROTON_MASS_EV, 324e6
    pts, ref = beams.gaussian_bunch(2000, seed=beams.SEED0 + 83, mass=mass, charge=1.0,
                                    ekin=3.35e6, current=0.0, freq=freq)
    vals = [2.5e6, freq, 222.0, 1.0, 0.0065]
    if etype == 101:
        vals += [0.02, 68.0, 0.02, -67.0]  # the drift-tube quadrupoles
    gaps = []
    for nseg in (40, 160):
        r1, _, b1 = orc.run([impz.elem(etype, 0.08, nseg, 20, vals, rf=table)], pts, 0.0, mass,
                            1.0, freq, ref, (16, 16, 32), flagmap=1)
        r2, _, b2 = orc.run([impz.elem(etype, 0.08, nseg, 20, vals, rf=coef)], pts, 0.0, mass,
                            1.0, freq, ref, (16, 16, 32), flagmap=2)
        gain1 = -b1.refptcl[5] + ref[5]
        gaps.append(abs((-b2.refptcl[5] + ref[5]) / gain1 - 1))
        assert gain1 > 1e-4
    assert gaps[0] > 8 * gaps[1] and gaps[1] < 1e-5, gaps
    for c in (7, 13, 21):
        assert abs(r2[-1, c] / r1[-1, c] - 1) < 1e-2


EXAMPLE1 = reference_path("examples", "Example1") or ""


@pytest.mark.skipif(not os.path.isdir(EXAMPLE1),
                    reason="IMPZ_REFERENCE_TREE unset (the reference's examples)")
def test_example1_dtl_cells_on_the_oracle():
    """The reference's Example1 (Flagmap=2: nine DTL cells over rfdata
    Fourier coefficients, quadrupoles and a drift) through the deck reader
    and the oracle's Lorentz integrator, without current: the reference
    particle's energy and phase at the end agree with an independent
    integration of d gamma/dz = qmcc Ez(z) cos(w phi + theta0), d phi/dz =
    1/(beta Scxl) over the same Fourier fields (the reference's
    default-real pi in the series and in theta0)."""
    from scipy.integrate import solve_ivp
    from impz_b200 import deck
    d = deck.read_deck(os.path.join(EXAMPLE1, "ImpactZ.in"))
    assert d.flagmap == 2
    pts = deck.read_particles(os.path.join(EXAMPLE1, "particle.in"))
    ref, z = d.refptcl(), 0.0
    for kind, item in deck.lattice_segments(d, EXAMPLE1):
        if kind == "run":
            rows, pts, beam = orc.run(item, pts, 0.0, d.bmass, d.bcharge, d.bfreq, ref,
                                      (d.nx, d.ny, d.nz), z, flagmap=d.flagmap)
            ref, z = np.array(beam.refptcl[:]), beam.z
            assert np.isfinite(rows).all()
    # the same reference particle by an adaptive RK45 at tight tolerance
    pi32 = float(np.float32(2) * np.arcsin(np.float32(1.0)))
    half_pi32 = float(np.arcsin(np.float32(1.0)))
    scxl = 299792458.0 / (2 * np.pi * d.bfreq)
    qmcc = d.bcharge / d.bmass
    y = np.array([-d.refptcl()[5], d.refptcl()[4]])
    for e in d.elements:
        if e.type < 0:
            continue
        if 101 <= e.type <= 104:
            coef = deck.read_rfcoef(os.path.join(EXAMPLE1, "rfdata%d.in" % int(e.vals[3] + 0.1)))
            n = (len(coef) - 1) // 2
            k = np.arange(1, n + 1)
            a, b = coef[1::2][:n], coef[2::2][:n]
            ww, th0 = e.vals[1] / d.bfreq, e.vals[2] * half_pi32 / 90
            L = e.length

            def rhs(s, yy):
                arg = k * 2 * pi32 * (s - L / 2) / L
                ez = e.vals[0] * (coef[0] / 2 + (a * np.cos(arg) + b * np.sin(arg)).sum())
                beta = np.sqrt(1 - 1 / yy[0] ** 2)
                return [qmcc * ez * np.cos(ww * yy[1] + th0), 1 / (beta * scxl)]
        else:
            def rhs(s, yy):
                return [0.0, 1 / (np.sqrt(1 - 1 / yy[0] ** 2) * scxl)]
        y = solve_ivp(rhs, (0.0, e.length), y, rtol=1e-12, atol=1e-14, method="DOP853").y[:, -1]
    gain = y[0] + d.refptcl()[5]
    assert gain > 1e-4  # the cells accelerate
    assert abs(-ref[5] - y[0]) < 1e-5 * gain
    assert abs(ref[4] - y[1]) < 1e-6 * y[1]


def solrf_two_series(length=0.2):
    """getfld_SolRF's two series: the cavity's Ez, then the solenoid's Bz
    profile (a constant 1 over the element, scaled by Param(12))."""
    from test_abi import solrf_coefficients
    rf = list(solrf_coefficients(length))
    return np.array(rf + [1, 0.0, length, length, 2.0])


@pytest.mark.parametrize("etype", [105, 106])
def test_solrf_and_tws_under_kick2_gain_the_map_integrators_energy(etype):
    """getfld_SolRF / getfld_TWS (SolRF.f90:482-628, TWS.f90) under kick2:
    the reference particle's energy gain converges, at second order, to
    maplinear_SolRF / maplinear_TWS's RK6 over the same coefficients."""
    from test_abi import tws_coefficients
    mass, freq = beams.PROTON_MASS_EV, 402.5e6
    pts, ref = beams.gaussian_bunch(2000, seed=beams.SEED0 + 85, mass=mass, charge=1.0,
                                    ekin=2.5e6, current=0.0, freq=freq)
    coef = solrf_two_series() if etype == 105 else tws_coefficients()
    vals = [1e6, freq, 60.0, 1.0, 1.0, 0, 0, 0, 0, 0, 0.2 if etype == 105 else 90.0]
    gaps = []
    for nseg in (40, 160):
        lat = [impz.elem(etype, 0.2, nseg, 20, vals, rf=coef)]
        _, _, b1 = orc.run(lat, pts, 0.0, mass, 1.0, freq, ref, (16, 16, 32), flagmap=1)
        _, _, b2 = orc.run(lat, pts, 0.0, mass, 1.0, freq, ref, (16, 16, 32), flagmap=2)
        gain1 = -b1.refptcl[5] + ref[5]
        assert abs(gain1) > 1e-5
        gaps.append(abs((-b2.refptcl[5] + ref[5]) / gain1 - 1))
    # the 0.2 m element spans about four beta-lambda, so the splitting error
    # is larger than in one DTL cell: 1e-2 at 40 steps, 6e-4 at 160
    assert gaps[0] > 8 * gaps[1] and gaps[1] < 1e-3, gaps


@pytest.mark.parametrize("idpole,g", [(2, 3.0e3), (3, 2.0e6), (4, 1.0e9)])
def test_multipole_kick_is_getfld_multipole(idpole, g):
    """One kick2 step of a 2 cm multipole without current: with only Bx,
    By the implicit update is exactly px -= c q/m tau By, py += c q/m tau
    Bx at the position after the first drift2 (getfld_Multipole's MAD
    fields, Multipole.f90:403-452); pt does not move."""
    cfg = beams.fodo_1e5(n=500, seed=beams.SEED0 + 87)
    p0, ref = cfg["pts"], cfg["refptcl"]
    tau, clight = 0.02, 299792458.0
    scxl = clight / (2 * np.pi * cfg["freq"])
    _, p1, _ = _lz_run([impz.elem(5, tau, 1, 1, [idpole, g, 0.0, 1.0])], cfg)
    g0 = -ref[5]
    pz = np.sqrt((g0 - p0[:, 5]) * (g0 - p0[:, 5]) - 1.0 - p0[:, 1] * p0[:, 1] -
                 p0[:, 3] * p0[:, 3])
    x = (p0[:, 0] + 0.5 * tau * p0[:, 1] / (scxl * pz)) * scxl
    y = (p0[:, 2] + 0.5 * tau * p0[:, 3] / (scxl * pz)) * scxl
    if idpole == 2:
        bx, by = g * y * x, g * (x * x - y * y) / 2
    elif idpole == 3:
        bx, by = g * (3 * (x * x) * y - y * y * y) / 6, g * (x * x * x - 3 * x * (y * y)) / 6
    else:
        bx = g * (x * x * x * y - x * (y * y * y)) / 6
        by = g * ((x * x) * (x * x) - 6 * (x * x) * (y * y) + (y * y) * (y * y)) / 24
    r7 = p0[:, 6]
    np.testing.assert_allclose(p1[:, 1], p0[:, 1] - clight * by * tau * r7, rtol=1e-14, atol=0)
    np.testing.assert_allclose(p1[:, 3], p0[:, 3] + clight * bx * tau * r7, rtol=1e-14, atol=0)
    np.testing.assert_array_equal(p1[:, 5], p0[:, 5])
    assert np.max(np.abs(p1[:, 1] - p0[:, 1])) > 0.05 * np.max(np.abs(p0[:, 1]))


# ---------------------------------------------------------------------------
# EMfld 110: discrete x-y-z field map (read4_Data, scatter2 FlagDisc 1, FlagCart 2)
def emfld_grid(fields, length, xr=(-8e-3, 8e-3, 16), yr=(-8e-3, 8e-3, 16), nz=10):
    """read4_Data's map of an element of `length`: nodes x fastest, then y,
    then z; fields(x, y, z) -> six complex arrays (Ex, Ey, Ez, Bx, By, Bz)."""
    xs = np.linspace(xr[0], xr[1], xr[2] + 1)
    ys = np.linspace(yr[0], yr[1], yr[2] + 1)
    zs = np.linspace(0.0, length, nz + 1)
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    comps = [np.broadcast_to(np.asarray(f, dtype=complex), X.shape).reshape(-1)
             for f in fields(X, Y, Z)]
    header = np.array([xr[0], xr[1], xr[2], yr[0], yr[1], yr[2], 0.0, length, nz], dtype=float)
    return header, np.stack(comps, axis=1)


def emfld(length, nseg, grid, scale=1.0, freq=0.0, theta0=0.0, radius=1.0):
    """A type 110 element: Param(2..14) = scale, frequency, theta0 [deg],
    file ID, x and y radius, errors (0), FlagDisc 1, FlagCart 2."""
    vals = [scale, freq, theta0, 1.0, radius, radius, 0, 0, 0, 0, 0, 1.0, 2.0]
    return impz.elem(110, length, nseg, 1, vals, grid=grid)


def quad_map(g):
    def f(x, y, z):
        zero = np.zeros_like(x)
        return zero, zero, zero, g * y, g * x, zero
    return f


@pytest.mark.parametrize("current", [0.0, 0.030])
def test_emfld_with_a_quadrupoles_field_tracks_like_the_quadrupole(current):
    """An EMfld 110 whose x-y-z map holds a hard-edge quadrupole's static
    field (B = G (y, x, 0), zero frequency) tracks like that quadrupole
    under the Lorentz integrator: the map's quadratic interpolation is exact
    for fields linear in x and y inside the grid, so the runs agree to
    rounding (1e-12 of each column's rms), with and without space charge."""
    cfg = beams.fodo_1e5(n=2000, seed=beams.SEED0 + 91)
    g, length = 20.0, 0.1
    drift = impz.elem(0, 0.1, 2, 1, [1.0])
    lat_q = [drift, impz.elem(1, length, 4, 1, [g, 0.0, 1.0]), drift]
    lat_e = [drift, emfld(length, 4, emfld_grid(quad_map(g), length)), drift]
    _, pq, bq = _lz_run(lat_q, cfg, current)
    _, pe, be = _lz_run(lat_e, cfg, current)
    assert pq.shape == pe.shape
    for c in range(6):
        scale = np.sqrt(np.mean(pq[:, c] ** 2))
        assert np.max(np.abs(pe[:, c] - pq[:, c])) / scale <= 1e-12, c
    np.testing.assert_allclose(be.refptcl[:], bq.refptcl[:], rtol=1e-15)


def test_emfld_rf_map_moves_the_reference_energy():
    """A uniform complex Ez map (E0 (1 + 0.2 i), escale 1.5, 402.5 MHz,
    theta0 30 deg): each kick changes gamma0 by tau qmcc ez0 with ez0 =
    Re(Ez escale e^{i(ww tg + theta0)}) at the reference time tg (kick2's
    refptcl(6) = -gam, scatter2's ez0 at x = y = 0), theta0 with the
    reference's single-precision asin(1.0)."""
    cfg = beams.fodo_1e5(n=500, seed=beams.SEED0 + 92)
    length, nseg, e0, scale, freq, th = 0.2, 5, 2.0e6, 1.5, 402.5e6, 30.0

    def uniform(x, y, z):
        zero = np.zeros_like(x)
        return zero, zero, e0 * (1 + 0.2j) + zero, zero, zero, zero
    lat = [emfld(length, nseg, emfld_grid(uniform, length), scale, freq, th)]
    _, _, beam = _lz_run(lat, cfg)
    scxl = 2.99792458e8 / (2 * np.pi * cfg["freq"])
    qmcc = cfg["charge"] / cfg["mass"]
    ww = freq / cfg["freq"]
    theta0 = th * float(np.arcsin(np.float32(1.0))) / 90
    tau, tg, gam = length / nseg, cfg["refptcl"][4], -cfg["refptcl"][5]
    for _ in range(nseg):
        tg += 0.5 * tau / (scxl * np.sqrt(1.0 - 1.0 / gam / gam))
        ph = ww * tg + theta0
        ez0 = e0 * (scale * np.cos(ph)) - 0.2 * e0 * (scale * np.sin(ph))
        gam = gam + tau * qmcc * ez0
        tg += 0.5 * tau / (scxl * np.sqrt(1.0 - 1.0 / gam / gam))
    np.testing.assert_allclose(-beam.refptcl[5], gam, rtol=1e-13)
    assert abs(-beam.refptcl[5] + cfg["refptcl"][5]) > 1e-4


def test_emfld_other_forms_are_refused():
    """EMfld's analytical and r-z forms read data the reference's driver
    never loads for type 110 under Flagmap=2: refused."""
    cfg = beams.fodo_1e5(n=200, seed=beams.SEED0 + 93)
    grid = emfld_grid(quad_map(1.0), 0.1)
    vals = [1.0, 0.0, 0.0, 1.0, 1.0, 1.0, 0, 0, 0, 0, 0, 1.0, 1.0]  # FlagCart 1 (r-z)
    with pytest.raises(RuntimeError):
        _lz_run([impz.elem(110, 0.1, 2, 1, vals, grid=grid)], cfg)
    vals[11], vals[12] = 3.0, 2.0  # analytical
    with pytest.raises(RuntimeError):
        _lz_run([impz.elem(110, 0.1, 2, 1, vals, grid=grid)], cfg)
