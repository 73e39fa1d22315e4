"""Read-in wakefield (type -41 elements) on the oracle, no GPU needed.

The reference convolves the line density with the wake table on a doubled
grid by FFT (wakefieldread_FieldQuant, src/Appl/Field.f90:783-1001); the
oracle (and the GPU path) evaluate the causal sum that convolution reduces
to.  These tests restate the reference's doubled-grid procedure with numpy's
real FFT and check the oracle's per-plane field against it, longitudinal and
transverse, then run the reference's Example3 with its wake controls."""
import ctypes
import os

import numpy as np
import pytest

from conftest import load_impz, load_oracle, reference_path

impz = load_impz()
orc = load_oracle()
from impz_b200 import deck  # noqa: E402

EXAMPLES = reference_path("examples") or ""


def synthetic_table(rows=5000, hwk=2.0e-6, seed=7):
    """A cavity-like wake table: z from 0 in steps of hwk, a decaying
    longitudinal wake of order 1e13-1e14 V/C/m and linear transverse ones."""
    rng = np.random.default_rng(seed)
    z = np.arange(rows) * hwk
    ez = 4.3e13 * np.exp(-z / 2.5e-3) + 3.0e12
    ex = 1.0e15 * z * np.exp(-z / 4.0e-3)
    ey = 0.8e15 * z * np.exp(-z / 5.0e-3)
    ez *= 1.0 + 1e-3 * rng.standard_normal(rows)
    return np.c_[z + 0.37, ez, ex, ey]  # z need not start at 0


def green_ref(col, table, nz, hz):
    """greenwake of Field.f90:818-830 for kz = 1..Nz+1 (index 0..Nz); rows
    past the table read zero (the reference's zero-filled module arrays)."""
    zd = table[:, 0] - table[0, 0]
    hwk = zd[1] - zd[0]

    def e(i1):
        return col[i1 - 1] if 1 <= i1 <= col.shape[0] else 0.0

    g = np.zeros(nz + 1)
    for kz in range(nz + 1):
        zwk = kz * hz - zd[0]
        iwk = int(zwk / hwk + 1)
        ab = iwk * hwk - zwk
        g[kz] = e(iwk) * ab + e(iwk + 1) * (1.0 - ab)
    return g


def fft_wake(table, recv, xbar, ybar, hz, transverse, greens=None):
    """Field.f90:783-1001 (or, with greens = (W_L, W_T) sampled at 0..Nz,
    Field.f90:590-782) with numpy's FFT: returns (exwake, eywake, ezwake)."""
    nz = recv.shape[0]
    n2 = 2 * nz

    def conv(dens, col, transverse_green):
        d2 = np.r_[dens, np.zeros(nz)]
        if greens is not None:
            w = greens[1 if transverse_green else 0]
        else:
            w = green_ref(col, table, nz, hz)
        g = np.zeros(n2)
        g[: nz + 1] = w
        g[0] = 0.5 * w[0]
        for kz in range(nz + 2, n2 + 1):  # greenwake(kz) = greenwake(2Nz-kz+2)
            g[kz - 1] = g[n2 - kz + 1]
        if transverse_green:
            g[:nz] = 0.0  # kz = 1..Nz
        else:
            g[1:nz] = 0.0  # kz = 2..Nz
        return np.fft.irfft(np.fft.rfft(d2) * np.fft.rfft(g), n2)[:nz]

    col = (lambda c: None) if table is None else (lambda c: table[:, c])  # noqa: E731
    ez = -conv(recv, col(1), False) * hz
    if not transverse:
        return np.zeros(nz), np.zeros(nz), ez
    ex = conv(recv * xbar, col(2), True) * hz
    ey = conv(recv * ybar, col(3), True) * hz
    return ex, ey, ez


def kick_consts(gam, curr, mass, chrg, freq):
    """kick1wake's constants (src/Appl/BeamBunch.f90:4989-5006)."""
    clight, pi = 299792458.0, 2 * np.arcsin(1.0)
    scxl = clight / (2 * pi * freq)
    fpei = clight * clight * float(np.float32(1.0e-7))
    bet = np.sqrt(gam * gam - 1.0) / gam
    gambet = gam * bet
    brho = gambet / (clight * chrg) * mass
    vz0 = bet * clight
    perv0 = 2.0 * curr * fpei / (brho * vz0 * vz0 * gam * gam)
    xycon = 0.5 * perv0 * gambet * (bet * scxl) * 2 * pi / (curr / freq)
    return xycon, bet * xycon * gam * gam, bet


@pytest.mark.parametrize("transverse", [False, True])
@pytest.mark.parametrize("nz", [32, 128])
def test_direct_wake_sum_equals_the_doubled_grid_fft(nz, transverse):
    L = orc.lib()
    table = synthetic_table()
    freq, curr, mass, chrg, gam, npt = 1.3e9, 0.13, 0.51099895e6, -1.0, 190.0, 20000
    orc.physconst(freq)
    t = np.ascontiguousarray(table.T)
    assert L.orc_wake_set(orc.dp(t[0]), orc.dp(t[1]), orc.dp(t[2]), orc.dp(t[3]), t.shape[1],
                          0.8, int(transverse)) == 0
    rng = np.random.default_rng(nz)
    # a line density with a bunch-like profile; z extent chosen so the
    # doubled grid reaches past the table's 1 cm
    densz = npt * np.exp(-0.5 * ((np.arange(nz) - nz / 2) / (nz / 6)) ** 2)
    densz *= 1 + 0.05 * rng.random(nz)
    densz[[0, -1]] = 0.0
    xsum = densz * 1e-4 * rng.standard_normal(nz)
    ysum = densz * 1e-4 * rng.standard_normal(nz)
    rng6 = np.array([-1e-3, 1e-3, -1e-3, 1e-3, -0.9, 1.1]) * (nz / 64)
    out = np.zeros(3 * nz)
    L.orc_wake_field(nz, orc.dp(densz), orc.dp(xsum), orc.dp(ysum), orc.dp(rng6), gam, curr,
                     npt, mass, chrg, orc.dp(out))
    L.orc_wake_off()
    # AccSimulator.f90:1297-1322: recvdensz, the centroids, hzwake / gamma
    hz = (rng6[5] - rng6[4]) / (nz - 1) / gam
    recv = densz * curr / freq / npt / hz * chrg / abs(chrg)
    with np.errstate(invalid="ignore", divide="ignore"):
        xbar = np.where(densz != 0, xsum / densz, 0.0)
        ybar = np.where(densz != 0, ysum / densz, 0.0)
    ex, ey, ez = fft_wake(table, recv, xbar, ybar, hz, transverse)
    xycon, tcon, bet = kick_consts(gam, curr, mass, chrg, freq)
    want = np.r_[chrg * 0.8 * ex / xycon / mass / bet / gam,
                 chrg * 0.8 * ey / xycon / mass / bet / gam,
                 chrg * 0.8 * ez / tcon / mass]
    assert np.abs(want[2 * nz:]).max() > 0
    scale = np.abs(want).max()
    np.testing.assert_allclose(out, want, rtol=0, atol=1e-12 * scale)
    if not transverse:
        assert not out[: 2 * nz].any()


def analytic_greens(aa, gg, leng, nz, hz):
    """Field.f90:623-641 and 694-700: the fits in default real literals."""
    f32 = lambda x: float(np.float32(x))  # noqa: E731
    pilc, clight = 2 * np.arcsin(1.0), 299792458.0
    z0 = f32(0.41) * (aa / leng) ** f32(0.8) * (gg / leng) ** f32(1.6) * aa
    z0_0 = 120 * pilc
    zz = np.arange(nz + 1) * hz
    wl = z0_0 * clight * np.exp(-np.sqrt(zz / z0)) / (pilc * aa * aa)
    z1 = f32(0.169) * aa * (aa / leng) ** f32(1.17) * (gg / aa) ** f32(0.38)
    coef1 = 4 * z0_0 * clight * z1 / (pilc * aa ** 4)
    wt = coef1 * (1.0 - (1.0 + np.sqrt(zz / z1)) * np.exp(-np.sqrt(zz / z1)))
    return wl, wt


@pytest.mark.parametrize("nz", [32, 128])
def test_analytic_wake_sum_equals_the_doubled_grid_fft(nz):
    """wakefield_FieldQuant (Field.f90:590-782): the short-range wakes of a
    periodic structure (iris radius 11.6 mm, gap 29 mm, period 35 mm), both
    planes, as the oracle's direct sums."""
    L = orc.lib()
    freq, curr, mass, chrg, gam, npt = 1.3e9, 0.13, 0.51099895e6, -1.0, 190.0, 20000
    aa, gg, leng = 0.0116, 0.029, 0.035
    orc.physconst(freq)
    rng = np.random.default_rng(nz + 1)
    densz = npt * np.exp(-0.5 * ((np.arange(nz) - nz / 2) / (nz / 6)) ** 2)
    densz[[0, -1]] = 0.0
    xsum = densz * 1e-4 * rng.standard_normal(nz)
    ysum = densz * 1e-4 * rng.standard_normal(nz)
    rng6 = np.array([-1e-3, 1e-3, -1e-3, 1e-3, -0.9e-3, 1.1e-3]) * 190
    out = np.zeros(3 * nz)
    L.orc_wake_field_analytic(nz, orc.dp(densz), orc.dp(xsum), orc.dp(ysum), orc.dp(rng6), gam,
                              curr, npt, mass, chrg, aa, gg, leng, orc.dp(out))
    hz = (rng6[5] - rng6[4]) / (nz - 1) / gam
    recv = densz * curr / freq / npt / hz * chrg / abs(chrg)
    with np.errstate(invalid="ignore", divide="ignore"):
        xbar = np.where(densz != 0, xsum / densz, 0.0)
        ybar = np.where(densz != 0, ysum / densz, 0.0)
    ex, ey, ez = fft_wake(None, recv, xbar, ybar, hz, True,
                          greens=analytic_greens(aa, gg, leng, nz, hz))
    xycon, tcon, bet = kick_consts(gam, curr, mass, chrg, freq)
    want = np.r_[chrg * ex / xycon / mass / bet / gam, chrg * ey / xycon / mass / bet / gam,
                 chrg * ez / tcon / mass]
    for part in range(3):
        w, o = want[part * nz:(part + 1) * nz], out[part * nz:(part + 1) * nz]
        assert np.abs(w).max() > 0
        np.testing.assert_allclose(o, w, rtol=0, atol=1e-11 * np.abs(w).max())


def test_wake_switch_of_the_element_loop():
    """AccSimulator.f90:865-875 with -41's flags: 105/106 with Param(15) > 0
    turns the (analytic, or the read-in if on) wake on, without it off; other
    elements turn off only a wake that is not a read-in one.  Observed
    through orc_run: a lattice of an RF structure with wake parameters then
    a drift, against the same with the parameters zeroed."""
    cfg_pts = np.zeros((1000, 9))
    rng = np.random.default_rng(5)
    cfg_pts[:, :6] = 1e-3 * rng.standard_normal((1000, 6))
    cfg_pts[:, 6] = -1.0 / 0.51099895e6
    cfg_pts[:, 7] = 1e-3 / 1.3e9 / 1000
    cfg_pts[:, 8] = np.arange(1000) + 1
    ref = np.array([0, 0, 0, 0, 0, -200.0])

    def rf(wake):
        v = [1.0e6, 1.3e9, 0.0, -1.0, 1.0] + [0.0] * 19
        if wake:
            v[11], v[12], v[13] = 0.0116, 0.029, 0.035
        return impz.elem(105, 0.2, 4, 1, v)

    drift = impz.elem(0, 0.2, 4, 1, [1.0])
    orc.wake_off()
    res = {}
    for name, lat in (("wake", [rf(True), drift]), ("plain", [rf(False), drift])):
        rows, p, _ = orc.run(lat, cfg_pts, 1.0, 0.51099895e6, -1.0, 1.3e9, ref, (8, 8, 32))
        res[name] = rows
    # identical through nothing, different after the structure's steps
    assert np.array_equal(res["wake"][0], res["plain"][0])
    assert not np.allclose(res["wake"][4, 21], res["plain"][4, 21], rtol=1e-12, atol=0)


def test_wake_line_density_sums_to_the_particle_count():
    """AccSimulator.f90:1279-1296: each particle adds ab and 1-ab."""
    L = orc.lib()
    rng = np.random.default_rng(3)
    n, nz = 5000, 40
    pts = np.zeros((n, 9))
    pts[:, 0] = 1e-3 * rng.standard_normal(n)
    pts[:, 2] = 1e-3 * rng.standard_normal(n)
    pts[:, 4] = 2e-3 * rng.standard_normal(n)
    lo, hi = pts[:, 4].min(), pts[:, 4].max()
    eps = (hi - lo) / (nz - 3)
    rng6 = np.array([-1, 1, -1, 1, lo - eps, hi + eps], dtype=np.float64)
    d, xs, ys = np.zeros(nz), np.zeros(nz), np.zeros(nz)
    L.orc_wake_line(orc.dp(np.ascontiguousarray(pts)), n, nz, orc.dp(rng6), orc.dp(d),
                    orc.dp(xs), orc.dp(ys))
    assert abs(d.sum() - n) < 1e-9 * n
    np.testing.assert_allclose(xs.sum(), pts[:, 0].sum(), rtol=1e-10, atol=1e-15)
    # the padded range leaves the end planes empty (to the rounding of 1 - ab)
    assert abs(d[0]) < 1e-12 and abs(d[-1]) < 1e-12


def test_deck_wake_controls():
    """-41 elements become wake controls (AccSimulator.f90:959-978): the
    table is read when Param(3) > 0, Param(4) > 0 turns the wake on, a
    Param(4) below 10 drops the transverse wake for good."""
    import tempfile

    with tempfile.TemporaryDirectory() as wd:
        np.savetxt(os.path.join(wd, "rfdata41.in"), synthetic_table(rows=50))
        z24 = lambda *v: list(v) + [0.0] * (24 - len(v))  # noqa: E731
        d = deck.Deck(nx=8, ny=8, nz=8)
        d.elements = [
            deck.Element(0.0, 0, 1, -41, z24(1.5, 41, 20.0)),
            deck.Element(0.5, 2, 1, 0, z24(1.0)),
            deck.Element(0.0, 0, 1, -41, z24(1.0, 0, -1.0)),
            deck.Element(0.0, 0, 1, -41, z24(2.0, 0, 1.0)),
            deck.Element(0.0, 0, 1, -41, z24(2.0, 0, 30.0)),
        ]
        segs = list(deck.lattice_segments(d, wd))
    kinds = [k for k, _ in segs]
    assert kinds == ["wake", "run", "wake", "wake", "wake", "skipped"]
    w = [item for k, item in segs if k == "wake"]
    assert w[0]["on"] and w[0]["transverse"] and w[0]["scale"] == 1.5
    assert w[0]["table"].shape == (50, 4)
    assert not w[1]["on"]
    assert w[2]["on"] and not w[2]["transverse"]
    assert w[3]["on"] and not w[3]["transverse"]  # flagbtw = 2 stays


@pytest.mark.skipif(not os.path.isdir(EXAMPLES),
                    reason="IMPZ_REFERENCE_TREE unset (the reference's examples)")
def test_example3_runs_with_its_wake_on_the_oracle():
    """Example3's ten -41 controls switch the cavities' read-in wake
    (rfdata41.in) on and off around the 1.3 GHz cavities, and its -52 laser
    heater kicks the energy: the oracle runs the whole deck, its slice
    tables (-8) are finite, and the wake changes the final energy spread."""
    wd = os.path.join(EXAMPLES, "Example3")
    d = deck.read_deck(os.path.join(wd, "ImpactZ.in"))
    pts0 = deck.read_particles(os.path.join(wd, "particle.in"))
    finals = {}
    for with_wake in (True, False):
        pts, ref, z, nwake = pts0, d.refptcl(), 0.0, 0
        skip = set() if with_wake else {-41}
        try:
            for kind, item in deck.lattice_segments(d, wd, skip):
                if kind == "run":
                    _, pts, beam = orc.run(item, pts, d.bcurr, d.bmass, d.bcharge, d.bfreq, ref,
                                           (d.nx, d.ny, d.nz), z)
                    ref, z = np.array(beam.refptcl[:]), beam.z
                elif kind == "wake":
                    nwake += 1
                    if item["on"]:
                        orc.wake_set(item["table"], item["scale"], item["transverse"])
                    else:
                        orc.wake_off()
                elif kind == "slices":
                    nslice, ax, bx, ay, by = deck.slice_params(item)
                    tab = deck.slice_output(pts, pts.shape[0], nslice, d.bcurr / d.bfreq, d.bmass,
                                            ax, bx, ay, by, -ref[5], 299792458.0 / (2 * np.pi *
                                                                                   d.bfreq))
                    # weights, current, <pt> and centroids are finite; the
                    # emittance of an edge slice of a few particles can be the
                    # square root of a rounding-level negative, as there
                    assert tab.shape == (nslice, 11)
                    assert np.all(np.isfinite(tab[:, [0, 1, 2, 5, 7, 8]]))
                    assert np.isfinite(tab[:, 3]).mean() > 0.9
                elif kind == "laser":
                    p = np.ascontiguousarray(pts)
                    orc.lib().orc_laser_heater(orc.dp(p), p.shape[0], p.shape[0], item["rsig"],
                                               item["wavelength"], item["ez"], d.bmass)
                    pts = p
        finally:
            orc.wake_off()
        assert nwake == (10 if with_wake else 0)
        assert np.all(np.isfinite(pts))
        finals[with_wake] = pts
    spread = {k: np.std(v[:, 5]) for k, v in finals.items()}
    assert abs(spread[True] - spread[False]) > 1e-3 * spread[False]
