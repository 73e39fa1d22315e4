"""Multiple charge states on the GPU, through the C ABI, against the oracle.

A bunch created with IMPZ_FLAG_SPECIES carries Pts1 rows 7 (q/m) and 8
(charge weight) per particle: the deposit weights each particle by its row 8
(deposit_BeamBunch, BeamBunch.f90:3749-3763), the K-map quadrupole, the bend
maps and the Lorentz kick use its row 7 (Quadrupole.f90:533, Dipole.f90:
466-788, BeamBunch.f90:3026-3035), and every record carries chgupdate's
count of each charge state (BeamBunch.f90:688-728) for fort.32.

Tolerances (plain FP64 form): per-record particle counts of each charge
state exact; rms columns after a lattice within 1e-8 of the column's
largest magnitude (the oracle sums the weighted charge in FP64, the GPU in
2^-40 fixed point); per-cell counts exact and one step's charge density
within the fixed point's rounding: a particle of fractional weight rounds
each of its eight corner quanta, the largest corner taking the remainder of
its rounded total, so a node is off by at most 4 quanta per particle
touching it (relative L2 1e-11 with a species of the other sign, whose
charge cancels).  A single-species bunch with the flag moves every particle
bit for bit as the bunch without it; the records agree to the rounding of
the moment sums, whose order follows the sort's atomics."""
import ctypes

import numpy as np
import pytest

from conftest import load_impz, load_oracle
from test_gpu_parity import rel_l2

pytestmark = pytest.mark.gpu

impz = load_impz()
orc = load_oracle()
from impz_b200 import beams, deck  # noqa: E402

NPT = [12000, 8000]
QSTATES = (33.0, 34.0)
CURR = [0.004, 0.003]
FREQ = 80.5e6
GRID = (32, 32, 64)
RMS_COLS = [7, 9, 11, 13, 15, 17, 19, 21, 23]


def ion_bunch(seed=beams.SEED0 + 111, npt=NPT, qstates=QSTATES, curr=CURR):
    return beams.charge_state_bunch(npt, qstates, curr, seed=seed, freq=FREQ)


def gpu_run(pts, ref, mass, lat, flagmap=1, species=True, form=impz.FORM_FP64):
    b = impz.Bunch(pts, sum(CURR), mass, QSTATES[0], FREQ, ref, GRID, form=form,
                   track_ids=True, species=species)
    try:
        b.set_integrator(flagmap)
        recs, zs = b.run(lat)
        refs = b.run_reference()
        counts = b.run_species() if species else None
        qm, _ = b.species()
        final = b.download()
    finally:
        b.close()
    rows = np.array([impz.diag_row(zs[i], recs[i], refs[i], mass, FREQ)
                     for i in range(len(recs))])
    return rows, counts, qm, final, recs


def oracle_run(pts, ref, mass, qmc, lat, flagmap=1):
    nrec = 1 + sum(e.nseg for e in lat)
    npl = np.array([(pts[:, 6] == q).sum() for q in qmc], dtype=np.int32)
    out = np.zeros((nrec, len(qmc)), dtype=np.int32)
    rows, p, _ = orc.run(lat, pts, sum(CURR), mass, QSTATES[0], FREQ, ref, GRID, flagmap=flagmap,
                         charge_states=(qmc, npl, out))
    return rows, out, p


def compare(rows_g, counts_g, qm_g, rows_o, cs_o, qmc):
    assert rows_g.shape == rows_o.shape
    np.testing.assert_array_equal(rows_g[:, 0], rows_o[:, 0])
    for c in RMS_COLS:
        scale = np.max(np.abs(rows_o[:, c])) + 1e-300
        err = np.max(np.abs(rows_g[:, c] - rows_o[:, c])) / scale
        assert err <= 1e-8, (c, err)
    np.testing.assert_array_equal(rows_g[:, 30:33], rows_o[:, 30:33])
    cs_g = deck.charge_state_counts(qm_g, counts_g, qmc)
    np.testing.assert_array_equal(cs_g, cs_o)


def test_map_integrator_two_charge_states_with_losses():
    """Drifts and K-map quadrupoles behind a 4 mm aperture (conv1st loses
    particles of both charge states), then a sector bend: every record's
    rms columns and charge-state counts against the oracle, and the final
    particles keep their rows 7 and 8."""
    pts, ref, mass, qmc = ion_bunch()
    lat = [impz.elem(0, 0.1, 4, 1, [0.004]),
           impz.elem(1, 0.1, 4, 1, [8.0, -1.0, 0.004]),
           impz.elem(0, 0.1, 4, 1, [0.004]),
           impz.elem(1, 0.1, 4, 1, [-8.0, -1.0, 0.004]),
           impz.elem(4, 0.2, 4, 1, [0.05, 0.0, 150.0, 0.01]),
           impz.elem(0, 0.1, 4, 1, [1.0])]
    rows_g, counts_g, qm_g, final, _ = gpu_run(pts, ref, mass, lat)
    rows_o, cs_o, p_o = oracle_run(pts, ref, mass, qmc, lat)
    np.testing.assert_array_equal(np.sort(qm_g), np.sort(qmc))
    assert cs_o[-1].sum() < sum(NPT) and np.all(cs_o[-1] < NPT)  # both lost particles
    compare(rows_g, counts_g, qm_g, rows_o, cs_o, qmc)
    by_id = pts[np.argsort(pts[:, 8])]
    ids = final[:, 8].astype(np.int64) - 1
    np.testing.assert_array_equal(final[:, 6:8], by_id[ids, 6:8])
    np.testing.assert_array_equal(np.sort(final[:, 8]), np.sort(p_o[:, 8]))


def test_lorentz_integrator_two_charge_states():
    """Flagmap=2 through DTL cells over Fourier coefficients and a
    quadrupole, with space charge: kick2 uses each particle's q/m."""
    from test_lorentz import rf_cell
    coef, _ = rf_cell()
    pts, ref, mass, qmc = ion_bunch(seed=beams.SEED0 + 113)
    cell = lambda th: impz.elem(101, 0.08, 12, 20, [2.5e6, FREQ, th, 1.0, 0.0065,  # noqa: E731
                                                    0.02, 68.0, 0.02, -67.0], rf=coef)
    lat = [cell(222.0), cell(218.0), impz.elem(1, 0.045, 8, 1, [-19.15, 0.0, 0.009]),
           impz.elem(0, 0.09, 8, 1, [0.009])]
    rows_g, counts_g, qm_g, _, _ = gpu_run(pts, ref, mass, lat, flagmap=2)
    rows_o, cs_o, _ = oracle_run(pts, ref, mass, qmc, lat, flagmap=2)
    compare(rows_g, counts_g, qm_g, rows_o, cs_o, qmc)


@pytest.mark.parametrize("form", [impz.FORM_FP64, impz.FORM_FP32CONV])
def test_single_species_flag_moves_particles_identically(form):
    """One charge state: with the species path (column, weights, counts)
    every particle ends bit for bit where it ends without it; the moment
    records agree to the rounding of their sums and the count of the one
    species is Nptlocal."""
    cfg = beams.fodo_1e5(n=20_000, seed=beams.SEED0 + 115)
    lat = beams.fodo(1)
    out = []
    for sp in (False, True):
        b = impz.Bunch(cfg["pts"], cfg["current"], cfg["mass"], cfg["charge"], cfg["freq"],
                       cfg["refptcl"], cfg["grid"], form=form, track_ids=True, species=sp)
        try:
            recs, _ = b.run(lat)
            p = b.download()
            cnt = b.run_species() if sp else None
        finally:
            b.close()
        out.append((recs, p[np.argsort(p[:, 8])], cnt))
    np.testing.assert_array_equal(out[0][1], out[1][1])
    r0, r1 = out[0][0], out[1][0]
    np.testing.assert_array_equal(r0[:, 44:], r1[:, 44:])  # Npt, Nptlocal, Current
    scale = np.max(np.abs(r0[:, :44]), axis=0) + 1e-300
    assert np.max(np.abs(r0[:, :44] - r1[:, :44]) / scale) <= 1e-12
    np.testing.assert_array_equal(out[1][2][:, 0], out[0][0][:, 45].astype(np.int32))


def test_per_step_deposit_and_chgupdate_three_species():
    """The per-step surface with a third, negatively charged species: after
    impz_sc_prepare (a 3 mm pipe loses particles), impz_chgupdate counts
    the particles conv1st kept in each charge state; the weighted deposit
    matches deposit_BeamBunch's sum of rays(8,i) weights, counts exact."""
    npt, qs, cur = [6000, 4000, 2000], (33.0, 34.0, -1.0), [0.004, 0.003, 0.002]
    pts, ref, mass, qmc = ion_bunch(seed=beams.SEED0 + 117, npt=npt, qstates=qs, curr=cur)
    cfg = dict(current=sum(cur), mass=mass, charge=qs[0], freq=FREQ, refptcl=ref, grid=GRID)
    e = impz.elem(0, 0.1, 4, 1, [0.003])
    tau = 0.025
    from test_gpu_parity import oracle_step
    o = oracle_step(pts, cfg, e, tau, 0.003)
    b = impz.Bunch(pts, sum(cur), mass, qs[0], FREQ, ref, GRID, form=impz.FORM_FP64,
                   track_ids=True, species=True)
    try:
        before = b.chgupdate(qmc)
        z, ih = b.map_half(e, 0.0, 0.0, tau / 2, 1, 0)
        nptot, ptrange, rng, msize = b.sc_prepare(0.003, 0.003)
        kept = b.chgupdate(qmc)
        rho, counts = b.deposit()
        qm, w = b.species()
    finally:
        b.close()
    np.testing.assert_array_equal(before, npt)
    assert nptot == o["nptot"] < sum(npt)
    np.testing.assert_array_equal(kept, [(o["pts"][:, 6] == q).sum() for q in qmc])
    np.testing.assert_array_equal(ptrange, o["ptrange"])
    np.testing.assert_array_equal(counts, o["counts"])
    wref = w[np.argmax(np.abs(w))]
    quantum = abs(wref) * 2.0 ** -40
    assert np.max(np.abs(rho - o["rho"])) <= 4 * quantum * 8 * counts.max()
    assert rel_l2(rho, o["rho"]) <= 1e-11
    assert np.all(np.sign(w) == np.sign(qm))  # the weight carries the charge sign
    # every kept particle deposits its own weight
    want = sum(kept[list(qmc).index(q)] * wk for q, wk in zip(qm, w))
    assert abs(rho.sum() - want) <= 1e-12 * np.abs(w).max() * sum(kept)


def test_non_uniform_rows_need_the_flag():
    pts, ref, mass, qmc = ion_bunch()
    with pytest.raises(impz.ImpzError):
        impz.Bunch(pts, sum(CURR), mass, QSTATES[0], FREQ, ref, GRID, species=False)
