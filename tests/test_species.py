"""Multiple charge states on the oracle and in the host code, no GPU needed:
Pts1 rows 7 (q/m) and 8 (charge weight) per particle, chgupdate_BeamBunch's
count of each charge state after every conv1st (BeamBunch.f90:688-728,
AccSimulator.f90:1130) and fort.32 (Output.f90:352)."""
import numpy as np

from conftest import load_impz, load_oracle

impz = load_impz()
orc = load_oracle()
from impz_b200 import beams, deck  # noqa: E402

NPT = [3000, 2000]
QSTATES = (33.0, 34.0)
CURR = [0.004, 0.003]


def ion_bunch(seed=beams.SEED0 + 101):
    return beams.charge_state_bunch(NPT, QSTATES, CURR, seed=seed)


def test_charge_state_bunch_rows():
    pts, ref, mass, qmc = ion_bunch()
    assert pts.shape == (sum(NPT), 9)
    for j in range(2):
        sel = pts[:, 6] == qmc[j]
        assert sel.sum() == NPT[j]
        np.testing.assert_array_equal(pts[sel, 7], CURR[j] / 80.5e6 / NPT[j])
    # interleaved, not in blocks
    assert 0 < np.argmax(pts[:, 6] == qmc[1]) < 20


def test_oracle_counts_charge_states_after_every_conv1st():
    """orc_run's chgupdate after each conv1st, copied at every record: the
    first record holds the list given (the deck's nptlist), the others sum
    to fort.28's particle count, and the last one matches the surviving
    particles' rows 7.  A narrow aperture makes conv1st lose particles."""
    pts, ref, mass, qmc = ion_bunch()
    lat = [impz.elem(0, 0.1, 4, 1, [0.004]),
           impz.elem(1, 0.1, 4, 1, [8.0, -1.0, 0.004]),   # K-map quadrupole
           impz.elem(0, 0.1, 4, 1, [0.004]),
           impz.elem(1, 0.1, 4, 1, [-8.0, -1.0, 0.004])]
    nrec = 1 + sum(e.nseg for e in lat)
    npl = np.array(NPT, dtype=np.int32)
    out = np.zeros((nrec, 2), dtype=np.int32)
    rows, p, beam = orc.run(lat, pts, sum(CURR), mass, QSTATES[0], 80.5e6, ref, (16, 16, 32),
                            charge_states=(qmc, npl, out))
    assert rows.shape[0] == nrec
    np.testing.assert_array_equal(out[0], NPT)
    np.testing.assert_array_equal(out[1:].sum(1), rows[1:, 32].astype(np.int32))
    assert rows[-1, 32] < sum(NPT)  # the aperture lost particles
    np.testing.assert_array_equal(out[-1], [(p[:, 6] == q).sum() for q in qmc])
    np.testing.assert_array_equal(npl, out[-1])  # nptlist updated in place (idchgold)


def test_oracle_lorentz_kick_uses_each_particles_charge_to_mass():
    """Without current the particles do not interact: under the Lorentz
    integrator through an RF cell (kick2's rays(7,n), BeamBunch.f90:3026-3035)
    each charge state of a mixed bunch ends exactly where a bunch of that
    charge state alone does, and the two charge states end differently."""
    from test_lorentz import rf_cell
    coef, _ = rf_cell()
    pts, ref, mass, qmc = ion_bunch()
    freq = 80.5e6
    lat = [impz.elem(101, 0.08, 20, 20, [2.5e6, freq, 222.0, 1.0, 0.0065], rf=coef)]
    run = lambda p: orc.run(lat, p, 0.0, mass, QSTATES[0], freq, ref, (16, 16, 32),  # noqa
                            flagmap=2)[1]
    mixed = run(pts)
    for j in range(2):
        alone = pts.copy()
        alone[:, 6] = qmc[j]
        out = run(alone)
        sel = pts[:, 6] == qmc[j]
        np.testing.assert_array_equal(mixed[sel], out[sel])
    a0, a1 = pts.copy(), pts.copy()
    a0[:, 6], a1[:, 6] = qmc[0], qmc[1]
    assert np.max(np.abs(run(a0)[:, 5] - run(a1)[:, 5])) > 0


def test_charge_state_counts_and_fort32(tmp_path):
    """fort.32: z and the particles of each charge state per record, a
    species counting for every qmcclist entry within relative 1e-4."""
    qm = np.array([33.0 / 2.2e11, 34.0 / 2.2e11, 33.0 / 2.2e11 * (1 + 5e-5)])
    per = np.array([[10, 20, 3], [9, 20, 2]])
    cs = deck.charge_state_counts(qm, per, [33.0 / 2.2e11, 34.0 / 2.2e11, 1.0])
    np.testing.assert_array_equal(cs, [[13, 20, 0], [11, 20, 0]])
    rows = np.zeros((2, impz.DIAG_LEN))
    rows[:, 0] = [0.0, 0.25]
    deck.write_diag(str(tmp_path), rows, cs)
    got = np.loadtxt(str(tmp_path / "fort.32"))
    np.testing.assert_array_equal(got, [[0.0, 13, 20, 0], [0.25, 11, 20, 0]])


def test_runner_accepts_several_charge_states():
    d = deck.Deck(np=5, nchrg=2, nptlist=[3, 2], currlist=[0.001, 0.001],
                  qmcclist=[1e-9, 2e-9], flagdist=19)
    deck.check_supported(d)


def test_species_footprint():
    """The species column costs one byte per particle in each of the two
    particle buffers (plus a 3 KB table); a run's tables add
    IMPZ_MAX_SPECIES counts per record.  Footprints are whole 2 MiB
    granules."""
    n, grid, g = 4_000_000, (32, 32, 64), 2 << 20
    a = impz.footprint(n, grid, impz.FORM_FP64)
    b = impz.footprint(n, grid, impz.FORM_FP64, species=True)
    assert abs((b - a) - 2 * n) <= g
    a1 = impz.footprint(n, grid, impz.FORM_FP64, nsteps=1000)
    b1 = impz.footprint(n, grid, impz.FORM_FP64, nsteps=1000, species=True)
    extra = 1024 * 128 * 4  # 1024 table rows (the power of two above 1002)
    assert abs((b1 - a1) - (b - a) - extra) <= g
