"""The reference's on-disk formats (impz_b200.deck): ImpactZ.in, particle.in,
rfdataN.in, fort.18/24-30.  The reference's own example decks are parsed
where its source tree is present (this container); round trips of the
writers always run.  No GPU needed."""
import os

import numpy as np
import pytest

from conftest import load_impz, load_oracle, reference_path

impz = load_impz()
from impz_b200 import beams, deck  # noqa: E402

EXAMPLES = reference_path("examples") or ""
have_examples = pytest.mark.skipif(not os.path.isdir(EXAMPLES),
                                   reason="IMPZ_REFERENCE_TREE unset (the reference's examples)")


@have_examples
def test_reads_the_reference_example_decks():
    d1 = deck.read_deck(os.path.join(EXAMPLES, "Example1", "ImpactZ.in"))
    assert (d1.np, d1.flagmap, d1.flagdist, d1.nx, d1.ny, d1.nz) == (200, 2, 19, 32, 32, 64)
    assert d1.bfreq == 324.0e6 and d1.qmcclist == [-1.064629e-9]
    d2 = deck.read_deck(os.path.join(EXAMPLES, "Example2", "ImpactZ.in"))
    assert (d2.np, d2.flagmap, d2.flagdist, d2.nchrg) == (160000, 1, 3, 1)
    assert d2.bkenergy == 230.0e6 and d2.bcharge == -1.0
    d3 = deck.read_deck(os.path.join(EXAMPLES, "Example3", "ImpactZ.in"))
    assert (d3.np, d3.flagmap, d3.flagbc, d3.flagdist) == (3134, 1, 1, 19)
    assert (d3.nx, d3.ny, d3.nz) == (32, 32, 32)
    types = [e.type for e in d3.elements]
    assert types.count(4) == 4 and types.count(103) == 5 and types.count(-41) == 10
    bend = next(e for e in d3.elements if e.type == 4)
    assert bend.nseg == 10 and bend.vals[2] == 150.0  # file ID: no CSR
    # "d" exponents and text after "/" are read as the reference reads them
    assert d3.qmcclist == [-1.95692801440299e-06] and d3.bfreq == 1.3e9
    p = deck.read_particles(os.path.join(EXAMPLES, "Example3", "particle.in"))
    assert p.shape == (3134, 9) and p[0, 8] == 1.0 and p[0, 6] == -1.956928e-06


@have_examples
def test_example3_lattice_runs_on_the_path_with_its_controls_skipped():
    """Example3 (map integrator, open BC, particle.in) maps onto the path's
    elements, its controls all handled (wake -41, laser heater -52, slice
    output -8); with them passed over the oracle runs its 138 steps."""
    orc = load_oracle()
    wd = os.path.join(EXAMPLES, "Example3")
    d = deck.read_deck(os.path.join(wd, "ImpactZ.in"))
    deck.check_supported(d)
    kinds = {k for k, _ in deck.lattice_segments(d, wd)}
    assert kinds == {"run", "dump", "wake", "laser", "slices", "skipped"}
    pts = deck.read_particles(os.path.join(wd, "particle.in"))
    ref, z, nrows, skipped = d.refptcl(), 0.0, 0, None
    for kind, item in deck.lattice_segments(d, wd, {-8, -41, -52}):
        if kind == "run":
            rows, pts, beam = orc.run(item, pts, d.bcurr, d.bmass, d.bcharge, d.bfreq, ref,
                                      (d.nx, d.ny, d.nz), z)
            ref, z = np.array(beam.refptcl[:]), beam.z
            nrows += len(rows) - (1 if nrows else 0)
        elif kind == "skipped":
            skipped = item
    assert nrows == 139 and sorted(set(skipped)) == [-52, -41, -8]
    assert np.all(np.isfinite(pts)) and pts.shape[0] == 3134
    assert -ref[5] * d.bmass > 1.5 * (d.bkenergy + d.bmass)  # the cavities accelerate


def test_deck_round_trip(tmp_path):
    d = deck.Deck(np=1000, nx=16, ny=16, nz=32, xrad=0.02, yrad=0.02, perdlen=0.1,
                  nptlist=[1000], currlist=[0.13], qmcclist=[-1.95692801440299e-06],
                  bcurr=0.13, bkenergy=98.169272e6, bmass=0.511005e6, bcharge=-1.0,
                  bfreq=1.3e9)
    d.elements = [deck.Element(0.0, 0, 1001, -2, [1.0] + [0.0] * 23),
                  deck.Element(0.5, 4, 1, 0, [0.014] + [0.0] * 23),
                  deck.Element(0.1, 4, 1, 1, [12.5, 0.0, 0.014] + [0.0] * 21),
                  deck.Element(0.0, 0, 0, -99, [0.0] * 24)]
    p = tmp_path / "ImpactZ.in"
    deck.write_deck(str(p), d)
    r = deck.read_deck(str(p))
    assert r == d


def test_particles_and_diag_files_round_trip(tmp_path):
    pts, _ = beams.gaussian_bunch(257, seed=beams.SEED0 + 3)
    deck.write_particles(str(tmp_path / "particle.in"), pts)
    np.testing.assert_array_equal(deck.read_particles(str(tmp_path / "particle.in")), pts)
    rows = np.random.default_rng(5).standard_normal((7, impz.DIAG_LEN))
    rows[:, 30:33] = np.abs(np.round(rows[:, 30:33] * 1000))
    deck.write_diag(str(tmp_path), rows)
    np.testing.assert_array_equal(deck.read_diag(str(tmp_path), "fort.24"),
                                  np.c_[rows[:, 0], rows[:, 6:12]])
    np.testing.assert_array_equal(deck.read_diag(str(tmp_path), "fort.18"),
                                  np.c_[rows[:, 0], rows[:, 1:6]])
    np.testing.assert_array_equal(deck.read_diag(str(tmp_path), "fort.28"),
                                  np.c_[rows[:, 0], rows[:, 30:33]])
    np.testing.assert_array_equal(deck.read_diag(str(tmp_path), "fort.30"),
                                  np.c_[rows[:, 0], rows[:, 39:45]])


GUI_READER = reference_path("GUI", "src", "ImpactFile.py") or ""


@pytest.mark.skipif(not os.path.exists(GUI_READER),
                    reason="IMPZ_REFERENCE_TREE unset (the reference's GUI deck reader)")
@pytest.mark.parametrize("example", ["Example1", "Example2", "Example3"])
def test_deck_reader_agrees_with_the_reference_gui_reader(example):
    """The reference's own Python deck reader (GUI/src/ImpactFile.py,
    conciseReadInput) gives the tokens of every non-comment line; the header
    values and each element's values up to its "/" equal read_deck's."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("impactz_gui_file", GUI_READER)
    gui = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gui)
    path = os.path.join(EXAMPLES, example, "ImpactZ.in")
    lines = gui.conciseReadInput(path)
    d = deck.read_deck(path)
    nums = lambda toks, k: [float(t) for t in toks[:k]]  # noqa: E731
    head = [nums(lines[0], 2), nums(lines[1], 5), nums(lines[2], 7), nums(lines[3], 4),
            nums(lines[4], d.nchrg), nums(lines[5], d.nchrg), nums(lines[6], d.nchrg),
            nums(lines[7], 7), nums(lines[8], 7), nums(lines[9], 7), nums(lines[10], 6)]
    mine = [[d.npcol, d.nprow], [d.dim, d.np, d.flagmap, d.flagerr, d.flagdiag],
            [d.nx, d.ny, d.nz, d.flagbc, d.xrad, d.yrad, d.perdlen],
            [d.flagdist, d.restart, d.subcycle, d.nchrg], d.nptlist, d.currlist, d.qmcclist,
            d.distparam[0:7], d.distparam[7:14], d.distparam[14:21],
            [d.bcurr, d.bkenergy, d.bmass, d.bcharge, d.bfreq, d.phsini]]
    assert head == mine
    elems = [toks for toks in lines[11:] if len(toks) >= 4]
    assert len(elems) == len(d.elements)
    for toks, e in zip(elems, d.elements):
        vals = []
        for t in toks:
            if t.startswith("/"):
                break
            vals.append(float(t.rstrip("/")))
            if t.endswith("/"):
                break
        assert vals[:4] == [e.length, e.nseg, e.mapstp, e.type]
        assert vals[4:] == e.vals[:len(vals) - 4]


def test_checkpoint_round_trip_and_records(tmp_path):
    """-7 checkpoints (outpoint_Output, Output.f90:1733-1774): nine gfortran
    unformatted records, read back unchanged."""
    rng = np.random.default_rng(9)
    pts = rng.standard_normal((37, 9))
    path = str(tmp_path / "fort.1234")
    deck.write_checkpoint(path, 1.25, 7, 3, 40, 40, [1e-4, 2e-4, 3e-4],
                          [-1, 1, -2, 2, -3, 3], (8, 16, 32), np.arange(6.0), pts)
    raw = open(path, "rb").read()
    assert np.frombuffer(raw[:4], "<i4")[0] == 8 and np.frombuffer(raw[12:16], "<i4")[0] == 8
    assert len(raw) == 9 * 8 + 8 + 16 + 24 + 48 + 8 + 32 + 4 + 48 + 72 * 37
    ck = deck.read_checkpoint(path)
    assert ck["z"] == 1.25 and (ck["inb"], ck["jstp"], ck["ibal"], ck["nstep"]) == (7, 3, 40, 40)
    np.testing.assert_array_equal(ck["pts"], pts)
    np.testing.assert_array_equal(ck["refptcl"], np.arange(6.0))
    np.testing.assert_array_equal(ck["range"], [-1, 1, -2, 2, -3, 3])


def test_checkpoint_controls_in_the_lattice(tmp_path):
    """A -7 element yields its counters; a restart skips the elements up to
    and including it."""
    z24 = lambda *v: list(v) + [0.0] * (24 - len(v))  # noqa: E731
    d = deck.Deck(nx=8, ny=8, nz=8)
    d.elements = [deck.Element(0.5, 3, 1, 0, z24(1.0)), deck.Element(0.0, 0, 1001, -7, z24()),
                  deck.Element(0.4, 2, 1, 0, z24(1.0)), deck.Element(0.0, 0, 1002, -7, z24())]
    segs = list(deck.lattice_segments(d, str(tmp_path)))
    cks = [item for k, item in segs if k == "checkpoint"]
    assert [(c["inb"], c["jstp"], c["nstep"]) for c in cks] == [(2, 4, 3), (4, 3, 5)]
    assert deck.checkpoint_file(d) == 1002
    rest = list(deck.lattice_segments(d, str(tmp_path), start=2))
    assert [k for k, _ in rest] == ["run", "checkpoint", "skipped"]
    assert rest[0][1][0].length == 0.4


def _slices_by_loop(pts, npt, nslice, qchg, pmass, ax0, bx0, ay0, by0, gam0, scxl):
    """sliceprocdep_Output (Output.f90:3002-3215) as plain loops."""
    import math
    f32 = lambda v: float(np.float32(v))  # noqa: E731
    sclcur = 2.99792e8 * qchg / npt
    gx0, gy0 = (1 + ax0 ** 2) / bx0, (1 + ay0 ** 2) / by0
    zmn, zmx = min(pts[:, 4]), max(pts[:, 4])
    zmin, zmax = zmn - (zmx - zmn) * f32(0.5e-5), zmx + (zmx - zmn) * f32(0.5e-5)
    hz = (zmax - zmin) / (nslice - 1)
    acc = [[0.0] * nslice for _ in range(12)]
    cells = []
    for p in pts:
        iz = min(max(int((p[4] - zmin) / hz + 1), 1), nslice - 1)
        ab = ((zmin - p[4]) + iz * hz) / hz
        cells.append((iz, ab))
        vals = (1.0, p[0], p[0] ** 2, p[1], p[1] ** 2, p[0] * p[1], p[2], p[2] ** 2, p[3],
                p[3] ** 2, p[2] * p[3], p[5])
        for k, v in enumerate(vals):
            acc[k][iz - 1] += v * ab
            acc[k][iz] += v * (1.0 - ab)
    out = []
    mean = [[acc[k][i] / acc[0][i] if acc[0][i] > 0 else 0.0 for i in range(nslice)]
            for k in range(12)]
    unc = [0.0] * nslice
    for p, (iz, ab) in zip(pts, cells):
        gz = mean[11][iz - 1] * ab + mean[11][iz] * (1 - ab)
        unc[iz - 1] += (p[5] - gz) ** 2 * ab
        unc[iz] += (p[5] - gz) ** 2 * (1 - ab)
    for i in range(nslice):
        c = acc[0][i]
        xx, xx2, px, px2, xpx, yy, yy2, py, py2, ypy, gam = (mean[k][i] for k in range(1, 12))
        epx = math.sqrt((xx2 - xx ** 2) * (px2 - px ** 2) - (xpx - xx * px) ** 2)
        epy = math.sqrt((yy2 - yy ** 2) * (py2 - py ** 2) - (ypy - yy * py) ** 2)
        gb = math.sqrt((gam0 - gam) ** 2 - 1)
        axx, bxx = -xpx / epx, (xx2 - xx ** 2) * gb / epx
        ayy, byy = -ypy / epy, (yy2 - yy ** 2) * gb / epy
        bmx = bxx * gx0 - 2 * axx * ax0 + (1 + axx ** 2) / bxx * bx0
        bmy = byy * gy0 - 2 * ayy * ay0 + (1 + ayy ** 2) / byy * by0
        out.append([-(zmin + i * hz) * scxl, c, c / (hz * scxl) * sclcur, epx * scxl,
                    epy * scxl, -gam / gam0, math.sqrt(unc[i] / c) * pmass, xx * scxl,
                    yy * scxl, bmx, bmy])
    return np.array(out)


def test_slice_output_matches_a_loop_restatement():
    """-8 slice tables (sliceprocdep_Output): the vectorised form = plain
    loops over a correlated bunch, every slice populated."""
    rng = np.random.default_rng(21)
    n = 3000
    pts = np.zeros((n, 9))
    pts[:, :6] = rng.standard_normal((n, 6)) * [1e-2, 1e-3, 1e-2, 1e-3, 0.05, 0.02]
    pts[:, 1] += 0.3 * pts[:, 0] * 1e-1
    pts[:, 5] += 0.5 * pts[:, 4]
    args = (n, 7, 1e-9, 0.511e6, 0.5, 2.0, -0.3, 3.0, 200.0, 0.118)
    got = deck.slice_output(pts, *args)
    want = _slices_by_loop(pts, *args)
    assert got.shape == (7, 11) and np.all(np.isfinite(got))
    np.testing.assert_allclose(got, want, rtol=1e-10, atol=0)
    assert abs(got[:, 1].sum() - n) < 1e-9 * n


def test_emfld_map_file_round_trip_and_deck_element(tmp_path):
    """An EMfld 110 map written in read4_Data's format (complex constants
    "(re,im)") reads back exactly, and a Flagmap=2 deck's 110 element built
    from it tracks on the oracle like the element built from the arrays."""
    from test_lorentz import emfld, emfld_grid, quad_map
    header, data = emfld_grid(quad_map(12.0), 0.1, nz=6)
    data = np.stack([data.real, data.imag], axis=-1).reshape(data.shape[0], 12)
    data[:, 4] += 1.0e5  # a uniform Ez as well
    data[:, 5] -= 2.0e4
    path = str(tmp_path / "rfdata7.in")
    deck.write_emfld(path, header, data)
    h2, d2 = deck.read_emfld(path)
    np.testing.assert_array_equal(h2, header)
    np.testing.assert_array_equal(d2, data)
    d = deck.Deck()
    d.flagmap = 2
    vals = [1.0, 402.5e6, 15.0, 7.0, 1.0, 1.0, 0, 0, 0, 0, 0, 1.0, 2.0]
    d.elements = [deck.Element(0.1, 4, 1, 110, vals + [0.0] * (24 - len(vals)))]
    runs = [item for kind, item in deck.lattice_segments(d, str(tmp_path)) if kind == "run"]
    cfg = beams.fodo_1e5(n=500, seed=beams.SEED0 + 95)
    args = (cfg["pts"], 0.0, cfg["mass"], cfg["charge"], cfg["freq"], cfg["refptcl"],
            (16, 16, 32))
    orc = load_oracle()
    _, p1, b1 = orc.run(runs[0], *args, flagmap=2)
    direct = emfld(0.1, 4, (header, data), 1.0, 402.5e6, 15.0)
    direct.val[3] = 7.0
    _, p2, b2 = orc.run([direct], *args, flagmap=2)
    np.testing.assert_array_equal(p1, p2)
    np.testing.assert_array_equal(b1.refptcl[:], b2.refptcl[:])
    assert b1.refptcl[5] != cfg["refptcl"][5]
