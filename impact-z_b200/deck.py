"""The reference's on-disk formats and a standalone runner over them.

* `read_deck` parses ImpactZ.in as in1_Input/in2_Input do
  (src/Contrl/Input.f90:37-385): Fortran list-directed records, lines whose
  first token starts with "!" are comments, a "/" ends a record (the rest
  of the line is free text, the missing values stay zero), "d" exponents.
* `read_particles` / `write_particles`: particle.in of readin_Dist
  (src/Appl/Distribution.f90:1666-1714): the count, then Pts1 one particle
  per line (9 values).
* `read_rfdata`: rfdataN.in of read1_Data (src/DataStruct/Data.f90:139-215):
  z, Ez, Ez', Ez'' per line, z shifted to start at 0.
* `write_diag`: fort.18 and fort.24-30 of diagnostic1_Output
  (src/Contrl/Output.f90:341-352), one record per line; the reference
  prints with `g0` (shortest width), here `%.17g` (the same digits).
* `write_phase`: the phase-space dump of a type -2 element, phase_Output
  (src/Contrl/Output.f90:1776-1855), fort.<mapstp>, every samplePeriod-th
  particle.
* `run_deck` runs a deck of the map integrator with open boundaries and a
  particle.in distribution (Flagmap=1, Flagbc=1, Flagdist=19) on the GPU
  runner, splitting the lattice at control elements (types < 0,
  `lattice_segments`): -2 dumps phase space, -7 writes a checkpoint, -8
  appends a slice table (`slice_output`, sliceprocdep_Output of
  src/Contrl/Output.f90:3002-3215), -41
  turns the read-in wake on or off, -52 applies the laser heater's energy
  kick, -99 ends the lattice, the types listed in `skip` are passed over
  (reported), any other is refused.
* `read_wake`: rfdataN.in as the wake table of a -41 element, read1wk_Data
  (src/DataStruct/Data.f90:559-633).
* `write_checkpoint` / `read_checkpoint`: the -7 checkpoint of
  outpoint_Output / inpoint_Output (src/Contrl/Output.f90:1733-1774,
  1371-1437), gfortran's unformatted sequential records; `run_deck` writes
  one at each -7 and, with the deck's restart flag set, continues from the
  last -7's file after that element.
"""
import os
import re
from dataclasses import dataclass, field

import numpy as np

_NUM = re.compile(r"([0-9.])[dD]([-+]?[0-9])")


def _values(line):
    """List-directed values of one record: text after '/' is ignored."""
    rec = line.split("/", 1)[0]
    rec = _NUM.sub(r"\1e\2", rec).replace(",", " ")
    return rec.split()


def _is_comment(line):
    t = line.strip()
    return t == "" or t.startswith("!")


@dataclass
class Element:
    length: float
    nseg: int
    mapstp: int
    type: int
    vals: list = field(default_factory=lambda: [0.0] * 24)


@dataclass
class Deck:
    npcol: int = 1
    nprow: int = 1
    dim: int = 6
    np: int = 0
    flagmap: int = 1
    flagerr: int = 0
    flagdiag: int = 1
    nx: int = 0
    ny: int = 0
    nz: int = 0
    flagbc: int = 1
    xrad: float = 0.0
    yrad: float = 0.0
    perdlen: float = 0.0
    flagdist: int = 19
    restart: int = 0
    subcycle: int = 0
    nchrg: int = 1
    nptlist: list = field(default_factory=list)
    currlist: list = field(default_factory=list)
    qmcclist: list = field(default_factory=list)
    distparam: list = field(default_factory=lambda: [0.0] * 21)
    bcurr: float = 0.0
    bkenergy: float = 0.0
    bmass: float = 0.0
    bcharge: float = 0.0
    bfreq: float = 0.0
    phsini: float = 0.0
    elements: list = field(default_factory=list)

    def refptcl(self):
        """construct_BeamBunch's reference particle (BeamBunch.f90:56-58)."""
        r = [0.0] * 6
        r[4] = self.phsini
        r[5] = -(1.0 + self.bkenergy / self.bmass)
        return np.array(r)


def read_deck(path):
    """ImpactZ.in -> Deck (in1_Input / in2_Input, Input.f90:37-385)."""
    with open(path) as f:
        lines = [ln for ln in f.read().splitlines() if not _is_comment(ln)]
    it = iter(lines)

    def record(n):
        # list-directed: a record may continue on the next lines until n values
        vals = []
        while len(vals) < n:
            ln = next(it)
            vals += _values(ln)
            if "/" in ln:
                break
        return vals + ["0"] * (n - len(vals))

    d = Deck()
    v = record(2)
    d.npcol, d.nprow = int(v[0]), int(v[1])
    v = record(5)
    d.dim, d.np, d.flagmap, d.flagerr, d.flagdiag = (int(float(x)) for x in v[:5])
    v = record(7)
    d.nx, d.ny, d.nz, d.flagbc = (int(float(x)) for x in v[:4])
    d.xrad, d.yrad, d.perdlen = (float(x) for x in v[4:7])
    v = record(4)
    d.flagdist, d.restart, d.subcycle, d.nchrg = (int(float(x)) for x in v[:4])
    d.nptlist = [int(float(x)) for x in record(d.nchrg)[: d.nchrg]]
    d.currlist = [float(x) for x in record(d.nchrg)[: d.nchrg]]
    d.qmcclist = [float(x) for x in record(d.nchrg)[: d.nchrg]]
    d.distparam = [float(x) for x in record(7)[:7] + record(7)[:7] + record(7)[:7]]
    v = record(6)
    d.bcurr, d.bkenergy, d.bmass, d.bcharge, d.bfreq, d.phsini = (float(x) for x in v[:6])
    for ln in it:
        v = _values(ln)
        if len(v) < 4:
            continue
        e = Element(float(v[0]), int(float(v[1])), int(float(v[2])), int(float(v[3])))
        vals = [float(x) for x in v[4:28]]
        e.vals = vals + [0.0] * (24 - len(vals))
        d.elements.append(e)
        if e.type == -99:
            break
    return d


def write_deck(path, d):
    """A Deck as ImpactZ.in (the layout read_deck and in1_Input read)."""
    g = lambda x: "%.17g" % x  # noqa: E731
    out = ["! written by impz_b200.deck", "%d %d" % (d.npcol, d.nprow),
           "%d %d %d %d %d" % (d.dim, d.np, d.flagmap, d.flagerr, d.flagdiag),
           "%d %d %d %d %s %s %s" % (d.nx, d.ny, d.nz, d.flagbc, g(d.xrad), g(d.yrad),
                                     g(d.perdlen)),
           "%d %d %d %d" % (d.flagdist, d.restart, d.subcycle, d.nchrg),
           " ".join(str(n) for n in d.nptlist), " ".join(g(c) for c in d.currlist),
           " ".join(g(q) for q in d.qmcclist)]
    for r in range(3):
        out.append(" ".join(g(x) for x in d.distparam[7 * r:7 * r + 7]))
    out.append(" ".join(g(x) for x in (d.bcurr, d.bkenergy, d.bmass, d.bcharge, d.bfreq,
                                       d.phsini)))
    for e in d.elements:
        last = max([i + 1 for i, x in enumerate(e.vals) if x != 0.0] or [0])
        out.append("%s %d %d %d %s /" % (g(e.length), e.nseg, e.mapstp, e.type,
                                         " ".join(g(x) for x in e.vals[:last])))
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")


def read_particles(path):
    """particle.in -> Pts1 as an (n, 9) array (readin_Dist)."""
    with open(path) as f:
        first = f.readline()
        n = int(float(_values(first)[0]))
        vals = np.array(_values(f.read().replace("\n", " ")), dtype=np.float64)
    if vals.size < 9 * n:
        raise ValueError("particle.in holds %d values for %d particles" % (vals.size, n))
    return vals[: 9 * n].reshape(n, 9)


def write_particles(path, pts, sample=1):
    """Pts1 rows as particle.in / a phase_Output dump (9(g0,1x))."""
    pts = np.asarray(pts)[:: max(1, sample)]
    with open(path, "w") as f:
        f.write("%d\n" % pts.shape[0])
        for row in pts:
            f.write(" ".join("%.17g" % x for x in row) + "\n")


def write_phase(path, pts, sample):
    """phase_Output for samplePeriod >= 0: every sample-th particle, 9 values
    per line, no count line (Output.f90:1776-1855)."""
    pts = np.asarray(pts)[:: max(1, int(sample))]
    with open(path, "w") as f:
        for row in pts:
            f.write(" ".join("%.17g" % x for x in row) + "\n")


def read_rfdata(path):
    """rfdataN.in -> (z, Ez, Ez', Ez'') with z shifted to start at 0."""
    rows = []
    with open(path) as f:
        for ln in f:
            v = _values(ln)
            if len(v) >= 4:
                rows.append([float(x) for x in v[:4]])
    tab = np.array(rows)
    tab[:, 0] -= tab[0, 0]
    return tab[:, 0].copy(), tab[:, 1].copy(), tab[:, 2].copy(), tab[:, 3].copy()


def read_rfcoef(path):
    """rfdataN.in as Fourier coefficients, read3_Data
    (src/DataStruct/Data.f90:348-408) for SolRF and TWS, and for every RF
    cavity under the Lorentz integrator: the first value of each line, a
    zero appended to make the count odd."""
    vals = []
    with open(path) as f:
        for ln in f:
            v = _values(ln)
            if v:
                vals.append(float(v[0]))
    if len(vals) % 2 == 0:
        vals.append(0.0)
    return np.array(vals)


_CPLX = None


def _fortran_tokens(line):
    """List-directed values of one line: "(re,im)" complex constants and
    plain numbers (Fortran d exponents allowed)."""
    import re
    global _CPLX
    if _CPLX is None:
        _CPLX = re.compile(r"\(\s*([^,()\s]+)\s*,\s*([^,()\s]+)\s*\)|([^\s,()]+)")
    out = []
    for m in _CPLX.finditer(line.replace("d", "e").replace("D", "e")):
        if m.group(1) is not None:
            out.append(complex(float(m.group(1)), float(m.group(2))))
        else:
            try:
                out.append(float(m.group(3)))
            except ValueError:
                break
    return out


def read_emfld(path):
    """rfdataN.in of an EMfld 110 element as read4_Data reads it
    (src/DataStruct/Data.f90:415-554): three records xmin, xmax, NxIntv /
    y / z (the bounds as complex constants, their real parts kept), then
    (Ex, Ey, Ez, Bx, By, Bz) complex per node, x fastest, nodes not given
    left zero.  Returns (header[9], data (nodes, 12) re/im pairs) for
    impz_b200.elem(..., grid=...)."""
    with open(path) as f:
        lines = [ln for ln in f if ln.strip() and not _is_comment(ln)]
    header = []
    for ln in lines[:3]:
        v = _fortran_tokens(ln)
        header += [complex(v[0]).real, complex(v[1]).real, float(complex(v[2]).real)]
    nx, ny, nz = (int(header[k] + 0.1) for k in (2, 5, 8))
    nodes = (nx + 1) * (ny + 1) * (nz + 1)
    data = np.zeros((nodes, 12))
    n = 0
    for ln in lines[3:]:
        v = _fortran_tokens(ln)
        if len(v) < 6 or n >= nodes:
            break
        for c in range(6):
            z = complex(v[c])
            data[n, 2 * c] = z.real
            data[n, 2 * c + 1] = z.imag
        n += 1
    return np.array(header), data


def write_emfld(path, header, data):
    """Writes an EMfld map in read4_Data's format (read_emfld's inverse)."""
    data = np.asarray(data, dtype=float).reshape(-1, 12)
    with open(path, "w") as f:
        for k in range(3):
            lo, hi, nint = header[3 * k], header[3 * k + 1], int(header[3 * k + 2] + 0.1)
            f.write("(%.17g,0.0) (%.17g,0.0) %d\n" % (lo, hi, nint))
        for row in data:
            f.write(" ".join("(%.17g,%.17g)" % (row[2 * c], row[2 * c + 1]) for c in range(6))
                    + "\n")


def read_wake(path):
    """rfdataN.in as a wake table, read1wk_Data (src/DataStruct/Data.f90:
    559-633): rows (z, longitudinal, x, y wake); z is shifted to start at 0
    by the bunch's wake call, as the reference does after reading."""
    rows = []
    with open(path) as f:
        for ln in f:
            v = _values(ln)
            if len(v) >= 4:
                rows.append([float(x) for x in v[:4]])
    return np.array(rows)


def _records(f):
    """Fortran unformatted sequential records as gfortran writes them: a
    4-byte little-endian length before and after each record."""
    while True:
        head = f.read(4)
        if not head:
            return
        n = int(np.frombuffer(head, "<i4")[0])
        body = f.read(n)
        tail = int(np.frombuffer(f.read(4), "<i4")[0])
        if tail != n or len(body) != n:
            raise ValueError("not a Fortran unformatted sequential file")
        yield body


def write_checkpoint(path, z, inb, jstp, ibal, nstep, msize, rng, grid, refptcl, pts):
    """The -7 checkpoint of one rank, outpoint_Output
    (src/Contrl/Output.f90:1733-1774): z; element index, segment, balance
    and step counters; mesh size; range; the local mesh table (Nz, Ny) and
    range table (zmin, zmax, ymin, ymax) of the single rank; Nptlocal;
    refptcl; Pts1(9, Nptlocal)."""
    pts = np.ascontiguousarray(pts, dtype="<f8")
    rng = np.asarray(rng, dtype="<f8")
    recs = [np.array([z], "<f8"), np.array([inb, jstp, ibal, nstep], "<i4"),
            np.asarray(msize, "<f8"), rng, np.array([grid[2], grid[1]], "<i4"),
            np.array([rng[4], rng[5], rng[2], rng[3]], "<f8"), np.array([pts.shape[0]], "<i4"),
            np.asarray(refptcl, "<f8"), pts]
    with open(path, "wb") as f:
        for r in recs:
            b = r.tobytes()
            n = np.array([len(b)], "<i4").tobytes()
            f.write(n + b + n)


def read_checkpoint(path):
    """A -7 checkpoint back (inpoint_Output, src/Contrl/Output.f90:
    1371-1437, one rank)."""
    with open(path, "rb") as f:
        r = list(_records(f))
    if len(r) != 9:
        raise ValueError("%s: %d records, a one-rank checkpoint has 9" % (path, len(r)))
    n = int(np.frombuffer(r[6], "<i4")[0])
    inb, jstp, ibal, nstep = (int(v) for v in np.frombuffer(r[1], "<i4"))
    return {"z": float(np.frombuffer(r[0], "<f8")[0]), "inb": inb, "jstp": jstp, "ibal": ibal,
            "nstep": nstep, "msize": np.frombuffer(r[2], "<f8").copy(),
            "range": np.frombuffer(r[3], "<f8").copy(),
            "refptcl": np.frombuffer(r[7], "<f8").copy(),
            "pts": np.frombuffer(r[8], "<f8").reshape(n, 9).copy()}


def slice_output(pts, npt, nslice, qchg, pmass, alphax0, betax0, alphay0, betay0, gam0, scxl):
    """The slice table of a type -8 element, sliceprocdep_Output
    (src/Contrl/Output.f90:3002-3215), for one rank: Pts1 (z frame) cut into
    nslice linearly weighted slices in phase over the bunch (its extent
    widened by 0.5e-5 at each end); per slice the columns -z [m], weight,
    current [A], rms emittances x, y [m rad], -<pt>/gamma0, uncorrelated
    energy spread [eV], centroids x, y [m] and the mismatch factors against
    (alpha0, beta0).  The reference's quirks are kept: its speed of light
    2.99792e8 in the current and the uncentred <x px> in alpha."""
    pts = np.asarray(pts, dtype=np.float64)
    f32 = lambda v: float(np.float32(v))  # noqa: E731
    clite = 2.99792e8
    sclcur = clite * qchg / npt
    with np.errstate(divide="ignore", invalid="ignore"):  # a zero beta0 gives inf, as there
        gamx0 = np.float64(1.0 + alphax0 ** 2) / np.float64(betax0)
        gamy0 = np.float64(1.0 + alphay0 ** 2) / np.float64(betay0)
    z = pts[:, 4]
    zmn, zmx = z.min(), z.max()
    zmin = zmn - (zmx - zmn) * f32(0.5e-5)
    zmax = zmx + (zmx - zmn) * f32(0.5e-5)
    hz = (zmax - zmin) / (nslice - 1)
    iz = np.trunc((z - zmin) / hz + 1).astype(np.int64)
    iz = np.where(iz < 1, 1, iz)
    iz = np.where(iz >= nslice, nslice - 1, iz)
    ab = ((zmin - z) + iz * hz) / hz
    # contributions in the reference's order: particle by particle, iz then iz+1
    idx = np.stack([iz - 1, iz], axis=1).ravel()
    wts = np.stack([ab, 1.0 - ab], axis=1).ravel()

    def acc(v):
        return np.bincount(idx, weights=np.repeat(v, 2) * wts, minlength=nslice)

    x, px, y, py, pt = pts[:, 0], pts[:, 1], pts[:, 2], pts[:, 3], pts[:, 5]
    count = np.bincount(idx, weights=wts, minlength=nslice)
    sums = [acc(v) for v in (x, x ** 2, px, px ** 2, x * px, y, y ** 2, py, py ** 2, y * py, pt)]
    with np.errstate(invalid="ignore", divide="ignore"):
        have = count > 0
        xx, xx2, pxm, px2, xpx, yy, yy2, pym, py2, ypy, gam = (
            np.where(have, sm / np.where(have, count, 1.0), 0.0) for sm in sums)
        epx = np.sqrt((xx2 - xx ** 2) * (px2 - pxm ** 2) - (xpx - xx * pxm) ** 2)
        epy = np.sqrt((yy2 - yy ** 2) * (py2 - pym ** 2) - (ypy - yy * pym) ** 2)
        alphax = -xpx / epx
        gambet = np.sqrt((gam0 - gam) ** 2 - 1.0)
        betax = (xx2 - xx ** 2) * gambet / epx
        gamx = (1.0 + alphax ** 2) / betax
        bmx = betax * gamx0 - 2 * alphax * alphax0 + gamx * betax0
        alphay = -ypy / epy
        betay = (yy2 - yy ** 2) * gambet / epy
        gamy = (1.0 + alphay ** 2) / betay
        bmy = betay * gamy0 - 2 * alphay * alphay0 + gamy * betay0
        epx, epy = np.where(have, epx, 0.0), np.where(have, epy, 0.0)
        bmx, bmy = np.where(have, bmx, 0.0), np.where(have, bmy, 0.0)
        gammaz = gam[iz - 1] * ab + gam[iz] * (1.0 - ab)
        dg2 = (-(pt - gammaz)) ** 2
        unc = np.sqrt(np.bincount(idx, weights=np.repeat(dg2, 2) * wts, minlength=nslice) / count)
        zz = zmin + np.arange(nslice) * hz
        return np.c_[-zz * scxl, count, count / (hz * scxl) * sclcur, epx * scxl, epy * scxl,
                     -gam / gam0, unc * pmass, xx * scxl, yy * scxl, bmx, bmy]


def slice_params(e):
    """nslice and the matching Twiss values of a -8 element
    (AccSimulator.f90:908-922), beta_y0's default as written there (it tests
    beta_x0 a second time, so a zero beta_y0 stays zero)."""
    nslice = int(e.vals[0] + 0.1)
    alphax0, betax0, alphay0, betay0 = e.vals[1], e.vals[2], e.vals[3], e.vals[4]
    if betax0 == 0.0:
        betax0 = 1.0
    if betax0 == 0.0:
        betay0 = 1.0
    return nslice, alphax0, betax0, alphay0, betay0


def write_slices(path, rows):
    """Appends a slice table (the reference writes to a unit it keeps open,
    so repeated -8 elements of one file number accumulate)."""
    with open(path, "a") as f:
        for r in rows:
            f.write(" ".join("%.17g" % v for v in r) + "\n")


def checkpoint_file(deck):
    """nfileout: the file number of the deck's last -7 element, which a
    restart reads (Input.f90:260, AccSimulator.f90:558-561)."""
    n = None
    for e in deck.elements:
        if e.type == -7:
            n = e.mapstp
    return n


# the 45 columns of impz_diag_row: z, then the files' columns in order
_FILES = (("fort.18", 1, 6), ("fort.24", 6, 12), ("fort.25", 12, 18), ("fort.26", 18, 24),
          ("fort.27", 24, 30), ("fort.28", 30, 33), ("fort.29", 33, 39), ("fort.30", 39, 45))


def write_diag(outdir, rows, charge_states=None):
    """fort.18 and fort.24-30 (diagnostic1_Output) from diag rows, and with
    `charge_states` (records x nchrg particle counts) fort.32: z and the
    count of each charge state (Output.f90:352)."""
    rows = np.asarray(rows)
    for name, a, b in _FILES:
        with open(os.path.join(outdir, name), "w") as f:
            for r in rows:
                if name == "fort.28":
                    f.write("%.17g %10d %10d %10d\n" % (r[0], int(r[30]), int(r[31]), int(r[32])))
                else:
                    f.write(" ".join("%.17g" % x for x in [r[0]] + list(r[a:b])) + "\n")
    if charge_states is not None:
        with open(os.path.join(outdir, "fort.32"), "w") as f:
            for r, c in zip(rows, np.asarray(charge_states)):
                f.write("%.17g " % r[0] + " ".join("%d" % int(x) for x in c) + "\n")


def charge_state_counts(species_qm, species_counts, qmcclist):
    """chgupdate_BeamBunch's counts (BeamBunch.f90:700-708): for each entry
    j of qmcclist, the particles of the species whose q/m lies within
    relative 1e-4 (a default-real literal) of it.  species_counts has one
    row per record and one column per species."""
    eps = float(np.float32(1.0e-4))
    qm = np.asarray(species_qm, dtype=np.float64)
    cnt = np.asarray(species_counts)
    out = np.zeros((cnt.shape[0], len(qmcclist)), dtype=np.int64)
    for j, q in enumerate(qmcclist):
        sel = np.abs((qm - q) / q) < eps
        out[:, j] = cnt[:, sel].sum(axis=1)
    return out


def read_diag(outdir, name):
    """One fort.* file back as an array of floats."""
    with open(os.path.join(outdir, name)) as f:
        return np.array([[float(x) for x in ln.split()] for ln in f if ln.strip()])


def lattice_segments(deck, workdir, skip=(), start=0):
    """The lattice cut at its control elements, for a runner: yields
    ("run", [impz_elem_t]) for each stretch of beam-line elements (RF tables
    read from workdir), ("dump", Element) for each type -2 phase dump,
    ("wake", {"on", "table", "scale", "transverse"}) for each type -41
    read-in wake control, ("checkpoint", {"element", "inb", "jstp", "nstep"})
    for each type -7 checkpoint, ("laser", {"rsig", "wavelength", "ez"}) for
    each type -52 laser heater, ("slices", Element) for each type -8 slice
    output, ("integrator", Flagmap) for each type -25 switch, and last ("skipped", [types]) for the
    control elements passed over because they are in `skip`.  -99 ends the
    lattice; any other control element is refused (ValueError).  `start`
    skips the first elements (a restart continues after element iend).

    A -41 element (src/Contrl/AccSimulator.f90:959-978) reads the table
    rfdata<Param(3)>.in when Param(3) > 0, turns the wake on with scale
    Param(2) when Param(4) > 0 and off otherwise; a Param(4) below 10 drops
    the transverse wake for the rest of the run (flagbtw = 2 is never
    reset)."""
    from . import elem

    flagmap = deck.flagmap

    def to_elem(e):
        # the RF data (AccSimulator.f90:820-848): under the map integrator
        # read1_Data's table, Fourier coefficients (read3_Data) for SolRF and
        # TWS; under the Lorentz integrator Fourier coefficients for all
        rf = None
        if e.type in (105, 106) and e.vals[3] >= 0.0:
            rf = read_rfcoef(os.path.join(workdir, "rfdata%d.in" % int(e.vals[3] + 0.1)))
        elif 101 <= e.type <= 104 and e.vals[3] >= 0.0 and flagmap == 2:
            rf = read_rfcoef(os.path.join(workdir, "rfdata%d.in" % int(e.vals[3] + 0.1)))
        elif 101 <= e.type <= 104 and e.vals[3] >= 0.0:
            rf = read_rfdata(os.path.join(workdir, "rfdata%d.in" % int(e.vals[3])))
        elif e.type == 1 and e.vals[1] > 1.0e-5:
            # a quadrupole's gradient profile (AccSimulator.f90:853-863)
            rf = read_rfdata(os.path.join(workdir, "rfdata%d.in" % int(e.vals[1] + 0.1)))
        elif e.type == 110 and flagmap == 2 and e.vals[3] >= 0.0:
            # EMfld's x-y-z map (read4_Data, AccSimulator.f90:841-842)
            grid = read_emfld(os.path.join(workdir, "rfdata%d.in" % int(e.vals[3] + 0.1)))
            return elem(e.type, e.length, e.nseg, e.mapstp, list(e.vals), grid=grid)
        return elem(e.type, e.length, e.nseg, e.mapstp, list(e.vals), rf=rf)

    seg, skipped = [], []
    table, no_transverse = None, False
    nstep, jlast = 0, 0
    for i, e in enumerate(deck.elements):
        if i < start:
            continue
        if e.type >= 0:
            seg.append(to_elem(e))
            nstep += e.nseg
            jlast = e.nseg + 1
            continue
        if seg:
            yield "run", seg
            seg = []
        if e.type == -99:
            break
        if e.type == -2:
            yield "dump", e
        elif e.type in skip:
            skipped.append(e.type)
        elif e.type == -8:
            yield "slices", e
        elif e.type == -25:
            # switch integrator: Flagmap = bmpstp (AccSimulator.f90:806-809)
            flagmap = e.mapstp
            yield "integrator", e.mapstp
        elif e.type == -52:
            # laser heater (AccSimulator.f90:982-1006): Param(2..4)
            yield "laser", {"rsig": e.vals[0], "wavelength": e.vals[1], "ez": e.vals[2]}
        elif e.type == -7:
            # outpoint_Output's counters: the element (1-based), the segment
            # loop index the previous element left, the steps so far
            yield "checkpoint", {"element": e, "inb": i + 1, "jstp": jlast, "nstep": nstep}
        elif e.type == -41:
            scale, rfile, onoff = e.vals[0], e.vals[1], e.vals[2]
            if rfile > 0.0:
                table = read_wake(os.path.join(workdir, "rfdata%d.in" % int(rfile + 0.1)))
            if onoff > 0.0:
                if table is None:
                    raise ValueError("a -41 element turns the wake on before any table is read")
                no_transverse = no_transverse or onoff < 10.0
                yield "wake", {"on": True, "table": table, "scale": scale,
                               "transverse": not no_transverse}
            else:
                yield "wake", {"on": False}
        else:
            raise ValueError("control element type %d is outside this path" % e.type)
    if seg:
        yield "run", seg
    yield "skipped", skipped


def check_supported(deck):
    """The runner covers open boundaries and a particle.in distribution
    (any number of charge states, rows 7 and 8 per particle), with the map
    integrator (Flagmap=1) or the Lorentz integrator (Flagmap=2)."""
    if deck.flagmap not in (1, 2) or deck.flagbc != 1 or deck.flagdist != 19:
        raise ValueError("this runner needs Flagmap=1 or 2, Flagbc=1 and Flagdist=19 (deck has "
                         "%d, %d, %d)" % (deck.flagmap, deck.flagbc, deck.flagdist))


def run_deck(workdir, outdir=None, form=None, skip=(), write=True):
    """Runs ImpactZ.in + particle.in of `workdir` on the GPU and writes
    fort.18/24-30, fort.32 and the -2 phase dumps into `outdir` (default:
    workdir).  A particle.in whose rows 7 and 8 differ between particles
    (multiple charge states) runs as a multi-species bunch.  Returns {"rows":
    diag rows, "charge_states": fort.32's counts, "skipped": [types passed
    over], "pts": final Pts1}."""
    from . import FORM_FP64, Bunch, diag_row
    from .beams import scxl
    outdir = outdir or workdir
    deck = read_deck(os.path.join(workdir, "ImpactZ.in"))
    check_supported(deck)
    start, z0, ref = 0, 0.0, deck.refptcl()
    if deck.restart == 1:
        # Rstartflg = 1: continue from the last -7 checkpoint
        ck = read_checkpoint(os.path.join(workdir, "fort.%d" % checkpoint_file(deck)))
        pts, ref, z0, start = ck["pts"], ck["refptcl"], ck["z"], ck["inb"]
    else:
        pts = read_particles(os.path.join(workdir, "particle.in"))
    multi = bool(np.any(pts[:, 6] != pts[0, 6]) or np.any(pts[:, 7] != pts[0, 7]))
    b = Bunch(pts, deck.bcurr, deck.bmass, deck.bcharge, deck.bfreq, ref,
              (deck.nx, deck.ny, deck.nz), form=FORM_FP64 if form is None else form,
              track_ids=True, species=multi)
    b.set_z(z0)
    b.set_integrator(deck.flagmap)
    rows, skipped, charges = [], [], []
    qmcc = list(deck.qmcclist) or [float(pts[0, 6])]
    # nptlist of the deck until the first space-charge step's chgupdate
    # (AccSimulator.f90:155-161, 1130); every step of a run with current has one
    npl0 = list(deck.nptlist)[: len(qmcc)] + [0] * max(0, len(qmcc) - len(deck.nptlist))
    sc = deck.bcurr >= 1.0e-10
    try:
        for kind, item in lattice_segments(deck, workdir, set(skip), start):
            if kind == "skipped":
                skipped = item
            elif kind == "wake":
                if item["on"]:
                    b.wake(item["table"], item["scale"], item["transverse"])
                else:
                    b.wake_off()
            elif kind == "laser":
                b.laser_heater(item["rsig"], item["wavelength"], item["ez"])
            elif kind == "integrator":
                b.set_integrator(item)
            elif kind == "slices":
                if write:
                    info = b.info()
                    nslice, ax, bx, ay, by = slice_params(item)
                    rows_s = slice_output(b.download(), info["npt"], nslice,
                                          info["current"] / deck.bfreq, deck.bmass, ax, bx, ay,
                                          by, -info["refptcl"][5], scxl(deck.bfreq))
                    write_slices(os.path.join(outdir, "fort.%d" % item.mapstp), rows_s)
            elif kind == "checkpoint":
                if write:
                    rng, ms = b.geom()
                    info = b.info()
                    write_checkpoint(os.path.join(outdir, "fort.%d" % item["element"].mapstp),
                                     info["z"], item["inb"], item["jstp"], item["nstep"],
                                     item["nstep"], ms, rng, (deck.nx, deck.ny, deck.nz),
                                     info["refptcl"], b.download())
            elif kind == "dump":
                if write:
                    write_phase(os.path.join(outdir, "fort.%d" % item.mapstp), b.download(),
                                max(1, int(item.vals[0])))
            else:
                recs, zs = b.run(item)
                refs = b.run_reference()
                seg = [diag_row(zs[i], recs[i], refs[i], deck.bmass, deck.bfreq)
                       for i in range(len(recs))]
                if multi:
                    per = b.run_species()
                else:  # one species: every live particle
                    per = np.array([[int(r[32])] for r in seg])
                cs = charge_state_counts(b.species()[0], per, qmcc)
                if not sc:
                    cs[:] = npl0
                if not rows:
                    cs[0] = npl0
                # a stretch's first record repeats the previous stretch's last
                rows += seg[1:] if rows else seg
                charges += list(cs[1:] if charges else cs)
        final = b.download()
    finally:
        b.close()
    rows = np.array(rows)
    charges = np.array(charges)
    if write:
        write_diag(outdir, rows, charges if len(charges) else None)
    return {"rows": rows, "charge_states": charges, "skipped": skipped, "pts": final}
