"""B200-native IMPACT-Z space-charge kick and element push: Python bindings.

The product is the C-ABI library ``libimpz_b200.so`` (include/impz_b200.h);
this module binds it with ctypes, mirroring the reference's call surface
(BeamBunch / CompDom / FieldQuant, src/Appl/BeamBunch.f90, CompDom.f90,
Field.f90) so that tests and the benchmark read like the reference's own
step loop.  There is no CPU fallback: every compute entry point runs the CUDA
kernels and raises ImpzError if the library or a GPU is missing.

The package directory is named ``impact-z_b200``; load it under the import
name ``impz_b200`` with :func:`load_package` helpers in the callers.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libimpz_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "impz_b200.h")

OK = 0
ERR_ARG, ERR_NOMEM, ERR_CUDA, ERR_UNSUPPORTED = -1, -2, -3, -4
ERR_NONUNIFORM, ERR_STATE, ERR_NONFINITE, ERR_NODEVICE, ERR_BUDGET = -5, -6, -7, -8, -9
ERR_LIMIT = -10
STATIC_MAX_CELLS = 1 << 19
FORM_FP64 = 0
FORM_FP32CONV = 1
FLAG_TRACK_IDS = 1
FLAG_SPECIES = 2
RAW_LEN = 44
DIAG_LEN = 45
MOMREC = 48


class ImpzError(RuntimeError):
    def __init__(self, code, what=""):
        self.code = code
        msg = "%s failed: %s (%d)" % (what, error_string(code), code)
        if code == ERR_CUDA:
            msg += ": " + last_cuda_error()
        super().__init__(msg)


class ElemStruct(ctypes.Structure):
    """impz_elem_t: one ImpactZ.in lattice line (src/Contrl/Input.f90:300-315)."""

    _fields_ = [
        ("type", ctypes.c_int),
        ("nseg", ctypes.c_int),
        ("mapstp", ctypes.c_int),
        ("ndata", ctypes.c_int),
        ("length", ctypes.c_double),
        ("val", ctypes.c_double * 24),
        ("zdat", ctypes.POINTER(ctypes.c_double)),
        ("edat", ctypes.POINTER(ctypes.c_double)),
        ("epdat", ctypes.POINTER(ctypes.c_double)),
        ("eppdat", ctypes.POINTER(ctypes.c_double)),
    ]


_lib = None
_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)
_LL = ctypes.POINTER(ctypes.c_longlong)
_E = ctypes.POINTER(ElemStruct)
_B = ctypes.c_void_p

_SIGS = {
    "impz_version": (ctypes.c_char_p, []),
    "impz_error_string": (ctypes.c_char_p, [ctypes.c_int]),
    "impz_last_cuda_error": (ctypes.c_char_p, []),
    "impz_set_device": (ctypes.c_int, [ctypes.c_int]),
    "impz_bunch_create": (ctypes.c_int, [_D, ctypes.c_longlong, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_double, _D, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                         ctypes.POINTER(_B)]),
    "impz_bunch_download": (ctypes.c_int, [_B, _D, ctypes.c_longlong, _LL]),
    "impz_bunch_destroy": (ctypes.c_int, [_B]),
    "impz_bunch_info": (ctypes.c_int, [_B, _D]),
    "impz_bunch_geom": (ctypes.c_int, [_B, _D, _D]),
    "impz_laser_heater": (ctypes.c_int, [_B, ctypes.c_double, ctypes.c_double, ctypes.c_double]),
    "impz_autotune": (ctypes.c_int, [_B, ctypes.c_int, _D]),
    "impz_step_params_size": (ctypes.c_int, []),
    "impz_set_integrator": (ctypes.c_int, [_B, ctypes.c_int]),
    "impz_bunch_set_z": (ctypes.c_int, [_B, ctypes.c_double]),
    "impz_bunch_stream": (ctypes.c_void_p, [_B]),
    "impz_map_half": (ctypes.c_int, [_B, _E, ctypes.c_double, _D, ctypes.c_double, ctypes.c_int,
                                     _I]),
    "impz_bend_entry": (ctypes.c_int, [_B, _E]),
    "impz_bend_sector": (ctypes.c_int, [_B, _D, ctypes.c_double]),
    "impz_bend_exit": (ctypes.c_int, [_B]),
    "impz_sc_prepare": (ctypes.c_int, [_B, ctypes.c_double, ctypes.c_double, _LL, _D, _D, _D]),
    "impz_deposit": (ctypes.c_int, [_B, _D, _I]),
    "impz_poisson_open": (ctypes.c_int, [_B, _D]),
    "impz_kick": (ctypes.c_int, [_B, ctypes.c_double, _D]),
    "impz_drift2": (ctypes.c_int, [_B, _D, ctypes.c_double]),
    "impz_kick2": (ctypes.c_int, [_B, _E, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                  _D]),
    "impz_moments": (ctypes.c_int, [_B, _D]),
    "impz_diag_row": (ctypes.c_int, [ctypes.c_double, _D, _D, ctypes.c_double, ctypes.c_double,
                                     _D]),
    "impz_run": (ctypes.c_int, [_B, _E, ctypes.c_int, _D, _D, ctypes.c_int, _I]),
    "impz_run_async": (ctypes.c_int, [_B, _E, ctypes.c_int]),
    "impz_run_fetch": (ctypes.c_int, [_B, _D, _D, ctypes.c_int, _I]),
    "impz_count_steps": (ctypes.c_int, [_E, ctypes.c_int]),
    "impz_maplinear": (ctypes.c_int, [_E, ctypes.c_double, ctypes.c_double, ctypes.c_double, _D,
                                      ctypes.c_double, ctypes.c_double, ctypes.c_double, _D]),
    "impz_profile_enable": (ctypes.c_int, [_B, ctypes.c_int]),
    "impz_profile_fetch": (ctypes.c_int, [_B, _D, _LL]),
    "impz_kernel_launches": (ctypes.c_longlong, []),
    "impz_bunch_upload": (ctypes.c_int, [_B, _D, ctypes.c_longlong, ctypes.c_double, _D]),
    "impz_bunching": (ctypes.c_int, [_B, ctypes.c_double, _D]),
    "impz_wake_set": (ctypes.c_int, [_B, _D, ctypes.c_int, ctypes.c_double, ctypes.c_int]),
    "impz_wake_off": (ctypes.c_int, [_B]),
    "impz_run_reference": (ctypes.c_int, [_B, _D, ctypes.c_int, _I]),
    "impz_bunch_species": (ctypes.c_int, [_B, _D, _D, ctypes.c_int]),
    "impz_chgupdate": (ctypes.c_int, [_B, ctypes.c_int, _D, _I]),
    "impz_run_species": (ctypes.c_int, [_B, _I, ctypes.c_int, _I]),
    "impz_run_batch": (ctypes.c_int, [ctypes.POINTER(_B), ctypes.POINTER(_E),
                                      ctypes.POINTER(ctypes.c_int), ctypes.c_int]),
    "impz_run_advance_packed": (ctypes.c_int, [ctypes.POINTER(_B), ctypes.c_int, ctypes.c_int,
                                               ctypes.POINTER(ctypes.c_int)]),
    "impz_run_begin": (ctypes.c_int, [_B, _E, ctypes.c_int]),
    "impz_run_advance": (ctypes.c_int, [_B, ctypes.c_int, _I]),
    "impz_bunch_footprint": (ctypes.c_longlong, [ctypes.c_longlong, ctypes.c_int, ctypes.c_int,
                                                 ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                 ctypes.c_int]),
    "impz_deposit_static": (ctypes.c_int, [ctypes.c_void_p] * 6 + [
        ctypes.c_longlong, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
        ctypes.c_double, _D, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
        ctypes.c_void_p]),
    "impz_server_create": (ctypes.c_int, [ctypes.c_double, ctypes.c_int, ctypes.POINTER(_B)]),
    "impz_server_submit": (ctypes.c_int, [_B, _D, ctypes.c_longlong, ctypes.c_double,
                                          ctypes.c_double, ctypes.c_double, ctypes.c_double, _D,
                                          ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                          _E, ctypes.c_int, _LL]),
    "impz_server_wait": (ctypes.c_int, [_B, ctypes.c_longlong, ctypes.c_double, _D, ctypes.c_int,
                                        _I, _D]),
    "impz_server_stats": (ctypes.c_int, [_B, _D]),
    "impz_server_destroy": (ctypes.c_int, [_B]),
}

PROF_NAMES = ("deposit", "scan", "green", "convolve", "efield", "push", "wake")


def kernel_launches():
    """Process-wide number of kernels the library has launched."""
    return int(lib().impz_kernel_launches())


def lib():
    """The loaded C-ABI library (raises ImpzError/OSError if it is not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError("libimpz_b200.so is not built; run impact-z_b200/build.py")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def declared_symbols():
    """Entry points declared in include/impz_b200.h."""
    import re
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"\b(impz_[a-z0-9_]+)\s*\(", txt)))


def error_string(code):
    return lib().impz_error_string(code).decode()


def last_cuda_error():
    return lib().impz_last_cuda_error().decode()


def _check(rc, what):
    if rc != OK:
        raise ImpzError(rc, what)


def _dp(a):
    return a.ctypes.data_as(_D) if a is not None else None


# ---------------------------------------------------------------------------
def elem(etype, length, nseg, mapstp=1, vals=(), rf=None, grid=None):
    """Build an impz_elem_t.  vals are the deck values v1..v24; rf is an
    optional (z, Ez, Ez', Ez'') on-axis table for linear RF maps, or the
    1-D array of read3_Data's Fourier coefficients for SolRF and TWS (105,
    106) and, under the Lorentz integrator, for types 101..104.  grid is
    EMfld 110's x-y-z field map as read4_Data reads it: (header, data) with
    header = (xmin, xmax, NxIntv, ymin, ymax, NyIntv, zmin, zmax, NzIntv) and
    data the complex (Ex, Ey, Ez, Bx, By, Bz) of every node, x fastest, as an
    array of shape (nodes, 6) complex or (nodes, 12) real (re, im pairs)."""
    e = ElemStruct()
    e.type = int(etype)
    e.nseg = int(nseg)
    e.mapstp = int(mapstp)
    e.length = float(length)
    for i, v in enumerate(vals):
        e.val[i] = float(v)
    e._keep = None
    if rf is not None and np.ndim(rf) == 1:
        coef = np.ascontiguousarray(rf, dtype=np.float64)
        e.ndata = len(coef)
        e.zdat = coef.ctypes.data_as(_D)
        e._keep = [coef]
    elif rf is not None:
        cols = [np.ascontiguousarray(c, dtype=np.float64) for c in rf]
        e.ndata = len(cols[0])
        e.zdat, e.edat, e.epdat, e.eppdat = [c.ctypes.data_as(_D) for c in cols]
        e._keep = cols
    if grid is not None:
        header = np.ascontiguousarray(grid[0], dtype=np.float64)
        data = np.asarray(grid[1])
        if np.iscomplexobj(data):
            data = np.stack([data.real, data.imag], axis=-1).reshape(data.shape[0], 12)
        data = np.ascontiguousarray(data, dtype=np.float64).reshape(-1)
        if header.shape != (9,) or data.size % 12:
            raise ValueError("grid: a 9-value header and 12 values per node")
        e.ndata = data.size // 12
        e.zdat = header.ctypes.data_as(_D)
        e.edat = data.ctypes.data_as(_D)
        e._keep = [header, data]
    return e


def elem_array(elems):
    arr = (ElemStruct * len(elems))()
    keep = []
    for i, e in enumerate(elems):
        arr[i] = e
        keep.append(getattr(e, "_keep", None))
    arr._keep = keep
    return arr


def count_steps(elems):
    arr = elem_array(elems)
    return lib().impz_count_steps(arr, len(elems))


def run_batch(bunches, lattices):
    """Runs every bunch over its own lattice with interleaved steps; returns
    [(records, zs)] in bunch order."""
    nb = len(bunches)
    arrs = [elem_array(l) for l in lattices]
    hs = (_B * nb)(*[b.h for b in bunches])
    ptrs = (_E * nb)(*[ctypes.cast(a, _E) for a in arrs])
    ns = (ctypes.c_int * nb)(*[len(l) for l in lattices])
    for b, l, a in zip(bunches, lattices, arrs):
        b._pending = (a, count_steps(l) + 1)
    _check(lib().impz_run_batch(hs, ptrs, ns, nb), "impz_run_batch")
    return [b.run_fetch() for b in bunches]


def run_packed(bunches, lattices, steps_per_call=8):
    """Runs every bunch over its own lattice (any lengths and grid sizes)
    with impz_run_advance_packed, `steps_per_call` steps per call; returns
    [(records, zs)] in bunch order."""
    arrs = [elem_array(l) for l in lattices]
    for b, l, a in zip(bunches, lattices, arrs):
        _check(lib().impz_run_begin(b.h, a, len(l)), "impz_run_begin")
        b._pending = (a, count_steps(l) + 1)
    left = list(bunches)
    while left:
        hs = (_B * len(left))(*[b.h for b in left])
        rem = (ctypes.c_int * len(left))()
        _check(lib().impz_run_advance_packed(hs, len(left), int(steps_per_call), rem),
               "impz_run_advance_packed")
        left = [b for b, r in zip(left, rem) if r > 0]
    return [b.run_fetch() for b in bunches]


def maplinear(e, zedge, t, tau, refpt, charge, mass, freq):
    ref = np.array(refpt, dtype=np.float64)
    xm = np.zeros(36)
    _check(lib().impz_maplinear(ctypes.byref(e), zedge, t, tau, _dp(ref), charge, mass, freq,
                                _dp(xm)), "impz_maplinear")
    return xm.reshape(6, 6, order="F"), ref


def diag_row(z, rec, refptcl, mass, freq):
    rec = np.ascontiguousarray(rec, dtype=np.float64)
    ref = np.ascontiguousarray(refptcl, dtype=np.float64)
    row = np.zeros(DIAG_LEN)
    _check(lib().impz_diag_row(z, _dp(rec), _dp(ref), mass, freq, _dp(row)), "impz_diag_row")
    return row


class Bunch:
    """A bunch resident on the GPU (BeamBunch + CompDom + FieldQuant of one rank)."""

    def __init__(self, pts, current, mass, charge, freq, refptcl, grid, form=FORM_FP64,
                 track_ids=True, species=False):
        """species=True: Pts1 rows 7 (q/m) and 8 (charge weight) may differ
        between particles (multiple charge states); otherwise they must not."""
        pts = np.ascontiguousarray(pts, dtype=np.float64)
        if pts.ndim != 2 or pts.shape[1] != 9:
            raise ValueError("pts must be (n, 9): Pts1 transposed")
        ref = np.ascontiguousarray(refptcl, dtype=np.float64)
        h = _B()
        nx, ny, nz = grid
        flags = (FLAG_TRACK_IDS if track_ids else 0) | (FLAG_SPECIES if species else 0)
        _check(lib().impz_bunch_create(_dp(pts), pts.shape[0], current, mass, charge, freq,
                                       _dp(ref), nx, ny, nz, form, flags, ctypes.byref(h)),
               "impz_bunch_create")
        self.h = h
        self.n0 = pts.shape[0]
        self.grid = (nx, ny, nz)
        self.mass, self.charge, self.freq, self.form = mass, charge, freq, form

    def close(self):
        if self.h:
            lib().impz_bunch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def stream(self):
        """The bunch's cudaStream_t as an integer handle."""
        return int(lib().impz_bunch_stream(self.h) or 0)

    def upload(self, pts, current, refptcl):
        pts = np.ascontiguousarray(pts, dtype=np.float64)
        ref = np.ascontiguousarray(refptcl, dtype=np.float64)
        _check(lib().impz_bunch_upload(self.h, _dp(pts), pts.shape[0], current, _dp(ref)),
               "impz_bunch_upload")

    def profile_enable(self, on=True):
        _check(lib().impz_profile_enable(self.h, 1 if on else 0), "impz_profile_enable")

    def profile_fetch(self):
        ms = np.zeros(len(PROF_NAMES))
        la = np.zeros(len(PROF_NAMES), dtype=np.int64)
        _check(lib().impz_profile_fetch(self.h, _dp(ms), la.ctypes.data_as(_LL)),
               "impz_profile_fetch")
        return {k: (float(ms[i]), int(la[i])) for i, k in enumerate(PROF_NAMES)}

    def info(self):
        out = np.zeros(11)
        _check(lib().impz_bunch_info(self.h, _dp(out)), "impz_bunch_info")
        return {"current": out[0], "npt": int(out[1]), "nlocal": int(out[2]),
                "refptcl": out[3:9].copy(), "z": out[9], "bytes": int(out[10])}

    def geom(self):
        """(range[6], msize[3]) of the last space-charge step."""
        rng, ms = np.zeros(6), np.zeros(3)
        _check(lib().impz_bunch_geom(self.h, _dp(rng), _dp(ms)), "impz_bunch_geom")
        return rng, ms

    def autotune(self, nsteps=8):
        """Picks deposit and push blocks and the z convolution's lines per
        block by timing this bunch; the bunch is left as it was."""
        out = np.zeros(4)
        _check(lib().impz_autotune(self.h, int(nsteps), _dp(out)), "impz_autotune")
        return {"deposit_blocks": int(out[0]), "push_blocks": int(out[1]),
                "z_lines": int(out[2]), "ms_per_step": float(out[3])}

    def laser_heater(self, rsig, wavelength, ez):
        """The energy kick of a type -52 laser heater element."""
        _check(lib().impz_laser_heater(self.h, float(rsig), float(wavelength), float(ez)),
               "impz_laser_heater")

    def set_integrator(self, flagmap):
        """1: the linear map integrator; 2: the Lorentz integrator."""
        _check(lib().impz_set_integrator(self.h, int(flagmap)), "impz_set_integrator")

    def set_z(self, z):
        _check(lib().impz_bunch_set_z(self.h, float(z)), "impz_bunch_set_z")

    def download(self):
        pts = np.zeros((self.n0, 9))
        n = ctypes.c_longlong()
        _check(lib().impz_bunch_download(self.h, _dp(pts), self.n0, ctypes.byref(n)),
               "impz_bunch_download")
        return pts[: n.value].copy()

    # --- the per-step surface -------------------------------------------
    def map_half(self, e, zedge, z, tau, nst, ihlf):
        zc = ctypes.c_double(z)
        ih = ctypes.c_int(ihlf)
        _check(lib().impz_map_half(self.h, ctypes.byref(e), zedge, ctypes.byref(zc), tau, nst,
                                   ctypes.byref(ih)), "impz_map_half")
        return zc.value, ih.value

    def bend_entry(self, e):
        _check(lib().impz_bend_entry(self.h, ctypes.byref(e)), "impz_bend_entry")

    def bend_sector(self, z, tau):
        zc = ctypes.c_double(z)
        _check(lib().impz_bend_sector(self.h, ctypes.byref(zc), tau), "impz_bend_sector")
        return zc.value

    def bend_exit(self):
        _check(lib().impz_bend_exit(self.h), "impz_bend_exit")

    def sc_prepare(self, piperad, piperad2):
        nptot = ctypes.c_longlong()
        ptrange, rng, msize = np.zeros(6), np.zeros(6), np.zeros(3)
        _check(lib().impz_sc_prepare(self.h, piperad, piperad2, ctypes.byref(nptot), _dp(ptrange),
                                     _dp(rng), _dp(msize)), "impz_sc_prepare")
        return nptot.value, ptrange, rng, msize

    def deposit(self, want_rho=True, want_counts=True):
        G = int(np.prod(self.grid))
        rho = np.zeros(G) if want_rho else None
        cnt = np.zeros(G, dtype=np.int32) if want_counts else None
        _check(lib().impz_deposit(self.h, _dp(rho),
                                  cnt.ctypes.data_as(_I) if cnt is not None else None),
               "impz_deposit")
        return rho, cnt

    def run_reference(self):
        """refptcl at each record of the last run, shape (records, 6)."""
        nrec = ctypes.c_int()
        lib().impz_run_reference(self.h, None, 0, ctypes.byref(nrec))
        out = np.zeros((max(nrec.value, 1), 6))
        _check(lib().impz_run_reference(self.h, _dp(out), nrec.value, ctypes.byref(nrec)),
               "impz_run_reference")
        return out[: nrec.value]

    def species(self):
        """(q/m, weight) arrays of the bunch's species (Pts1 rows 7 and 8), in
        order of first appearance in the uploaded particles."""
        ns = lib().impz_bunch_species(self.h, None, None, 0)
        if ns < 0:
            raise ImpzError(ns, "impz_bunch_species")
        qm, w = np.zeros(ns), np.zeros(ns)
        _check(min(0, lib().impz_bunch_species(self.h, _dp(qm), _dp(w), ns)),
               "impz_bunch_species")
        return qm, w

    def chgupdate(self, qmcclist):
        """chgupdate_BeamBunch: particles per charge state of qmcclist (q/m
        within relative 1e-4) that the latest conv1st kept."""
        q = np.ascontiguousarray(qmcclist, dtype=np.float64)
        out = np.zeros(len(q), dtype=np.int32)
        _check(lib().impz_chgupdate(self.h, len(q), _dp(q), out.ctypes.data_as(_I)),
               "impz_chgupdate")
        return out

    def run_species(self):
        """Per-species particle counts at each record of the last run,
        shape (records, species); multi-species bunches only."""
        ns = len(self.species()[0])
        nrec = ctypes.c_int()
        _check(lib().impz_run_species(self.h, None, 0, ctypes.byref(nrec)), "impz_run_species")
        out = np.zeros((max(nrec.value, 1), ns), dtype=np.int32)
        _check(lib().impz_run_species(self.h, out.ctypes.data_as(_I), nrec.value,
                                      ctypes.byref(nrec)), "impz_run_species")
        return out[: nrec.value]

    def bunching(self, wavenumber):
        """(1/N) sum exp(-i k z) of the live particles (complex); abs() is the
        bunching factor at wavenumber k [1/m]."""
        out = np.zeros(2)
        _check(lib().impz_bunching(self.h, wavenumber, _dp(out)), "impz_bunching")
        return complex(out[0], out[1])

    def wake(self, table, scale=1.0, transverse=False):
        """Read-in wakefield on for the space-charge steps that follow (a
        type -41 element with Param(4) > 0): table rows (z, Ez wake, x wake,
        y wake) as in rfdataN.in, scale = Param(2), transverse False when
        Param(4) < 10."""
        t = np.ascontiguousarray(table, dtype=np.float64)
        if t.ndim != 2 or t.shape[1] != 4:
            raise ValueError("wake table: rows of (z, Ez, Ex, Ey) wake")
        _check(lib().impz_wake_set(self.h, _dp(t), t.shape[0], float(scale),
                                   int(bool(transverse))), "impz_wake_set")

    def wake_off(self):
        _check(lib().impz_wake_off(self.h), "impz_wake_off")

    def poisson(self, want_phi=True):
        phi = np.zeros(int(np.prod(self.grid))) if want_phi else None
        _check(lib().impz_poisson_open(self.h, _dp(phi)), "impz_poisson_open")
        return phi

    def kick(self, tau, want_e=False):
        eg = np.zeros(3 * int(np.prod(self.grid))) if want_e else None
        _check(lib().impz_kick(self.h, tau, _dp(eg)), "impz_kick")
        return eg

    def drift2(self, z, tau):
        """drift2_BeamBunch by tau/2 (the Lorentz integrator's half step);
        returns the new z."""
        zc = ctypes.c_double(z)
        _check(lib().impz_drift2(self.h, ctypes.byref(zc), tau), "impz_drift2")
        return zc.value

    def kick2(self, e, zedge, z, tau, want_e=False):
        """kick2_BeamBunch in element e at z (scatter2 after a solve, or
        scatter20 for a bunch without current)."""
        eg = np.zeros(3 * int(np.prod(self.grid))) if want_e else None
        _check(lib().impz_kick2(self.h, ctypes.byref(e), zedge, z, tau, _dp(eg)), "impz_kick2")
        return eg

    def moments(self):
        rec = np.zeros(MOMREC)
        _check(lib().impz_moments(self.h, _dp(rec)), "impz_moments")
        return rec

    # --- whole lattice ------------------------------------------------------
    def run(self, elems):
        arr = elem_array(elems)
        nrec_cap = count_steps(elems) + 1
        recs = np.zeros((nrec_cap, MOMREC))
        zs = np.zeros(nrec_cap)
        nrec = ctypes.c_int()
        _check(lib().impz_run(self.h, arr, len(elems), _dp(recs), _dp(zs), nrec_cap,
                              ctypes.byref(nrec)), "impz_run")
        return recs[: nrec.value], zs[: nrec.value]

    def run_async(self, elems):
        arr = elem_array(elems)
        self._pending = (arr, count_steps(elems) + 1)
        _check(lib().impz_run_async(self.h, arr, len(elems)), "impz_run_async")

    def run_fetch(self):
        arr, cap = self._pending
        recs = np.zeros((cap, MOMREC))
        zs = np.zeros(cap)
        nrec = ctypes.c_int()
        _check(lib().impz_run_fetch(self.h, _dp(recs), _dp(zs), cap, ctypes.byref(nrec)),
               "impz_run_fetch")
        self._pending = None
        return recs[: nrec.value], zs[: nrec.value]


def footprint(n, grid, form=FORM_FP32CONV, track_ids=False, nsteps=0, species=False):
    """Device bytes of a bunch running nsteps steps (the serving loop admits by it)."""
    nx, ny, nz = grid
    return int(lib().impz_bunch_footprint(n, nx, ny, nz, form,
                                          (FLAG_TRACK_IDS if track_ids else 0)
                                          | (FLAG_SPECIES if species else 0), nsteps))


class Server:
    """The serving loop: submitted jobs share the GPU with continuous batching
    under an HBM budget (impz_server_*)."""

    def __init__(self, budget_bytes=160e9, max_active=64):
        h = _B()
        _check(lib().impz_server_create(budget_bytes, max_active, ctypes.byref(h)),
               "impz_server_create")
        self.h = h
        self._caps = {}

    def submit(self, pts, current, mass, charge, freq, refptcl, grid, lattice,
               form=FORM_FP32CONV):
        pts = np.ascontiguousarray(pts, dtype=np.float64)
        ref = np.ascontiguousarray(refptcl, dtype=np.float64)
        arr = elem_array(lattice)
        job = ctypes.c_longlong()
        nx, ny, nz = grid
        _check(lib().impz_server_submit(self.h, _dp(pts), pts.shape[0], current, mass, charge,
                                        freq, _dp(ref), nx, ny, nz, form, arr, len(lattice),
                                        ctypes.byref(job)), "impz_server_submit")
        self._caps[job.value] = count_steps(lattice) + 1
        return job.value

    def wait(self, job, timeout=-1.0):
        """Returns (records, latency_s, queued_s, measured_bytes) or None if
        the timeout expired."""
        cap = self._caps[job]
        recs = np.zeros((cap, MOMREC))
        nrec = ctypes.c_int()
        times = np.zeros(3)
        rc = lib().impz_server_wait(self.h, job, timeout, _dp(recs), cap, ctypes.byref(nrec),
                                    _dp(times))
        if rc == 1:
            return None
        _check(rc, "impz_server_wait")
        del self._caps[job]
        return recs[: nrec.value], float(times[0]), float(times[1]), int(times[2])

    def stats(self):
        out = np.zeros(8)
        _check(lib().impz_server_stats(self.h, _dp(out)), "impz_server_stats")
        keys = ("completed", "failed", "particle_steps", "span_s", "admitted_bytes",
                "peak_admitted_bytes", "peak_measured_job_bytes", "queued")
        return dict(zip(keys, out.tolist()))

    def close(self):
        if self.h:
            lib().impz_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
