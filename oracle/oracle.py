"""ctypes bindings of the CPU oracle (oracle/impz_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() as
the checker, and by bench.py's CPU-baseline leg.  The product never imports
it.  PARITY UNPINNED: the oracle restates the reference's Fortran (no
Fortran compiler or golden output exists to run it against); it is pinned by
known-answer tests in tests/test_oracle_kat.py.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle_impz.so")
DIAG_LEN = 45
RAW_LEN = 44

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)
_LL = ctypes.POINTER(ctypes.c_longlong)


class OrcElem(ctypes.Structure):
    _fields_ = [
        ("type", ctypes.c_int),
        ("nseg", ctypes.c_int),
        ("mapstp", ctypes.c_int),
        ("length", ctypes.c_double),
        ("val", ctypes.c_double * 24),
        ("ndata", ctypes.c_int),
        ("zdat", _D), ("edat", _D), ("epdat", _D), ("eppdat", _D),
    ]


class OrcBeam(ctypes.Structure):
    _fields_ = [
        ("current", ctypes.c_double), ("mass", ctypes.c_double), ("charge", ctypes.c_double),
        ("freq", ctypes.c_double), ("npt", ctypes.c_int), ("nlocal", ctypes.c_int),
        ("pts", _D), ("refptcl", ctypes.c_double * 6), ("z", ctypes.c_double),
        ("zbleng", ctypes.c_double), ("sentr", ctypes.c_double),
        ("bendlencsr", ctypes.c_double), ("r0", ctypes.c_double),
        ("flagbendcsr", ctypes.c_int),
        ("flagmap", ctypes.c_int),
    ]

CSR_FIELDS = ("zbleng", "sentr", "bendlencsr", "r0", "flagbendcsr")


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-s", "-C", HERE], check=True)
        L = ctypes.CDLL(LIB_PATH)
        v = None
        sig = {
            "orc_physconst": (v, [ctypes.c_double]),
            "orc_get_physconst": (v, [_D]),
            "orc_set_threads": (v, [ctypes.c_int]),
            "orc_set_field_probe": (v, [_D, _D, ctypes.c_int]),
            "orc_set_charge_states": (v, [_D, ctypes.c_int, _I, _I, ctypes.c_int]),
            "orc_drift_exact": (v, [_D, ctypes.c_int, _D, ctypes.c_double]),
            "orc_maplinear_quad": (v, [ctypes.c_double, ctypes.c_double, _D, _D, ctypes.c_double,
                                       ctypes.c_int, ctypes.c_double, ctypes.c_double]),
            "orc_maplinear_ccl": (v, [ctypes.c_double, ctypes.c_double, _D, _D, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_int, _D, _D, _D, _D]),
            "orc_maplinear_dtl": (v, [ctypes.c_double, ctypes.c_double, _D, _D, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_int, _D, _D, _D, _D, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_double]),
            "orc_maplinear_solrf": (v, [ctypes.c_double, ctypes.c_double, _D, _D,
                                        ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                        ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_int, _D]),
            "orc_maplinear_tws": (v, [ctypes.c_double, ctypes.c_double, _D, _D,
                                      ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_int, _D]),
            "orc_maplinear_quad_fringe": (v, [ctypes.c_double, ctypes.c_double, _D, _D,
                                              ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                              ctypes.c_double, ctypes.c_int, _D, _D]),
            "orc_undulator": (v, [ctypes.c_double, ctypes.c_double, _D, _D, ctypes.c_int]),
            "orc_maplinear_sol": (v, [ctypes.c_double, ctypes.c_double, _D, _D,
                                      ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                      ctypes.c_double]),
            "orc_maplinear_constfoc": (v, [ctypes.c_double, ctypes.c_double, _D, _D, _D,
                                           ctypes.c_int]),
            "orc_apply_xm": (v, [_D, ctypes.c_int, _D]),
            "orc_transfmapK": (v, [ctypes.c_double, ctypes.c_double, _D, _D, ctypes.c_int,
                                   ctypes.c_double]),
            "orc_conv1st": (ctypes.c_int, [_D, ctypes.c_int, _D, _I, _D, ctypes.c_double,
                                           ctypes.c_double, _D]),
            "orc_update_compdom": (v, [_D, _I, _D, _D]),
            "orc_deposit": (v, [_D, ctypes.c_int, _I, _D, _D, _D, _I, _LL]),
            "orc_igf": (v, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                            ctypes.c_double, ctypes.c_double, _D]),
            "orc_poisson_open": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                ctypes.c_double, ctypes.c_double,
                                                ctypes.c_double, _D]),
            "orc_poisson_direct": (v, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                       ctypes.c_double, ctypes.c_double, _D, _D]),
            "orc_cvbkforth1st": (v, [_D, ctypes.c_int, _D]),
            "orc_kick1": (v, [_D, ctypes.c_int, _D, _I, _D, _D, ctypes.c_double, ctypes.c_double,
                              ctypes.c_double, ctypes.c_double, ctypes.c_double, _D]),
            "orc_kick1w": (v, [_D, ctypes.c_int, _D, _I, _D, _D, ctypes.c_double,
                               ctypes.c_double, ctypes.c_double, ctypes.c_double,
                               ctypes.c_double, _D, _D]),
            "orc_wake_set": (ctypes.c_int, [_D, _D, _D, _D, ctypes.c_int, ctypes.c_double,
                                            ctypes.c_int]),
            "orc_wake_off": (v, []),
            "orc_wake_elem": (v, [ctypes.c_int, _D]),
            "orc_wake_field_analytic": (v, [ctypes.c_int, _D, _D, _D, _D, ctypes.c_double,
                                            ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                            ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                            ctypes.c_double, _D]),
            "orc_wake_line": (v, [_D, ctypes.c_int, ctypes.c_int, _D, _D, _D, _D]),
            "orc_wake_field": (v, [ctypes.c_int, _D, _D, _D, _D, ctypes.c_double,
                                   ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                   ctypes.c_double, _D]),
            "orc_csr_wake": (v, [ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                 ctypes.c_double, ctypes.c_double, _D, ctypes.c_double, _D]),
            "orc_csr_field": (v, [ctypes.c_int, _D, _D, ctypes.c_double, ctypes.c_double,
                                  ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                  ctypes.c_double, ctypes.c_double, ctypes.c_double, _D]),
            "orc_laser_heater": (v, [_D, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                     ctypes.c_double, ctypes.c_double, ctypes.c_double]),
            "orc_moment_sums": (v, [_D, ctypes.c_int, _D]),
            "orc_diag_row": (v, [ctypes.c_double, _D, ctypes.c_int, ctypes.c_int, _D,
                                 ctypes.c_double, _D]),
            "orc_run": (ctypes.c_int, [ctypes.POINTER(OrcElem), ctypes.c_int,
                                       ctypes.POINTER(OrcBeam), _I, _D, ctypes.c_int]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def dp(a):
    return a.ctypes.data_as(_D) if a is not None else None


def physconst(freq):
    lib().orc_physconst(freq)
    out = np.zeros(5)
    lib().orc_get_physconst(dp(out))
    return dict(Pi=out[0], Clight=out[1], Scxl=out[2], Rad2deg=out[3], Scfreq=out[4])


def wake_set(table, scale=1.0, transverse=False):
    """Turns the read-in wake on (a type -41 element with Param(4) > 0):
    table rows (z, Ez wake, x wake, y wake) as in rfdataN.in."""
    t = np.ascontiguousarray(np.asarray(table, dtype=np.float64).T)
    r = lib().orc_wake_set(dp(t[0]), dp(t[1]), dp(t[2]), dp(t[3]), t.shape[1], float(scale),
                           int(bool(transverse)))
    if r:
        raise ValueError("orc_wake_set: %d" % r)


def wake_off():
    lib().orc_wake_off()


def set_threads(n):
    lib().orc_set_threads(int(n))


def elem_from(e):
    """Converts an impz_b200 ElemStruct (or any object with the same fields)."""
    o = OrcElem()
    o.type, o.nseg, o.mapstp, o.length = e.type, e.nseg, e.mapstp, e.length
    for i in range(24):
        o.val[i] = e.val[i]
    o.ndata = getattr(e, "ndata", 0)
    if o.ndata:
        o.zdat, o.edat, o.epdat, o.eppdat = e.zdat, e.edat, e.epdat, e.eppdat
    return o


def run(elems, pts, current, mass, charge, freq, refptcl, grid, z=0.0, state=None, flagmap=1,
        probe=None, charge_states=None):
    """orc_run over a lattice: returns (rows, final pts, final beam).  `state`
    (a beam returned by an earlier call) carries the CSR bend bookkeeping
    across calls, as one element loop of the reference would.  `probe` =
    (phi, eg) float64 arrays of shape (S, G) and (S, 3G) (either may be None)
    receive the potential and kick1's field of the first S space-charge
    steps of the map integrator.  `charge_states` = (qmcclist, nptlist,
    out): chgupdate's counts per charge state (nptlist, int32, updated in
    place) copied to out[r] (int32, shape (records, nchrg)) at every record."""
    physconst(freq)
    if probe is not None:
        phi, eg = probe
        steps = (phi if phi is not None else eg).shape[0]
        lib().orc_set_field_probe(dp(phi), dp(eg), steps)
    if charge_states is not None:
        qmc, npl, cs_out = charge_states
        qmc = np.ascontiguousarray(qmc, dtype=np.float64)
        assert npl.dtype == np.int32 and cs_out.dtype == np.int32 and cs_out.flags.c_contiguous
        lib().orc_set_charge_states(dp(qmc), len(qmc), npl.ctypes.data_as(_I),
                                    cs_out.ctypes.data_as(_I), cs_out.shape[0])
    arr = (OrcElem * len(elems))(*[elem_from(e) for e in elems])
    keep = [getattr(e, "_keep", None) for e in elems]
    p = np.ascontiguousarray(pts, dtype=np.float64).copy()
    beam = OrcBeam()
    beam.current, beam.mass, beam.charge, beam.freq = current, mass, charge, freq
    beam.npt = beam.nlocal = p.shape[0]
    beam.pts = dp(p)
    for i in range(6):
        beam.refptcl[i] = refptcl[i]
    beam.z = z
    beam.flagmap = int(flagmap)
    if state is not None:
        for f in CSR_FIELDS:
            setattr(beam, f, getattr(state, f))
    mesh = np.array(grid, dtype=np.int32)
    nsteps = sum(e.nseg for e in elems)
    rows = np.zeros((nsteps + 1, DIAG_LEN))
    try:
        n = lib().orc_run(arr, len(elems), ctypes.byref(beam), mesh.ctypes.data_as(_I), dp(rows),
                          nsteps + 1)
    finally:
        if probe is not None:
            lib().orc_set_field_probe(None, None, 0)
        if charge_states is not None:
            lib().orc_set_charge_states(None, 0, None, None, 0)
    del keep
    if n < 0:
        raise RuntimeError("orc_run failed: %d" % n)
    return rows[:n], p[: beam.nlocal].copy(), beam
