"""Writes tests/golden/step_*.npz: one space-charge step of small seeded
bunches computed by the CPU oracle (oracle/impz_oracle.c).

The reference ships no golden outputs and cannot be compiled here (no
Fortran compiler), so these fixtures pin the oracle's own restatement
against regressions and give the GPU tests fixed vectors to meet.

    python tests/golden/make_golden.py
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
from conftest import load_impz, load_oracle  # noqa: E402

IP = ctypes.POINTER(ctypes.c_int)

CASES = {
    # name: (particles, grid, first element (type, length, nseg, vals), seed offset)
    "step_drift_8x8x16": (2048, (8, 8, 16), (0, 0.1, 4, [1.0]), 1),
    "step_quad_16x16x32": (4096, (16, 16, 32), (1, 0.1, 4, [20.0, 0.0, 1.0]), 2),
}


def oracle_step(orc, pts, cfg, e, tau):
    """half map -> conv1st -> update_CompDom -> deposit -> openBC3D ->
    cvbkforth1st -> kick1 -> half map (AccSimulator.f90:1109-1430)."""
    L = orc.lib()
    orc.physconst(cfg["freq"])
    p = np.ascontiguousarray(pts).copy()
    n = p.shape[0]
    ref = np.array(cfg["refptcl"], dtype=np.float64)
    xm = np.zeros(36)

    def half():
        if e.type == 0:
            L.orc_drift_exact(orc.dp(p), p.shape[0], orc.dp(ref), tau / 2)
        else:
            L.orc_maplinear_quad(0.0, tau / 2, orc.dp(xm), orc.dp(ref), e.val[0], e.mapstp,
                                 cfg["charge"], cfg["mass"])
            L.orc_apply_xm(orc.dp(p), p.shape[0], orc.dp(xm))

    half()
    cur = ctypes.c_double(cfg["current"])
    npt = ctypes.c_int(n)
    ptrange = np.zeros(6)
    nl = L.orc_conv1st(orc.dp(p), n, ctypes.byref(cur), ctypes.byref(npt), orc.dp(ref), 1.0,
                       1.0, orc.dp(ptrange))
    p = p[:nl].copy()
    mesh = np.array(cfg["grid"], dtype=np.int32)
    rng, msize = np.zeros(6), np.zeros(3)
    L.orc_update_compdom(orc.dp(ptrange), mesh.ctypes.data_as(IP), orc.dp(rng), orc.dp(msize))
    G = int(np.prod(cfg["grid"]))
    rho = np.zeros(G)
    counts = np.zeros(G, dtype=np.int32)
    L.orc_deposit(orc.dp(p), nl, mesh.ctypes.data_as(IP), orc.dp(rng), orc.dp(msize),
                  orc.dp(rho), counts.ctypes.data_as(IP), None)
    phi = rho.copy()
    L.orc_poisson_open(int(mesh[0]), int(mesh[1]), int(mesh[2]), msize[0], msize[1], msize[2],
                       orc.dp(phi))
    L.orc_cvbkforth1st(orc.dp(p), nl, orc.dp(ref))
    eg = np.zeros(3 * G)
    L.orc_kick1(orc.dp(p), nl, orc.dp(phi), mesh.ctypes.data_as(IP), orc.dp(rng), orc.dp(msize),
                -ref[5], cur.value, tau, cfg["mass"], cfg["charge"], orc.dp(eg))
    half()
    raw = np.zeros(orc.RAW_LEN)
    L.orc_moment_sums(orc.dp(p), nl, orc.dp(raw))
    return dict(ptrange=ptrange, range=rng, msize=msize, counts=counts, rho=rho, phi=phi, eg=eg,
                pts=p, raw=raw, refptcl=ref, current=np.array([cur.value]))


def build(name):
    impz = load_impz()
    orc = load_oracle()
    from impz_b200 import beams
    n, grid, (etype, length, nseg, vals), seed = CASES[name]
    pts, ref = beams.gaussian_bunch(n, seed=beams.SEED0 + 100 + seed)
    cfg = dict(pts=pts, refptcl=ref, current=0.030, mass=beams.PROTON_MASS_EV, charge=1.0,
               freq=402.5e6, grid=grid)
    e = impz.elem(etype, length, nseg, 1, vals)
    out = oracle_step(orc, pts, cfg, e, length / nseg)
    return pts, ref, cfg, e, out


def main():
    for name in CASES:
        pts, ref, cfg, e, out = build(name)
        # the input bunch is regenerated from its Philox seed by build()
        np.savez_compressed(os.path.join(HERE, name + ".npz"), grid=np.array(cfg["grid"]), **out)
        print(name, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
