"""impz_deposit_static: the charge deposit for callers that may not allocate
device memory.

Host codes that hand out all GPU memory from their own pool, or timed loops
that cannot take the device-wide synchronization of cudaMalloc/cudaFree,
cannot use impz_deposit, whose bunch allocates its grids.  impz_deposit_static
takes particles and output in caller-owned device memory and keeps its only
scratch, the int64 accumulator, in a fixed array of the library's device
image, shared by every call.  These tests check it against impz_deposit on
the same particles and mesh box, on two calls in a row with different beams
(the second call must clear the first call's sums), and that grids above the
array are refused.  The tolerance is the charge-density tolerance of the
parity tests (relative L2 1e-12); both paths form the same integer sums, so
in practice the grids are identical.

The file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

from conftest import load_impz

impz = load_impz()
from impz_b200 import beams  # noqa: E402

RTOL = 1e-12


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def bunch_deposit(cfg, piperad):
    """Charge density and mesh box from the bunch path (impz_sc_prepare +
    impz_deposit) for the particles as given."""
    b = impz.Bunch(cfg["pts"], cfg["current"], cfg["mass"], cfg["charge"], cfg["freq"],
                   cfg["refptcl"], cfg["grid"], form=impz.FORM_FP64, track_ids=False)
    nptot, _, rng, _ = b.sc_prepare(piperad, piperad)
    rho, _ = b.deposit(want_counts=False)
    b.close()
    return rho, rng, nptot


def static_deposit(cfg, rng, piperad, stream=0):
    """The same deposit through impz_deposit_static, device buffers owned by
    the caller (torch here)."""
    import torch
    pts = cfg["pts"]
    cols = [torch.from_numpy(np.ascontiguousarray(pts[:, c])).to("cuda") for c in range(6)]
    nx, ny, nz = cfg["grid"]
    out = torch.full((nx * ny * nz,), float("nan"), dtype=torch.float64, device="cuda")
    rng = np.ascontiguousarray(rng, dtype=np.float64)
    torch.cuda.synchronize()  # the inputs are ready before a call on another stream
    rc = impz.lib().impz_deposit_static(
        *[c.data_ptr() for c in cols], pts.shape[0], -cfg["refptcl"][5], piperad, piperad,
        cfg["freq"], float(pts[0, 7]) if pts.shape[0] else 1.0,
        rng.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
        nx, ny, nz, out.data_ptr(), stream)
    assert rc == impz.OK, impz.error_string(rc)
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.gpu
def test_static_deposit_equals_bunch_deposit_on_two_calls_in_a_row():
    first = beams.fodo_1e5(n=30_000, seed=beams.SEED0 + 21)
    second = beams.fodo_1e5(n=12_000, seed=beams.SEED0 + 22)
    # the second beam meets a pipe narrow enough that conv1st loses particles
    p = second["pts"]
    narrow = 2.0 * float(np.sqrt(np.mean(p[:, 0] ** 2 + p[:, 2] ** 2))) * beams.scxl(
        second["freq"])
    for cfg, piperad, lossy in ((first, 1.0, False), (second, narrow, True)):
        rho, rng, nptot = bunch_deposit(cfg, piperad)
        assert (nptot < cfg["pts"].shape[0]) == lossy
        got = static_deposit(cfg, rng, piperad)
        assert np.all(np.isfinite(got))
        assert rel_l2(got, rho) <= RTOL
        # the same integer sums: in practice the grids are identical
        np.testing.assert_array_equal(got, rho)
        w = float(cfg["pts"][0, 7])
        assert abs(got.sum() - nptot * w) <= 1e-12 * nptot * abs(w)


def test_static_deposit_refuses_grids_above_its_scratch():
    rng = np.array([-1.0, 1.0, -1.0, 1.0, -1.0, 1.0])
    r = rng.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    L = impz.lib()
    # refused before any device call: no GPU needed
    assert L.impz_deposit_static(None, None, None, None, None, None, 0, 2.0, 1.0, 1.0, 402.5e6,
                                 1.0, r, 128, 128, 64, 1, None) == impz.ERR_LIMIT
    assert L.impz_deposit_static(None, None, None, None, None, None, 0, 2.0, 1.0, 1.0, 402.5e6,
                                 1.0, r, 1, 64, 64, 1, None) == impz.ERR_ARG
    assert 64 * 64 * 128 <= impz.STATIC_MAX_CELLS
    assert impz.error_string(impz.ERR_LIMIT) != "unknown error"


def oracle_deposit(cfg, rng, piperad):
    """The oracle's conv1st + deposit_BeamBunch on a given mesh box
    (BeamBunch.f90:1285-1352, 3736-3764): particles outside it skipped."""
    from conftest import load_oracle
    orc = load_oracle()
    orc.physconst(cfg["freq"])
    L = orc.lib()
    p = np.ascontiguousarray(cfg["pts"], dtype=np.float64).copy()
    n = p.shape[0]
    ref = np.array(cfg["refptcl"], dtype=np.float64)
    cur = ctypes.c_double(cfg["current"])
    npt = ctypes.c_int(n)
    ptrange = np.zeros(6)
    nl = L.orc_conv1st(orc.dp(p), n, ctypes.byref(cur), ctypes.byref(npt), orc.dp(ref),
                       piperad, piperad, orc.dp(ptrange))
    mesh = np.array(cfg["grid"], dtype=np.int32)
    rng = np.ascontiguousarray(rng, dtype=np.float64)
    msize = np.array([(rng[2 * k + 1] - rng[2 * k]) / (mesh[k] - 1) for k in range(3)])
    rho = np.zeros(int(np.prod(mesh)))
    L.orc_deposit(orc.dp(p), nl, mesh.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), orc.dp(rng),
                  orc.dp(msize), orc.dp(rho), None, None)
    return rho


@pytest.mark.gpu
def test_static_deposit_skips_particles_outside_the_callers_box():
    """A box narrower than the beam (the outer particles fall outside it) and
    a few particles 1e12 cells away: those are skipped, never written out of
    bounds, and the grid equals the oracle's deposit on the same box."""
    cfg = beams.fodo_1e5(n=20_000, seed=beams.SEED0 + 23)
    rho, rng, nptot = bunch_deposit(cfg, 1.0)
    mid = 0.5 * (rng[0::2] + rng[1::2])
    half = 0.5 * (rng[1::2] - rng[0::2])
    box = np.empty(6)
    box[0::2] = mid - 0.4 * half
    box[1::2] = mid + 0.4 * half
    far = dict(cfg)
    far["pts"] = cfg["pts"].copy()
    far["pts"][:5, 0] = 1e12 * half[0] / beams.scxl(cfg["freq"])
    far["pts"][5:10, 2] = -1e12 * half[1] / beams.scxl(cfg["freq"])
    got = static_deposit(far, box, 1e30)
    near = dict(cfg)
    near["pts"] = cfg["pts"][10:]
    want = oracle_deposit(near, box, 1e30)
    assert np.all(np.isfinite(got))
    assert 0.3 * rho.sum() < got.sum() < 0.95 * rho.sum()
    # the oracle adds FP64 weights; the library rounds each corner to 2^-40 of
    # a particle, so on a box this narrow (few particles per node) the two
    # differ by up to ~1e-12 of a node's charge
    assert rel_l2(got, want) <= 1e-11


@pytest.mark.gpu
def test_static_deposit_empty_beam_and_side_stream():
    """n = 0 gives an all-zero grid after a call that left sums behind; a
    call on a torch side stream equals the default-stream call."""
    import torch
    cfg = beams.fodo_1e5(n=15_000, seed=beams.SEED0 + 24)
    rho, rng, _ = bunch_deposit(cfg, 1.0)
    first = static_deposit(cfg, rng, 1.0)
    assert rel_l2(first, rho) <= RTOL
    empty = dict(cfg)
    empty["pts"] = cfg["pts"][:0]
    zero = static_deposit(empty, rng, 1.0)
    assert np.all(zero == 0.0)
    side = torch.cuda.Stream()
    got = static_deposit(cfg, rng, 1.0, stream=side.cuda_stream)
    np.testing.assert_array_equal(got, first)
