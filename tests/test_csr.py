"""CSR wake of bends (csrwakeTrIGF_FieldQuant, src/Appl/Field.f90:1003-1303)
on the oracle, no GPU needed: the steady-state regime against the standard
steady-state CSR field of a Gaussian bunch, and the bend bookkeeping that
decides where CSR acts (src/Contrl/AccSimulator.f90:1035-1051, 1131-1138)."""
import numpy as np
import pytest

from conftest import load_impz, load_oracle

impz = load_impz()
orc = load_oracle()
from impz_b200 import beams  # noqa: E402

EPS0 = 8.854187817e-12


def steady_state(s, sig, q, r0, s_mid):
    """E(s) = -2 / (3^(1/3) R^(2/3)) / (4 pi eps0) int lambda'(s') (s-s')^(-1/3) ds'
    for a Gaussian line charge, with u = (s-s')^(2/3) removing the
    singularity."""
    k = 2 / (3 ** (1 / 3) * r0 ** (2 / 3)) / (4 * np.pi * EPS0)
    u = np.linspace(0, (14 * sig) ** (2 / 3), 20001)
    out = []
    for si in s:
        sp = si - u ** 1.5
        dl = q / (np.sqrt(2 * np.pi) * sig) * np.exp(-0.5 * ((sp - s_mid) / sig) ** 2)
        dl *= -(sp - s_mid) / sig ** 2
        out.append(-k * np.trapezoid(1.5 * dl, u))
    return np.array(out)


@pytest.mark.parametrize("nz,tol", [(128, 5e-2), (512, 2.5e-2)])
def test_csr_steady_state_in_a_long_bend(nz, tol):
    """5 m into a 100 m bend of radius 10 m, gamma 1000, a 100 um Gaussian:
    the entrance transient has passed (case B only) and the IGF field
    approaches the steady-state formula as the grid refines."""
    L = orc.lib()
    sig, r0, gam, q = 1e-4, 10.0, 1000.0, 1e-9
    ptmin = 5.0 - 6 * sig
    hx = 12 * sig / (nz - 1)
    s = ptmin + np.arange(nz) * hx
    lam = q / (np.sqrt(2 * np.pi) * sig) * np.exp(-0.5 * ((s - 5.0) / sig) ** 2)
    ez = np.zeros(nz)
    L.orc_csr_wake(nz, r0, ptmin, hx, 100.0, orc.dp(lam), gam, orc.dp(ez))
    want = steady_state(s, sig, q, r0, 5.0)
    assert np.linalg.norm(ez - want) / np.linalg.norm(want) < tol
    # the most negative field sits where the formula puts it, to a cell
    assert ez[np.argmin(want)] < 0 and abs(int(np.argmin(ez)) - int(np.argmin(want))) <= 1


def test_csr_exit_transient_decays_downstream():
    """Past the exit (cases C and D) the field decays with the distance from
    the bend: 0.1 m after a 0.2 m bend it is below the field at the exit."""
    L = orc.lib()
    nz, sig, r0, gam, q = 128, 1e-4, 5.0, 500.0, 1e-9
    peak = []
    for after in (0.0, 0.02, 0.1, 1.0):
        ptmin = 0.2 + after - 6 * sig
        hx = 12 * sig / (nz - 1)
        s = ptmin + np.arange(nz) * hx
        lam = q / (np.sqrt(2 * np.pi) * sig) * np.exp(-0.5 * ((s - 0.2 - after) / sig) ** 2)
        ez = np.zeros(nz)
        L.orc_csr_wake(nz, r0, ptmin, hx, 0.2, orc.dp(lam), gam, orc.dp(ez))
        assert np.all(np.isfinite(ez))
        peak.append(np.abs(ez).max())
    assert peak[0] > peak[2] > peak[3] > 0


def test_csr_bookkeeping_on_a_chicane():
    """File ID 150: no CSR; above 200: CSR inside the bends; above 500: also
    the transient downstream of each bend, which leaves flagbendcsr set and
    sentr at the distance from the last bend's entrance."""
    pts, ref = beams.flat_top_bunch(5000, seed=beams.SEED0 + 31, current=10.0)
    res = {}
    for fid in (150.0, 300.0, 600.0):
        lat = beams.chicane(ldrift_in=0.5, drift_steps_in=4, nseg_bend=4, nseg_drift=2,
                            file_id=fid)
        lat.append(impz.elem(0, 0.3, 2, 1, [1.0]))
        rows, p, beam = orc.run(lat, pts, 10.0, beams.ELECTRON_MASS_EV, -1.0, 1.3e9, ref,
                                (16, 16, 32))
        assert np.all(np.isfinite(p))
        res[fid] = (p, beam)
    assert res[150.0][1].flagbendcsr == 0 and res[300.0][1].flagbendcsr == 0
    assert res[600.0][1].flagbendcsr == 1
    assert abs(res[600.0][1].sentr - 0.5) < 1e-12 and abs(res[600.0][1].bendlencsr - 0.2) < 1e-15
    spread = {k: np.std(v[0][:, 5]) for k, v in res.items()}
    assert spread[300.0] > 1.5 * spread[150.0]
    assert abs(spread[600.0] - spread[300.0]) > 1e-2 * spread[300.0]  # the drift transients
