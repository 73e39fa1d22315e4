"""Golden fixtures (tests/golden/, written by make_golden.py from the oracle):
the oracle must keep reproducing them bit for bit (CPU), and the GPU path,
called through the C ABI, must meet them at the parity tolerances."""
import os
import sys

import numpy as np
import pytest

from conftest import load_impz, load_oracle

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden  # noqa: E402

impz = load_impz()
orc = load_oracle()

CASES = sorted(make_golden.CASES)


def fixture(name):
    return dict(np.load(os.path.join(HERE, "golden", name + ".npz")))


@pytest.mark.parametrize("name", CASES)
def test_oracle_reproduces_golden(name):
    gold = fixture(name)
    pts, ref, cfg, e, out = make_golden.build(name)
    for k, v in out.items():
        np.testing.assert_array_equal(v, gold[k], err_msg=k)


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_gpu_meets_golden(name):
    gold = fixture(name)
    n, grid, (etype, length, nseg, vals), seed = make_golden.CASES[name]
    pts, ref, cfg, e, _ = make_golden.build(name)
    tau = length / nseg
    b = impz.Bunch(pts, cfg["current"], cfg["mass"], cfg["charge"], cfg["freq"], ref, grid,
                   form=impz.FORM_FP64, track_ids=True)
    z, ih = b.map_half(e, 0.0, 0.0, tau / 2, 1, 0)
    nptot, ptrange, rng, msize = b.sc_prepare(1.0, 1.0)
    rho, counts = b.deposit()
    phi = b.poisson()
    eg = b.kick(tau, want_e=True)
    b.map_half(e, 0.0, z, tau / 2, 1, ih)
    p = b.download()
    rec = b.moments()
    b.close()
    np.testing.assert_array_equal(ptrange, gold["ptrange"])
    np.testing.assert_array_equal(rng, gold["range"])
    np.testing.assert_array_equal(msize, gold["msize"])
    np.testing.assert_array_equal(counts, gold["counts"])
    for k, v in (("rho", rho), ("phi", phi), ("eg", eg)):
        err = np.linalg.norm(v - gold[k]) / np.linalg.norm(gold[k])
        assert err <= 1e-12, (k, err)
    gp = p[np.argsort(p[:, 8])]
    op = gold["pts"][np.argsort(gold["pts"][:, 8])]
    np.testing.assert_array_equal(gp[:, 8], op[:, 8])
    for c in range(6):
        s = np.sqrt(np.mean(op[:, c] ** 2))
        assert np.max(np.abs(gp[:, c] - op[:, c])) <= 1e-11 * s, c
    np.testing.assert_allclose(rec[:37], gold["raw"][:37], rtol=1e-10, atol=1e-300)
