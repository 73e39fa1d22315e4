"""The autotuner (impz_autotune): it leaves the bunch as it found it, and a
tuned bunch gives the results of an untuned one (per-particle arithmetic
does not depend on the launch shape; the moment sums only change their
partition into blocks: 1e-12)."""
import numpy as np
import pytest

from conftest import load_impz

pytestmark = pytest.mark.gpu

impz = load_impz()
from impz_b200 import beams  # noqa: E402


@pytest.mark.parametrize("form", [impz.FORM_FP64, impz.FORM_FP32CONV])
def test_autotune_restores_the_bunch_and_keeps_results(form):
    cfg = beams.fodo_1e5(n=50_000, seed=beams.SEED0 + 61)
    mk = lambda: impz.Bunch(cfg["pts"], cfg["current"], cfg["mass"], cfg["charge"],  # noqa: E731
                            cfg["freq"], cfg["refptcl"], cfg["grid"], form=form, track_ids=True)
    lat = beams.fodo(1)
    a, b = mk(), mk()
    try:
        a.run(lat)  # a bunch in the middle of its life
        b.run(lat)
        before = a.download()
        info0 = a.info()
        t = a.autotune(6)
        assert t["ms_per_step"] > 0 and t["deposit_blocks"] >= 1 and t["push_blocks"] >= 1
        after = a.download()
        by_id = lambda p: p[np.argsort(p[:, 8])]  # noqa: E731
        np.testing.assert_array_equal(by_id(after), by_id(before))
        info1 = a.info()
        assert info1["z"] == info0["z"] and np.array_equal(info1["refptcl"], info0["refptcl"])
        ra, za = a.run(lat)
        rb, zb = b.run(lat)
        np.testing.assert_array_equal(za, zb)
        np.testing.assert_allclose(ra[:, :44], rb[:, :44], rtol=1e-12, atol=1e-300)
        pa, pb = by_id(a.download()), by_id(b.download())
        np.testing.assert_array_equal(pa[:, :6], pb[:, :6])
    finally:
        a.close()
        b.close()
