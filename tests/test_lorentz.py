"""The Lorentz integrator (Flagmap=2) on the oracle, no GPU needed:
drift2 half steps around kick2/scatter2 (BeamBunch.f90:467-509,
2187-3071).  Through a FODO lattice its second-order splitting of the
quadrupoles' focusing converges to the linear map integrator's result as
the steps shrink."""
import numpy as np

from conftest import load_impz, load_oracle

impz = load_impz()
orc = load_oracle()
from impz_b200 import beams  # noqa: E402


def test_lorentz_integrator_converges_to_the_map_integrator():
    cfg = beams.fodo_1e5(n=5000, seed=beams.SEED0 + 71)
    gaps = []
    for nseg in (4, 16, 64):
        lat = beams.fodo(1, nseg=nseg)
        run = lambda fm: orc.run(lat, cfg["pts"], cfg["current"], cfg["mass"],  # noqa: E731
                                 cfg["charge"], cfg["freq"], cfg["refptcl"], (16, 16, 32),
                                 flagmap=fm)[0]
        r1, r2 = run(1), run(2)
        np.testing.assert_array_equal(r1[:, 0], r2[:, 0])  # the same steps and z
        gaps.append(max(abs(r2[-1, c] - r1[-1, c]) / abs(r1[-1, c]) for c in (7, 13)))
    # the splitting error falls fast with the step (the space-charge kicks
    # of the two integrators also differ slightly, which leaves a small floor)
    assert gaps[0] > 8 * gaps[1] > 0 and gaps[1] > 2 * gaps[2] and gaps[2] < 1e-3


def test_lorentz_integrator_refuses_elements_outside_it():
    cfg = beams.fodo_1e5(n=500)
    bend = impz.elem(4, 0.2, 4, 1, [0.05, 0.0, 150.0, 0.01])
    try:
        orc.run([bend], cfg["pts"], cfg["current"], cfg["mass"], cfg["charge"], cfg["freq"],
                cfg["refptcl"], (16, 16, 32), flagmap=2)
    except RuntimeError as e:
        assert "-10" in str(e)
    else:
        raise AssertionError("a bend under the Lorentz integrator must be refused")


def test_lorentz_integrator_without_current_converges_too():
    """Zero current: kick2 is scatter20, the quadrupoles' field alone on the
    stored coordinates (BeamBunch.f90:3075-3531)."""
    cfg = beams.fodo_1e5(n=2000, seed=beams.SEED0 + 73)
    gaps = []
    for nseg in (4, 32):
        lat = beams.fodo(1, nseg=nseg)
        run = lambda fm: orc.run(lat, cfg["pts"], 0.0, cfg["mass"], cfg["charge"],  # noqa: E731
                                 cfg["freq"], cfg["refptcl"], (16, 16, 32), flagmap=fm)[0]
        r1, r2 = run(1), run(2)
        gaps.append(max(abs(r2[-1, c] - r1[-1, c]) / abs(r1[-1, c]) for c in (7, 13)))
    assert gaps[0] > 8 * gaps[1] and gaps[1] < 2e-3
