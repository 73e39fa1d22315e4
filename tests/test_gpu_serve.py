"""Batched scans and the serving loop: a bunch's result does not depend on
what else shares the GPU.

Per-particle arithmetic is independent of other bunches; only the order of
the per-step particle sort (and so the summation order of the moment sums)
can differ between runs, so records agree to relative 1e-10.  Admission
never exceeds the HBM budget, and a job above the budget is refused.
"""
import numpy as np
import pytest

from conftest import load_impz

pytestmark = pytest.mark.gpu

impz = load_impz()
from impz_b200 import beams  # noqa: E402

TOL = 1e-10


def close(a, b):
    a = np.asarray(a)[:, :44]
    b = np.asarray(b)[:, :44]
    scale = np.maximum(np.abs(b), 1e-300)
    err = np.abs(a - b) / scale
    # sums that cancel (centroids near zero) are compared against their column scale
    colscale = np.maximum(np.max(np.abs(b), axis=0, keepdims=True), 1e-300)
    err = np.minimum(err, np.abs(a - b) / colscale)
    return float(np.max(err))


def small_jobs():
    jobs = beams.scan_jobs(nbunch=6, nmin=2e3, nmax=6e4, steps_periods=3)
    return jobs


def alone(job, form):
    pts, ref = beams.make_scan_bunch(job)
    b = impz.Bunch(pts, job["current"], beams.PROTON_MASS_EV, 1.0, 402.5e6, ref, job["grid"],
                   form=form, track_ids=False)
    recs, zs = b.run(job["lattice"])
    b.close()
    return recs


@pytest.mark.parametrize("form", [impz.FORM_FP64, impz.FORM_FP32CONV])
def test_batch_equals_one_by_one(form):
    jobs = small_jobs()
    ref = [alone(j, form) for j in jobs]
    bunches = []
    for j in jobs:
        pts, r = beams.make_scan_bunch(j)
        bunches.append(impz.Bunch(pts, j["current"], beams.PROTON_MASS_EV, 1.0, 402.5e6, r,
                                  j["grid"], form=form, track_ids=False))
    out = impz.run_batch(bunches, [j["lattice"] for j in jobs])
    for b in bunches:
        b.close()
    for (recs, zs), r in zip(out, ref):
        assert recs.shape == r.shape
        assert close(recs, r) <= TOL


@pytest.mark.parametrize("form", [impz.FORM_FP64, impz.FORM_FP32CONV])
def test_packed_runs_of_different_lengths_equal_solo_runs(form):
    """impz_run_advance_packed over bunches of three grid sizes whose
    lattices have different lengths (each bunch at its own step, runs ending
    at different calls): each bunch's records equal its solo run."""
    jobs = small_jobs()
    for i, j in enumerate(jobs):
        j["lattice"] = beams.fodo_steps(16 + 7 * i, nseg=4)
    ref = [alone(j, form) for j in jobs]
    bunches = []
    for j in jobs:
        pts, r = beams.make_scan_bunch(j)
        bunches.append(impz.Bunch(pts, j["current"], beams.PROTON_MASS_EV, 1.0, 402.5e6, r,
                                  j["grid"], form=form, track_ids=False))
    out = impz.run_packed(bunches, [j["lattice"] for j in jobs], steps_per_call=5)
    for b in bunches:
        b.close()
    for (recs, zs), r in zip(out, ref):
        assert recs.shape == r.shape
        assert close(recs, r) <= TOL


def test_server_result_alone_equals_result_in_mix():
    jobs = small_jobs()
    target = jobs[2]
    pts, ref = beams.make_scan_bunch(target)
    with impz.Server(budget_bytes=4e9, max_active=8) as srv:
        jid = srv.submit(pts, target["current"], beams.PROTON_MASS_EV, 1.0, 402.5e6, ref,
                         target["grid"], target["lattice"])
        solo = srv.wait(jid)[0]
    with impz.Server(budget_bytes=4e9, max_active=8) as srv:
        ids = []
        for j in jobs:
            p, r = beams.make_scan_bunch(j)
            ids.append(srv.submit(p, j["current"], beams.PROTON_MASS_EV, 1.0, 402.5e6, r,
                                  j["grid"], j["lattice"]))
        res = [srv.wait(i) for i in ids]
        st = srv.stats()
    assert st["completed"] == len(jobs) and st["failed"] == 0
    assert close(res[2][0], solo) <= TOL
    for (recs, lat, queued, measured), j in zip(res, jobs):
        assert recs.shape[0] == impz.count_steps(j["lattice"]) + 1
        assert lat >= queued >= 0.0
        assert measured <= impz.footprint(j["n"], j["grid"],
                                          nsteps=impz.count_steps(j["lattice"]))


def test_server_admits_within_budget_and_refuses_oversize():
    jobs = small_jobs()
    fp = max(impz.footprint(j["n"], j["grid"], nsteps=impz.count_steps(j["lattice"]))
             for j in jobs)
    budget = 2.2 * fp  # at most two jobs resident at a time
    with impz.Server(budget_bytes=budget, max_active=16) as srv:
        ids = []
        for j in jobs:
            p, r = beams.make_scan_bunch(j)
            ids.append(srv.submit(p, j["current"], beams.PROTON_MASS_EV, 1.0, 402.5e6, r,
                                  j["grid"], j["lattice"]))
        for i in ids:
            srv.wait(i)
        st = srv.stats()
        assert st["completed"] == len(jobs)
        assert st["peak_admitted_bytes"] <= budget
    big, r = beams.gaussian_bunch(1000)
    with impz.Server(budget_bytes=1e6, max_active=2) as srv:
        with pytest.raises(impz.ImpzError) as ei:
            srv.submit(big, 0.03, beams.PROTON_MASS_EV, 1.0, 402.5e6, r, (64, 64, 128),
                       beams.fodo(1), form=impz.FORM_FP64)
        assert ei.value.code == impz.ERR_BUDGET


def test_server_admits_a_job_that_arrives_while_others_run():
    """Continuous batching: two long jobs are on the GPU when a short job is
    submitted; it is admitted at once (slots and budget are free), finishes
    while both long jobs are still running, and its records equal its solo
    run within the module tolerance."""
    import time
    # each long job runs for about a second (4e6 particles, 2400 steps),
    # the short one for milliseconds
    long_jobs = [dict(n=4_000_000, seed=beams.SEED0 + 600 + k, current=0.03 + 0.01 * k,
                      grid=(64, 64, 128), lattice=beams.fodo_steps(2400, nseg=4))
                 for k in range(2)]
    short = dict(n=20_000, seed=beams.SEED0 + 610, current=0.02, grid=(32, 32, 64),
                 lattice=beams.fodo_steps(40, nseg=4))
    pts_s, ref_s = beams.make_scan_bunch(short)
    with impz.Server(budget_bytes=8e9, max_active=8) as srv:
        solo = srv.wait(srv.submit(pts_s, short["current"], beams.PROTON_MASS_EV, 1.0, 402.5e6,
                                   ref_s, short["grid"], short["lattice"]))[0]
    with impz.Server(budget_bytes=8e9, max_active=8) as srv:
        ids = []
        for j in long_jobs:
            p, r = beams.make_scan_bunch(j)
            ids.append(srv.submit(p, j["current"], beams.PROTON_MASS_EV, 1.0, 402.5e6, r,
                                  j["grid"], j["lattice"]))
        t0 = time.perf_counter()
        while srv.stats()["queued"] > 0 and time.perf_counter() - t0 < 30:
            time.sleep(0.002)
        st = srv.stats()
        assert st["queued"] == 0 and st["completed"] == 0 and st["admitted_bytes"] > 0
        sid = srv.submit(pts_s, short["current"], beams.PROTON_MASS_EV, 1.0, 402.5e6, ref_s,
                         short["grid"], short["lattice"])
        recs, latency, queued, _ = srv.wait(sid)
        during = srv.stats()
        long_res = [srv.wait(i) for i in ids]
        end = srv.stats()
    assert during["completed"] == 1, during  # only the short job had finished
    assert queued <= latency
    assert end["completed"] == 3 and end["failed"] == 0
    assert all(r[0].shape[0] == 2401 for r in long_res)
    assert recs.shape == solo.shape
    assert close(recs, solo) <= TOL
