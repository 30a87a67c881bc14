"""Serving loop (php_serve.h): jobs admitted as memory and slots free up,
advanced together, each result identical to the same simulation run alone."""
import numpy as np
import pytest

from php_fdtd_b200 import PhpError, Simulation
from php_fdtd_b200.serving import DftSpec, Server, estimate_bytes
from php_fdtd_b200.workloads import request_desc, serving_requests

pytestmark = pytest.mark.gpu


def _requests(n, seed=1):
    # small grids and step counts of the serving mix
    return serving_requests(n, seed=seed, edge_range=(20, 40), steps_range=(150, 420), pml=4)


def _alone(req, precision):
    holder, dft = request_desc(req, precision)
    with Simulation(holder) as sim:
        pid = sim.dft_add(dft["component"], dft["z_plane"], dft["freqs"])
        sim.step(req["steps"])
        sim.sync()
        return sim.dft_read(pid)[0]


def _serve(reqs, precisions, **kw):
    out = {}
    with Server(**kw) as srv:
        ids = {}
        for q, (req, prec) in enumerate(zip(reqs, precisions)):
            holder, dft = request_desc(req, prec)
            ids[srv.submit(holder, req["steps"], DftSpec(dft["component"], dft["z_plane"], dft["freqs"]), tag=q)] = q
        while len(out) < len(reqs):
            for info in srv.poll(timeout_ms=20000):
                assert info["status"] == 0, info["error"]
                assert info["steps"] == reqs[info["tag"]]["steps"]
                assert info["t_submit"] <= info["t_admit"] <= info["t_done"]
                out[info["tag"]] = srv.fetch_dft(info)
        stats = srv.stats()
    return out, stats


def test_results_in_the_mix_equal_results_alone():
    reqs = _requests(6)
    # a longer first job, so that the others run beside it
    reqs[0] = dict(reqs[0], grid=(64, 64, 64), steps=12000)
    precs = ["fp32", "fp64", "fp32", "fp32", "fp64", "fp32"]
    got, stats = _serve(reqs, precs, memory_budget=8 << 30, chunk_steps=64)
    assert stats["completed"] == 6 and stats["peak_running"] >= 2
    for q, (req, prec) in enumerate(zip(reqs, precs)):
        np.testing.assert_array_equal(got[q], _alone(req, prec), err_msg=f"job {q}")


def test_memory_budget_and_slots_limit_admission():
    # one grid for all five, so that the budget holds exactly one at a time
    reqs = [dict(r, grid=(36, 30, 28)) for r in _requests(5, seed=2)]
    biggest = max(estimate_bytes(request_desc(r, "fp32")[0]) for r in reqs)
    # room for one job at a time
    got, stats = _serve(reqs, ["fp32"] * 5, memory_budget=int(biggest * 1.5), chunk_steps=128)
    assert stats["peak_running"] == 1 and stats["peak_bytes"] <= int(biggest * 1.5)
    # two slots
    got2, stats2 = _serve(reqs, ["fp32"] * 5, memory_budget=8 << 30, max_active=2)
    assert stats2["peak_running"] <= 2
    for q in range(5):
        np.testing.assert_array_equal(got[q], got2[q])


def test_failing_job_does_not_disturb_the_others():
    reqs = _requests(3, seed=3)
    with Server(memory_budget=8 << 30) as srv:
        holder, dft = request_desc(reqs[0], "fp32")
        good = srv.submit(holder, reqs[0]["steps"], DftSpec(dft["component"], dft["z_plane"], dft["freqs"]))
        bad_holder, _ = request_desc(reqs[1], "fp32")
        # a DFT plane outside the grid makes php_dft_add fail inside the server
        bad = srv.submit(bad_holder, 10, DftSpec("Ez", 10 ** 6, [1e13]))
        done = {}
        while len(done) < 2:
            for info in srv.poll(timeout_ms=20000):
                done[info["job"]] = info
        assert done[bad]["status"] != 0 and done[bad]["error"]
        assert done[good]["status"] == 0
        np.testing.assert_array_equal(srv.fetch_dft(done[good]), _alone(reqs[0], "fp32"))
        srv.release(bad)
        with pytest.raises(PhpError):
            srv.release(bad)


def test_job_larger_than_budget_is_refused_at_submit():
    req = _requests(1)[0]
    holder, _ = request_desc(req, "fp32")
    with Server(memory_budget=1 << 20) as srv:
        with pytest.raises(PhpError) as e:
            srv.submit(holder, 10)
        assert e.value.code == -2


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_memory_estimate_covers_the_context(precision):
    for req in _requests(3, seed=4):
        holder, _ = request_desc(req, precision)
        est = estimate_bytes(holder)
        with Simulation(holder) as sim:
            used = sim.memory_bytes
        assert used <= est <= 1.1 * used + (2 << 20), (used, est)
