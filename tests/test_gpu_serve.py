"""The serving loop on the device: solves that overlap on the GPU give the same result
as each solve alone, and the precision form stays within |dE/L| <= 1e-8 of FP64."""

import pytest
import torch

from tenet import _lib, serve

pytestmark = pytest.mark.gpu

TOL_PER_SITE = 1e-8


@pytest.fixture(autouse=True)
def _device_error_clear():
    yield
    torch.cuda.synchronize()
    assert _lib.device_error(0) == 0, "a kernel raised the device error word"


REQUESTS = [serve.SolveRequest(0, 8, 0.0, 16, sweeps=3, arrival=0.0, seed=11),
            serve.SolveRequest(1, 10, 0.3, 32, sweeps=3, arrival=0.0, seed=12),
            serve.SolveRequest(2, 12, 0.2, 24, sweeps=3, arrival=0.0, seed=13),
            serve.SolveRequest(3, 8, 0.4, 16, sweeps=3, arrival=0.05, seed=14),
            serve.SolveRequest(4, 16, 0.1, 32, sweeps=2, arrival=0.1, seed=15)]


@pytest.mark.parametrize("precision,tc_min", [("f64", None), ("3xbf16", 0)])
def test_served_solves_equal_the_same_solves_alone(precision, tc_min):
    srv = serve.Server(max_active=3, hbm_budget=8 << 30, precision=precision,
                       tc_min_flops=tc_min)
    results = srv.run(REQUESTS)
    assert sorted(r.rid for r in results) == [r.rid for r in REQUESTS]
    assert srv.peak_active >= 2, "the solves did not overlap"
    for r in results:
        e, hist = serve.solve_alone(r.request, precision=precision, tc_min_flops=tc_min)
        assert len(hist) == len(r.history)
        for a, b in zip(hist, r.history):
            assert abs(a - b) / r.request.L <= TOL_PER_SITE
        if precision != "f64":
            e64, _ = serve.solve_alone(r.request, precision="f64")
            assert abs(e - e64) / r.request.L <= TOL_PER_SITE, \
                f"request {r.rid}: |dE/L| = {abs(e - e64) / r.request.L:.2e} against FP64"


def test_admission_by_footprint_serialises_what_does_not_fit_together():
    reqs = REQUESTS[:3]
    one = max(serve.footprint_bytes(r) for r in reqs)
    srv = serve.Server(max_active=3, hbm_budget=one, precision="f64")
    results = srv.run(reqs)
    assert srv.peak_active == 1
    assert len(results) == 3
    for r in results:
        assert r.admitted >= 0.0 and r.finished >= r.admitted


def test_solves_served_by_worker_processes_equal_the_same_solves_alone():
    """Host-parallel serving (two spawned workers on the same GPU): every result is the
    same as the solve alone in this process."""
    with serve.ProcessServer(workers=2, hbm_budget=8 << 30, precision="f64") as srv:
        assert len(srv.pids) == 2
        results = srv.run(REQUESTS[:4])
    assert sorted(r.rid for r in results) == [0, 1, 2, 3]
    assert srv.peak_active == 2
    for r in results:
        e, hist = serve.solve_alone(r.request, precision="f64")
        assert len(hist) == len(r.history)
        for a, b in zip(hist, r.history):
            assert abs(a - b) / r.request.L <= TOL_PER_SITE
