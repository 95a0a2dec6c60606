"""Host-side logic of the serving loop: the request stream, footprint estimates and
admission refusals (no device needed)."""

import numpy as np
import pytest

from tenet import serve


def test_request_stream_is_seeded_and_drawn_from_the_named_sets():
    a = serve.request_stream(64, 2.0, seed=5)
    b = serve.request_stream(64, 2.0, seed=5)
    assert a == b
    assert {r.L for r in a} <= {16, 32, 64, 128}
    assert {r.chi for r in a} <= {32, 64, 128, 256}
    assert all(0.0 <= r.j2 <= 0.4 and r.sweeps == 8 for r in a)
    arr = np.array([r.arrival for r in a])
    assert (np.diff(arr) >= 0).all() and arr[0] > 0
    # Poisson: mean gap ~ 1/rate
    assert 0.3 < np.diff(arr).mean() < 0.8
    burst = serve.request_stream(8, float("inf"), seed=1)
    assert all(r.arrival == 0.0 for r in burst)


def test_footprint_grows_with_length_and_bond_dimension():
    f = serve.footprint_bytes
    base = serve.SolveRequest(0, 16, 0.1, 32)
    assert f(serve.SolveRequest(0, 32, 0.1, 32)) > f(base)
    assert f(serve.SolveRequest(0, 16, 0.1, 64)) > f(base)
    assert f(serve.SolveRequest(0, 128, 0.1, 256)) < 8 << 30  # many fit in 180 GB


def test_a_request_larger_than_the_budget_is_refused_before_any_work():
    srv = serve.Server(hbm_budget=1 << 20, precision="f64")
    with pytest.raises(ValueError, match="more HBM than the whole budget"):
        srv.run([serve.SolveRequest(0, 16, 0.0, 32)])
    with pytest.raises(ValueError):
        serve.Server(max_active=0, hbm_budget=1 << 30)
