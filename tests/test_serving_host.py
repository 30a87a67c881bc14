"""Host-side parts of the serving loop that need no GPU: the request
stream, the device-memory estimate used for admission, and the server's
refusal to start without a device."""
import numpy as np
import pytest

from php_fdtd_b200 import PhpError
from php_fdtd_b200.serving import Server, estimate_bytes
from php_fdtd_b200.workloads import request_desc, serving_requests


def test_request_stream_follows_the_configuration():
    reqs = serving_requests(256)
    arr = np.array([r["arrival"] for r in reqs])
    assert np.all(np.diff(arr) > 0)
    assert 40 < arr[-1] < 100            # 256 arrivals at 4 per second
    edges = np.array([r["grid"] for r in reqs]).ravel()
    assert edges.min() >= 64 and edges.max() <= 192
    steps = np.array([r["steps"] for r in reqs])
    assert steps.min() >= 3000 and steps.max() <= 12000
    assert all(700 <= r["wavenumber"] <= 1600 and 5 <= r["tip_height_nm"] <= 50 for r in reqs)
    assert serving_requests(8, seed=5) == serving_requests(8, seed=5)


def test_memory_estimate_scales_with_grid_and_precision():
    r = serving_requests(1)[0]
    small = dict(r, grid=(32, 32, 32))
    big = dict(r, grid=(64, 64, 64))
    e32 = estimate_bytes(request_desc(small, "fp32")[0])
    e64 = estimate_bytes(request_desc(small, "fp64")[0])
    b32 = estimate_bytes(request_desc(big, "fp32")[0])
    # nine fields alone: 9 x 32 x 32 x 34 words
    assert e32 > 9 * 32 * 32 * 34 * 4
    assert 1.5 < (e64 - (1 << 20)) / (e32 - (1 << 20)) < 2.1
    assert b32 > 6 * (e32 - (1 << 20))


def test_server_needs_a_device():
    try:
        srv = Server(memory_budget=1 << 30)
    except PhpError as e:
        assert e.code == -8
        return
    srv.close()
    pytest.skip("a CUDA device is visible")
