"""The device failure path, without a GPU fault.

Every wait of the sweep kernels on a plane load is bounded: after its limit
the block records an error flag, waits (bounded again) for its own loads
still in flight and leaves, and the host reports PHP_ERR_TIMEOUT.  With
PHP_TEST_STALL_WAIT=1 at php_create the first block of every H sweep (or of
every one-launch step) waits on a barrier that nothing ever arrives on, with
a short limit: the test checks
that the status comes back, that the context still answers, and that a new
context on the same device steps correctly afterwards.
"""
import numpy as np
import pytest

import harness as H
from php_fdtd_b200 import Config, PhpError, Simulation

pytestmark = pytest.mark.gpu

PHP_ERR_TIMEOUT = -5


def _holder(golden_case, precision):
    with H.chdir(golden_case("vacuum_pml")):
        cfg = Config.load("case.cfg")
        return cfg.desc(cfg.load_medium(), precision)


@pytest.mark.parametrize("fused", ["1", "0"])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_bounded_wait_gives_up_with_a_timeout_status(precision, fused, golden_case, monkeypatch):
    holder = _holder(golden_case, precision)
    monkeypatch.setenv("PHP_TEST_STALL_WAIT", "1")
    monkeypatch.setenv("PHP_FUSED", fused)
    stalled = Simulation(holder)
    monkeypatch.delenv("PHP_TEST_STALL_WAIT")
    monkeypatch.delenv("PHP_FUSED")
    stalled.step(3)
    with pytest.raises(PhpError) as e:
        stalled.sync()
    assert e.value.code == PHP_ERR_TIMEOUT and "gave up" in str(e.value)
    # the context still answers: reads and its own destruction work
    assert stalled.read_volume("Ex").shape == (holder.nx, holder.ny, holder.nz)
    stalled.close()
    # the device is healthy: a new context advances exactly like another
    a, b = Simulation(holder), Simulation(holder)
    a.step(9)
    b.step(4)
    b.step(5)
    for comp in ("Ex", "Ez", "Hy"):
        np.testing.assert_array_equal(a.read_volume(comp), b.read_volume(comp))
    a.sync()
    assert np.abs(a.read_volume("Ez")).max() > 0
    a.close()
    b.close()
