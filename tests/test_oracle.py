"""CPU tests of the oracle: the C restatement (oracle/php_oracle.c) reproduces
the reference solver bit for bit on every golden case, and the golden
fixtures still equal what the reference binary in oracle/_ref produces."""
import numpy as np
import pytest

from conftest import golden_cases
import harness as H
from oracle import reference_binary


def _compare_exact(res, g):
    steps = list(g["slice_steps"])
    assert sorted(res["slices"]) == steps
    for s, ref in zip(steps, g["slices"]):
        np.testing.assert_array_equal(res["slices"][s], ref, err_msg=f"slice at step {s}")
    np.testing.assert_array_equal(res["monitor"], g["monitor"])
    if g["full"].size:
        np.testing.assert_array_equal(res["full"], g["full"])


@pytest.mark.parametrize("name", golden_cases())
def test_oracle_equals_reference_bitwise(name, golden_case):
    d = golden_case(name)
    res = H.run_inprocess(d, "oracle")
    _compare_exact(res, np.load(d / "golden.npz"))


@pytest.mark.parametrize("threads", [1, 3])
def test_oracle_thread_count_does_not_change_results(threads, golden_case):
    d = golden_case("ions2")
    res = H.run_inprocess(d, "oracle", threads=threads)
    _compare_exact(res, np.load(d / "golden.npz"))


@pytest.mark.skipif(not reference_binary("wide").exists(), reason="reference not built here")
@pytest.mark.parametrize("name", ["ions2", "lossy_rot"])
def test_golden_fixtures_are_the_reference_outputs(name, golden_case):
    d = golden_case(name)
    live = H.run_reference(d, "wide")
    assert live["returncode"] == 0
    _compare_exact(live, np.load(d / "golden.npz"))


def test_oracle_diagnostics_match_reference_progress_line(golden_case):
    """|E|_max and r_max printed by the reference (fdtd.c:3563, 3597)."""
    import re
    d = golden_case("ions2")
    res = H.run_inprocess(d, "oracle")
    out = (d / "reference_stdout.txt").read_text()
    lines = re.findall(r"it (\d+)/\d+ .*?\|E\|_max = (\S+) V/m,r_max = (\S+) A,", out)
    assert lines
    for t, emax, rmax in lines:
        dg = res["diag"][int(t)]
        assert f"{dg['max_e']:.2e}" == emax
        assert f"{dg['max_r'] / 1e-10:.2e}" == rmax
