"""GPU parity: the CUDA path against the reference's own outputs.

  fp64-strict  bit-identical to the reference (golden fixtures and the drop-in
               executable's files byte for byte)
  fp64         relative L2 <= 1e-10 on every output (the plain-path bound)
  fp32         relative L2 <= 5e-4 on slices with signal (mixed precision)
"""
import filecmp

import numpy as np
import pytest

from conftest import golden_cases
import harness as H

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10   # relative L2, plain FP64 path vs the reference
FP32_TOL = 5e-4    # relative L2, FP32 path vs the reference (fields with signal)


def _golden(d):
    return np.load(d / "golden.npz")


@pytest.mark.parametrize("name", golden_cases())
def test_strict_fp64_is_bit_identical_to_reference(name, golden_case):
    d = golden_case(name)
    g = _golden(d)
    res = H.run_inprocess(d, "device", "fp64-strict")
    steps = list(g["slice_steps"])
    assert sorted(res["slices"]) == steps
    for s, ref in zip(steps, g["slices"]):
        np.testing.assert_array_equal(res["slices"][s], ref, err_msg=f"{name} slice step {s}")
    np.testing.assert_array_equal(res["monitor"], g["monitor"])
    if g["full"].size:
        np.testing.assert_array_equal(res["full"], g["full"])


def _groups(ncols, natom_cols):
    """Column groups of a monitor table: E, D, H, then the lattice columns."""
    g = [slice(1, 4), slice(4, 7), slice(7, 10)]
    if ncols > 10:
        g.append(slice(10, ncols))
    return g


@pytest.mark.parametrize("name", golden_cases())
def test_fp64_within_1e10_of_reference(name, golden_case):
    d = golden_case(name)
    g = _golden(d)
    res = H.run_inprocess(d, "device", "fp64")
    for s, ref in zip(list(g["slice_steps"]), g["slices"]):
        assert H.rel_l2(res["slices"][s], ref) <= FP64_TOL, (name, s)
    for table in ("monitor", "full"):
        ref = g[table]
        if not ref.size:
            continue
        np.testing.assert_array_equal(res[table][:, 0], ref[:, 0])
        for grp in _groups(ref.shape[1], 0):
            assert H.rel_l2(res[table][:, grp], ref[:, grp]) <= FP64_TOL, (name, table, grp)


@pytest.mark.parametrize("name", golden_cases())
def test_fp32_close_to_reference(name, golden_case):
    d = golden_case(name)
    g = _golden(d)
    res = H.run_inprocess(d, "device", "fp32")
    errs = []
    for s, ref in zip(list(g["slice_steps"]), g["slices"]):
        if np.abs(ref).max() > 0:
            errs.append(H.rel_l2(res["slices"][s], ref))
    # the first samples of a pulse are a few cells wide and dominated by
    # round-off; the check takes the slices of the last half of the run
    tail = errs[len(errs) // 2:]
    assert tail and max(tail) <= FP32_TOL, (name, errs)


@pytest.mark.parametrize("name", golden_cases())
def test_dropin_executable_writes_reference_files(name, golden_case):
    """fdtd_b200 <cfg> fp64-strict writes the reference's files byte for byte
    (float32 slices, %e monitors, source.txt)."""
    d = golden_case(name)
    res = H.run_cli(d, "fp64-strict")
    assert res["returncode"] == 0, res["stdout"][-3000:]
    plain = d / "plain"
    ref_files = sorted(p.name for p in plain.iterdir())
    assert ref_files
    for fn in ref_files:
        assert (d / fn).exists(), fn
        assert filecmp.cmp(d / fn, plain / fn, shallow=False), f"{name}: {fn} differs"
    produced = sorted(p.name for p in d.glob("field_slice_*.bin"))
    assert produced == sorted(p for p in ref_files if p.startswith("field_slice_"))
