"""GPU parity at the benchmark workloads' own sizes, against the reference's
own outputs (tests/golden/baseline, made by tests/golden/make_golden.py
--baseline):

  cfg0_full     96^3, 2000 steps, two-atom polar slab: the whole run
  cfg1_200      256^3, Drude-Lorentz tip (tensor ADE) over a rotated lossy
                slab: the first 200 of its 8000 steps
  cfg2_200      512 x 512 x 256, 16-atom lattice (the ion pass): the first
                200 of its 10000 steps
  blocks_mixed  96 x 64 x 64 with every block class of the sweeps

The inputs are regenerated from the seeded generator and checked against the
SHA-256 the fixture recorded when the reference ran on them.  The plain FP64
path must be within 1e-10 relative L2 of the reference on every slice and
every monitor column group; the strict mode bit-identical; the FP32 path's
error against the reference is printed beside it (and bounded where the
fields carry signal).
"""
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

import harness as H
from conftest import GOLDEN
from php_fdtd_b200.workloads import parity_baseline_case, write_case

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10   # relative L2, plain FP64 path vs the reference
FP32_TOL = 1e-3    # relative L2, FP32 path vs the reference, slices of the last half of the run
BASE = GOLDEN / "baseline"


def _cases():
    return sorted(p.name for p in BASE.iterdir() if (p / "golden.npz").exists()) if BASE.exists() else []


def _inputs(name: str, tmp_path: Path):
    g = np.load(BASE / name / "golden.npz")
    d = tmp_path / name
    write_case(parity_baseline_case(name), d)
    want = json.loads(str(g["inputs"]))
    got = {p.name: hashlib.sha256(p.read_bytes()).hexdigest() for p in sorted(d.iterdir()) if p.is_file()}
    assert got == want, "regenerated inputs differ from those the reference ran on"
    return d, g


def _groups(ncols):
    """Column groups of a monitor table: E, D, H, then the lattice columns."""
    g = [slice(1, 4), slice(4, 7), slice(7, 10)]
    if ncols > 10:
        g.append(slice(10, ncols))
    return g


def _close(res):
    sim = res.pop("sim", None)
    if sim is not None:
        sim.close()


def _compare(res, g, name):
    """worst relative L2 over slices and monitor groups"""
    steps = list(g["slice_steps"])
    assert sorted(res["slices"]) == steps, name
    worst = {"slice": 0.0}
    for s, ref in zip(steps, g["slices"]):
        if np.abs(ref).max() > 0:
            worst["slice"] = max(worst["slice"], H.rel_l2(res["slices"][s], ref))
        else:
            assert np.abs(res["slices"][s]).max() == 0, (name, s)
    for table in ("monitor", "full"):
        ref = g[table]
        if not ref.size:
            continue
        assert res[table].shape == ref.shape, (name, table)
        np.testing.assert_array_equal(res[table][:, 0], ref[:, 0])
        for grp in _groups(ref.shape[1]):
            key = f"{table}[{grp.start}:{grp.stop}]"
            worst[key] = H.rel_l2(res[table][:, grp], ref[:, grp]) if np.abs(ref[:, grp]).max() > 0 else 0.0
    return worst


@pytest.mark.parametrize("name", _cases())
def test_fp64_within_1e10_of_reference_at_workload_size(name, tmp_path):
    d, g = _inputs(name, tmp_path)
    res = H.run_inprocess(d, "device", "fp64")
    census = res["sim"].block_census()
    _close(res)
    worst = _compare(res, g, name)
    print(f"\n{name} fp64 vs reference: " + ", ".join(f"{k} {v:.2e}" for k, v in worst.items()) + f"; blocks {census}")
    for k, v in worst.items():
        assert v <= FP64_TOL, (name, k, v)


@pytest.mark.parametrize("name", [n for n in _cases() if n != "cfg2_200"])
def test_strict_fp64_bit_identical_at_workload_size(name, tmp_path):
    d, g = _inputs(name, tmp_path)
    res = H.run_inprocess(d, "device", "fp64-strict")
    _close(res)
    for s, ref in zip(list(g["slice_steps"]), g["slices"]):
        np.testing.assert_array_equal(res["slices"][s], ref, err_msg=f"{name} slice step {s}")
    np.testing.assert_array_equal(res["monitor"], g["monitor"])
    if g["full"].size:
        np.testing.assert_array_equal(res["full"], g["full"])


@pytest.mark.parametrize("name", _cases())
def test_fp32_error_against_reference_at_workload_size(name, tmp_path):
    d, g = _inputs(name, tmp_path)
    res = H.run_inprocess(d, "device", "fp32")
    _close(res)
    steps = list(g["slice_steps"])
    errs = [H.rel_l2(res["slices"][s], ref) for s, ref in zip(steps, g["slices"]) if np.abs(ref).max() > 0]
    mon = g["monitor"]
    mon_err = {f"monitor[{grp.start}:{grp.stop}]": H.rel_l2(res["monitor"][:, grp], mon[:, grp])
               for grp in _groups(mon.shape[1]) if np.abs(mon[:, grp]).max() > 0} if mon.size else {}
    print(f"\n{name} fp32 vs reference: slices " + " ".join(f"{e:.2e}" for e in errs) + "; " +
          ", ".join(f"{k} {v:.2e}" for k, v in mon_err.items()))
    assert all(np.isfinite(errs)) and all(np.isfinite(list(mon_err.values())))
    tail = errs[len(errs) // 2:]
    assert tail and max(tail) <= FP32_TOL, (name, errs)


def test_every_block_class_engages_in_the_mixed_case(tmp_path):
    """blocks_mixed: each code path of the sweeps has blocks, and (above) all
    of them together match the reference at 1e-10."""
    from php_fdtd_b200 import Config, Simulation
    d, _ = _inputs("blocks_mixed", tmp_path)
    with H.chdir(d):
        cfg = Config.load("case.cfg")
        medium = cfg.load_medium()
    for prec in ("fp64", "fp32"):
        sim = Simulation(cfg.desc(medium, prec))
        c = sim.block_census()
        sim.close()
        print(f"\nblocks_mixed {prec} census: {c}")
        for k in ("e_plain", "e_plain_cpml", "e_tensor", "e_atoms", "e_general", "h_plain", "h_general"):
            assert c[k] > 0, (prec, k, c)
        assert sum(c[k] for k in ("e_plain", "e_plain_cpml", "e_tensor", "e_atoms", "e_general")) == c["blocks"]
        assert c["h_plain"] + c["h_general"] == c["blocks"]
    sim = Simulation(cfg.desc(medium, "fp64-strict"))
    c = sim.block_census()
    sim.close()
    assert c["e_general"] == c["h_general"] == c["blocks"]
