"""Generates the golden fixtures under tests/golden/<case>/.

For every parity case of php_fdtd_b200.workloads.SMALL_CASES this writes the
inputs (case.cfg, medium_map.bin, lattice / OUTCAR / dielectric files) and
runs the reference solver compiled from its own sources (oracle/_ref,
``make -C oracle ref``) twice:
  - the widened build (float64 slices, %.17e monitors): golden.npz
  - the plain build (the reference's exact file formats): plain/
so the fixtures hold the reference's own outputs on these inputs.

    python tests/golden/make_golden.py [case ...]
"""
from __future__ import annotations

import shutil
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

from php_fdtd_b200.workloads import SMALL_CASES, write_case  # noqa: E402
import harness as H  # noqa: E402


def make(name: str):
    d = HERE / name
    if d.exists():
        shutil.rmtree(d)
    spec = SMALL_CASES[name]
    write_case(spec, d)
    if spec.expect_abort:
        # the divergence abort: the plain outputs written before it and the
        # reference's report; no golden.npz (not a solver parity case)
        plain = H.run_reference(d, "plain")
        assert plain["returncode"] == 1, plain["stdout"][-2000:]
        assert "ERROR: r field too large" in plain["stdout"]
        pd = d / "plain"
        pd.mkdir()
        for p in list(d.glob("field_slice_*.bin")) + [d / n for n in ("monitor_point.dat", "full_monitor.dat", "source.txt")]:
            if p.exists():
                shutil.move(str(p), pd / p.name)
        (d / "reference_stdout.txt").write_text(plain["stdout"])
        print(f"{name}: abort, {len(list(pd.glob('field_slice_*')))} slices")
        return
    wide = H.run_reference(d, "wide")
    assert wide["returncode"] == 0, wide["stdout"][-2000:]
    steps = sorted(wide["slices"])
    np.savez_compressed(d / "golden.npz", slice_steps=np.array(steps, dtype=np.int64),
                        slices=np.stack([wide["slices"][s] for s in steps]) if steps else np.zeros((0, 0, 0)),
                        monitor=wide["monitor"], full=wide["full"], source=wide["source"])
    plain = H.run_reference(d, "plain")
    assert plain["returncode"] == 0
    pd = d / "plain"
    pd.mkdir()
    for p in list(d.glob("field_slice_*.bin")) + [d / n for n in ("monitor_point.dat", "full_monitor.dat", "source.txt")]:
        if p.exists():
            shutil.move(str(p), pd / p.name)
    (d / "reference_stdout.txt").write_text(plain["stdout"])
    print(f"{name}: {len(steps)} slices, monitor {wide['monitor'].shape}, full {wide['full'].shape}")


if __name__ == "__main__":
    for n in (sys.argv[1:] or list(SMALL_CASES)):
        make(n)
