"""Generates the golden fixtures under tests/golden/<case>/.

For every parity case of php_fdtd_b200.workloads.SMALL_CASES this writes the
inputs (case.cfg, medium_map.bin, lattice / OUTCAR / dielectric files) and
runs the reference solver compiled from its own sources (oracle/_ref,
``make -C oracle ref``) twice:
  - the widened build (float64 slices, %.17e monitors): golden.npz
  - the plain build (the reference's exact file formats): plain/
so the fixtures hold the reference's own outputs on these inputs.

The parity cases at the benchmark workloads' sizes
(php_fdtd_b200.workloads.PARITY_BASELINE_CASES) go to
tests/golden/baseline/<case>/: their inputs (up to 268 MB of medium map) are
not committed but regenerated from the seeded generator by the tests, so
golden.npz holds the SHA-256 of every input file beside the reference's wide
outputs.  The large ones run through the multi-rank reference build
(fdtd_ref_mp_wide, the shared-memory MPI stand-in): its ranks split z as the
reference does, and the ranks are chosen so that no output plane sits at a
rank's top plane (where the reference reads a neighbour's halo for its z
slice and monitor); on such planes its outputs equal the one-rank run's
byte for byte.

    python tests/golden/make_golden.py [case ...]
    python tests/golden/make_golden.py --baseline [case ...]
"""
from __future__ import annotations

import hashlib
import json
import shutil
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

from php_fdtd_b200.workloads import (PARITY_BASELINE_CASES, SMALL_CASES, parity_baseline_case,  # noqa: E402
                                     write_case)
import harness as H  # noqa: E402

# reference ranks per baseline case (1 = the one-rank wide build)
BASELINE_RANKS = {"cfg0_full": 1, "cfg1_200": 1, "cfg2_200": 8, "cfg4_half_200": 8, "blocks_mixed": 1}


def input_hashes(d: Path) -> dict:
    return {p.name: hashlib.sha256(p.read_bytes()).hexdigest() for p in sorted(d.iterdir()) if p.is_file()}


def make_baseline(name: str):
    spec = parity_baseline_case(name)
    out = HERE / "baseline" / name
    out.mkdir(parents=True, exist_ok=True)
    ranks = BASELINE_RANKS[name]
    with tempfile.TemporaryDirectory(prefix=f"golden_{name}_") as tmp:
        work = Path(tmp)
        write_case(spec, work)
        hashes = input_hashes(work)
        t0 = time.time()
        res = H.run_reference(work, "wide" if ranks == 1 else "mp_wide", timeout=6 * 3600, ranks=ranks)
        assert res["returncode"] == 0, res["stdout"][-2000:]
        steps = sorted(res["slices"])
        np.savez_compressed(out / "golden.npz", slice_steps=np.array(steps, dtype=np.int64),
                            slices=np.stack([res["slices"][s] for s in steps]), monitor=res["monitor"],
                            full=res["full"], source=res["source"], inputs=json.dumps(hashes), ranks=ranks)
        lines = res["stdout"].splitlines()
        (out / "reference_stdout_tail.txt").write_text("\n".join(lines[-40:]) + "\n")
    print(f"{name}: {len(steps)} slices, monitor {res['monitor'].shape}, full {res['full'].shape}, "
          f"{ranks} rank(s), {time.time() - t0:.0f} s")


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
    if name in POST_CASES:
        post(d, wide)
    print(f"{name}: {len(steps)} slices, monitor {wide['monitor'].shape}, full {wide['full'].shape}")


# cases whose slices also go through the reference's post-processor
POST_CASES = ("spectra_dft",)


def post(d: Path, wide: dict):
    """The reference's post-processor (frequency_analysis.c) on the
    reference's own slices of case d: on the float32 files (its frequency
    slice files, committed under post/) and on float64 ones (its %.17e
    values of every written row, spectra.npz)."""
    import subprocess
    from oracle import reference_binary
    pd = d / "post"
    pd.mkdir()
    for p in (d / "plain").glob("field_slice_*.bin"):
        shutil.copy(p, pd / p.name)
    shutil.copy(d / "case.cfg", pd / "case.cfg")
    r = subprocess.run([str(reference_binary("post")), "case.cfg"], cwd=pd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    (pd / "post_stdout.txt").write_text(r.stdout)
    for p in list(pd.glob("field_slice_*.bin")) + [pd / "case.cfg"]:
        p.unlink()
    with tempfile.TemporaryDirectory(prefix="post_wide_") as tmp:
        w = Path(tmp)
        for step, a in wide["slices"].items():
            n0, n1 = a.shape
            name = next(p.name for p in (d / "plain").glob(f"field_slice_*_{step:08d}.bin"))
            (w / name).write_bytes(np.array([n0, n1], np.int32).tobytes() + np.ascontiguousarray(a).tobytes())
        shutil.copy(d / "case.cfg", w / "case.cfg")
        r = subprocess.run([str(reference_binary("post_wide")), "case.cfg"], cwd=w, capture_output=True, text=True)
        assert r.returncode == 0, r.stdout + r.stderr
        names, index, freq, rows = [], [], [], []
        for p in sorted(w.glob("frequency_slice_*.txt"), key=lambda q: int(q.name.split("_")[2])):
            names.append(p.name)
            index.append(int(p.name.split("_")[2]))
            head = [l for l in p.read_text().splitlines() if l.startswith("#")]
            freq.append(float(head[0].split()[4]))
            rows.append(np.array([[float(x) for x in l.split()] for l in p.read_text().splitlines()
                                  if l.strip() and not l.startswith("#")]))
        np.savez_compressed(d / "spectra.npz", names=np.array(names), index=np.array(index), freq=np.array(freq),
                            rows=np.stack(rows))


if __name__ == "__main__":
    args = sys.argv[1:]
    if args and args[0] == "--baseline":
        for n in (args[1:] or list(PARITY_BASELINE_CASES)):
            make_baseline(n)
    else:
        for n in (args or list(SMALL_CASES)):
            make(n)
