"""Runs one case through the reference solver, the oracle restatement or the
CUDA path and returns the outputs in a common form:

  {"slices": {step: 2-D float64}, "monitor": [steps, cols], "full": [rows, cols],
   "source": [rows, cols], "diag": {step: dict}}

The reference writes its files into the case directory; the two in-process
runners reproduce the reference's output cadence and index conventions
(monitor fields at z+1 and atoms at z, z slices at position+1).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from contextlib import contextmanager
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

from php_fdtd_b200 import Config, Simulation  # noqa: E402
from php_fdtd_b200._abi import COMPONENTS  # noqa: E402


@contextmanager
def chdir(path):
    old = os.getcwd()
    os.chdir(path)
    try:
        yield
    finally:
        os.chdir(old)


def read_slice_file(path: Path, wide: bool) -> np.ndarray:
    raw = path.read_bytes()
    a, b = np.frombuffer(raw[:8], dtype=np.int32)
    data = np.frombuffer(raw[8:], dtype=np.float64 if wide else np.float32)
    assert data.size == a * b, (path, a, b, data.size)
    return data.reshape(a, b).astype(np.float64)


def read_table(path: Path) -> np.ndarray:
    if not path.exists():
        return np.zeros((0, 0))
    rows = [l.split() for l in path.read_text().splitlines() if l.strip() and not l.startswith("#")]
    return np.array(rows, dtype=np.float64) if rows else np.zeros((0, 0))


def collect_files(case_dir: Path, wide: bool) -> dict:
    out = {"slices": {}, "monitor": read_table(case_dir / "monitor_point.dat"),
           "full": read_table(case_dir / "full_monitor.dat"), "source": read_table(case_dir / "source.txt")}
    for p in sorted(case_dir.glob("field_slice_*.bin")):
        step = int(p.stem.rsplit("_", 1)[1])
        out["slices"][step] = read_slice_file(p, wide)
    return out


def clean_outputs(case_dir: Path):
    for p in list(case_dir.glob("field_slice_*.bin")) + [case_dir / n for n in
                                                         ("monitor_point.dat", "full_monitor.dat", "source.txt")]:
        if p.exists():
            p.unlink()


def run_reference(case_dir: Path, kind: str = "wide", timeout: int = 600, ranks: int = 1) -> dict:
    """kind: plain / wide / fast (one rank), mp / mp_wide (``ranks`` ranks
    through the shared-memory MPI stand-in)."""
    from oracle import reference_binary
    exe = reference_binary(kind)
    if not exe.exists():
        raise FileNotFoundError(exe)
    clean_outputs(case_dir)
    env = dict(os.environ, PHP_MPI_NP=str(ranks))
    p = subprocess.run([str(exe), "case.cfg"], cwd=case_dir, capture_output=True, text=True, timeout=timeout, env=env)
    res = collect_files(case_dir, wide=kind in ("wide", "mp_wide"))
    res["returncode"] = p.returncode
    res["stdout"] = p.stdout
    return res


def run_cli(case_dir: Path, precision: str = "fp64", timeout: int = 600) -> dict:
    exe = ROOT / "php_fdtd_b200" / "fdtd_b200"
    clean_outputs(case_dir)
    p = subprocess.run([str(exe), "case.cfg", precision], cwd=case_dir, capture_output=True, text=True, timeout=timeout)
    res = collect_files(case_dir, wide=False)
    res["returncode"] = p.returncode
    res["stdout"] = p.stdout + p.stderr
    return res


def run_inprocess(case_dir: Path, runner: str = "oracle", precision: str = "fp64-strict", steps: int | None = None,
                  threads: int = 0) -> dict:
    """runner 'oracle' (C restatement) or 'device' (libphpfdtd)."""
    with chdir(case_dir):
        cfg = Config.load("case.cfg")
        medium = cfg.load_medium()
        holder = cfg.desc(medium, precision)
        if runner == "oracle":
            from oracle import Oracle
            sim = Oracle(holder, threads=threads)
        else:
            sim = Simulation(holder)
    nx, ny, nz = cfg.nx, cfg.ny, cfg.nz
    oi, tsteps = cfg.output_interval, steps if steps is not None else cfg.tsteps
    comp = COMPONENTS.get(cfg.output_component, 0)
    axis, pos = cfg.output_slice_axis, cfg.output_slice_position
    mx, my, mz = cfg.monitor_x, cfg.monitor_y, cfg.monitor_z
    mon_ok = cfg.monitor_enabled and 0 <= mx < nx and 0 <= my < ny and 0 <= mz < nz
    mon_natom = int(cfg.materials[int(medium[mx, my, mz])].natom) if mon_ok else 0
    with_rv = mon_ok and cfg.monitor_atom < mon_natom
    full_on = cfg.full_monitor_enabled or (mon_ok and mon_natom > 0)
    res = {"slices": {}, "monitor": [], "full": [], "source": [], "diag": {}}
    for t in range(tsteps):
        sim.step(1)
        if t % oi == 0:
            res["diag"][t] = sim.diagnostics()
            try:
                res["slices"][t] = sim.read_slice(comp, axis, pos, f64=True)
            except Exception:
                pass
            if full_on and mon_ok:
                f9 = sim.read_point(mx, my, mz + 1)
                st = sim.read_cell_state(mx, my, mz)
                row = [t * cfg.dt, *f9]
                for a in range(st["natom"]):
                    row += list(st["r"][3 * a:3 * a + 3]) + list(st["v"][3 * a:3 * a + 3])
                res["full"].append(row)
        if mon_ok:
            f9 = sim.read_point(mx, my, mz + 1)
            row = [t * cfg.dt, *f9]
            if with_rv:
                st = sim.read_cell_state(mx, my, mz)
                q = cfg.monitor_atom * 3 + cfg.monitor_dir
                row += [st["r"][q], st["v"][q]]
            res["monitor"].append(row)
    res["monitor"] = np.array(res["monitor"]) if res["monitor"] else np.zeros((0, 0))
    res["full"] = np.array(res["full"]) if res["full"] else np.zeros((0, 0))
    res["sim"] = sim
    res["cfg"] = cfg
    return res


def rel_l2(a, b) -> float:
    """||a - b|| / ||b||; complex inputs keep their imaginary parts (a
    running-DFT accumulator is checked in amplitude and phase)."""
    a = np.asarray(a)
    b = np.asarray(b)
    if not (np.iscomplexobj(a) or np.iscomplexobj(b)):
        a = a.astype(np.float64)
        b = b.astype(np.float64)
    den = np.linalg.norm(b)
    num = np.linalg.norm(a - b)
    if den == 0.0:
        return 0.0 if num == 0.0 else float("inf")
    return float(num / den)


def copy_case(src: Path, dst: Path) -> Path:
    if dst.exists():
        shutil.rmtree(dst)
    shutil.copytree(src, dst)
    return dst
