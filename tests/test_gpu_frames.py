"""Asynchronous output frames (php_frame_begin / wait / release) and the
drop-in executable's writer thread built on them.

  - a frame holds exactly what the synchronous reads return at that step
    (diagnostics, slice, probe rows, point and cell state);
  - frames taken while the device runs ahead come back in order, each with
    the state of its own step;
  - fdtd_b200 writes the same files with its writer thread as with
    --sync-output, and both match the reference byte for byte;
  - the divergence abort (fdtd.c:3626-3668) prints the reference's report,
    from the frame of the aborting step, and leaves the reference's files.
"""
from __future__ import annotations

import filecmp
import subprocess

import numpy as np
import pytest

import harness as H
from conftest import golden_cases
from php_fdtd_b200 import Config, Simulation

pytestmark = pytest.mark.gpu


def _sim(d, precision="fp64-strict"):
    with H.chdir(d):
        cfg = Config.load("case.cfg")
        holder = cfg.desc(cfg.load_medium(), precision)
        sim = Simulation(holder)
    return cfg, sim


@pytest.mark.parametrize("name", ["ions2", "ade_metal", "lossy_rot"])
def test_frame_equals_synchronous_reads(name, golden_case):
    d = golden_case(name)
    cfg, a = _sim(d)
    _, b = _sim(d)
    mx, my, mz = cfg.monitor_x, cfg.monitor_y, cfg.monitor_z
    for s in (a, b):
        s.probe_set(mx, my, mz + 1, mz)
    axis, pos = cfg.output_slice_axis, cfg.output_slice_position
    comp = cfg.output_component
    for chunk in (1, 7, 12):
        a.step(chunk)
        b.step(chunk)
        tk = a.frame_begin(diag=True, slice=(comp, axis, pos), probe=True, point=(mx, my, mz + 1), cell=(mx, my, mz))
        fr = a.frame_wait(tk)
        assert fr["step"] == b.t
        assert fr["diag"] == b.diagnostics()
        np.testing.assert_array_equal(fr["slice"], b.read_slice(comp, axis, pos).ravel())
        np.testing.assert_array_equal(fr["rows"], b.probe_read())
        np.testing.assert_array_equal(fr["point"], b.read_point(mx, my, mz + 1))
        st = b.read_cell_state(mx, my, mz)
        assert fr["cell"]["natom"] == st["natom"]
        np.testing.assert_array_equal(fr["cell"]["r"], st["r"])
        np.testing.assert_array_equal(fr["cell"]["v"], st["v"])
        dg = fr["diag"]
        if dg["max_r"] > 0:
            i, j, k = dg["argmax_r"][:3]
            np.testing.assert_array_equal(fr["diag_cell"]["point"], b.read_point(i, j, k))
            st = b.read_cell_state(i, j, k)
            np.testing.assert_array_equal(fr["diag_cell"]["r"], st["r"])
            np.testing.assert_array_equal(fr["diag_cell"]["v"], st["v"])
    a.close()
    b.close()


def test_frames_in_flight_keep_their_steps(golden_case):
    """Three frames taken back to back while the device runs ahead: each
    holds its own step's slice and probe rows."""
    d = golden_case("ions2")
    cfg, a = _sim(d, "fp64")
    _, b = _sim(d, "fp64")
    mx, my, mz = cfg.monitor_x, cfg.monitor_y, cfg.monitor_z
    for s in (a, b):
        s.probe_set(mx, my, mz + 1, mz)
    tickets = []
    for n in (3, 5, 4):
        a.step(n)
        tickets.append(a.frame_begin(slice=("Ez", "z", 5), probe=True))
    ref = []
    for n in (3, 5, 4):
        b.step(n)
        ref.append((b.read_slice("Ez", "z", 5).ravel(), b.probe_read()))
    for tk, (sl, rows) in zip(tickets, ref):
        fr = a.frame_wait(tk)
        np.testing.assert_array_equal(fr["slice"], sl)
        np.testing.assert_array_equal(fr["rows"], rows)
    a.close()
    b.close()


def _cli(d, *args):
    exe = H.ROOT / "php_fdtd_b200" / "fdtd_b200"
    H.clean_outputs(d)
    p = subprocess.run([str(exe), "case.cfg", *args], cwd=d, capture_output=True, text=True, timeout=600)
    files = {f.name: f.read_bytes() for f in sorted(d.iterdir())
             if f.name.startswith("field_slice_") or f.name in ("monitor_point.dat", "full_monitor.dat", "source.txt")}
    return p, files


@pytest.mark.parametrize("name", [n for n in golden_cases() if n in ("ions2", "ade_metal", "multi_source_ragged")])
def test_writer_thread_matches_sync_output(name, golden_case):
    d = golden_case(name)
    p1, f1 = _cli(d, "fp64-strict")
    p2, f2 = _cli(d, "fp64-strict", "--sync-output")
    assert p1.returncode == 0 and p2.returncode == 0, (p1.stdout + p1.stderr)[-2000:]
    assert f1.keys() == f2.keys()
    for k in f1:
        assert f1[k] == f2[k], k


def _report(text):
    lines = text.splitlines()
    i = next(n for n, l in enumerate(lines) if l.startswith("ERROR: r field too large"))
    return lines[i:i + 6]


@pytest.mark.parametrize("mode", [(), ("--sync-output",)])
def test_divergence_abort_matches_reference(mode, golden_case):
    d = golden_case("ions2_diverge")
    p, _ = _cli(d, "fp64-strict", *mode)
    assert p.returncode == 1, (p.stdout + p.stderr)[-2000:]
    ref = (d / "reference_stdout.txt").read_text()
    assert _report(p.stdout) == _report(ref)
    plain = d / "plain"
    for f in plain.iterdir():
        assert filecmp.cmp(d / f.name, f, shallow=False), f.name
    assert sorted(x.name for x in d.glob("field_slice_*")) == sorted(x.name for x in plain.glob("field_slice_*"))
