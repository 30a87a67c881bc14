"""The one-launch step (he_sweep_tma: H, D, sources, E, ADE and ions of a
time step in one sweep, with E, H and the H CPML state double buffered)
against the two sweeps (the default; PHP_FUSED=1 at create selects the one
launch).  The arithmetic per cell is the same,
so every field, the CPML state, the ADE pools and the lattice state must come
out bit-identical: over odd and even step counts (the buffers swap every
step), step calls that split graph chunks, every block class of the sweeps
(blocks_mixed) and the golden cases' materials, sources and CPML layers.
"""
import os
from contextlib import contextmanager

import numpy as np
import pytest

import harness as H
from conftest import golden_cases
from php_fdtd_b200 import Config, Simulation
from php_fdtd_b200.workloads import parity_baseline_case, write_case

pytestmark = pytest.mark.gpu


@contextmanager
def _env(**kv):
    old = {k: os.environ.get(k) for k in kv}
    os.environ.update(kv)
    try:
        yield
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


def _pair(holder):
    """(one-launch step, two sweeps) contexts of one description"""
    with _env(PHP_FUSED="1"):
        a = Simulation(holder)
    with _env(PHP_FUSED="0"):
        b = Simulation(holder)
    return a, b


def _same(a, b, cfg, what):
    for comp in range(9):
        np.testing.assert_array_equal(a.read_volume(comp), b.read_volume(comp), err_msg=f"{what}: component {comp}")
    for cell in [(cfg.nx // 2, cfg.ny // 2, cfg.nz // 2), (1, 1, 1), (cfg.nx - 2, cfg.ny - 2, cfg.nz - 2)]:
        sa, sb = a.read_cell_state(*cell), b.read_cell_state(*cell)
        for k in sa:
            np.testing.assert_array_equal(np.asarray(sa[k]), np.asarray(sb[k]), err_msg=f"{what}: {k} at {cell}")


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("name", golden_cases())
def test_one_launch_step_equals_two_sweeps(name, precision, golden_case):
    with H.chdir(golden_case(name)):
        cfg = Config.load("case.cfg")
        holder = cfg.desc(cfg.load_medium(), precision)
    a, b = _pair(holder)
    try:
        a.step(7)
        b.step(7)
        _same(a, b, cfg, f"{name} {precision} after 7 steps")
        # one launch fewer per step (the ion pass of many-atom cells, where it
        # runs apart, is one more in both)
        assert b.last_launch_count - a.last_launch_count == 7
        a.step(6)
        a.step(1)
        b.step(7)
        _same(a, b, cfg, f"{name} {precision} after 14 steps")
    finally:
        a.close()
        b.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_every_block_class_and_graph_chunks(precision, tmp_path):
    """blocks_mixed (96 x 64 x 64: plain, plain with CPML, tensor, atom and
    general blocks in both parts of the step) over a step count that spans a
    recorded graph chunk (256 steps) and ends on an odd level"""
    d = tmp_path / "blocks_mixed"
    write_case(parity_baseline_case("blocks_mixed"), d)
    with H.chdir(d):
        cfg = Config.load("case.cfg")
        holder = cfg.desc(cfg.load_medium(), precision)
    a, b = _pair(holder)
    try:
        census = a.block_census()
        assert census["h_plain"] > 0 and census["e_plain"] > 0
        a.prepare(41)
        a.step(41)
        a.step(256)
        b.step(297)
        a.sync()
        b.sync()
        _same(a, b, cfg, f"blocks_mixed {precision} after 297 steps")
    finally:
        a.close()
        b.close()


def test_probe_and_dft_read_the_new_level(golden_case):
    """the probe rows and running DFT recorded after each one-launch step read
    the buffers that step wrote"""
    with H.chdir(golden_case("ade_metal")):
        cfg = Config.load("case.cfg")
        holder = cfg.desc(cfg.load_medium(), "fp64")
    a, b = _pair(holder)
    try:
        for s in (a, b):
            s.probe_set(cfg.nx // 2, cfg.ny // 2, cfg.nz // 2, cfg.nz // 2)
        pa = a.dft_add("Ez", cfg.nz // 2, [cfg.unique_source_frequency], first_step=0, interval=1, cast_f32=False)
        pb = b.dft_add("Ez", cfg.nz // 2, [cfg.unique_source_frequency], first_step=0, interval=1, cast_f32=False)
        a.step(9)
        b.step(9)
        np.testing.assert_array_equal(a.probe_read(), b.probe_read())
        np.testing.assert_array_equal(a.dft_read(pa)[0], b.dft_read(pb)[0])
    finally:
        a.close()
        b.close()


def test_profile_reports_the_one_launch_step(golden_case):
    """php_profile_read: the one-launch step under its own kind, no H or E
    sweep launches; the two sweeps under theirs"""
    with H.chdir(golden_case("vacuum_pml")):
        cfg = Config.load("case.cfg")
        holder = cfg.desc(cfg.load_medium(), "fp32")
    a, b = _pair(holder)
    try:
        for s in (a, b):
            s.profile(True)
            s.step(5)
        pa, pb = a.profile_read(), b.profile_read()
        assert pa["step"]["launches"] == 5 and pa["h_sweep"]["launches"] == 0 and pa["e_sweep"]["launches"] == 0
        assert pb["step"]["launches"] == 0 and pb["h_sweep"]["launches"] == 5 and pb["e_sweep"]["launches"] == 5
        assert pa["step"]["ms"] > 0 and pb["e_sweep"]["ms"] > 0
    finally:
        a.close()
        b.close()
