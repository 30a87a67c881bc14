"""Running-DFT planes of E and D components are sampled by the E sweep itself
(after each block's z march, from the values it stored) instead of by a
dft_sample launch per plane and step; PHP_DFT_FOLD=0 at create keeps the
launches.  Both take the same samples with the same arithmetic, so the
accumulators must be bit-identical: E and D components, several planes (one
on a z-chunk boundary), sampling from a later step every few steps, the
float32 cast, FP64, FP32 and strict, z slabs and the one-launch step.  H
planes still take the launch.  The monitor row likewise (PHP_PROBE_FOLD=0
keeps probe_record_counted) where its field and atom cells share a z chunk.
"""
import os
from contextlib import contextmanager

import numpy as np
import pytest

import harness as H
from php_fdtd_b200 import Config, Simulation
from php_fdtd_b200.slab import LocalSlabs

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


def _planes(cfg):
    f = cfg.unique_source_frequency
    return [("Ez", cfg.nz // 2, [f, 1.3 * f], 0, 1, True),
            ("Dx", 4, [0.7 * f], 3, 2, False),      # plane 4: the first plane of a z chunk of 4
            ("Ex", cfg.nz - 2, [f], 1, 3, False),
            ("Hy", cfg.nz // 2, [f], 0, 1, False)]  # an H plane: a dft_sample launch either way


def _run(holder, cfg, steps, **env):
    with _env(**env):
        sim = Simulation(holder)
    ids = [sim.dft_add(c, z, fr, first_step=s0, interval=iv, cast_f32=cast) for c, z, fr, s0, iv, cast in _planes(cfg)]
    sim.step(steps[0])
    sim.step(steps[1])
    out = [sim.dft_read(p) for p in ids]
    launches = sim.last_launch_count
    sim.close()
    return out, launches


@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp64-strict"])
@pytest.mark.parametrize("name", ["ade_metal", "ions2", "lossy_rot"])
def test_folded_dft_equals_the_launched_samples(name, precision, golden_case):
    with H.chdir(golden_case(name)):
        cfg = Config.load("case.cfg")
        holder = cfg.desc(cfg.load_medium(), precision)
    holder.desc.z_chunk = 4
    folded, n_f = _run(holder, cfg, (9, 8), PHP_DFT_FOLD="1")
    launched, n_l = _run(holder, cfg, (9, 8), PHP_DFT_FOLD="0")
    for q, ((acc_f, ns_f), (acc_l, ns_l)) in enumerate(zip(folded, launched)):
        assert ns_f == ns_l > 0, q
        np.testing.assert_array_equal(acc_f, acc_l, err_msg=f"plane {q}")
    assert np.abs(folded[0][0]).max() > 0
    # the three E and D planes no longer launch (8 steps in the last call)
    assert n_l - n_f == 8 * 3


@pytest.mark.parametrize("fused", ["1", "0"])
def test_folded_dft_in_slabs_and_the_one_launch_step(fused, golden_case):
    with H.chdir(golden_case("ade_metal")):
        cfg = Config.load("case.cfg")
        holder = cfg.desc(cfg.load_medium(), "fp64")
    holder.desc.z_chunk = 3
    launched, _ = _run(holder, cfg, (6, 5), PHP_DFT_FOLD="0")
    with _env(PHP_FUSED=fused):
        one, _ = _run(holder, cfg, (6, 5), PHP_DFT_FOLD="1")
    for q in range(4):
        np.testing.assert_array_equal(one[q][0], launched[q][0], err_msg=f"one domain, plane {q}")
    slabs = LocalSlabs(holder, 2)
    c, z, fr, s0, iv, cast = _planes(cfg)[0]
    owner = [s for s in slabs.slabs if s.z0 <= z < s.z0 + s.nz][0]
    pid = owner.dft_add(c, z - owner.z0, fr, first_step=s0, interval=iv, cast_f32=cast)
    slabs.step(11)
    acc, ns = owner.dft_read(pid)
    slabs.close()
    assert ns == launched[0][1]
    np.testing.assert_array_equal(acc, launched[0][0])


def _probe_rows(holder, cell, steps, **env):
    with _env(**env):
        sim = Simulation(holder)
    sim.probe_set(*cell)
    sim.step(steps)
    rows = sim.probe_read()
    launches = sim.last_launch_count
    sim.close()
    return rows, launches


@pytest.mark.parametrize("precision", ["fp64", "fp32", "fp64-strict"])
@pytest.mark.parametrize("name,kf,ka", [("ions2", 9, 8), ("ions2", 8, 7), ("ade_metal", 5, 5), ("ions2", 16, 15),
                                        ("ions16", 9, 8)])
def test_monitor_row_recorded_by_the_sweep_equals_the_probe_launch(name, kf, ka, precision, golden_case):
    """The monitor row (fields at k_field, r and v at k_atom) recorded by the
    E sweep after its march equals probe_record_counted's: field and atom cell
    in one z chunk of 4 planes (recorded by the sweep), in two chunks (8 / 7)
    and the field cell on the high halo plane (16 of 16; both keep the
    launch), and the many-atom lattice whose ion pass runs apart (launch)."""
    with H.chdir(golden_case(name)):
        cfg = Config.load("case.cfg")
        holder = cfg.desc(cfg.load_medium(), precision)
    holder.desc.z_chunk = 4
    cell = (cfg.nx // 2, cfg.ny // 2, kf, ka)
    folded, n_f = _probe_rows(holder, cell, 13, PHP_PROBE_FOLD="1")
    launched, n_l = _probe_rows(holder, cell, 13, PHP_PROBE_FOLD="0")
    assert folded.shape == launched.shape and folded.shape[0] == 13
    np.testing.assert_array_equal(folded, launched)
    # ions16 runs its ion pass apart, except in the strict mode
    same_chunk = kf < cfg.nz and kf // 4 == ka // 4 and (name != "ions16" or precision == "fp64-strict")
    assert n_l - n_f == (13 if same_chunk else 0)


def test_monitor_row_of_the_one_launch_step(golden_case):
    with H.chdir(golden_case("ions2")):
        cfg = Config.load("case.cfg")
        holder = cfg.desc(cfg.load_medium(), "fp64")
    holder.desc.z_chunk = 4
    cell = (cfg.nx // 2, cfg.ny // 2, 9, 8)
    launched, _ = _probe_rows(holder, cell, 11, PHP_PROBE_FOLD="0")
    one, n = _probe_rows(holder, cell, 11, PHP_PROBE_FOLD="1", PHP_FUSED="1")
    np.testing.assert_array_equal(one, launched)
    assert n == 11  # the one launch per step, nothing else
