"""GPU tests of the read-out paths and the C ABI behaviour against the
oracle restatement (itself bit-identical to the reference)."""
import numpy as np
import pytest

from conftest import golden_cases
import harness as H
from php_fdtd_b200 import Config, PhpError, Simulation
from oracle import Oracle

pytestmark = pytest.mark.gpu


def _pair(d, precision="fp64-strict"):
    with H.chdir(d):
        cfg = Config.load("case.cfg")
        medium = cfg.load_medium()
        holder = cfg.desc(medium, precision)
        return cfg, Simulation(holder), Oracle(holder)


@pytest.mark.parametrize("name", ["ions2", "ade_metal", "lossy_rot", "multi_source_ragged"])
def test_full_state_bitwise_after_steps(name, golden_case):
    """Every field component, ADE current and ion coordinate of every cell."""
    cfg, sim, orc = _pair(golden_case(name))
    sim.step(17)
    orc.step(17)
    for comp in range(9):
        np.testing.assert_array_equal(sim.read_volume(comp), orc.read_volume(comp), err_msg=f"component {comp}")
    medium = cfg.load_medium() if False else None
    for (i, j, k) in [(0, 0, 0), (cfg.nx // 2, cfg.ny // 2, 2), (cfg.nx // 2, cfg.ny // 2, cfg.nz // 3),
                      (cfg.nx - 1, cfg.ny - 1, cfg.nz - 1), (5, 6, 4)]:
        a, b = sim.read_cell_state(i, j, k), orc.read_cell_state(i, j, k)
        assert a["natom"] == b["natom"]
        np.testing.assert_array_equal(a["r"], b["r"])
        np.testing.assert_array_equal(a["v"], b["v"])
        np.testing.assert_array_equal(a["P"], b["P"])
        np.testing.assert_array_equal(a["P_old"], b["P_old"])


@pytest.mark.parametrize("precision", ["fp64-strict", "fp64", "fp32"])
def test_chunked_stepping_equals_single_steps(precision, golden_case):
    """Graph replays of different chunk lengths advance the same state."""
    d = golden_case("ions2")
    with H.chdir(d):
        cfg = Config.load("case.cfg")
        holder = cfg.desc(cfg.load_medium(), precision)
    a, b = Simulation(holder), Simulation(holder)
    a.step(23)
    for n in (1, 5, 1, 16):
        b.step(n)
    assert a.t == b.t == 23
    for comp in range(9):
        np.testing.assert_array_equal(a.read_volume(comp), b.read_volume(comp))


def test_slices_every_axis_component_and_top_plane(golden_case):
    cfg, sim, orc = _pair(golden_case("aniso_lossy"))
    sim.step(12)
    orc.step(12)
    for comp in list(range(9)) + [9]:
        for axis, n in (("x", cfg.nx), ("y", cfg.ny), ("z", cfg.nz)):
            for pos in (0, n // 2, n - 1):
                ref = orc.read_slice(comp, axis, pos)
                np.testing.assert_array_equal(sim.read_slice(comp, axis, pos, f64=True), ref)
                np.testing.assert_array_equal(sim.read_slice(comp, axis, pos), ref.astype(np.float32))
    # z = nz-1 reads the zero halo plane, as a single-rank reference run does
    assert not sim.read_slice("Ez", "z", cfg.nz - 1, f64=True).any()
    for axis, bad in (("x", cfg.nx), ("y", -1), ("z", cfg.nz), ("q", 0)):
        with pytest.raises(PhpError) as e:
            sim.read_slice("Ex", axis, bad)
        assert e.value.code == -1


@pytest.mark.parametrize("name", ["ions2", "ions16"])
def test_diagnostics_and_argmax(name, golden_case):
    cfg, sim, orc = _pair(golden_case(name))
    for n in (1, 9, 10):
        sim.step(n)
        orc.step(n)
        a, b = sim.diagnostics(), orc.diagnostics()
        assert a["max_e"] == b["max_e"] and a["max_ex"] == b["max_ex"] and a["max_r"] == b["max_r"]
        assert a["argmax_r"] == b["argmax_r"]


def test_diagnostics_without_atoms_report_no_argmax(golden_case):
    cfg, sim, orc = _pair(golden_case("vacuum_pml"))
    sim.step(5)
    orc.step(5)
    a, b = sim.diagnostics(), orc.diagnostics()
    assert a == b and a["argmax_r"] == (-1, -1, -1, -1, -1)


def test_probe_rows_match_point_reads(golden_case):
    cfg, sim, orc = _pair(golden_case("ions2"))
    sim.probe_set(8, 8, 5, 4)
    rows = []
    for n in (3, 1, 6):
        sim.step(n)
        rows.append(sim.probe_read())
    rows = np.concatenate(rows)
    assert rows.shape == (10, 9 + 12)
    for t in range(10):
        orc.step(1)
        np.testing.assert_array_equal(rows[t, :9], orc.read_point(8, 8, 5))
        st = orc.read_cell_state(8, 8, 4)
        np.testing.assert_array_equal(rows[t, 9:15], st["r"])
        np.testing.assert_array_equal(rows[t, 15:21], st["v"])


def test_running_dft_matches_direct_sum(golden_case):
    """F(f) = sum_t x(t) exp(-2 pi i f t dt) over the samples taken, the sum
    frequency_analysis.c evaluates with FFTW (frequency_analysis.c:548-570)."""
    cfg, sim, orc = _pair(golden_case("vacuum_pml"))
    z = 7
    freqs = [1370 * 0.03e12, 1.1e13, 4.4e13]
    pid = sim.dft_add("Ez", z, freqs, first_step=2, interval=3)
    pid32 = sim.dft_add("Ex", z, freqs[:1], first_step=0, interval=1, cast_f32=True)
    acc = np.zeros((3, cfg.nx, cfg.ny), complex)
    acc32 = np.zeros((1, cfg.nx, cfg.ny), complex)
    n = 0
    for t in range(40):
        orc.step(1)
        plane = orc.read_volume("Ez")[:, :, z]
        if t >= 2 and (t - 2) % 3 == 0:
            n += 1
            for q, f in enumerate(freqs):
                acc[q] += plane * np.exp(-2j * np.pi * f * (t * cfg.dt))
        p32 = orc.read_volume("Ex")[:, :, z].astype(np.float32).astype(np.float64)
        acc32[0] += p32 * np.exp(-2j * np.pi * freqs[0] * (t * cfg.dt))
    sim.step(17)
    sim.step(23)
    got, ns = sim.dft_read(pid)
    assert ns == n
    assert np.iscomplexobj(got) and np.abs(acc.imag).max() > 0
    assert H.rel_l2(got, acc) < 1e-12
    # the sine part on its own: its sign is the transform's direction
    assert H.rel_l2(got.imag, acc.imag) < 1e-12
    got32, _ = sim.dft_read(pid32)
    assert H.rel_l2(got32, acc32) < 1e-12
    assert H.rel_l2(got32.imag, acc32.imag) < 1e-12


def test_device_rejects_bad_descriptions(golden_case):
    d = golden_case("vacuum_pml")
    with H.chdir(d):
        cfg = Config.load("case.cfg")
        medium = cfg.load_medium()
    bad = medium.copy()
    bad[1, 1, 1] = 99
    with pytest.raises(PhpError) as e:
        Simulation(cfg.desc(bad, "fp64"))
    assert e.value.code == -1 and "outside the material table" in str(e.value)
    holder = cfg.desc(medium, "fp64")
    holder.desc.dt = -1.0
    with pytest.raises(PhpError):
        Simulation(holder)


def test_launch_count_and_memory(golden_case):
    d = golden_case("ions2")
    with H.chdir(d):
        cfg = Config.load("case.cfg")
        sim = Simulation(cfg.desc(cfg.load_medium(), "fp64"))
    sim.step(7)
    assert sim.last_launch_count == 14
    assert sim.memory_bytes > 9 * cfg.nx * cfg.ny * cfg.nz * 8
