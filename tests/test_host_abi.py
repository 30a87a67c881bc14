"""CPU tests: the C ABI libraries load and export every declared entry
point, the ctypes layouts match, and the host layer parses inputs the way
the reference does (checked against the reference's own printout and
outputs stored in tests/golden)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, golden_cases
import harness as H
from php_fdtd_b200 import Config, PhpError, _abi


def declared_functions(header: Path):
    text = header.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:[A-Za-z_][\w\s\*]*?)\b(php_\w+|oracle_\w+)\s*\(", text, flags=re.M)
    return sorted(set(n for n in names if not n.startswith("php_") or not n.endswith("_H")))


@pytest.mark.parametrize("header,lib", [
    ("include/php_fdtd.h", "php_fdtd_b200/libphpfdtd.so"),
    ("include/php_serve.h", "php_fdtd_b200/libphpfdtd.so"),
    ("include/php_host.h", "php_fdtd_b200/libphphost.so"),
    ("oracle/php_oracle.h", "oracle/liboracle.so"),
])
def test_library_exports_every_declared_symbol(header, lib):
    names = declared_functions(ROOT / header)
    assert len(names) >= 5, names
    so = C.CDLL(str(ROOT / lib))  # loads without a GPU: the CUDA driver is only touched by php_create
    missing = [n for n in names if not hasattr(so, n)]
    assert not missing, f"{lib} lacks {missing}"


def test_ctypes_layouts_match_c():
    lib = _abi.host_lib()
    for name, st in _abi._STRUCTS.items():
        assert lib.php_host_sizeof(name.encode()) == C.sizeof(st), name


def test_device_calls_fail_without_device_or_with_bad_input():
    lib = _abi.device_lib()
    d = _abi.Desc()
    d.abi_version = 999
    ctx = C.c_void_p()
    rc = lib.php_create(C.byref(d), C.byref(ctx))
    assert rc == _abi.PHP_ERR_INPUT
    assert b"abi_version" in lib.php_last_error(None)
    assert lib.php_step(None, 1) == _abi.PHP_ERR_INPUT


@pytest.mark.parametrize("name", golden_cases())
def test_config_matches_reference_printout(name, golden_case):
    d = golden_case(name)
    with H.chdir(d):
        cfg = Config.load("case.cfg")
    out = (d / "reference_stdout.txt").read_text()
    m = re.search(r"Grid size: (\d+) x (\d+) x (\d+)", out)
    assert (cfg.nx, cfg.ny, cfg.nz) == tuple(map(int, m.groups()))
    m = re.search(r"Time steps: (\d+), dt=(\S+) s", out)
    assert cfg.tsteps == int(m.group(1)) and f"{cfg.dt:.4e}" == m.group(2)
    # material table as printed by the reference (fdtd.c:2827-2874)
    blocks = re.findall(r"Material (\d+): (\S.*)\n    Dielectric tensor \(real\):\n(.*)\n(.*)\n(.*)\n"
                        r"    Dielectric tensor \(imag\) should be >= 0:\n(.*)\n(.*)\n(.*)\n", out)
    assert len(blocks) == cfg.num_materials
    for b in blocks:
        mid = int(b[0])
        mat = cfg.materials[mid]
        assert mat.name.decode() == b[1].strip()
        re_rows = [list(map(float, r.strip()[1:-1].split(","))) for r in b[2:5]]
        im_rows = [list(map(float, r.strip()[1:-1].split(","))) for r in b[5:8]]
        for q in range(9):
            assert f"{mat.eps_re[q]:.4f}" == f"{re_rows[q // 3][q % 3]:.4f}"
            assert f"{mat.eps_im[q]:.4f}" == f"{im_rows[q // 3][q % 3]:.4f}"
    m = re.search(r"use_ADE: (\d+)", out)
    assert m


@pytest.mark.parametrize("name", golden_cases())
def test_source_values_match_reference_source_txt(name, golden_case):
    """source.txt rows (fdtd.c:3359-3400, widened to %.17e) equal the host
    waveform bit for bit."""
    d = golden_case(name)
    g = np.load(d / "golden.npz")
    with H.chdir(d):
        cfg = Config.load("case.cfg")
    src = g["source"]
    assert src.shape[0] == len(range(0, cfg.tsteps, cfg.output_interval))
    for row_i, t in enumerate(range(0, cfg.tsteps, cfg.output_interval)):
        assert src[row_i, 0] == t * cfg.dt
        for s in range(cfg.num_sources):
            assert src[row_i, 1 + s] == cfg.source_value(s, t * cfg.dt)


def test_plain_reference_files_use_float32_and_e_format():
    """The plain fixtures are the reference's own file formats: 2 int32 dims +
    float32 slices, %e monitor text (fdtd.c:1080-1093, 3839)."""
    d = GOLDEN / "vacuum_pml" / "plain"
    files = sorted(d.glob("field_slice_*.bin"))
    assert files
    raw = files[-1].read_bytes()
    a, b = np.frombuffer(raw[:8], dtype=np.int32)
    assert len(raw) == 8 + 4 * a * b
    line = (d / "monitor_point.dat").read_text().splitlines()[2]
    assert re.fullmatch(r"(-?\d\.\d{6}e[+-]\d\d\t){9}-?\d\.\d{6}e[+-]\d\d", line)


def test_cfg_errors_are_returned_not_exit(tmp_path):
    bad = tmp_path / "bad.cfg"
    bad.write_text("nx = 4\nny = 4\nnz = 4\nsource type=dipole, x=1,y=1,z=1, frequency=1e13, wavenumber=900\n")
    with pytest.raises(PhpError) as e:
        Config.load(str(bad))
    assert "both frequency and wavenumber" in str(e.value)
    with pytest.raises(PhpError):
        Config.load(str(tmp_path / "missing.cfg"))
    ok = tmp_path / "ok.cfg"
    ok.write_text("nx = 4\nny = 4\nnz = 4\nmaterial id=5, natom=2, QeZV=nope.txt\n")
    with pytest.raises(PhpError) as e:
        Config.load(str(ok))
    assert "nope.txt" in str(e.value) or "QeZM" in str(e.value)


def test_medium_dimension_mismatch(tmp_path):
    from php_fdtd_b200.workloads import write_medium
    write_medium(tmp_path / "m.bin", np.zeros((3, 4, 5), np.int32))
    cfgp = tmp_path / "c.cfg"
    cfgp.write_text("nx = 3\nny = 4\nnz = 6\nmedium_file = m.bin\n")
    with H.chdir(tmp_path):
        cfg = Config.load("c.cfg")
        with pytest.raises(PhpError) as e:
            cfg.load_medium()
    assert "do not match" in str(e.value)


def test_cfg_defaults_follow_reference_quirks(tmp_path):
    """Pass-one source defaults use the default grid (nx/2, ny/2, nz/3 of 50)
    and dt = -1 (fdtd.c:1420-1429, 1755); the slice position default is 25."""
    p = tmp_path / "q.cfg"
    p.write_text("nx = 10\nny = 12\nnz = 14\ndelta_x = 1e-8\ndelta_y = 1e-8\ndelta_z = 1e-8\n"
                 "source type=gaussian, component=x\n")
    cfg = Config.load(str(p))
    s = cfg.sources[0]
    assert (s.x, s.y, s.z) == (25, 25, 16)
    assert s.t0 == -40.0 and s.tau == -15.0
    assert s.end_time == cfg.tsteps * cfg.dt
    assert cfg.output_slice_position == 25
    assert cfg.dt == 1e-8 / (3e8 * np.sqrt(3.0)) * 0.99


def test_slab_parts_and_census_reject_bad_arguments():
    lib = _abi.device_lib()
    counts = (C.c_int64 * 8)()
    assert lib.php_step_part(None, 0, None) == _abi.PHP_ERR_INPUT
    assert lib.php_block_census(None, counts) == _abi.PHP_ERR_INPUT


def test_bench_bytes_count_p_ion_when_the_ion_pass_runs_apart(golden_case):
    """bench.py's algorithmic bytes: with the ion pass apart the fused sweep
    reads P_ion (3 words per atom cell) instead of r and v (12 N words)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench_mod", ROOT / "bench.py")
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    d = golden_case("ions16")
    with H.chdir(d):
        cfg = Config.load("case.cfg")
        medium = cfg.load_medium()
    c = bench.census(cfg, medium)
    assert c["atom_cells"] == int(np.sum(medium == 10)) and c["atom_words"] == 12 * 16 * c["atom_cells"]
    for s in (4, 8):
        h0, e0 = bench.algorithmic_bytes(c, s)
        h1, e1 = bench.algorithmic_bytes(c, s, ion_pass=True)
        assert h0 == h1
        assert e0 - e1 == s * (c["atom_words"] - 3 * c["atom_cells"])


def test_bench_rooflines_count_the_folded_dft(golden_case):
    """bench.py: with no dft_sample launch the E sweep's bytes include the
    running DFT it sampled itself (a word read and 32 bytes per frequency of
    each sampled cell); with the launches they do not."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench_mod", ROOT / "bench.py")
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    d = golden_case("ade_metal")
    with H.chdir(d):
        cfg = Config.load("case.cfg")
        medium = cfg.load_medium()
    c = bench.census(cfg, medium)
    prof = {k: {"ms": 0.1, "launches": 10} for k in ("h_sweep", "e_sweep", "probe", "dft", "ion")}
    prof["step"] = {"ms": 0.0, "launches": 0}
    launched = bench.sweep_rooflines(prof, c, 8, 6500.0, dft_cells=300, dft_freqs=3)
    prof["dft"]["launches"] = 0
    folded = bench.sweep_rooflines(prof, c, 8, 6500.0, dft_cells=300, dft_freqs=3)
    assert set(folded) == {"e_sweep", "h_sweep"}
    de = folded["e_sweep"]["algorithmic_bytes_per_launch"] - launched["e_sweep"]["algorithmic_bytes_per_launch"]
    assert de == 300 * (8 + 32 * 3)
    assert folded["h_sweep"] == launched["h_sweep"]
