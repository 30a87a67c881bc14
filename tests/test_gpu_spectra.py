"""Near-field spectra and the running DFT against the reference's own
post-processor (frequency_analysis.c, compiled unmodified against the FFTW
stand-in of oracle/fftw_stub), run on the reference's own slices of the
spectra_dft golden case (tests/golden/make_golden.py):

  - fdtd_b200 --spectra writes frequency_slice_*.txt from its running DFT;
    the files must match the post-processor's (golden post/) header for
    header and row for row, values within the %.6e text precision;
  - the running-DFT accumulators (php_dft_read, FP64 samples, no float32
    cast) over N samples, divided by N, must equal the post-processor's
    values on the reference's float64 slices (golden spectra.npz, printed
    %.17e) to relative L2 <= 1e-10, real and imaginary parts (amplitude and
    phase).
"""
import subprocess
from pathlib import Path

import numpy as np
import pytest

import harness as H
from oracle import spectra
from php_fdtd_b200 import Config, Simulation

pytestmark = pytest.mark.gpu
EXE = Path(__file__).resolve().parents[1] / "php_fdtd_b200" / "fdtd_b200"
CASE = "spectra_dft"


@pytest.mark.parametrize("precision,tol", [("fp64-strict", 2e-6), ("fp64", 2e-6), ("fp32", 1e-3)])
def test_spectra_files_match_the_reference_post_processor(precision, tol, golden_case):
    d = golden_case(CASE)
    r = subprocess.run([str(EXE), "case.cfg", precision, "--spectra"], cwd=d, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    want = sorted(p.name for p in (d / "post").glob("frequency_slice_*.txt"))
    got = sorted(p.name for p in d.glob("frequency_slice_*.txt"))
    assert got == want and len(got) == 9
    for name in want:
        head_ref, rows_ref = spectra.read_frequency_slice(d / "post" / name)
        head, rows = spectra.read_frequency_slice(d / name)
        assert head == head_ref, name
        assert rows.shape == rows_ref.shape
        np.testing.assert_array_equal(rows[:, :2], rows_ref[:, :2])
        scale = float(np.abs(rows_ref[:, 2:4]).max())
        assert float(np.abs(rows[:, 2:4] - rows_ref[:, 2:4]).max()) <= tol * scale, (name, precision)


def _crop(a):
    nx, ny = a.shape
    return np.array([a[i, j] for i in range(nx) for j in range(ny) if nx * 0.25 < i < nx * 0.75 and ny * 0.25 < j < ny * 0.75])


@pytest.mark.parametrize("precision", ["fp64-strict", "fp64"])
def test_running_dft_matches_the_reference_post_processor(precision, golden_case):
    d = golden_case(CASE)
    ref = np.load(d / "spectra.npz")
    with H.chdir(d):
        cfg = Config.load("case.cfg")
        sim = Simulation(cfg.desc(cfg.load_medium(), precision))
    oi = cfg.output_interval
    N = (cfg.tsteps - 1) // oi + 1
    times = [s * oi * cfg.dt for s in range(N)]
    fs = 1.0 / ((times[-1] - times[0]) / (N - 1))        # frequency_analysis.c:371-373
    idx = [int(k) for k in ref["index"]]
    freqs = [k * fs / N for k in idx]                     # frequency_analysis.c:381-390
    pid = sim.dft_add("Ez", cfg.output_slice_position + 1, freqs, first_step=0, interval=oi, cast_f32=False)
    sim.step(cfg.tsteps)
    acc, ns = sim.dft_read(pid)
    sim.close()
    assert ns == N
    worst = 0.0
    for q in range(len(idx)):
        got = _crop(acc[q] / N)
        rows = ref["rows"][q]
        want = rows[:, 2] + 1j * rows[:, 3]
        e = H.rel_l2(got, want)
        worst = max(worst, e)
        assert e <= 1e-10, (precision, idx[q], e)
        assert H.rel_l2(got.imag, want.imag) <= 1e-10, (precision, idx[q])
    print(f"\n{precision} running DFT vs reference post-processor: worst rel L2 {worst:.2e} over {len(idx)} bins")
