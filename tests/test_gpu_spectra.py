"""Near-field spectra (fdtd_b200 --spectra): the frequency_slice_*.txt files
the solver writes from its running DFT, against the reference's
post-processor restated with NumPy's FFT over the slice files of the same
run (oracle/spectra.py)."""
import math
import subprocess
from pathlib import Path

import numpy as np
import pytest

from oracle import spectra
from php_fdtd_b200.workloads import CaseSpec, write_case

pytestmark = pytest.mark.gpu
EXE = Path(__file__).resolve().parents[1] / "php_fdtd_b200" / "fdtd_b200"


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_spectra_match_the_post_processor(precision, tmp_path):
    dl = 10e-9
    dt = dl / (299792458.0 * math.sqrt(3.0)) * 0.99
    spec = CaseSpec("spectra", 24, 22, 20, 201, delta=(dl, dl, dl), pml=4, output_interval=2,
                    output_component="Ez", slice_axis="z", slice_pos=9, dt=dt,
                    sources=["type=sinusoidal, x=12,y=11,z=13, amplitude=1.0, frequency=1.2e15, component=z"],
                    materials=["id=4, name=slab, eps_xx=4.0, eps_yy=4.0, eps_zz=3.0"],
                    medium_fn=lambda nx, ny, nz: np.pad(np.full((nx, ny, 4), 4, np.int32), ((0, 0), (0, 0), (0, nz - 4))))
    write_case(spec, tmp_path)
    r = subprocess.run([str(EXE), "case.cfg", precision, "--spectra"], cwd=tmp_path, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    text = (tmp_path / "case.cfg").read_text()
    want = spectra.analyse(tmp_path, dt, spectra.source_frequency(text))
    got = sorted(p.name for p in tmp_path.glob("frequency_slice_*.txt"))
    assert got == sorted(want) and len(got) == 9
    for name, (f, k, fs, N, re, im) in want.items():
        head, rows = spectra.read_frequency_slice(tmp_path / name)
        assert head[0] == f"# Frequency slice at {f:.3e} Hz (index: {k})"
        assert head[4] == f"#   Time points: {N}"
        exp = spectra.expected_rows(spec.nx, spec.ny, re, im)
        assert rows.shape == exp.shape
        np.testing.assert_array_equal(rows[:, :2], exp[:, :2])
        scale = max(float(np.abs(exp[:, 2:4]).max()), 1e-30)
        # %.6e text against the FFT of the same float32 samples
        assert float(np.abs(rows[:, 2:4] - exp[:, 2:4]).max()) <= 2e-6 * scale, name
