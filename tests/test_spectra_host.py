"""Host side of the near-field spectra: the source frequency and DFT bins the
solver picks (php_spectra_source_frequency / php_spectra_bins) equal those of
the reference's post-processor as restated in oracle/spectra.py."""
import ctypes as C
import math

import numpy as np
import pytest

from oracle import spectra
from php_fdtd_b200 import _abi


def _bins(n, interval, dt, f):
    lib = _abi.host_lib()
    idx = (C.c_int32 * 9)()
    fr = (C.c_double * 9)()
    fs = C.c_double()
    k = lib.php_spectra_bins(n, interval, dt, f, idx, fr, C.byref(fs))
    return list(idx[:k]), list(fr[:k]), fs.value


@pytest.mark.parametrize("n,interval,f", [(101, 2, 1.2e15), (6, 10, 4.1e13), (400, 20, 2.7e13), (2, 5, 1e14),
                                          (1000, 1, 9e15)])
def test_bins_follow_the_post_processor(n, interval, f):
    dt = 1.9e-17
    idx, fr, fs = _bins(n, interval, dt, f)
    times = [s * interval * dt for s in range(n)]
    fs_ref = 1.0 / ((times[-1] - times[0]) / (n - 1))
    target = min(range(n // 2), key=lambda i: (abs(i * fs_ref / n - f), i))
    want = [target + o for o in range(-4, 5) if 0 <= target + o < n // 2]
    assert idx == want and fs == fs_ref
    assert fr == [k * fs_ref / n for k in want]


def test_source_frequency_from_cfg(tmp_path):
    p = tmp_path / "c.cfg"
    text = ("[grid]\nnx = 4\n# source type=sinusoidal, frequency=9e9\n"
            "source type=sinusoidal, x=1,y=1,z=1, frequency=1.2e15, component=z\n"
            "source type=dipole, x=1,y=1,z=1, wavenumber=1370, component=x\n"
            "source type=gaussian, x=1,y=1,z=1, component=x\n")
    p.write_text(text)
    v, dt = C.c_double(), C.c_double()
    assert _abi.host_lib().php_spectra_config(str(p).encode(), C.byref(v), C.byref(dt)) == 0
    assert v.value == spectra.source_frequency(text) == 1370 * 0.03e12
    assert dt.value == -1.0
    p.write_text(text + "dt = 1.5e-17\n")
    assert _abi.host_lib().php_spectra_config(str(p).encode(), C.byref(v), C.byref(dt)) == 0
    assert dt.value == 1.5e-17
    p.write_text("source type=gaussian, x=1\n")
    assert _abi.host_lib().php_spectra_config(str(p).encode(), C.byref(v), C.byref(dt)) != 0


def test_numpy_restatement_matches_the_reference_post_processor():
    """oracle/spectra.py (the NumPy restatement) on the reference's own
    float32 slices of the spectra_dft case gives the rows the reference's
    post-processor (frequency_analysis.c, built against the FFTW stand-in)
    wrote for them: same files, headers and indices, values within the
    %.6e text precision."""
    from conftest import GOLDEN
    d = GOLDEN / "spectra_dft"
    text = (d / "case.cfg").read_text()
    dt = float(next(l.split("=", 1)[1] for l in text.splitlines() if l.startswith("dt")))
    want = spectra.analyse(d / "plain", dt, spectra.source_frequency(text))
    ref = sorted(p.name for p in (d / "post").glob("frequency_slice_*.txt"))
    assert sorted(want) == ref and len(ref) == 9
    for name, (f, k, fs, N, re, im) in want.items():
        head, rows = spectra.read_frequency_slice(d / "post" / name)
        assert head[0] == f"# Frequency slice at {f:.3e} Hz (index: {k})"
        assert head[4] == f"#   Time points: {N}"
        exp = spectra.expected_rows(re.shape[0], re.shape[1], re, im)
        np.testing.assert_array_equal(rows[:, :2], exp[:, :2])
        scale = float(np.abs(exp[:, 2:4]).max())
        assert float(np.abs(rows[:, 2:4] - exp[:, 2:4]).max()) <= 1e-6 * scale, name
