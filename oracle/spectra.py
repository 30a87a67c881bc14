"""Test infrastructure only: a NumPy restatement of the reference's
post-processor frequency_analysis.c (which needs FFTW, absent here), used to
check the near-field spectra the solver writes with --spectra.

It follows frequency_analysis.c: the source frequency of the last source
line (:56-104), the field_slice_*.bin files sorted by step (:180-230), sample
times step * dt and fs = (N - 1) / (t_last - t_first) (:363-377), the bin
nearest the source frequency below N / 2 and four on each side (:380-421),
X_k / N of an unnormalised forward DFT per cell (:532-570), and the rows of
save_frequency_result (:275-314)."""
from __future__ import annotations

import math
import re
from pathlib import Path

import numpy as np


def source_frequency(cfg_text: str) -> float:
    found = 0.0
    for line in cfg_text.splitlines():
        if line.startswith("#") or not line.startswith("source"):
            continue
        fr = wn = None
        for tok in line.split(","):
            if "=" not in tok:
                continue
            if "frequency" in tok:
                fr = float(tok.split("=", 1)[1].split()[0])
            elif "wavenumber" in tok:
                wn = float(tok.split("=", 1)[1].split()[0])
        if wn is not None:
            fr = wn * 0.03e12
        if fr is not None:
            found = fr
    return found


def read_slice(path: Path) -> np.ndarray:
    raw = path.read_bytes()
    n0, n1 = np.frombuffer(raw[:8], dtype=np.int32)
    return np.frombuffer(raw[8:8 + 4 * n0 * n1], dtype=np.float32).reshape(n0, n1)


def analyse(run_dir: Path, dt: float, f_src: float):
    """{file name: (freq_hz, index, fs, N, re[nx,ny], im[nx,ny])}"""
    files = sorted(Path(run_dir).glob("field_slice_*.bin"), key=lambda p: int(p.stem.rsplit("_", 1)[1]))
    steps = [int(p.stem.rsplit("_", 1)[1]) for p in files]
    N = len(files)
    times = [s * dt for s in steps]
    fs = 1.0 / ((times[-1] - times[0]) / (N - 1))
    target, best = -1, 1e100
    for i in range(N // 2):
        d = abs(i * fs / N - f_src)
        if d < best:
            best, target = d, i
    idx = [target + o for o in range(-4, 5) if 0 <= target + o < N // 2][:9]
    data = np.stack([read_slice(p).astype(np.float64) for p in files])   # [N][nx][ny]
    spec = np.fft.fft(data, axis=0) / N
    out = {}
    for k in idx:
        f = k * fs / N
        name = f"frequency_slice_{k}_{f:.3e}Hz_{f / 0.03e12:.3e}cm-1.txt"
        out[name] = (f, k, fs, N, spec[k].real, spec[k].imag)
    return out


def read_frequency_slice(path: Path):
    """(header lines, rows [i, j, re, im, mag, phase, phase_deg])"""
    head, rows = [], []
    for line in Path(path).read_text().splitlines():
        if line.startswith("#"):
            head.append(line)
        elif line.strip():
            rows.append([float(x) for x in line.split()])
    return head, np.array(rows)


def expected_rows(nx: int, ny: int, re: np.ndarray, im: np.ndarray) -> np.ndarray:
    rows = []
    for i in range(nx):
        for j in range(ny):
            if nx * 0.25 < i < nx * 0.75 and ny * 0.25 < j < ny * 0.75:
                mag = math.hypot(re[i, j], im[i, j])
                ph = math.atan2(im[i, j], re[i, j])
                rows.append([i, j, re[i, j], im[i, j], mag, ph, ph * 180.0 / math.pi])
    return np.array(rows)
