"""Serving loop: a stream of independent simulations on one GPU
(php_serve.h).  Thin ctypes layer; the admission and stepping threads are
the library's own (C++)."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from . import _abi
from .solver import DescHolder, PhpError, _comp


@dataclass
class DftSpec:
    """Running DFT of one xy plane (php_dft_add arguments)."""
    component: object
    z_plane: int
    freqs: Sequence[float]
    first_step: int = 0
    interval: int = 1
    cast_f32: bool = False


def estimate_bytes(holder: DescHolder) -> int:
    v = C.c_uint64()
    lib = _abi.device_lib()
    rc = lib.php_estimate_bytes(C.byref(holder.desc), C.byref(v))
    if rc != 0:
        raise PhpError(rc, "php_estimate_bytes rejected the description")
    return v.value


class Server:
    def __init__(self, memory_budget: int, device: int = 0, max_active: int = 0, chunk_steps: int = 0):
        self._lib = _abi.device_lib()
        d = _abi.ServerDesc()
        d.abi_version = _abi.PHP_ABI_VERSION
        d.device = device
        d.memory_budget = int(memory_budget)
        d.max_active = int(max_active)
        d.chunk_steps = int(chunk_steps)
        s = C.c_void_p()
        rc = self._lib.php_server_create(C.byref(d), C.byref(s))
        if rc != 0:
            raise PhpError(rc, "php_server_create failed")
        self._s = s
        self._keep = {}

    def _ck(self, rc):
        if rc != 0:
            raise PhpError(rc, self._lib.php_server_last_error(self._s).decode())

    def submit(self, holder: DescHolder, nsteps: int, dft: Optional[DftSpec] = None, tag: int = 0) -> int:
        req = None
        if dft is not None:
            f = np.ascontiguousarray(np.asarray(dft.freqs, dtype=np.float64))
            req = _abi.DftRequest()
            req.component = _comp(dft.component)
            req.z_plane = int(dft.z_plane)
            req.first_step = int(dft.first_step)
            req.interval = int(dft.interval)
            req.nfreq = int(f.size)
            req.cast_f32 = int(bool(dft.cast_f32))
            req.freq_hz = f.ctypes.data_as(C.POINTER(C.c_double))
        job = C.c_int64()
        self._ck(self._lib.php_batch_submit(self._s, C.byref(holder.desc), int(nsteps),
                                            C.byref(req) if req is not None else None, int(tag), C.byref(job)))
        return job.value

    def poll(self, max_jobs: int = 256, timeout_ms: int = 0) -> List[dict]:
        buf = (_abi.JobInfo * max_jobs)()
        n = C.c_int32()
        self._ck(self._lib.php_batch_poll(self._s, buf, max_jobs, int(timeout_ms), C.byref(n)))
        out = []
        for k in range(n.value):
            b = buf[k]
            out.append({"job": b.job, "tag": b.tag, "status": b.status, "steps": b.steps, "t_submit": b.t_submit,
                        "t_admit": b.t_admit, "t_start": b.t_start, "t_done": b.t_done, "device_bytes": b.device_bytes, "nx": b.nx,
                        "ny": b.ny, "nfreq": b.nfreq, "dft_samples": b.dft_samples,
                        "error": b.error.decode(errors="replace")})
        return out

    def fetch_dft(self, info: dict) -> np.ndarray:
        out = np.empty((info["nfreq"], info["nx"], info["ny"], 2), dtype=np.float64)
        self._ck(self._lib.php_batch_fetch_dft(self._s, int(info["job"]), out.ctypes.data_as(C.POINTER(C.c_double))))
        return out[..., 0] + 1j * out[..., 1]

    def release(self, job: int):
        self._ck(self._lib.php_batch_release(self._s, int(job)))

    def stats(self) -> dict:
        st = _abi.ServerStats()
        self._ck(self._lib.php_server_stats_read(self._s, C.byref(st)))
        return {k: getattr(st, k) for k, _ in _abi.ServerStats._fields_}

    def clock(self) -> float:
        t = C.c_double()
        self._ck(self._lib.php_server_clock(self._s, C.byref(t)))
        return t.value

    def close(self):
        if getattr(self, "_s", None):
            self._lib.php_server_destroy(self._s)
            self._s = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
