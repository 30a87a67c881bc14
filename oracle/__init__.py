"""TEST INFRASTRUCTURE -- Python binding of the oracle.

``Oracle`` runs the C restatement of PhP_FDTD's time-step loop
(oracle/php_oracle.c) on the same php_desc the CUDA path consumes, with the
same read-out methods as ``php_fdtd_b200.Simulation``.  ``reference_binary``
locates the reference solver compiled from its own sources (oracle/_ref).
Only tests, the smoke check and the benchmark's CPU-baseline leg use this
package; the product never imports it.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from php_fdtd_b200 import _abi
from php_fdtd_b200._abi import COMPONENTS

HERE = Path(__file__).resolve().parent
_lib = None


def lib():
    global _lib
    if _lib is None:
        path = HERE / "liboracle.so"
        if not path.exists():
            raise RuntimeError(f"{path} is not built; run `make -C oracle restatement`")
        L = C.CDLL(str(path))
        vp, i, dp = C.c_void_p, C.c_int, C.POINTER(C.c_double)
        sig = {
            "oracle_create": (i, [C.POINTER(_abi.Desc), C.POINTER(vp)]),
            "oracle_destroy": (None, [vp]),
            "oracle_last_error": (C.c_char_p, []),
            "oracle_set_threads": (None, [i]),
            "oracle_step": (i, [vp, i]),
            "oracle_get_step": (i, [vp]),
            "oracle_read_volume": (i, [vp, i, dp]),
            "oracle_read_slice_f64": (i, [vp, i, C.c_char, i, dp]),
            "oracle_read_point": (i, [vp, i, i, i, dp]),
            "oracle_read_cell_state": (i, [vp, i, i, i, C.POINTER(i), dp, dp, dp, dp]),
            "oracle_diagnostics": (i, [vp, C.POINTER(_abi.Diag)]),
        }
        for n, (r, a) in sig.items():
            f = getattr(L, n)
            f.restype, f.argtypes = r, a
        _lib = L
    return _lib


def reference_binary(kind: str = "wide") -> Path:
    """oracle/_ref/fdtd_ref{,_wide,_fast,_mp,_mp_wide}: the reference solver
    itself (_mp: release flags, PHP_MPI_NP ranks through the shared-memory
    MPI stand-in of mpi_shm/mpi.h; _mp_wide: the same ranks with the strict
    flags and wide outputs), or its post-processor (``post``, ``post_wide``:
    frequency_analysis.c against the FFTW stand-in)."""
    name = {"plain": "fdtd_ref", "wide": "fdtd_ref_wide", "fast": "fdtd_ref_fast", "mp": "fdtd_ref_mp",
            "mp_wide": "fdtd_ref_mp_wide", "post": "frequency_analysis", "post_wide": "frequency_analysis_wide"}[kind]
    return HERE / "_ref" / name


def _comp(c):
    return COMPONENTS[c] if isinstance(c, str) else int(c)


class Oracle:
    def __init__(self, holder, threads: int = 0):
        self._lib = lib()
        if threads:
            self._lib.oracle_set_threads(threads)
        self.holder = holder
        self.nx, self.ny, self.nz = holder.desc.nx, holder.desc.ny, holder.desc.nz
        ctx = C.c_void_p()
        rc = self._lib.oracle_create(C.byref(holder.desc), C.byref(ctx))
        if rc:
            raise RuntimeError(f"oracle_create: {self._lib.oracle_last_error().decode()}")
        self._ctx = ctx

    def close(self):
        if getattr(self, "_ctx", None):
            self._lib.oracle_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, n: int = 1):
        rc = self._lib.oracle_step(self._ctx, int(n))
        if rc:
            raise RuntimeError(self._lib.oracle_last_error().decode())

    @property
    def t(self):
        return self._lib.oracle_get_step(self._ctx)

    def read_volume(self, comp):
        out = np.empty((self.nx, self.ny, self.nz))
        assert self._lib.oracle_read_volume(self._ctx, _comp(comp), out.ctypes.data_as(C.POINTER(C.c_double))) == 0
        return out

    def read_slice(self, comp, axis, pos, f64=True):
        shape = {"z": (self.nx, self.ny), "x": (self.ny, self.nz), "y": (self.nx, self.nz)}[axis]
        out = np.empty(shape)
        rc = self._lib.oracle_read_slice_f64(self._ctx, _comp(comp), axis.encode(), int(pos),
                                             out.ctypes.data_as(C.POINTER(C.c_double)))
        if rc:
            raise ValueError("invalid slice")
        return out if f64 else out.astype(np.float32)

    def read_point(self, i, j, k):
        out = np.empty(9)
        assert self._lib.oracle_read_point(self._ctx, i, j, k, out.ctypes.data_as(C.POINTER(C.c_double))) == 0
        return out

    def read_cell_state(self, i, j, k, max_natom=64):
        na = C.c_int()
        r, v, p, po = np.zeros(3 * max_natom), np.zeros(3 * max_natom), np.zeros(3), np.zeros(3)
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
        assert self._lib.oracle_read_cell_state(self._ctx, i, j, k, C.byref(na), dp(r), dp(v), dp(p), dp(po)) == 0
        n = 3 * na.value
        return {"natom": na.value, "r": r[:n].copy(), "v": v[:n].copy(), "P": p, "P_old": po}

    def diagnostics(self):
        d = _abi.Diag()
        self._lib.oracle_diagnostics(self._ctx, C.byref(d))
        return {"max_e": d.max_e, "max_ex": d.max_ex, "max_r": d.max_r, "argmax_r": tuple(d.argmax_r)}
