"""Python face of libphpfdtd: configurations, descriptions and a simulation
handle over the C ABI of include/php_fdtd.h.

The reference (PhP_FDTD) is driven by a .cfg file and a medium map; the same
path exists here (``Config.load`` -> ``Simulation.from_config``).  Tests and
benchmarks also build descriptions directly from arrays (``make_desc``).
Every compute call goes through libphpfdtd.so on the GPU; if the CUDA
library is missing or no device is present the calls raise.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _abi
from ._abi import COMPONENTS, PREC


class PhpError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def _check_host(rc: int, err: bytes | str):
    if rc != 0:
        if isinstance(err, (bytes, bytearray)):
            err = err.split(b"\0", 1)[0].decode(errors="replace")
        raise PhpError(rc, err)


# ------------------------------------------------------------------ configs


class Config:
    """A parsed .cfg (php_cfg_load): the reference's Config after all
    material files are read."""

    def __init__(self, ptr):
        self._ptr = ptr
        self._lib = _abi.host_lib()

    @classmethod
    def load(cls, path: str) -> "Config":
        lib = _abi.host_lib()
        ptr = C.POINTER(_abi.Cfg)()
        err = C.create_string_buffer(1024)
        rc = lib.php_cfg_load(str(path).encode(), C.byref(ptr), err, len(err))
        _check_host(rc, err.raw)
        return cls(ptr)

    def __del__(self):
        try:
            if self._ptr:
                self._lib.php_cfg_free(self._ptr)
                self._ptr = None
        except Exception:
            pass

    @property
    def c(self) -> _abi.Cfg:
        return self._ptr.contents

    def __getattr__(self, name):
        if name.startswith("_"):
            raise AttributeError(name)
        v = getattr(self._ptr.contents, name)
        return v.decode() if isinstance(v, bytes) else v

    @property
    def sources(self):
        return [self.c.sources[i] for i in range(self.c.num_sources)]

    @property
    def materials(self):
        return [self.c.materials[i] for i in range(self.c.num_materials)]

    def load_medium(self, path: Optional[str] = None) -> np.ndarray:
        lib = self._lib
        p = C.POINTER(C.c_int32)()
        err = C.create_string_buffer(1024)
        rc = lib.php_medium_load((path or self.medium_file).encode(), self.nx, self.ny, self.nz, C.byref(p), err, len(err))
        _check_host(rc, err.raw)
        n = self.nx * self.ny * self.nz
        arr = np.ctypeslib.as_array(p, shape=(n,)).copy().reshape(self.nx, self.ny, self.nz)
        C.CDLL(None).free(p)
        return arr

    def source_value(self, s: int, time: float) -> float:
        return self._lib.php_source_value(C.byref(self.c.sources[s]), time)

    def desc(self, medium: np.ndarray, precision: str = "fp64") -> "DescHolder":
        medium = np.ascontiguousarray(medium, dtype=np.int32)
        d = _abi.Desc()
        rc = self._lib.php_cfg_to_desc(self._ptr, medium.ctypes.data_as(C.POINTER(C.c_int32)), PREC[precision], C.byref(d))
        _check_host(rc, "php_cfg_to_desc failed")
        return DescHolder(d, [self, medium])


@dataclass
class DescHolder:
    """A php_desc plus the Python objects its pointers point into."""
    desc: _abi.Desc
    keep: list = field(default_factory=list)

    @property
    def nx(self):
        return self.desc.nx

    @property
    def ny(self):
        return self.desc.ny

    @property
    def nz(self):
        return self.desc.nz


@dataclass
class Material:
    eps_re: Sequence[float] = (1, 0, 0, 0, 1, 0, 0, 0, 1)
    eps_im: Sequence[float] = (0,) * 9
    sigma: float = 0.0
    anglez: float = 0.0
    anglex: float = 0.0
    use_ade: int = 0
    natom: int = 0
    qezv: Optional[np.ndarray] = None
    qezm: Optional[np.ndarray] = None
    dmm: Optional[np.ndarray] = None


@dataclass
class Source:
    type: int = 3
    x: int = 0
    y: int = 0
    z: int = 0
    component: str = "z"
    amplitude: float = 1.0
    frequency: float = 1e13
    t0: float = 0.0
    tau: float = 1e-15
    start_time: float = 0.0
    end_time: float = 1.0


def make_desc(medium: np.ndarray, materials: Sequence[Material], sources: Sequence[Source], *, dx: float, dy: float,
              dz: float, dt: float, pml_thickness: int, pml_reflection: float = 1e-6, source_frequency: Optional[float] = None,
              precision: str = "fp64", epsilon0: float = 8.854e-12, mu0: float = np.pi * 4e-7, z_chunk: int = 0,
              device: int = 0) -> DescHolder:
    """Builds a php_desc from arrays (medium is [nx][ny][nz] int32, file order)."""
    medium = np.ascontiguousarray(medium, dtype=np.int32)
    nx, ny, nz = medium.shape
    keep: list = [medium]
    mats = (_abi.MaterialDesc * len(materials))()
    for k, m in enumerate(materials):
        md = mats[k]
        md.eps_re[:] = [float(x) for x in m.eps_re]
        md.eps_im[:] = [float(x) for x in m.eps_im]
        md.sigma, md.anglez, md.anglex = m.sigma, m.anglez, m.anglex
        md.use_ade, md.natom = m.use_ade, m.natom
        if m.natom > 0:
            arrs = []
            for a, n in ((m.qezv, 9 * m.natom), (m.qezm, 9 * m.natom), (m.dmm, 9 * m.natom * m.natom)):
                a = np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel())
                if a.size != n:
                    raise ValueError(f"material {k}: expected {n} values, got {a.size}")
                keep.append(a)
                arrs.append(a.ctypes.data_as(C.POINTER(C.c_double)))
            md.qezv, md.qezm, md.dmm = arrs
    srcs = (_abi.SourceDesc * max(1, len(sources)))()
    for k, s in enumerate(sources):
        sd = srcs[k]
        sd.type, sd.x, sd.y, sd.z = s.type, s.x, s.y, s.z
        sd.component = ord(s.component)
        sd.amplitude, sd.frequency, sd.t0, sd.tau = s.amplitude, s.frequency, s.t0, s.tau
        sd.start_time, sd.end_time = s.start_time, s.end_time
    keep += [mats, srcs]
    d = _abi.Desc()
    d.abi_version = _abi.PHP_ABI_VERSION
    d.nx, d.ny, d.nz = nx, ny, nz
    d.dx, d.dy, d.dz, d.dt = dx, dy, dz, dt
    d.epsilon0, d.mu0 = epsilon0, mu0
    d.pml_thickness, d.pml_reflection = pml_thickness, pml_reflection
    d.precision = PREC[precision]
    d.source_frequency = source_frequency if source_frequency is not None else (sources[0].frequency if sources else -1.0)
    d.num_materials = len(materials)
    d.materials = C.cast(mats, C.POINTER(_abi.MaterialDesc))
    d.medium = medium.ctypes.data_as(C.POINTER(C.c_int32))
    d.num_sources = len(sources)
    d.sources = C.cast(srcs, C.POINTER(_abi.SourceDesc))
    d.z_chunk = z_chunk
    d.device = device
    return DescHolder(d, keep)


def with_precision(h: DescHolder, precision: str) -> DescHolder:
    d = _abi.Desc.from_buffer_copy(h.desc)
    d.precision = PREC[precision]
    return DescHolder(d, list(h.keep))


# --------------------------------------------------------------- simulation


def _comp(c) -> int:
    return COMPONENTS[c] if isinstance(c, str) else int(c)


class Simulation:
    """One device-resident domain (php_create ... php_destroy)."""

    def __init__(self, holder: DescHolder):
        self._lib = _abi.device_lib()
        self.holder = holder
        self.nx, self.ny, self.nz = holder.desc.nx, holder.desc.ny, holder.desc.nz
        ctx = C.c_void_p()
        rc = self._lib.php_create(C.byref(holder.desc), C.byref(ctx))
        if rc != 0:
            raise PhpError(rc, self._lib.php_last_error(None).decode())
        self._ctx = ctx

    @classmethod
    def from_config(cls, cfg: Config, precision: str = "fp64", medium: Optional[np.ndarray] = None) -> "Simulation":
        if medium is None:
            medium = cfg.load_medium()
        return cls(cfg.desc(medium, precision))

    def _ck(self, rc):
        if rc != 0:
            raise PhpError(rc, self._lib.php_last_error(self._ctx).decode())

    def close(self):
        if getattr(self, "_ctx", None):
            self._lib.php_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # stepping
    def step(self, n: int = 1):
        self._ck(self._lib.php_step(self._ctx, int(n)))

    def prepare(self, n: int):
        """Records the step graphs of step(n) ahead of its first call (php_prepare)."""
        self._ck(self._lib.php_prepare(self._ctx, int(n)))

    def sync(self):
        self._ck(self._lib.php_sync(self._ctx))

    @property
    def t(self) -> int:
        v = C.c_int32()
        self._ck(self._lib.php_get_step(self._ctx, C.byref(v)))
        return v.value

    # read-outs
    def read_volume(self, comp) -> np.ndarray:
        out = np.empty((self.nx, self.ny, self.nz), dtype=np.float64)
        self._ck(self._lib.php_read_volume(self._ctx, _comp(comp), out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def _slice_shape(self, axis: str):
        # an unknown axis still goes to the library, which rejects it
        return {"z": (self.nx, self.ny), "x": (self.ny, self.nz), "y": (self.nx, self.nz)}.get(axis, (1, 1))

    def read_slice(self, comp, axis: str, pos: int, f64: bool = False) -> np.ndarray:
        shape = self._slice_shape(axis)
        if f64:
            out = np.empty(shape, dtype=np.float64)
            self._ck(self._lib.php_read_slice_f64(self._ctx, _comp(comp), axis.encode(), int(pos),
                                                  out.ctypes.data_as(C.POINTER(C.c_double))))
        else:
            out = np.empty(shape, dtype=np.float32)
            self._ck(self._lib.php_read_slice(self._ctx, _comp(comp), axis.encode(), int(pos),
                                              out.ctypes.data_as(C.POINTER(C.c_float))))
        return out

    def read_point(self, i: int, j: int, k: int) -> np.ndarray:
        out = np.empty(9, dtype=np.float64)
        self._ck(self._lib.php_read_point(self._ctx, i, j, k, out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def read_cell_state(self, i: int, j: int, k: int, max_natom: int = 64):
        na = C.c_int32()
        r = np.zeros(3 * max_natom)
        v = np.zeros(3 * max_natom)
        p = np.zeros(3)
        po = np.zeros(3)
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
        self._ck(self._lib.php_read_cell_state(self._ctx, i, j, k, C.byref(na), dp(r), dp(v), dp(p), dp(po)))
        n = 3 * na.value
        return {"natom": na.value, "r": r[:n].copy(), "v": v[:n].copy(), "P": p, "P_old": po}

    def diagnostics(self) -> dict:
        d = _abi.Diag()
        self._ck(self._lib.php_diagnostics(self._ctx, C.byref(d)))
        return {"max_e": d.max_e, "max_ex": d.max_ex, "max_r": d.max_r, "argmax_r": tuple(d.argmax_r)}

    def probe_set(self, i: int, j: int, k_field: int, k_atom: int):
        self._ck(self._lib.php_probe_set(self._ctx, i, j, k_field, k_atom))

    def probe_read(self, max_rows: int = 8192) -> np.ndarray:
        n = C.c_int32()
        rl = C.c_int32()
        buf = np.empty(max_rows * (9 + 6 * 64), dtype=np.float64)
        self._ck(self._lib.php_probe_read(self._ctx, buf.ctypes.data_as(C.POINTER(C.c_double)), max_rows, C.byref(n),
                                          C.byref(rl)))
        return buf[: n.value * rl.value].reshape(n.value, rl.value).copy()

    def frame_begin(self, diag: bool = False, slice=None, probe: bool = False, point=None, cell=None) -> int:
        """Enqueues an output frame behind the steps enqueued so far
        (php_frame_begin) and returns its ticket at once.  slice is
        (component, axis, position); point and cell are (i, j, k)."""
        q = _abi.FrameReq()
        q.diag = int(bool(diag))
        q.slice_comp = -1
        if slice is not None:
            comp, axis, pos = slice
            q.slice_comp, q.slice_axis, q.slice_pos = _comp(comp), ord(axis), int(pos)
        q.probe = int(bool(probe))
        q.point[:] = tuple(point) if point is not None else (-1, 0, 0)
        q.cell[:] = tuple(cell) if cell is not None else (-1, 0, 0)
        tk = C.c_int32()
        self._ck(self._lib.php_frame_begin(self._ctx, C.byref(q), C.byref(tk)))
        return tk.value

    def frame_wait(self, ticket: int, release: bool = True) -> dict:
        """Waits for frame `ticket` and returns copies of its parts
        (php_frame_wait); releases the frame unless release is False."""
        f = _abi.Frame()
        try:
            self._ck(self._lib.php_frame_wait(self._ctx, int(ticket), C.byref(f)))
            out = {"step": f.step}
            d = f.diag
            out["diag"] = {"max_e": d.max_e, "max_ex": d.max_ex, "max_r": d.max_r, "argmax_r": tuple(d.argmax_r)}
            n = 3 * f.diag_natom
            out["diag_cell"] = {"natom": f.diag_natom, "point": np.array(f.diag_point[:]),
                                "r": np.array(f.diag_r[:n]), "v": np.array(f.diag_v[:n])}
            out["point"] = np.array(f.point[:])
            n = 3 * f.cell_natom
            out["cell"] = {"natom": f.cell_natom, "r": np.array(f.cell_r[:n]), "v": np.array(f.cell_v[:n])}
            out["slice"] = (np.ctypeslib.as_array(f.slice, shape=(f.slice_len,)).copy() if f.slice_len else None)
            out["rows"] = (np.ctypeslib.as_array(f.rows, shape=(f.nrows * f.row_len,)).reshape(f.nrows, f.row_len).copy()
                           if f.nrows else np.empty((0, f.row_len)))
        finally:
            if release:
                self._lib.php_frame_release(self._ctx, int(ticket))
        return out

    def dft_add(self, comp, z_plane: int, freqs: Sequence[float], first_step: int = 0, interval: int = 1,
                cast_f32: bool = False) -> int:
        f = np.ascontiguousarray(np.asarray(freqs, dtype=np.float64))
        pid = C.c_int32()
        self._ck(self._lib.php_dft_add(self._ctx, _comp(comp), int(z_plane), int(first_step), int(interval), int(f.size),
                                       f.ctypes.data_as(C.POINTER(C.c_double)), int(bool(cast_f32)), C.byref(pid)))
        self._dft_nf = getattr(self, "_dft_nf", {})
        self._dft_nf[pid.value] = f.size
        return pid.value

    def dft_read(self, pid: int):
        nf = self._dft_nf[pid]
        out = np.empty((nf, self.nx, self.ny, 2), dtype=np.float64)
        ns = C.c_int32()
        self._ck(self._lib.php_dft_read(self._ctx, pid, out.ctypes.data_as(C.POINTER(C.c_double)), C.byref(ns)))
        return out[..., 0] + 1j * out[..., 1], ns.value

    @property
    def memory_bytes(self) -> int:
        v = C.c_uint64()
        self._ck(self._lib.php_memory_bytes(self._ctx, C.byref(v)))
        return v.value

    @property
    def last_launch_count(self) -> int:
        v = C.c_int32()
        self._ck(self._lib.php_last_launch_count(self._ctx, C.byref(v)))
        return v.value

    CENSUS_KEYS = ("e_plain", "e_plain_cpml", "e_tensor", "e_atoms", "e_general", "h_plain", "h_general", "blocks")

    def block_census(self) -> dict:
        """Blocks per sweep code path (php_block_census)."""
        n = (C.c_int64 * 8)()
        self._ck(self._lib.php_block_census(self._ctx, n))
        return {k: int(n[q]) for q, k in enumerate(self.CENSUS_KEYS)}

    def profile(self, enable: bool = True):
        """Per-kernel device timing of the following steps (php_profile_enable)."""
        self._ck(self._lib.php_profile_enable(self._ctx, int(bool(enable))))

    def profile_read(self) -> dict:
        ms = np.zeros(6)
        n = (C.c_int64 * 6)()
        self._ck(self._lib.php_profile_read(self._ctx, ms.ctypes.data_as(C.POINTER(C.c_double)), n))
        names = ("h_sweep", "e_sweep", "probe", "dft", "ion", "step")
        return {k: {"ms": float(ms[q]), "launches": int(n[q])} for q, k in enumerate(names)}

    @property
    def stream(self) -> int:
        v = C.c_void_p()
        self._ck(self._lib.php_stream(self._ctx, C.byref(v)))
        return v.value or 0
