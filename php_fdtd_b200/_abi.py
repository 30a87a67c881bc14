"""ctypes mirror of include/php_fdtd.h and include/php_host.h.

Struct layouts are checked against the C sizes at load time
(``php_host_sizeof``), so a header change that is not mirrored here fails
loudly instead of corrupting memory.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

PKG = Path(__file__).resolve().parent

PHP_ABI_VERSION = 1

PHP_OK = 0
PHP_ERR_INPUT = -1
PHP_ERR_OOM = -2
PHP_ERR_CUDA = -3
PHP_ERR_DIVERGED = -4
PHP_ERR_TIMEOUT = -5
PHP_ERR_STATE = -6
PHP_ERR_UNSUPPORTED = -7
PHP_ERR_NODEVICE = -8

PREC = {"fp64-strict": 0, "fp64": 1, "fp32": 2}
COMPONENTS = {"Ex": 0, "Ey": 1, "Ez": 2, "Dx": 3, "Dy": 4, "Dz": 5, "Hx": 6, "Hy": 7, "Hz": 8, "E": 9}

_d = C.c_double
_i = C.c_int32
_dp = C.POINTER(C.c_double)


class MaterialDesc(C.Structure):
    _fields_ = [("eps_re", _d * 9), ("eps_im", _d * 9), ("sigma", _d), ("anglez", _d), ("anglex", _d),
                ("use_ade", _i), ("natom", _i), ("qezv", _dp), ("qezm", _dp), ("dmm", _dp)]


class SourceDesc(C.Structure):
    _fields_ = [("type", _i), ("x", _i), ("y", _i), ("z", _i), ("component", _i), ("pad_", _i),
                ("amplitude", _d), ("frequency", _d), ("t0", _d), ("tau", _d), ("start_time", _d), ("end_time", _d)]


class Desc(C.Structure):
    _fields_ = [("abi_version", _i), ("nx", _i), ("ny", _i), ("nz", _i),
                ("dx", _d), ("dy", _d), ("dz", _d), ("dt", _d), ("epsilon0", _d), ("mu0", _d),
                ("pml_thickness", _i), ("precision", _i), ("pml_reflection", _d), ("source_frequency", _d),
                ("num_materials", _i), ("num_sources", _i),
                ("materials", C.POINTER(MaterialDesc)), ("medium", C.POINTER(C.c_int32)),
                ("sources", C.POINTER(SourceDesc)), ("z_chunk", _i), ("device", _i)]


class Diag(C.Structure):
    _fields_ = [("max_e", _d), ("max_ex", _d), ("max_r", _d), ("argmax_r", _i * 5), ("pad_", _i)]


FRAME_MAX_N3 = 192


class FrameReq(C.Structure):
    _fields_ = [("diag", _i), ("slice_comp", _i), ("slice_axis", _i), ("slice_pos", _i), ("probe", _i),
                ("point", _i * 3), ("cell", _i * 3)]


class Frame(C.Structure):
    _fields_ = [("step", _i), ("nrows", _i), ("row_len", _i), ("diag_natom", _i), ("cell_natom", _i), ("pad_", _i),
                ("diag", Diag), ("diag_point", _d * 9), ("diag_r", _d * FRAME_MAX_N3), ("diag_v", _d * FRAME_MAX_N3),
                ("point", _d * 9), ("cell_r", _d * FRAME_MAX_N3), ("cell_v", _d * FRAME_MAX_N3),
                ("slice", C.POINTER(C.c_float)), ("slice_len", C.c_int64), ("rows", C.POINTER(C.c_double))]


class ServerDesc(C.Structure):
    _fields_ = [("abi_version", _i), ("device", _i), ("memory_budget", C.c_uint64), ("max_active", _i),
                ("chunk_steps", _i)]


class DftRequest(C.Structure):
    _fields_ = [("component", _i), ("z_plane", _i), ("first_step", _i), ("interval", _i), ("nfreq", _i),
                ("cast_f32", _i), ("freq_hz", _dp)]


class JobInfo(C.Structure):
    _fields_ = [("job", C.c_int64), ("tag", C.c_uint64), ("status", _i), ("steps", _i), ("t_submit", _d),
                ("t_admit", _d), ("t_done", _d), ("t_start", _d), ("device_bytes", C.c_uint64), ("nx", _i), ("ny", _i), ("nfreq", _i),
                ("dft_samples", _i), ("error", C.c_char * 256)]


class ServerStats(C.Structure):
    _fields_ = [("queued", _i), ("running", _i), ("finished_unpolled", _i), ("peak_running", _i),
                ("bytes_in_use", C.c_uint64), ("peak_bytes", C.c_uint64), ("submitted", C.c_int64),
                ("completed", C.c_int64)]


class HostMaterial(C.Structure):
    _fields_ = [("name", C.c_char * 64), ("eps_re", _d * 9), ("eps_im", _d * 9), ("sigma", _d), ("sigma_m", _d),
                ("anglez", _d), ("anglex", _d), ("use_ade", _i), ("natom", _i), ("switchxz", _i),
                ("use_born_file_for_eps", _i), ("use_dielectric_file", _i), ("qezv_set", _i), ("qezm_set", _i),
                ("dmm_set", _i), ("born_file", C.c_char * 1024), ("qezv_file", C.c_char * 1024),
                ("qezm_file", C.c_char * 1024), ("dmm_file", C.c_char * 1024), ("dielectric_file", C.c_char * 1024),
                ("born", _dp), ("qezv", _dp), ("qezm", _dp), ("dmm", _dp)]


class Cfg(C.Structure):
    _fields_ = [("nx", _i), ("ny", _i), ("nz", _i), ("tsteps", _i),
                ("delta_x", _d), ("delta_y", _d), ("delta_z", _d), ("dt", _d), ("c", _d), ("epsilon0", _d), ("mu0", _d),
                ("pml_thickness", _i), ("pml_reflection", _d), ("output_interval", _i),
                ("medium_file", C.c_char * 1024), ("output_component", C.c_char * 10), ("output_slice_axis", C.c_char),
                ("output_slice_position", _i), ("monitor_enabled", _i), ("monitor_x", _i), ("monitor_y", _i),
                ("monitor_z", _i), ("monitor_atom", _i), ("monitor_dir", _i), ("monitor_output_file", C.c_char * 1024),
                ("full_monitor_enabled", _i), ("full_monitor_output_file", C.c_char * 1024),
                ("unique_source_frequency", _d), ("num_sources", _i), ("sources", C.POINTER(SourceDesc)),
                ("num_materials", _i), ("materials", C.POINTER(HostMaterial)),
                ("desc_materials", C.POINTER(MaterialDesc)), ("warnings", C.c_char * 2048)]


DEVICE_SYMBOLS = {
    "php_create": (_i, [C.POINTER(Desc), C.POINTER(C.c_void_p)]),
    "php_destroy": (_i, [C.c_void_p]),
    "php_last_error": (C.c_char_p, [C.c_void_p]),
    "php_step": (_i, [C.c_void_p, _i]),
    "php_sync": (_i, [C.c_void_p]),
    "php_get_step": (_i, [C.c_void_p, C.POINTER(_i)]),
    "php_read_slice": (_i, [C.c_void_p, _i, C.c_char, _i, C.POINTER(C.c_float)]),
    "php_read_slice_f64": (_i, [C.c_void_p, _i, C.c_char, _i, _dp]),
    "php_read_volume": (_i, [C.c_void_p, _i, _dp]),
    "php_read_point": (_i, [C.c_void_p, _i, _i, _i, _dp]),
    "php_read_cell_state": (_i, [C.c_void_p, _i, _i, _i, C.POINTER(_i), _dp, _dp, _dp, _dp]),
    "php_diagnostics": (_i, [C.c_void_p, C.POINTER(Diag)]),
    "php_probe_set": (_i, [C.c_void_p, _i, _i, _i, _i]),
    "php_probe_read": (_i, [C.c_void_p, _dp, _i, C.POINTER(_i), C.POINTER(_i)]),
    "php_frame_begin": (_i, [C.c_void_p, C.POINTER(FrameReq), C.POINTER(_i)]),
    "php_frame_wait": (_i, [C.c_void_p, _i, C.POINTER(Frame)]),
    "php_frame_release": (_i, [C.c_void_p, _i]),
    "php_dft_add": (_i, [C.c_void_p, _i, _i, _i, _i, _i, _dp, _i, C.POINTER(_i)]),
    "php_dft_read": (_i, [C.c_void_p, _i, _dp, C.POINTER(_i)]),
    "php_memory_bytes": (_i, [C.c_void_p, C.POINTER(C.c_uint64)]),
    "php_last_launch_count": (_i, [C.c_void_p, C.POINTER(_i)]),
    "php_block_census": (_i, [C.c_void_p, C.POINTER(C.c_int64)]),
    "php_stream": (_i, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "php_profile_enable": (_i, [C.c_void_p, _i]),
    "php_profile_read": (_i, [C.c_void_p, _dp, C.POINTER(C.c_int64)]),
    "php_estimate_bytes": (_i, [C.POINTER(Desc), C.POINTER(C.c_uint64)]),
    "php_create_slab": (_i, [C.POINTER(Desc), _i, _i, C.POINTER(C.c_void_p)]),
    "php_halo_planes": (_i, [C.c_void_p, _i, C.POINTER(C.c_void_p), C.POINTER(C.c_uint64)]),
    "php_step_half": (_i, [C.c_void_p, _i]),
    "php_step_part": (_i, [C.c_void_p, _i, C.c_void_p]),
    "php_prepare": (_i, [C.c_void_p, _i]),
    "php_server_create": (_i, [C.POINTER(ServerDesc), C.POINTER(C.c_void_p)]),
    "php_server_destroy": (_i, [C.c_void_p]),
    "php_server_last_error": (C.c_char_p, [C.c_void_p]),
    "php_server_clock": (_i, [C.c_void_p, _dp]),
    "php_server_stats_read": (_i, [C.c_void_p, C.POINTER(ServerStats)]),
    "php_batch_submit": (_i, [C.c_void_p, C.POINTER(Desc), _i, C.POINTER(DftRequest), C.c_uint64,
                              C.POINTER(C.c_int64)]),
    "php_batch_poll": (_i, [C.c_void_p, C.POINTER(JobInfo), _i, _i, C.POINTER(_i)]),
    "php_batch_fetch_dft": (_i, [C.c_void_p, C.c_int64, _dp]),
    "php_batch_release": (_i, [C.c_void_p, C.c_int64]),
}

HOST_SYMBOLS = {
    "php_cfg_load": (_i, [C.c_char_p, C.POINTER(C.POINTER(Cfg)), C.c_char_p, C.c_size_t]),
    "php_cfg_free": (None, [C.POINTER(Cfg)]),
    "php_cfg_to_desc": (_i, [C.POINTER(Cfg), C.POINTER(C.c_int32), _i, C.POINTER(Desc)]),
    "php_medium_load": (_i, [C.c_char_p, _i, _i, _i, C.POINTER(C.POINTER(C.c_int32)), C.c_char_p, C.c_size_t]),
    "php_source_value": (_d, [C.POINTER(SourceDesc), _d]),
    "php_slice_filename": (None, [C.c_char_p, C.c_size_t, C.c_char, _i, _i]),
    "php_write_slice_file": (_i, [C.c_char_p, C.c_char, _i, _i, _i, C.POINTER(C.c_float)]),
    "php_component_from_name": (_i, [C.c_char_p]),
    "php_write_frequency_slice": (_i, [C.c_char_p, _d, _i, _d, _d, _i, _i, _i, _dp, _dp]),
    "php_host_sizeof": (C.c_uint64, [C.c_char_p]),
    "php_spectra_config": (_i, [C.c_char_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "php_spectra_bins": (_i, [_i, _i, _d, _d, C.POINTER(C.c_int32), _dp, _dp]),
}

_STRUCTS = {"php_desc": Desc, "php_material_desc": MaterialDesc, "php_source_desc": SourceDesc, "php_diag": Diag,
            "php_server_desc": ServerDesc, "php_dft_request": DftRequest, "php_job_info": JobInfo,
            "php_server_stats": ServerStats, "php_frame_req": FrameReq, "php_frame": Frame,
            "php_cfg": Cfg, "php_host_material": HostMaterial}

_host = None
_device = None


def _bind(lib, table):
    for name, (res, args) in table.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


def host_lib():
    """libphphost.so (no CUDA needed)."""
    global _host
    if _host is None:
        path = PKG / "libphphost.so"
        if not path.exists():
            raise RuntimeError(f"{path} is not built; run `python -m php_fdtd_b200.build`")
        lib = _bind(C.CDLL(str(path)), HOST_SYMBOLS)
        for name, st in _STRUCTS.items():
            n = lib.php_host_sizeof(name.encode())
            if n != C.sizeof(st):
                raise RuntimeError(f"ctypes layout of {name} is {C.sizeof(st)} bytes, C says {n}")
        _host = lib
    return _host


def device_lib():
    """libphpfdtd.so: the CUDA path.  Raises if the extension is not built;
    there is no fallback."""
    global _device
    if _device is None:
        path = PKG / "libphpfdtd.so"
        if not path.exists():
            raise RuntimeError(f"{path} is not built; run `python -m php_fdtd_b200.build` (CUDA path required)")
        _device = _bind(C.CDLL(str(path)), DEVICE_SYMBOLS)
    return _device
