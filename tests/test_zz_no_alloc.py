"""GPU test of php_field_maxima_noalloc, the allocation-free variant of the
field-maxima reduction.

It exists for callers that cannot allocate device memory when they need the
maxima -- a divergence check on a device whose memory is full, a host whose
allocator owns all device memory, a latency-critical loop where cudaMalloc
would synchronise -- so its output must match what php_diagnostics (which
reduces through a scratch buffer php_create allocates) reports for the same
fields, on consecutive calls that reuse the library's fixed scratch array.
This file is collected last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import ROOT
from php_fdtd_b200 import Material, Simulation, Source, make_desc

pytestmark = pytest.mark.gpu

NOALLOC_MAX_CELLS = 67108864  # PHP_NOALLOC_MAX_CELLS in include/php_fdtd.h


def _entry():
    lib = C.CDLL(str(ROOT / "php_fdtd_b200" / "libphpfdtd.so"))
    f = lib.php_field_maxima_noalloc
    f.restype = C.c_int32
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]
    return f


def _domain(n: int):
    medium = np.zeros((n, n, n), np.int32)
    medium[:, :, : n // 3] = 1
    mats = [Material(), Material(eps_re=(6.0, 0.3, 0, 0.3, 3.5, 0, 0, 0, 2.8), eps_im=(0.4, 0, 0, 0, 0.2, 0, 0, 0, 0.1),
                                 anglez=0.5)]
    srcs = [Source(type=3, x=n // 2, y=n // 2, z=n // 2, component="z", frequency=1370 * 0.03e12, t0=3e-16, tau=1e-16),
            Source(type=1, x=n // 3, y=n // 2, z=n // 2 + 2, component="x", frequency=2.5e13)]
    dl = 10e-9
    return make_desc(medium, mats, srcs, dx=dl, dy=dl, dz=dl, dt=dl / (3e8 * 3 ** 0.5) * 0.99, pml_thickness=4,
                     precision="fp64")


@pytest.mark.parametrize("n", [24, 64])
def test_noalloc_maxima_match_diagnostics_on_consecutive_calls(n):
    import torch
    f = _entry()
    sim = Simulation(_domain(n))
    stream = torch.cuda.current_stream()
    for call in range(2):
        sim.step(9 + 7 * call)
        fields = [torch.from_numpy(np.ascontiguousarray(sim.read_volume(c))).cuda() for c in ("Ex", "Ey", "Ez")]
        out = torch.full((2,), -1.0, dtype=torch.float64, device="cuda")
        rc = f(fields[0].data_ptr(), fields[1].data_ptr(), fields[2].data_ptr(), fields[0].numel(), out.data_ptr(),
               stream.cuda_stream)
        assert rc == 0
        torch.cuda.synchronize()
        ref = sim.diagnostics()
        assert ref["max_e"] > 0
        got = out.cpu().numpy()
        assert got[0] == ref["max_e"], (call, got[0], ref["max_e"])
        assert got[1] == ref["max_ex"], (call, got[1], ref["max_ex"])
    sim.close()


def test_noalloc_rejects_sizes_above_its_scratch():
    import torch
    f = _entry()
    buf = torch.zeros(4, dtype=torch.float64, device="cuda")
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    p = buf.data_ptr()
    # rejected on the host before anything is launched
    assert f(p, p, p, NOALLOC_MAX_CELLS + 1, out.data_ptr(), None) == -1
    assert f(p, p, p, -1, out.data_ptr(), None) == -1
    assert f(p, p, p, 4, None, None) == -1
    assert f(p, p, p, 0, out.data_ptr(), None) == 0
    torch.cuda.synchronize()
    assert out.cpu().numpy().tolist() == [0.0, 0.0]
