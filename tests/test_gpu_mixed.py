"""The FP32 (mixed) path against the FP64 path on a metal-tip case: the
required error bounds (1e-4 relative L2 on the fields, 1e-3 on the
running-DFT near-field plane) and the read-back of the ADE state, which the
FP32 path keeps in increment form."""
import math

import numpy as np
import pytest

from php_fdtd_b200 import Material, Simulation, Source, make_desc
from php_fdtd_b200.workloads import cone_tip_mask, drude_lorentz_eps

pytestmark = pytest.mark.gpu

N, DL = 64, 5e-9
DT = DL / (299792458.0 * math.sqrt(3.0)) * 0.99
F_SRC = 900 * 0.03e12


def _case(precision):
    e_tip = drude_lorentz_eps(900.0)
    mats = [Material(),
            Material(eps_re=(6.0, 0, 0, 0, 3.5, 0, 0, 0, 2.8), eps_im=(0.4, 0, 0, 0, 0.2, 0, 0, 0, 0.1),
                     anglez=0.5235987756),
            Material(eps_re=(e_tip.real, 0, 0, 0, e_tip.real, 0, 0, 0, e_tip.real),
                     eps_im=(e_tip.imag, 0, 0, 0, e_tip.imag, 0, 0, 0, e_tip.imag), use_ade=1)]
    med = np.zeros((N, N, N), np.int32)
    med[:, :, :16] = 1
    med[cone_tip_mask(N, N, N, DL, DL, (N // 2, N // 2), 18, 20e-9, 15.0, top_k=N - 10)] = 2
    src = [Source(type=1, x=N // 2, y=N // 2, z=N - 14, component="z", frequency=F_SRC)]
    return make_desc(med, mats, src, dx=DL, dy=DL, dz=DL, dt=DT, pml_thickness=8, precision=precision,
                     source_frequency=F_SRC), med


def _run(precision, steps):
    holder, med = _case(precision)
    with Simulation(holder) as sim:
        pid = sim.dft_add("Ez", 18, [F_SRC])
        sim.step(steps)
        sim.sync()
        E = [sim.read_volume(c) for c in ("Ex", "Ey", "Ez")]
        tip = np.argwhere(med == 2)
        cell = tuple(int(x) for x in tip[len(tip) // 2])
        return E, sim.dft_read(pid)[0][0], sim.read_cell_state(*cell), med


def test_fp32_fields_and_nearfield_within_bounds():
    e64, f64, s64, med = _run("fp64", 3000)
    e32, f32, s32, _ = _run("fp32", 3000)
    assert (med == 2).sum() > 100
    num = sum(float(np.sum((a - b) ** 2)) for a, b in zip(e32, e64))
    den = sum(float(np.sum(b ** 2)) for b in e64)
    field_err = math.sqrt(num / den)
    near_err = float(np.linalg.norm(f32 - f64) / np.linalg.norm(f64))
    assert field_err <= 1e-4, field_err
    assert near_err <= 1e-3, near_err
    # ADE state read back in the reference's terms (P, P_old)
    for key in ("P", "P_old"):
        scale = float(np.max(np.abs(s64["P"])))
        assert scale > 0
        np.testing.assert_allclose(s32[key], s64[key], rtol=0, atol=1e-3 * scale, err_msg=key)

