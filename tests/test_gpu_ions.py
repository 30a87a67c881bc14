"""The ion pass of many-atom cells (php_ions.cuh): selected for 16-atom
lattices in the fast paths, equal to the fused in-sweep update in FP64, and
within the FP32 error bound with DMM . r on the tensor cores (BF16 x 3)."""
import math
import os

import numpy as np
import pytest

import harness as H
from php_fdtd_b200 import Config, Simulation

pytestmark = pytest.mark.gpu


def _holder(d, precision):
    with H.chdir(d):
        cfg = Config.load("case.cfg")
        return cfg, cfg.desc(cfg.load_medium(), precision)


def _sim(holder, fused=False):
    old = os.environ.get("PHP_IONS")
    if fused:
        os.environ["PHP_IONS"] = "fused"
    try:
        return Simulation(holder)
    finally:
        if old is None:
            os.environ.pop("PHP_IONS", None)
        else:
            os.environ["PHP_IONS"] = old


def _atom_cells(cfg):
    # inside and at the edges of the 16-atom block of the case
    return [(cfg.nx // 2, cfg.ny // 2, 2), (3, 3, 1), (cfg.nx - 4, cfg.ny - 4, 4), (5, 7, 3)]


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_ion_pass_is_one_extra_launch(precision, golden_case):
    cfg, holder = _holder(golden_case("ions16"), precision)
    with _sim(holder) as a, _sim(holder, fused=True) as b:
        a.step(3)
        b.step(3)
        assert a.last_launch_count == 3 * 3
        assert b.last_launch_count == 3 * 2


def test_fp64_ion_pass_equals_fused_update(golden_case):
    cfg, holder = _holder(golden_case("ions16"), "fp64")
    with _sim(holder) as a, _sim(holder, fused=True) as b:
        a.step(40)
        b.step(40)
        for comp in range(9):
            x, y = a.read_volume(comp), b.read_volume(comp)
            scale = max(float(np.max(np.abs(y))), 1e-300)
            assert float(np.max(np.abs(x - y))) <= 1e-12 * scale, comp
        for cell in _atom_cells(cfg):
            sa, sb = a.read_cell_state(*cell), b.read_cell_state(*cell)
            assert sa["natom"] == sb["natom"]
            if sa["natom"]:
                scale = max(float(np.max(np.abs(sb["r"]))), 1e-300)
                assert float(np.max(np.abs(sa["r"] - sb["r"]))) <= 1e-12 * scale


def test_fp32_tensor_ion_pass_against_fp64(golden_case):
    """BF16 x 3 DMM . r with FP32 accumulation, against the FP64 path."""
    d = golden_case("ions16")
    cfg, h64 = _holder(d, "fp64")
    _, h32 = _holder(d, "fp32")
    with _sim(h64) as a, _sim(h32) as b:
        a.step(40)
        b.step(40)
        num = den = 0.0
        for comp in ("Ex", "Ey", "Ez"):
            x, y = b.read_volume(comp), a.read_volume(comp)
            num += float(np.sum((x - y) ** 2))
            den += float(np.sum(y ** 2))
        assert math.sqrt(num / den) <= 1e-4
        for cell in _atom_cells(cfg):
            s64, s32 = a.read_cell_state(*cell), b.read_cell_state(*cell)
            if s64["natom"]:
                scale = float(np.max(np.abs(s64["r"])))
                if scale > 0:
                    assert float(np.max(np.abs(s32["r"] - s64["r"]))) <= 1e-3 * scale
