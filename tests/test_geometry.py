"""Medium-map generator (php_fdtd_b200.geometry) against the medium map the
reference's generator wrote for the same [medium] section, and the tip
shape against the workload generator's."""
import struct
from pathlib import Path

import numpy as np

from php_fdtd_b200 import geometry
from php_fdtd_b200.workloads import cone_tip_mask

GOLD = Path(__file__).resolve().parent / "golden" / "medium"


def test_shapes_match_the_reference_generator():
    g = np.load(GOLD / "medium_golden.npz")
    med = geometry.medium_from_cfg((GOLD / "case.cfg").read_text())
    assert med.shape == tuple(g["shape"])
    np.testing.assert_array_equal(med, g["medium"])


def test_file_format_and_cli(tmp_path):
    out = tmp_path / "m.bin"
    assert geometry.main(["geometry", str(GOLD / "case.cfg"), str(out)]) == 0
    raw = out.read_bytes()
    nx, ny, nz = struct.unpack("iii", raw[:12])
    med = np.frombuffer(raw[12:], dtype=np.int32).reshape(nx, ny, nz)
    np.testing.assert_array_equal(med, np.load(GOLD / "medium_golden.npz")["medium"])


def test_no_medium_section_is_vacuum():
    med = geometry.medium_from_cfg("nx = 5\nny = 4\nnz = 3\n")
    assert med.shape == (5, 4, 3) and not med.any()


def test_cone_tip_and_sphere():
    text = """nx = 64
ny = 64
nz = 48
delta_x = 5e-09
delta_y = 5e-09
delta_z = 5e-09
[medium]
cubes = [ {"xrange": (0, 63), "yrange": (0, 63), "zrange": (0, 9), "material": 4} ]
cones = [ {"apex": (32, 32, 12), "radius": 2e-08, "half_angle": 15.0, "top": 40, "material": 5} ]
spheres = [ {"center": (10, 10, 30), "radius": 1.2e-08, "material": 6} ]
"""
    med = geometry.medium_from_cfg(text)
    tip = cone_tip_mask(64, 64, 48, 5e-9, 5e-9, (32, 32), 12, 20e-9, 15.0, top_k=40)
    np.testing.assert_array_equal(med == 5, tip)
    assert (med[:, :, :10] == 4).all()
    ball = med == 6
    assert ball.sum() > 0 and ball[10, 10, 30] and not ball[10, 10, 34]
