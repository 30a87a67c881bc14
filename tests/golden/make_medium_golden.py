"""Makes tests/golden/medium/: a .cfg whose [medium] section uses every
shape of the reference's medium generator (cubes, hexahedra, cylinders, an
anisotropic grid spacing) and the medium map that generator writes for it.

    python tests/golden/make_medium_golden.py [/path/to/reference]

Runs the reference's generate_medium5.py itself (it needs only numpy); the
result is committed as medium_golden.npz so that tests never need the reference.
"""
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent / "medium"
CFG = """[grid]
nx = 40
ny = 36
nz = 30
delta_x = 1e-08
delta_y = 1.5e-08
delta_z = 8e-09

[medium]
# a slab, an oblique block, a tilted rod and a vertical rod
cubes = [ {"xrange": (0, 39), "yrange": (0, 35), "zrange": (0, 5), "material": 4},
          {"xrange": (30, 45), "yrange": (2, 9), "zrange": (20, 29), "material": 2} ]
hexahedra = [ {"vertices": [(5, 5, 8), (15, 7, 8), (17, 15, 8), (7, 13, 8),
                            (6, 6, 14), (16, 8, 14), (18, 16, 14), (8, 14, 14)], "material": 3} ]
cylinders = [ {"p1": (20, 18, 6), "p2": (34, 30, 26), "radius": 3.2e-08, "material": 5},
              {"p1": (8, 28, 6), "p2": (8, 28, 29), "radius": 2.5e-08, "material": 6} ]
"""


def main(ref: Path):
    HERE.mkdir(parents=True, exist_ok=True)
    (HERE / "case.cfg").write_text(CFG)
    out = HERE / "reference_medium_map.bin"
    subprocess.run([sys.executable, str(ref / "generate_medium5.py"), "case.cfg", out.name], cwd=HERE, check=True,
                   capture_output=True)
    raw = out.read_bytes()
    shape = np.frombuffer(raw[:12], dtype=np.int32)
    med = np.frombuffer(raw[12:], dtype=np.int32).reshape(shape)
    np.savez_compressed(HERE / "medium_golden.npz", shape=shape, medium=med)
    out.unlink()
    print("wrote", HERE / "medium_golden.npz", shape.tolist(), np.unique(med).tolist())


if __name__ == "__main__":
    import os
    arg = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PHP_REFERENCE_DIR", "")
    if not arg:
        sys.exit("usage: make_medium_golden.py <reference checkout>  (or set PHP_REFERENCE_DIR)")
    main(Path(arg))
