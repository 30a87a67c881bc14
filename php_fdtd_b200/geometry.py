"""Medium-map generator: the ``[medium]`` section of a .cfg to the
``medium_map.bin`` the solver reads (header of three int32 nx, ny, nz, then
int32 material ids in [nx][ny][nz] order, z fastest; fdtd.c:808-817).

The section grammar and fill rules are those of the reference's generator
(generate_medium5.py:8-372), applied in its order:

  cubes     = [ {"xrange": (x0, x1), "yrange": (y0, y1), "zrange": (z0, z1), "material": m}, ... ]
              inclusive cell ranges, clipped to the grid
  hexahedra = [ {"vertices": [v0 .. v7], "material": m}, ... ]
              parallelepiped spanned by v1-v0, v3-v0, v4-v0 (cell indices);
              a cell is inside when its affine coordinates lie in [0, 1]
  cylinders = [ {"p1": (i, j, k), "p2": (i, j, k), "radius": r, "material": m}, ... ]
              axis between two cell positions, radius in metres (cell
              spacing from delta_x/y/z)

and two shapes the benchmark tips need, applied after those:

  spheres   = [ {"center": (i, j, k), "radius": r, "material": m}, ... ]
  cones     = [ {"apex": (i, j, k), "radius": r, "half_angle": deg, "top": k1, "material": m}, ... ]
              a cone opening towards +z whose apex is rounded by a sphere of
              radius r tangent to the cone (an AFM/s-SNOM tip), cut at plane k1

Usage: ``python -m php_fdtd_b200.geometry case.cfg [medium_map.bin]``.
"""
from __future__ import annotations

import ast
import math
import re
import struct
import sys
from pathlib import Path
from typing import Dict, List

import numpy as np


def _grid(text: str):
    def num(key, default, conv):
        m = re.search(key + r"\s*=\s*([\d.eE+-]+)", text)
        return conv(m.group(1)) if m else default
    n = tuple(num(k, 50, int) for k in (r"nx", r"ny", r"nz"))
    d = tuple(num(k, 1.0, float) for k in (r"delta_x", r"delta_y", r"delta_z"))
    return n, d


def _section(text: str) -> str:
    m = re.search(r"\[medium\](.*?)(?=\n\[|\Z)", text, re.S | re.I)
    return m.group(1) if m else ""


def _literal_list(sec: str, key: str) -> list:
    """The bracketed Python list after `key =` (comments removed)."""
    sec = re.sub(r"#.*", "", sec)
    m = re.search(key + r"\s*=", sec, re.I)
    if not m:
        return []
    rest = sec[m.end():]
    start = rest.find("[")
    if start < 0:
        return []
    depth = 0
    for i in range(start, len(rest)):
        depth += {"[": 1, "]": -1}.get(rest[i], 0)
        if depth == 0:
            try:
                val = ast.literal_eval(rest[start:i + 1])
            except (ValueError, SyntaxError):
                return []
            return [v for v in val if isinstance(v, dict)]
    return []


_CUBE = re.compile(r'\{\s*"xrange"\s*:\s*\(\s*(\d+)\s*,\s*(\d+)\s*\),\s*"yrange"\s*:\s*\(\s*(\d+)\s*,\s*(\d+)\s*\),'
                   r'\s*"zrange"\s*:\s*\(\s*(\d+)\s*,\s*(\d+)\s*\),\s*"material"\s*:\s*(\d+)\s*\}')


def parse_shapes(text: str) -> Dict[str, list]:
    sec = _section(text)
    shapes: Dict[str, list] = {"cubes": [], "hexahedra": [], "cylinders": [], "spheres": [], "cones": []}
    m = re.search(r"cubes\s*=\s*\[(.*?)\]", sec, re.S)
    if m:
        body = re.sub(r"\s+", " ", re.sub(r"#.*", "", m.group(1)).replace("\n", " "))
        for c in _CUBE.finditer(body):
            x0, x1, y0, y1, z0, z1, mat = map(int, c.groups())
            shapes["cubes"].append({"xrange": (x0, x1), "yrange": (y0, y1), "zrange": (z0, z1), "material": mat})
    for h in _literal_list(sec, "hexahedra"):
        if "vertices" in h and "material" in h and len(h["vertices"]) == 8:
            shapes["hexahedra"].append({"vertices": [tuple(float(c) for c in v) for v in h["vertices"]],
                                        "material": int(h["material"])})
    for c in _literal_list(sec, "cylinders"):
        if all(k in c for k in ("p1", "p2", "radius", "material")):
            shapes["cylinders"].append({"p1": tuple(float(x) for x in c["p1"]), "p2": tuple(float(x) for x in c["p2"]),
                                        "radius": float(c["radius"]), "material": int(c["material"])})
    for s in _literal_list(sec, "spheres"):
        if all(k in s for k in ("center", "radius", "material")):
            shapes["spheres"].append({"center": tuple(float(x) for x in s["center"]), "radius": float(s["radius"]),
                                      "material": int(s["material"])})
    for c in _literal_list(sec, "cones"):
        if all(k in c for k in ("apex", "radius", "half_angle", "material")):
            shapes["cones"].append({"apex": tuple(float(x) for x in c["apex"]), "radius": float(c["radius"]),
                                    "half_angle": float(c["half_angle"]), "top": c.get("top"),
                                    "material": int(c["material"])})
    return shapes


def _box(lo, hi, n):
    return max(0, int(math.floor(lo))), min(n - 1, int(math.ceil(hi)))


def _grid_points(b0, b1, b2):
    return np.meshgrid(np.arange(b0[0], b0[1] + 1), np.arange(b1[0], b1[1] + 1), np.arange(b2[0], b2[1] + 1),
                       indexing="ij")


def build_medium(shape, delta, shapes: Dict[str, list]) -> np.ndarray:
    nx, ny, nz = shape
    dx, dy, dz = delta
    med = np.zeros((nx, ny, nz), dtype=np.int32)
    for c in shapes.get("cubes", []):
        (x0, x1), (y0, y1), (z0, z1) = c["xrange"], c["yrange"], c["zrange"]
        med[max(x0, 0):min(x1 + 1, nx), max(y0, 0):min(y1 + 1, ny), max(z0, 0):min(z1 + 1, nz)] = c["material"]
    for h in shapes.get("hexahedra", []):
        v = np.array(h["vertices"], dtype=np.float64)
        basis = np.column_stack((v[1] - v[0], v[3] - v[0], v[4] - v[0]))
        if abs(np.linalg.det(basis)) < 1e-300:
            continue
        inv = np.linalg.inv(basis)
        bx, by, bz = (_box(v[:, a].min(), v[:, a].max(), n) for a, n in zip(range(3), (nx, ny, nz)))
        X, Y, Z = _grid_points(bx, by, bz)
        p = np.stack((X.ravel(), Y.ravel(), Z.ravel())).astype(np.float64) - v[0][:, None]
        f = inv @ p
        tol = 1e-9
        inside = np.all((f >= -tol) & (f <= 1 + tol), axis=0).reshape(X.shape)
        med[X[inside], Y[inside], Z[inside]] = h["material"]
    for c in shapes.get("cylinders", []):
        p1, p2 = np.array(c["p1"]), np.array(c["p2"])
        sc = np.array([dx, dy, dz])
        a = p1 * sc
        axis = p2 * sc - a  # in this order, as the reference rounds it
        length = float(np.linalg.norm(axis))
        if length < 1e-12:
            continue
        u = axis / length
        r = c["radius"]
        bounds = [_box(min(p1[q], p2[q]) - r / sc[q], max(p1[q], p2[q]) + r / sc[q], n)
                  for q, n in zip(range(3), (nx, ny, nz))]
        X, Y, Z = _grid_points(*bounds)
        wx, wy, wz = X * dx - a[0], Y * dy - a[1], Z * dz - a[2]
        t = wx * u[0] + wy * u[1] + wz * u[2]
        perp2 = (wx - t * u[0]) ** 2 + (wy - t * u[1]) ** 2 + (wz - t * u[2]) ** 2
        inside = (t >= 0.0) & (t <= length) & (perp2 <= r * r)
        med[X[inside], Y[inside], Z[inside]] = c["material"]
    I, J, K = (np.arange(n) for n in (nx, ny, nz))
    for s in shapes.get("spheres", []):
        ci, cj, ck = s["center"]
        d2 = (((I - ci) * dx)[:, None, None] ** 2 + ((J - cj) * dy)[None, :, None] ** 2
              + ((K - ck) * dz)[None, None, :] ** 2)
        med[d2 <= s["radius"] ** 2] = s["material"]
    for c in shapes.get("cones", []):
        ai, aj, ak = c["apex"]
        r, ang = c["radius"], math.radians(c["half_angle"])
        x = ((I - ai) * dx)[:, None, None]
        y = ((J - aj) * dy)[None, :, None]
        z = ((K - ak) * dz)[None, None, :]
        rho2 = x * x + y * y
        in_cap = rho2 + (z - r) ** 2 <= r * r                 # sphere of radius r resting on the apex plane
        z_t = r - r * math.sin(ang)                           # where the cone touches that sphere
        r_cone = r * math.cos(ang) + (z - z_t) * math.tan(ang)
        in_cone = (z >= z_t) & (rho2 <= r_cone * r_cone) & (r_cone >= 0)
        mask = in_cap | in_cone
        if c.get("top") is not None:
            mask &= (K <= int(c["top"]))[None, None, :]
        med[np.broadcast_to(mask, med.shape)] = c["material"]
    return med


def medium_from_cfg(text: str) -> np.ndarray:
    shape, delta = _grid(text)
    return build_medium(shape, delta, parse_shapes(text))


def write_medium_map(path, med: np.ndarray):
    med = np.ascontiguousarray(med, dtype=np.int32)
    with open(path, "wb") as f:
        f.write(struct.pack("iii", *med.shape))
        f.write(med.tobytes())


def main(argv: List[str]) -> int:
    if len(argv) < 2:
        print("usage: python -m php_fdtd_b200.geometry <config_file> [output_file]")
        return 1
    cfg = Path(argv[1])
    if not cfg.exists():
        print(f"Error: Config file '{cfg}' not found")
        return 1
    out = argv[2] if len(argv) > 2 else "medium_map.bin"
    med = medium_from_cfg(cfg.read_text())
    write_medium_map(out, med)
    ids, counts = np.unique(med, return_counts=True)
    for i, n in zip(ids, counts):
        print(f"  material {i}: {n} cells ({100.0 * n / med.size:.2f}%)")
    print(f"{out}: {med.shape[0]}x{med.shape[1]}x{med.shape[2]}")
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
