"""Seeded synthetic inputs in the reference's file formats.

``write_case`` writes a .cfg, a medium_map.bin and any QeZV / QeZM / DMM /
OUTCAR / dielectric-table files into a directory, so that the reference
solver, the oracle and the GPU path can all run the very same inputs.
``SMALL_CASES`` are the parity cases (each material class, source type and
output form of the reference); ``baseline_case`` builds the benchmark
workloads (grid, PML, materials and sources of the five benchmark
configurations) at any step count.

Lattice data follow the physical definitions of the reference's data files
(README section 7.2): QeZV = Z* e / Omega, QeZM = Z* e / m, DMM = Q Lambda Q^T
with Lambda the squared mode frequencies (omega = 2 pi 0.03e12 nu~, the
reference's wavenumber convention).
"""
from __future__ import annotations

import math
import struct
from dataclasses import dataclass, field
from pathlib import Path
from typing import Dict, List, Optional, Sequence

import numpy as np

E_CHARGE = 1.602176634e-19
AMU = 1.66053906660e-27
C_CM = 0.03e12  # Hz per cm^-1, fdtd.c:1504


def omega_of_wavenumber(nu_cm: float) -> float:
    return 2.0 * math.pi * C_CM * nu_cm


# ------------------------------------------------------------ lattice data


def lattice_data(zstar: np.ndarray, masses_amu: Sequence[float], mode_wavenumbers: Sequence[float], seed: int,
                 omega_cell_A3: float):
    """QeZV, QeZM ([natom][iE][idir]) and DMM ([3N][3N]) of a synthetic
    lattice.  zstar is [natom][3][3] in units of e."""
    zstar = np.asarray(zstar, dtype=np.float64)
    natom = zstar.shape[0]
    n3 = 3 * natom
    rng = np.random.default_rng(seed)
    q, _ = np.linalg.qr(rng.standard_normal((n3, n3)))
    lam = np.array([omega_of_wavenumber(w) ** 2 for w in mode_wavenumbers], dtype=np.float64)
    if lam.size != n3:
        raise ValueError(f"need {n3} mode wavenumbers, got {lam.size}")
    dmm = (q * lam) @ q.T
    dmm = 0.5 * (dmm + dmm.T)
    omega = omega_cell_A3 * 1e-30
    m = np.asarray(masses_amu, dtype=np.float64) * AMU
    qezv = zstar * E_CHARGE / omega
    qezm = zstar * E_CHARGE / m[:, None, None]
    return qezv, qezm, dmm


def lattice_2atom(seed: int = 0):
    """The 2-atom polar lattice of the benchmark's config 0: masses 10.8 and
    14.0 amu, Z* = +-diag(2.7, 2.7, 0.9) e, TO modes at 1370 (x2) and
    780 cm^-1 plus three zeros, cell volume 17.31 A^3."""
    z = np.zeros((2, 3, 3))
    z[0] = np.diag([2.7, 2.7, 0.9])
    z[1] = -np.diag([2.7, 2.7, 0.9])
    return lattice_data(z, [10.8, 14.0], [1370.0, 1370.0, 780.0, 0.0, 0.0, 0.0], seed, 17.31)


def lattice_16atom(seed: int = 0):
    """The 16-atom cell of the benchmark's config 2: 12 x 16.0 + 4 x 95.95 amu,
    Born diagonals uniform in +-[1, 6] e, off-diagonals in +-0.5 e, shifted to
    satisfy the acoustic sum rule; 45 modes uniform in 300-1000 cm^-1 plus
    three zeros."""
    rng = np.random.default_rng(seed + 1000)
    z = rng.uniform(-0.5, 0.5, size=(16, 3, 3))
    for a in range(16):
        d = rng.uniform(1.0, 6.0, size=3) * rng.choice([-1.0, 1.0], size=3)
        z[a][np.arange(3), np.arange(3)] = d
    z -= z.mean(axis=0, keepdims=True)  # acoustic sum rule: sum_a Z*_a = 0
    masses = [16.0] * 12 + [95.95] * 4
    modes = list(np.sort(rng.uniform(300.0, 1000.0, size=45))) + [0.0, 0.0, 0.0]
    return lattice_data(z, masses, modes, seed, 200.54)


def write_numbers(path: Path, arr: np.ndarray):
    with open(path, "w") as f:
        for v in np.asarray(arr, dtype=np.float64).ravel():
            f.write(f"{v:.17g}\n")


def write_outcar(path: Path, eps: np.ndarray, born: np.ndarray):
    """A VASP OUTCAR fragment with the two blocks read_born_from_file parses
    (fdtd.c:423-552)."""
    lines = [" MACROSCOPIC STATIC DIELECTRIC TENSOR (including local field effects)",
             " ------------------------------------------------------"]
    for r in range(3):
        lines.append("  " + "  ".join(f"{eps[r, c]:12.6f}" for c in range(3)))
    lines += [" ------------------------------------------------------", "", "",
              " BORN EFFECTIVE CHARGES (including local field effects) (in |e|, cummulative output)",
              " ---------------------------------------------------------------------------------"]
    for a in range(born.shape[0]):
        lines.append(f" ion {a + 1:4d}")
        for r in range(3):
            lines.append(f"    {r + 1}  " + "  ".join(f"{born[a, r, c]:11.5f}" for c in range(3)))
    path.write_text("\n".join(lines) + "\n")


def write_dielectric_table(path: Path, freqs_hz: Sequence[float], eps_fn):
    """15-column table of read_dielectric_from_file (fdtd.c:346-401):
    f, wavelength, wavenumber, Re xx xy xz yy yz zz, Im xx xy xz yy yz zz."""
    with open(path, "w") as f:
        f.write("# synthetic dielectric table\n")
        for fr in freqs_hz:
            e = np.asarray(eps_fn(fr), dtype=np.complex128)
            vals = [fr, 0.0, fr / C_CM, e[0, 0].real, e[0, 1].real, e[0, 2].real, e[1, 1].real, e[1, 2].real,
                    e[2, 2].real, e[0, 0].imag, e[0, 1].imag, e[0, 2].imag, e[1, 1].imag, e[1, 2].imag, e[2, 2].imag]
            f.write("  ".join(f"{v:.10g}" for v in vals) + "\n")


def write_medium(path: Path, medium: np.ndarray):
    medium = np.ascontiguousarray(medium, dtype=np.int32)
    nx, ny, nz = medium.shape
    with open(path, "wb") as f:
        f.write(struct.pack("iii", nx, ny, nz))
        medium.tofile(f)


# ------------------------------------------------------------------- cases


@dataclass
class CaseSpec:
    name: str
    nx: int
    ny: int
    nz: int
    tsteps: int
    delta: Sequence[float] = (10e-9, 10e-9, 10e-9)
    pml: int = 4
    pml_reflection: float = 1e-6
    output_interval: int = 10
    output_component: str = "Ez"
    slice_axis: str = "z"
    slice_pos: int = 0
    dt: Optional[float] = None
    sources: List[str] = field(default_factory=list)     # cfg source lines (after "source")
    materials: List[str] = field(default_factory=list)   # cfg material lines (after "material")
    monitor: Optional[str] = None                         # monitor_point value
    full_monitor: int = 0
    medium_fn: Optional[object] = None                    # (nx,ny,nz) -> int32 array
    files_fn: Optional[object] = None                     # (dir) -> None, writes data files
    expect_abort: bool = False                            # the run ends in the divergence abort (exit 1)


def write_case(spec: CaseSpec, out: Path) -> Path:
    out = Path(out)
    out.mkdir(parents=True, exist_ok=True)
    medium = spec.medium_fn(spec.nx, spec.ny, spec.nz) if spec.medium_fn else np.zeros((spec.nx, spec.ny, spec.nz), np.int32)
    write_medium(out / "medium_map.bin", medium)
    if spec.files_fn:
        spec.files_fn(out)
    L = [f"# {spec.name}", "[grid]", f"nx = {spec.nx}", f"ny = {spec.ny}", f"nz = {spec.nz}",
         f"delta_x = {spec.delta[0]!r}", f"delta_y = {spec.delta[1]!r}", f"delta_z = {spec.delta[2]!r}",
         f"tsteps = {spec.tsteps}"]
    if spec.dt is not None:
        L.append(f"dt = {spec.dt!r}")
    L += [f"pml_thickness = {spec.pml}", f"pml_reflection = {spec.pml_reflection!r}",
          f"output_interval = {spec.output_interval}", f"output_component = {spec.output_component}",
          f"output_slice_axis = {spec.slice_axis}", f"output_slice_position = {spec.slice_pos}"]
    for s in spec.sources:
        L.append("source " + s)
    for m in spec.materials:
        L.append("material " + m)
    L.append("medium_file = ./medium_map.bin")
    if spec.monitor:
        L += [f"monitor_point = {spec.monitor}", "monitor_output_file = monitor_point.dat"]
    if spec.full_monitor:
        L += ["full_monitor = 1", "full_monitor_output_file = full_monitor.dat"]
    (out / "case.cfg").write_text("\n".join(L) + "\n")
    return out / "case.cfg"


def _slab(k_max: int, mat: int, base=None):
    def fn(nx, ny, nz):
        m = np.zeros((nx, ny, nz), np.int32) if base is None else base(nx, ny, nz)
        m[:, :, :k_max] = mat
        return m
    return fn


def _blocks(*blocks):
    """blocks of (x0, x1, y0, y1, z0, z1, mat), inclusive like generate_medium5's cubes"""
    def fn(nx, ny, nz):
        m = np.zeros((nx, ny, nz), np.int32)
        for x0, x1, y0, y1, z0, z1, mat in blocks:
            m[x0:x1 + 1, y0:y1 + 1, z0:z1 + 1] = mat
        return m
    return fn


def _ions2_files(d: Path, seed: int = 0):
    qv, qm, dmm = lattice_2atom(seed)
    write_numbers(d / "QeZV.txt", qv)
    write_numbers(d / "QeZM.txt", qm)
    write_numbers(d / "DMM.txt", dmm)


def _ions16_files(d: Path, seed: int = 0):
    qv, qm, dmm = lattice_16atom(seed)
    write_numbers(d / "QeZV16.txt", qv)
    write_numbers(d / "QeZM16.txt", qm)
    write_numbers(d / "DMM16.txt", dmm)
    born = qv * 200.54e-30 / E_CHARGE
    write_outcar(d / "OUTCAR.txt", np.array([[5.8, 0.0, 0.0], [0.0, 6.6, 0.0], [0.0, 0.0, 4.4]]), born)


def _drude_table(d: Path):
    def eps(fr):
        w = omega_of_wavenumber(fr / C_CM)
        e = []
        for wp, g in ((9.0e14, 2.0e13), (8.0e14, 3.0e13), (7.5e14, 1.0e13)):
            e.append(1.0 - wp * wp / (w * w + 1j * g * w))
        return np.diag(e)
    write_dielectric_table(d / "drude.txt", [C_CM * w for w in np.arange(600.0, 1600.0, 37.0)], eps)


MAT_ANISO = "id=4, name=aniso, eps_xx=4.0, eps_xy=0.7, eps_xz=0.2, eps_yx=0.7, eps_yy=3.0, eps_yz=-0.3, eps_zx=0.2, eps_zy=-0.3, eps_zz=2.5"
MAT_LOSSY_ROTZ = ("id=5, name=lossyrot, eps_xx=6.0, eps_yy=3.5, eps_zz=2.8, eps_xxi=0.4, eps_yyi=0.2, eps_zzi=0.1, "
                  "eps_xyi=0.05, eps_yxi=0.05, anglez=0.5235987756")
MAT_ROTX = "id=6, name=rotx, eps_xx=5.0, eps_yy=2.0, eps_zz=3.0, eps_yzi=0.1, eps_zyi=0.1, anglex=0.3490658504"
MAT_METAL = ("id=7, name=metal, use_ADE=1, eps_xx=-300, eps_yy=-300, eps_zz=-300, eps_xxi=150, eps_yyi=150, "
             "eps_zzi=150, sigma=2000")
MAT_IONS2 = "id=8, name=polar2, natom=2, QeZV=QeZV.txt, QeZM=QeZM.txt, DMM=DMM.txt, eps_xx=4.9, eps_yy=4.9, eps_zz=2.95"
MAT_IONS2_ROT = ("id=9, name=polar2x, natom=2, QeZV=QeZV.txt, QeZM=QeZM.txt, DMM=DMM.txt, eps_xx=4.9, eps_yy=4.9, "
                 "eps_zz=2.95, anglex=0.3490658504")
MAT_IONS16 = "id=10, name=moo3like, natom=16, born=OUTCAR.txt, QeZV=QeZV16.txt, QeZM=QeZM16.txt, DMM=DMM16.txt, switchxz=1"
MAT_DRUDE_TABLE = "id=11, name=drude, dielectric=drude.txt, use_ADE=1, switchxz=1"

DIPOLE = "type=dipole, x={x},y={y},z={z}, amplitude=1.0, wavenumber={wn}, component={c}, t0={t0}, tau={tau}"


def _dip(x, y, z, c="z", wn=1370, t0=3e-16, tau=1e-16):
    return DIPOLE.format(x=x, y=y, z=z, c=c, wn=wn, t0=t0, tau=tau)


def _all_files(d: Path):
    _ions2_files(d)
    _ions16_files(d)
    _drude_table(d)


SMALL_CASES: Dict[str, CaseSpec] = {}


def _add(spec: CaseSpec):
    SMALL_CASES[spec.name] = spec


_add(CaseSpec("vacuum_pml", 20, 18, 16, 60, pml=4, output_interval=10, slice_pos=7,
              sources=[_dip(10, 9, 8)], monitor="x=10,y=9,z=6,atom=0,dir=z"))
_add(CaseSpec("aniso_lossy", 19, 17, 15, 50, pml=3, output_component="Ex", slice_pos=6,
              sources=[_dip(9, 8, 10, c="x", wn=1100)], materials=[MAT_ANISO],
              medium_fn=_blocks((3, 15, 3, 13, 0, 5, 4), (5, 9, 5, 9, 6, 8, 3), (10, 13, 6, 10, 6, 8, 2)),
              monitor="x=8,y=8,z=4,atom=0,dir=x"))
_add(CaseSpec("lossy_rot", 18, 18, 16, 50, pml=4, output_component="E", slice_axis="x", slice_pos=9,
              sources=["type=sinusoidal, x=9,y=9,z=11, amplitude=1.0, frequency=2.7e13, component=y"],
              materials=[MAT_LOSSY_ROTZ, MAT_ROTX],
              medium_fn=_blocks((2, 15, 2, 15, 0, 6, 5), (4, 12, 4, 12, 7, 8, 6)),
              monitor="x=9,y=9,z=5,atom=0,dir=y"))
_add(CaseSpec("ade_metal", 18, 16, 18, 60, pml=4, output_component="Dx", slice_axis="y", slice_pos=8,
              sources=["type=gaussian, x=9,y=8,z=13, amplitude=1.0, component=x, t0=2e-16, tau=0.8e-16",
                       "type=ricker, x=7,y=8,z=12, amplitude=0.5, frequency=3.0e13, component=z, t0=3e-16"],
              materials=[MAT_METAL], medium_fn=_blocks((5, 12, 4, 11, 3, 9, 7)),
              monitor="x=9,y=8,z=6,atom=0,dir=z"))
_add(CaseSpec("ions2", 16, 16, 16, 60, pml=4, output_component="Ez", slice_pos=5,
              sources=[_dip(8, 8, 11, wn=1370, t0=2e-16, tau=1e-16)], materials=[MAT_IONS2, MAT_IONS2_ROT],
              medium_fn=_blocks((0, 15, 0, 15, 0, 5, 8), (4, 11, 4, 11, 6, 7, 9)), files_fn=_all_files,
              monitor="x=8,y=8,z=4,atom=1,dir=z"))
# ions2 driven hard enough that |r| passes 1e-10 m at step 20: the
# reference's divergence report and abort (fdtd.c:3626-3668)
_add(CaseSpec("ions2_diverge", 16, 16, 16, 60, pml=4, output_component="Ez", slice_pos=5,
              sources=[_dip(8, 8, 11, wn=1370, t0=2e-16, tau=1e-16).replace("amplitude=1.0", "amplitude=1e24")],
              materials=[MAT_IONS2, MAT_IONS2_ROT],
              medium_fn=_blocks((0, 15, 0, 15, 0, 5, 8), (4, 11, 4, 11, 6, 7, 9)), files_fn=_all_files,
              monitor="x=8,y=8,z=4,atom=1,dir=z", expect_abort=True))
_add(CaseSpec("ions16", 14, 13, 12, 40, pml=3, output_component="Ey", slice_pos=4,
              sources=[_dip(7, 6, 9, c="x", wn=820, t0=2e-16, tau=1e-16)], materials=[MAT_IONS16],
              medium_fn=_blocks((2, 11, 2, 10, 1, 5, 10)), files_fn=_all_files,
              monitor="x=6,y=6,z=3,atom=5,dir=y"))
_add(CaseSpec("drude_table", 16, 16, 14, 50, pml=3, output_component="Ez", slice_axis="x", slice_pos=8,
              sources=[_dip(8, 8, 10, wn=950, t0=2e-16, tau=1e-16)], materials=[MAT_DRUDE_TABLE, "id=1"],
              medium_fn=_blocks((4, 11, 4, 11, 2, 6, 11), (0, 15, 0, 15, 0, 1, 1)), files_fn=_all_files,
              monitor="x=8,y=8,z=5,atom=0,dir=x"))
_add(CaseSpec("multi_source_ragged", 21, 11, 9, 40, pml=2, output_component="Ey", slice_axis="z", slice_pos=4,
              delta=(8e-9, 12e-9, 10e-9),
              sources=[_dip(10, 5, 4, c="y", wn=1500), "type=sinusoidal, x=3,y=3,z=3, frequency=2e13, component=x",
                       "type=gaussian, x=30,y=3,z=3, component=z, t0=1e-16, tau=1e-16",
                       _dip(10, 5, 4, c="y", wn=900)],
              materials=[MAT_ANISO], medium_fn=_blocks((5, 15, 2, 8, 2, 6, 4)),
              monitor="x=10,y=5,z=3,atom=0,dir=x"))
_add(CaseSpec("no_pml_tiny", 3, 3, 2, 12, pml=0, output_interval=3, output_component="Ex", slice_axis="y", slice_pos=1,
              sources=[_dip(1, 1, 0, c="x", wn=1200, t0=1e-16, tau=0.5e-16)], materials=[MAT_ANISO],
              medium_fn=_blocks((0, 2, 0, 2, 0, 0, 4)), monitor="x=1,y=1,z=0,atom=0,dir=x"))
# a sine-driven run with an explicit dt and 101 z slices above a two-atom
# slab: the input of the reference's post-processor (frequency_analysis.c),
# whose spectra pin the running DFT
_add(CaseSpec("spectra_dft", 24, 22, 20, 201, pml=4, output_interval=2, output_component="Ez", slice_axis="z",
              slice_pos=9, dt=10e-9 / (299792458.0 * math.sqrt(3.0)) * 0.99,
              sources=["type=sinusoidal, x=12,y=11,z=13, amplitude=1.0, frequency=1.2e15, component=z"],
              materials=[MAT_IONS2, MAT_ANISO], medium_fn=_blocks((0, 23, 0, 21, 0, 3, 8), (6, 17, 5, 16, 4, 5, 4)),
              files_fn=_all_files, monitor="x=12,y=11,z=2,atom=0,dir=z"))


MAT_GLASS = "id=12, name=glass, eps_xx=2.25, eps_yy=2.25, eps_zz=2.25"


def blocks_mixed_case(tsteps: int = 100) -> CaseSpec:
    """A 96 x 64 x 64 grid in which every block class of the device sweeps
    occurs: a two-atom polar slab (z < 16) whose tiles hold the lattice alone,
    a lossy rotated anisotropic layer (16 <= z < 24) filling whole tiles,
    vacuum interior tiles and vacuum tiles in the CPML or on the domain edge,
    whole tiles of an isotropic dielectric, and mixed tiles: a Drude metal
    block (ADE) cutting through tiles, a rotated two-atom inclusion in the
    slab, and the tile of the source."""
    def medium(nx, ny, nz):
        m = np.zeros((nx, ny, nz), np.int32)
        m[:, :, :16] = 8
        m[:, :, 16:24] = 5
        m[20:44, 20:28, 2:6] = 9          # rotated lattice inside the slab
        m[32:64, 16:32, 30:34] = 12       # whole 32 x 8 tiles of glass
        m[40:56, 36:44, 26:40] = 7        # ADE metal, partial tiles
        return m
    return CaseSpec("blocks_mixed", 96, 64, 64, tsteps, pml=6, output_interval=10, output_component="Ez",
                    slice_axis="z", slice_pos=22,
                    sources=[_dip(48, 32, 50, wn=1370, t0=3e-16, tau=1e-16),
                             "type=sinusoidal, x=70,y=40,z=28, amplitude=0.5, frequency=3.0e13, component=x"],
                    materials=[MAT_IONS2, MAT_IONS2_ROT, MAT_LOSSY_ROTZ, MAT_METAL, MAT_GLASS], medium_fn=medium,
                    files_fn=_all_files, monitor="x=48,y=32,z=12,atom=1,dir=z")


# -------------------------------------------------------- benchmark configs


def cone_tip_box(nx, ny, nz, dx, dz, apex_xy, apex_k, radius_m, half_angle_deg, top_k=None):
    """Cone along +z with a spherical cap at its apex (apex cell apex_k):
    cells whose centre is inside the cap sphere or the cone above it.
    Returns (box, mask): the index box (three slices) holding every such
    cell and the mask over that box, so large grids are painted without
    whole-grid temporaries."""
    a = math.radians(half_angle_deg)
    # sphere tangent to the cone, touching z = 0 at the apex
    zc = radius_m
    zt = zc - radius_m * math.sin(a)  # height where cone and sphere meet
    k_top = nz - 1 if top_k is None else min(nz - 1, top_k)
    k0 = max(0, apex_k)                # sphere and cone lie at z >= 0
    z_max = (k_top - apex_k) * dz
    rho_max = max(radius_m, radius_m * math.cos(a) + max(0.0, z_max - zt) * math.tan(a))
    reach = int(math.ceil(rho_max / dx)) + 1
    i0, i1 = max(0, apex_xy[0] - reach), min(nx, apex_xy[0] + reach + 1)
    j0, j1 = max(0, apex_xy[1] - reach), min(ny, apex_xy[1] + reach + 1)
    k1 = k_top + 1
    box = (slice(i0, max(i0, i1)), slice(j0, max(j0, j1)), slice(k0, max(k0, k1)))
    i = np.arange(box[0].start, box[0].stop)[:, None, None]
    j = np.arange(box[1].start, box[1].stop)[None, :, None]
    k = np.arange(box[2].start, box[2].stop)[None, None, :]
    x = (i - apex_xy[0]) * dx
    y = (j - apex_xy[1]) * dx
    z = (k - apex_k) * dz
    rho = np.sqrt(x * x + y * y)
    in_sphere = (x * x + y * y + (z - zc) ** 2) <= radius_m ** 2
    r_cone = radius_m * math.cos(a) + (z - zt) * math.tan(a)
    in_cone = (z >= zt) & (rho <= r_cone)
    return box, in_sphere | in_cone


def cone_tip_mask(nx, ny, nz, dx, dz, apex_xy, apex_k, radius_m, half_angle_deg, top_k=None):
    """The cone tip of cone_tip_box as a mask over the whole grid."""
    m = np.zeros((nx, ny, nz), bool)
    box, sub = cone_tip_box(nx, ny, nz, dx, dz, apex_xy, apex_k, radius_m, half_angle_deg, top_k)
    m[box] = sub
    return m


def drude_lorentz_eps(nu_cm: float) -> complex:
    """Drude-Lorentz metal of the benchmark tip: eps_inf = 1, plasma energy
    9.0 eV, damping 0.07 eV, Lorentz poles at 2.6 and 3.9 eV with strengths
    0.5 and 1.2.  The reference's ADE is single-frequency: only eps(omega_src)
    enters (fdtd.c:2478-2528)."""
    hbar_ev = 6.582119569e-16
    w = omega_of_wavenumber(nu_cm)
    wp, g = 9.0 / hbar_ev, 0.07 / hbar_ev
    e = 1.0 - wp * wp / (w * w + 1j * g * w)
    for w0_ev, f in ((2.6, 0.5), (3.9, 1.2)):
        w0 = w0_ev / hbar_ev
        e += f * wp * wp / (w0 * w0 - w * w - 1j * g * w)
    return e


CONFIG_NAMES = ["cfg0_polar_slab_96", "cfg1_tip_ade_256", "cfg2_lattice16_512x512x256", "cfg3_serving_request",
                  "cfg4_largest_1024x1024x512"]


def baseline_case(idx: int, tsteps: Optional[int] = None, seed: int = 0, scale: float = 1.0) -> CaseSpec:
    """Benchmark workload idx (0..4) as a CaseSpec.  scale < 1 shrinks the
    grid (for tests) keeping proportions."""
    if idx == 0:
        n = max(8, int(round(96 * scale)))
        dl = 10e-9
        f0 = 1370 * C_CM
        tau = 1.0 / (math.pi * 300 * C_CM)
        return CaseSpec(
            "cfg0_polar_slab_96", n, n, n, tsteps or 2000, delta=(dl, dl, dl), pml=max(2, int(10 * scale)),
            output_interval=20, output_component="Ez", slice_axis="z", slice_pos=int(42 * n / 96),
            sources=[_dip(n // 2, n // 2, int(60 * n / 96), wn=1370, t0=5 * tau, tau=tau)],
            materials=[f"id=4, name=polar2, natom=2, QeZV=QeZV.txt, QeZM=QeZM.txt, DMM=DMM.txt, born=OUTCAR2.txt"],
            medium_fn=_slab(int(40 * n / 96), 4),
            files_fn=lambda d: (_ions2_files(d, seed),
                                write_outcar(d / "OUTCAR2.txt", np.diag([4.9, 4.9, 2.95]),
                                             np.stack([np.diag([2.7, 2.7, 0.9]), -np.diag([2.7, 2.7, 0.9])]))),
            monitor=f"x={n // 2},y={n // 2},z={int(45 * n / 96)},atom=0,dir=z")
    if idx == 1:
        n = max(16, int(round(256 * scale)))
        dl = 5e-9
        slab = max(2, int(round(40 * n / 256)))
        apex = slab + 2
        eps_tip = drude_lorentz_eps(900.0)
        # the reference ADE needs Re eps < EPS_INF (20) on the diagonal: true for this metal
        tip = (f"id=5, name=tip, use_ADE=1, eps_xx={eps_tip.real!r}, eps_yy={eps_tip.real!r}, eps_zz={eps_tip.real!r}, "
               f"eps_xxi={eps_tip.imag!r}, eps_yyi={eps_tip.imag!r}, eps_zzi={eps_tip.imag!r}")
        slabm = ("id=4, name=sample, eps_xx=6.0, eps_yy=3.5, eps_zz=2.8, eps_xxi=0.4, eps_yyi=0.2, eps_zzi=0.1, "
                 "anglez=0.5235987756")

        def medium(nx, ny, nz):
            m = np.zeros((nx, ny, nz), np.int32)
            m[:, :, :slab] = 4
            tipm = cone_tip_mask(nx, ny, nz, dl, dl, (nx // 2, ny // 2), apex, 20e-9 * max(scale, 0.25), 15.0,
                                 top_k=nz - max(2, int(12 * scale)) - 2)
            m[tipm] = 5
            return m
        return CaseSpec(
            "cfg1_tip_ade_256", n, n, n, tsteps or 8000, delta=(dl, dl, dl), pml=max(2, int(12 * scale)),
            output_interval=50, output_component="Ez", slice_axis="z", slice_pos=slab + 1,
            sources=[f"type=sinusoidal, x={n // 2},y={n // 2},z={min(n - 3, apex + n // 4)}, amplitude=1.0, "
                     f"frequency={900 * C_CM!r}, component=z"],
            materials=[slabm, tip], medium_fn=medium,
            monitor=f"x={n // 2},y={n // 2},z={slab + 1},atom=0,dir=z")
    if idx == 2:
        nx = max(16, int(round(512 * scale)))
        nz = max(8, int(round(256 * scale)))
        dl = 10e-9
        return CaseSpec(
            "cfg2_lattice16_512x512x256", nx, nx, nz, tsteps or 10000, delta=(dl, dl, dl), pml=max(2, int(10 * scale)),
            output_interval=100, output_component="Ex", slice_axis="z", slice_pos=nz // 2 + 2,
            sources=[f"type=ricker, x={nx // 2},y={nx // 2},z={nz // 2 + 8}, amplitude=1.0, frequency={820 * C_CM!r}, "
                     f"component=x, t0=6e-14"],
            materials=["id=10, name=lattice16, natom=16, born=OUTCAR.txt, QeZV=QeZV16.txt, QeZM=QeZM16.txt, DMM=DMM16.txt"],
            medium_fn=_slab(nz // 2, 10), files_fn=lambda d: _ions16_files(d, seed),
            monitor=f"x={nx // 2},y={nx // 2},z={nz // 2 - 2},atom=0,dir=x")
    if idx == 4:
        nx = max(16, int(round(1024 * scale)))
        nz = max(8, int(round(512 * scale)))
        dl = 8e-9
        slab = max(2, int(round(64 * nz / 512)))
        tau = 1.0 / (math.pi * 400 * C_CM)
        eps_tip = drude_lorentz_eps(1400.0)
        tip = (f"id=5, name=tip, use_ADE=1, eps_xx={eps_tip.real!r}, eps_yy={eps_tip.real!r}, eps_zz={eps_tip.real!r}, "
               f"eps_xxi={eps_tip.imag!r}, eps_yyi={eps_tip.imag!r}, eps_zzi={eps_tip.imag!r}")

        def medium(nx_, ny_, nz_):
            m = np.zeros((nx_, ny_, nz_), np.int32)
            m[:, :, :slab] = 4
            box, sub = cone_tip_box(nx_, ny_, nz_, dl, dl, (nx_ // 2, ny_ // 2), slab + 2, 20e-9, 15.0,
                                    top_k=nz_ - max(2, int(16 * scale)) - 2)
            m[box][sub] = 5
            return m
        return CaseSpec(
            "cfg4_largest_1024x1024x512", nx, nx, nz, tsteps or 20000, delta=(dl, dl, dl), pml=max(2, int(16 * scale)),
            output_interval=100, output_component="Ez", slice_axis="z", slice_pos=slab + 1,
            sources=[_dip(nx // 2, nx // 2, slab + nz // 8, wn=1400, t0=5 * tau, tau=tau)],
            materials=[f"id=4, name=polar2x, natom=2, QeZV=QeZV.txt, QeZM=QeZM.txt, DMM=DMM.txt, born=OUTCAR2.txt, "
                       f"anglex=0.3490658504", tip],
            medium_fn=medium,
            files_fn=lambda d: (_ions2_files(d, seed),
                                write_outcar(d / "OUTCAR2.txt", np.diag([4.9, 4.9, 2.95]),
                                             np.stack([np.diag([2.7, 2.7, 0.9]), -np.diag([2.7, 2.7, 0.9])]))),
            monitor=f"x={nx // 2},y={nx // 2},z={slab + 1},atom=0,dir=z")
    raise ValueError(f"no single-domain workload {idx}")


# parity cases at the benchmark workloads' own sizes: the full-length
# config 0, 200-step truncations of configs 1 and 2, config 4 at half its
# edge (512 x 512 x 256: its rotated two-atom slab, Drude-Lorentz tip and
# three-wavenumber source) for 200 steps, and the block-class mix
PARITY_BASELINE_CASES = ("cfg0_full", "cfg1_200", "cfg2_200", "cfg4_half_200", "blocks_mixed")


def parity_baseline_case(name: str) -> CaseSpec:
    if name == "cfg0_full":
        return baseline_case(0)
    if name == "cfg1_200":
        return baseline_case(1, tsteps=200)
    if name == "cfg2_200":
        return baseline_case(2, tsteps=200)
    if name == "cfg4_half_200":
        return baseline_case(4, tsteps=200, scale=0.5)
    if name == "blocks_mixed":
        return blocks_mixed_case()
    raise ValueError(f"no baseline parity case {name}")


# ------------------------------------------------------ serving requests


def serving_requests(n: int = 256, seed: int = 0, rate_per_s: float = 4.0, edge_range=(64, 192),
                     steps_range=(3000, 12000), pml: int = 8):
    """The request stream of the serving configuration: Poisson arrivals at
    rate_per_s; each grid edge log-uniform in edge_range per axis; 8-cell
    CPML; steps uniform in steps_range; the 2-atom polar slab of config 0
    (10 nm cells, slab thickness 40/96 of nz); a sine source at a wavenumber
    uniform in 700-1600 cm^-1; a Drude-Lorentz tip (config 1 metal at that
    wavenumber, single-frequency ADE) whose apex sits 5-50 nm above the slab;
    a running DFT of Ez at the source frequency on the plane two cells above
    the slab.  Returns dicts with the arrival time and the parameters;
    ``request_desc`` turns one into a php_desc."""
    rng = np.random.default_rng(seed + 3000)
    t = 0.0
    out = []
    lo, hi = math.log(edge_range[0]), math.log(edge_range[1])
    for q in range(n):
        t += rng.exponential(1.0 / rate_per_s)
        nx, ny, nz = (int(round(math.exp(rng.uniform(lo, hi)))) for _ in range(3))
        out.append({"index": q, "arrival": t, "grid": (nx, ny, nz), "pml": pml,
                    "steps": int(rng.integers(steps_range[0], steps_range[1] + 1)),
                    "wavenumber": float(rng.uniform(700.0, 1600.0)),
                    "tip_height_nm": float(rng.uniform(5.0, 50.0))})
    return out


def request_desc(req: dict, precision: str = "fp32", device: int = 0, seed: int = 0):
    """php_desc (DescHolder) and DFT plane of one serving request."""
    from .solver import Material, Source, make_desc
    nx, ny, nz = req["grid"]
    L = req["pml"]
    dl = 10e-9
    dt = dl / (299792458.0 * math.sqrt(3.0)) * 0.99
    slab = max(1, int(round(40 * nz / 96)))
    qv, qm, dmm = lattice_2atom(seed)
    wn = req["wavenumber"]
    e_tip = drude_lorentz_eps(wn)
    mats = [Material(),
            Material(eps_re=(4.9, 0, 0, 0, 4.9, 0, 0, 0, 2.95), natom=2, qezv=qv, qezm=qm, dmm=dmm),
            Material(eps_re=(e_tip.real, 0, 0, 0, e_tip.real, 0, 0, 0, e_tip.real),
                     eps_im=(e_tip.imag, 0, 0, 0, e_tip.imag, 0, 0, 0, e_tip.imag), use_ade=1)]
    med = np.zeros((nx, ny, nz), np.int32)
    med[:, :, :slab] = 1
    apex = slab + max(1, int(round(req["tip_height_nm"] * 1e-9 / dl)))
    top = nz - L - 2
    if apex < top:
        med[cone_tip_mask(nx, ny, nz, dl, dl, (nx // 2, ny // 2), apex, 20e-9, 15.0, top_k=top)] = 2
    f = wn * C_CM
    zs = min(nz - L - 2, apex + max(2, nz // 4))
    src = [Source(type=1, x=nx // 2, y=ny // 2, z=max(0, zs), component="z", frequency=f)]
    holder = make_desc(med, mats, src, dx=dl, dy=dl, dz=dl, dt=dt, pml_thickness=L, precision=precision,
                       source_frequency=f, device=device)
    return holder, {"component": "Ez", "z_plane": min(nz - 1, slab + 2), "freqs": [f]}
