"""Plain blocks of the fused sweep.  Tiles of one plain isotropic material
away from the CPML, the domain edge and the sources take a path without the
per-cell material, CPML and source handling, and tiles of the lossy rotated
tensor layer one with that material's coefficients in the kernel
parameters; their result must be that of the general path (PHP_PLAIN=0
turns the plain paths off)."""
import os

import numpy as np
import pytest

from php_fdtd_b200 import Material, Simulation, Source, make_desc

pytestmark = pytest.mark.gpu


def _desc(precision, rotation):
    nx, ny, nz = 130, 72, 40
    med = np.zeros((nx, ny, nz), np.int32)
    med[:, :, :12] = 1                        # plain isotropic dielectric
    med[40:90, 20:50, 12:20] = 2              # anisotropic block (general path)
    med[:, :, 20:36] = 3                      # lossy rotated tensor layer, into the z CPML
    dl = 10e-9
    dt = dl / (299792458.0 * np.sqrt(3.0)) * 0.99
    mats = [Material(), Material(eps_re=(2.5, 0, 0, 0, 2.5, 0, 0, 0, 2.5)),
            Material(eps_re=(4.0, 0, 0, 0, 3.0, 0, 0, 0, 2.0)),
            Material(eps_re=(6.0, 0, 0, 0, 3.5, 0, 0, 0, 2.8), eps_im=(0.4, 0, 0, 0, 0.2, 0, 0, 0, 0.1),
                     **{rotation: 0.5235987756})]
    src = [Source(type=1, x=65, y=36, z=26, component="z", frequency=3.0e13),
           Source(type=1, x=100, y=20, z=6, component="x", frequency=2.0e13)]
    return make_desc(med, mats, src, dx=dl, dy=dl, dz=dl, dt=dt, pml_thickness=6, precision=precision,
                     source_frequency=3.0e13)


def _run(precision, rotation, plain):
    old = os.environ.get("PHP_PLAIN")
    os.environ["PHP_PLAIN"] = "1" if plain else "0"
    try:
        sim = Simulation(_desc(precision, rotation))
    finally:
        if old is None:
            os.environ.pop("PHP_PLAIN", None)
        else:
            os.environ["PHP_PLAIN"] = old
    sim.step(60)
    out = [sim.read_volume(c) for c in range(9)]
    sim.close()
    return out


@pytest.mark.parametrize("rotation", ["anglez", "anglex"])
@pytest.mark.parametrize("precision,rtol", [("fp64", 1e-12), ("fp32", 1e-5)])
def test_plain_blocks_match_general_path(precision, rtol, rotation):
    a, b = _run(precision, rotation, True), _run(precision, rotation, False)
    for c in range(9):
        scale = max(np.abs(b[c]).max(), 1e-300)
        assert np.abs(b[c]).max() > 0
        np.testing.assert_allclose(a[c], b[c], rtol=0, atol=rtol * scale, err_msg=f"component {c}")


def _desc_atoms(precision, natom, lossy):
    from php_fdtd_b200.workloads import lattice_2atom, lattice_data
    nx, ny, nz = 130, 72, 40
    med = np.zeros((nx, ny, nz), np.int32)
    med[:, :, :16] = 1                        # few-atom layer, into the z CPML
    med[40:90, 20:50, 16:20] = 2              # isotropic block above it
    dl = 10e-9
    dt = dl / (299792458.0 * np.sqrt(3.0)) * 0.99
    if natom == 2:
        qv, qm, dmm = lattice_2atom(0)
    else:
        z = np.zeros((4, 3, 3))
        for q, s in enumerate((1.0, -1.0, 0.6, -0.6)):
            z[q] = s * np.diag([2.7, 2.4, 0.9])
        qv, qm, dmm = lattice_data(z, [10.8, 14.0, 16.0, 24.3], [1370.0, 1300.0, 780.0, 900.0, 850.0, 700.0,
                                                               600.0, 500.0, 450.0, 0.0, 0.0, 0.0], 1, 40.0)
    extra = dict(eps_im=(0.2, 0, 0, 0, 0.1, 0, 0, 0, 0.05), anglez=0.4) if lossy else {}
    mats = [Material(), Material(eps_re=(4.9, 0, 0, 0, 4.9, 0, 0, 0, 2.95), natom=natom, qezv=qv, qezm=qm, dmm=dmm,
                                 **extra),
            Material(eps_re=(2.5, 0, 0, 0, 2.5, 0, 0, 0, 2.5))]
    src = [Source(type=1, x=65, y=36, z=26, component="z", frequency=4.0e13),
           Source(type=1, x=100, y=20, z=8, component="x", frequency=4.0e13)]
    return make_desc(med, mats, src, dx=dl, dy=dl, dz=dl, dt=dt, pml_thickness=6, precision=precision,
                     source_frequency=4.0e13)


def _run_atoms(precision, natom, lossy, plain):
    old = os.environ.get("PHP_PLAIN")
    os.environ["PHP_PLAIN"] = "1" if plain else "0"
    try:
        sim = Simulation(_desc_atoms(precision, natom, lossy))
    finally:
        if old is None:
            os.environ.pop("PHP_PLAIN", None)
        else:
            os.environ["PHP_PLAIN"] = old
    sim.step(80)
    out = [sim.read_volume(c) for c in range(9)]
    sim.close()
    return out


@pytest.mark.parametrize("natom,lossy", [(2, False), (2, True), (4, False)])
@pytest.mark.parametrize("precision,rtol", [("fp64", 1e-12), ("fp32", 1e-5)])
def test_atom_blocks_match_general_path(precision, rtol, natom, lossy):
    """Blocks of the few-atom layer take its material record from the kernel
    parameters with the fused ion update; fields after 80 steps equal the
    general path's."""
    a, b = _run_atoms(precision, natom, lossy, True), _run_atoms(precision, natom, lossy, False)
    for c in range(9):
        scale = max(np.abs(b[c]).max(), 1e-300)
        assert np.abs(b[c]).max() > 0
        np.testing.assert_allclose(a[c], b[c], rtol=0, atol=rtol * scale, err_msg=f"component {c}")
