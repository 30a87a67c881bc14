"""z slabs (php_create_slab / php_halo_planes / php_step_half) on one GPU:
a domain split into 2 or 3 slabs, with the halo planes copied between the
halves of every step, advances exactly like the undecomposed domain."""
import numpy as np
import pytest

import harness as H
from php_fdtd_b200 import Config, Simulation
from php_fdtd_b200.slab import LocalSlabs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,nslabs,precision", [("vacuum_pml", 2, "fp64-strict"), ("ions2", 3, "fp64-strict"),
                                                   ("ade_metal", 2, "fp64-strict"), ("lossy_rot", 3, "fp64"),
                                                   ("ions16", 2, "fp32"), ("aniso_lossy", 2, "fp32")])
def test_slabs_equal_single_domain(name, nslabs, precision, golden_case):
    with H.chdir(golden_case(name)):
        cfg = Config.load("case.cfg")
        holder = cfg.desc(cfg.load_medium(), precision)
    one = Simulation(holder)
    one.step(14)
    slabs = LocalSlabs(holder, nslabs)
    slabs.step(14)
    for comp in range(9):
        np.testing.assert_array_equal(slabs.read_volume(comp), one.read_volume(comp), err_msg=f"component {comp}")
    # atom state of a cell in every slab
    for s in slabs.slabs:
        k = s.nz // 2
        a, b = s.read_cell_state(cfg.nx // 2, cfg.ny // 2, k), one.read_cell_state(cfg.nx // 2, cfg.ny // 2, s.z0 + k)
        np.testing.assert_array_equal(a["r"], b["r"])
    slabs.close()
    one.close()
