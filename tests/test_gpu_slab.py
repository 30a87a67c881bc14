"""z slabs (php_create_slab / php_halo_planes / php_step_part) on one GPU.

  - LocalSlabs: a domain split into 2 or 3 slabs in one process, each step
    run in parts on two streams per slab with the halo planes copied device
    to device, all ordered by events, advances exactly like the
    undecomposed domain (one z chunk per block, and four planes per chunk,
    where the boundary parts and the interior parts are different launches).
  - DistSlab: two processes, each holding a real slab on this GPU, exchange
    their halo planes over gloo through page-locked host buffers
    (HostTransport) while the interior parts run; the assembled volume is
    bit-identical to the undecomposed domain.  The processes' kernels never
    wait on each other: every exchange is a host-side send and receive.
"""
import os
import socket

import numpy as np
import pytest

import harness as H
from conftest import GOLDEN
from php_fdtd_b200 import Config, Simulation
from php_fdtd_b200.slab import LocalSlabs, slab_ranges

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,nslabs,precision,zchunk", [
    ("vacuum_pml", 2, "fp64-strict", 0), ("ions2", 3, "fp64-strict", 0), ("ade_metal", 2, "fp64-strict", 0),
    ("lossy_rot", 3, "fp64", 0), ("ions16", 2, "fp32", 0), ("aniso_lossy", 2, "fp32", 0),
    ("ions2", 2, "fp64", 4), ("ade_metal", 2, "fp32", 3), ("vacuum_pml", 3, "fp64-strict", 2)])
def test_slabs_equal_single_domain(name, nslabs, precision, zchunk, golden_case):
    with H.chdir(golden_case(name)):
        cfg = Config.load("case.cfg")
        holder = cfg.desc(cfg.load_medium(), precision)
    holder.desc.z_chunk = zchunk
    one = Simulation(holder)
    one.step(14)
    slabs = LocalSlabs(holder, nslabs)
    slabs.step(9)
    slabs.step(5)
    for comp in range(9):
        np.testing.assert_array_equal(slabs.read_volume(comp), one.read_volume(comp), err_msg=f"component {comp}")
    # atom state of a cell in every slab
    for s in slabs.slabs:
        k = s.nz // 2
        a, b = s.read_cell_state(cfg.nx // 2, cfg.ny // 2, k), one.read_cell_state(cfg.nx // 2, cfg.ny // 2, s.z0 + k)
        np.testing.assert_array_equal(a["r"], b["r"])
    assert all(s.t == 14 for s in slabs.slabs)
    slabs.close()
    one.close()


STEPS = 12


def _holder(name, precision, zchunk):
    with H.chdir(GOLDEN / name):
        cfg = Config.load("case.cfg")
        holder = cfg.desc(cfg.load_medium(), precision)
    holder.desc.z_chunk = zchunk
    return holder


def _rank(rank, size, port, name, precision, zchunk, q):
    import datetime
    import torch
    import torch.distributed as dist
    from php_fdtd_b200.slab import DistSlab
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=size, timeout=datetime.timedelta(seconds=60))
    torch.cuda.set_device(0)
    ds = DistSlab(_holder(name, precision, zchunk), rank, size, transport="host")
    ds.step(7)
    ds.step(STEPS - 7)
    ds.sync()
    vols = [ds.slab.read_volume(c) for c in range(9)]
    ds.close()
    q.put((rank, vols))
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("name,size,precision,zchunk", [("ions2", 2, "fp64-strict", 0), ("ade_metal", 2, "fp32", 3),
                                                        ("lossy_rot", 3, "fp64", 2)])
def test_dist_slabs_over_host_staged_gloo_equal_single_domain(name, size, precision, zchunk):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, size, port, name, precision, zchunk, q)) for r in range(size)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    one = Simulation(_holder(name, precision, zchunk))
    one.step(STEPS)
    for comp in range(9):
        whole = np.concatenate([got[r][comp] for r in range(size)], axis=2)
        np.testing.assert_array_equal(whole, one.read_volume(comp), err_msg=f"component {comp}")
    one.close()
    assert [n for _, n in slab_ranges(one.nz, size)] == [got[r][0].shape[2] for r in range(size)]
