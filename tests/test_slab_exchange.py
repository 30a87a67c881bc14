"""The z-slab exchange of php_fdtd_b200.slab on CPU ranks (gloo, world size
2 and 3): a z-leapfrog pair with the Yee stencil's plane dependencies (H at
k reads E at k+1, E at k reads H at k-1), decomposed like the reference and
exchanged with exchange_e / exchange_h, must equal the undecomposed run."""
import os
import socket

import numpy as np
import pytest

from php_fdtd_b200.slab import exchange_e, exchange_h, slab_ranges

NX, NZ, STEPS = 6, 13, 9


def _single():
    E = np.zeros((NZ + 2, NX))   # planes -1 .. NZ (zero halos)
    H = np.zeros((NZ + 2, NX))
    for t in range(STEPS):
        for k in range(NZ):
            H[k + 1] += 0.5 * (E[k + 2] - E[k + 1])
        for k in range(NZ):
            E[k + 1] += 0.5 * (H[k + 1] - H[k])
        E[5 + 1, 2] += np.sin(0.7 * t)        # source at z = 5
    return E[1:-1], H[1:-1]


def _rank(rank, size, port, q):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=size)
    z0, n = slab_ranges(NZ, size)[rank]
    E = torch.zeros((n + 2, NX), dtype=torch.float64)
    H = torch.zeros((n + 2, NX), dtype=torch.float64)
    for t in range(STEPS):
        exchange_e(rank, size, [E[1]], [E[n + 1]], dist)
        for k in range(n):
            H[k + 1] += 0.5 * (E[k + 2] - E[k + 1])
        exchange_h(rank, size, [H[n]], [H[0]], dist)
        for k in range(n):
            E[k + 1] += 0.5 * (H[k + 1] - H[k])
        if z0 <= 5 < z0 + n:
            E[5 - z0 + 1, 2] += np.sin(0.7 * t)
    q.put((rank, E[1:-1].numpy().copy(), H[1:-1].numpy().copy()))
    dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("size", [2, 3])
def test_slab_exchange_reproduces_the_single_domain(size):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, size, port, q)) for r in range(size)]
    for p in procs:
        p.start()
    got = dict((r, (e, h)) for r, e, h in (q.get(timeout=120) for _ in procs))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    E = np.concatenate([got[r][0] for r in range(size)])
    H = np.concatenate([got[r][1] for r in range(size)])
    E1, H1 = _single()
    np.testing.assert_array_equal(E, E1)
    np.testing.assert_array_equal(H, H1)


def test_ranges_follow_the_reference_split():
    assert slab_ranges(10, 3) == [(0, 4), (4, 3), (7, 3)]
    assert slab_ranges(256, 8) == [(32 * r, 32) for r in range(8)]
    r = slab_ranges(97, 5)
    assert sum(n for _, n in r) == 97 and all(r[i][0] + r[i][1] == r[i + 1][0] for i in range(4))
