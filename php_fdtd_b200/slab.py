"""z-slab decomposition of one domain over several GPUs.

The reference splits z across MPI ranks (fdtd.c:2761-2771) and exchanges the
boundary planes each half step (fdtd.c:3120, 3235).  Here a slab is a
device context for its planes (php_create_slab); per time step each slab

    sends E plane 0 down, receives E into its halo plane nz  (exchange_e)
    runs the H sweep                                        (half 0)
    sends H plane nz-1 up, receives H into its halo plane -1 (exchange_h)
    runs the D/E sweep, ion pass, probe and DFT             (half 1)

Only plane data crosses between GPUs: three planes per neighbour and half
step, device to device (NCCL send/receive between processes, or copies
between the slabs of one process).  No collective is on the data path.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Sequence, Tuple

import numpy as np

from . import _abi
from .solver import DescHolder, PhpError, Simulation


def slab_ranges(nz: int, size: int) -> List[Tuple[int, int]]:
    """(z0, nz_local) of every rank: the first nz % size ranks get one plane
    more (fdtd.c:2761-2771)."""
    base, rem = divmod(nz, size)
    out, z0 = [], 0
    for r in range(size):
        n = base + 1 if r < rem else base
        out.append((z0, n))
        z0 += n
    return out


def exchange_e(rank: int, size: int, send_down: Sequence, recv_up: Sequence, dist) -> None:
    """E plane 0 to rank-1; the halo plane nz from rank+1."""
    ops = []
    if rank > 0:
        ops += [dist.P2POp(dist.isend, t, rank - 1) for t in send_down]
    if rank < size - 1:
        ops += [dist.P2POp(dist.irecv, t, rank + 1) for t in recv_up]
    if ops:
        for w in dist.batch_isend_irecv(ops):
            w.wait()


def exchange_h(rank: int, size: int, send_up: Sequence, recv_down: Sequence, dist) -> None:
    """H plane nz-1 to rank+1; the halo plane -1 from rank-1."""
    ops = []
    if rank < size - 1:
        ops += [dist.P2POp(dist.isend, t, rank + 1) for t in send_up]
    if rank > 0:
        ops += [dist.P2POp(dist.irecv, t, rank - 1) for t in recv_down]
    if ops:
        for w in dist.batch_isend_irecv(ops):
            w.wait()


class _DevicePlane:
    """A device byte range as a CUDA array (for torch.as_tensor)."""

    def __init__(self, ptr: int, n: int, typestr: str, device: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (ptr, False), "version": 3}
        self.device = device


class Slab(Simulation):
    """One z slab of a domain (php_create_slab); read-outs take local z."""

    def __init__(self, holder: DescHolder, z0: int, nz_local: int):
        self._lib = _abi.device_lib()
        self.holder = holder
        self.nx, self.ny, self.nz = holder.desc.nx, holder.desc.ny, nz_local
        self.z0 = z0
        ctx = C.c_void_p()
        rc = self._lib.php_create_slab(C.byref(holder.desc), int(z0), int(nz_local), C.byref(ctx))
        if rc != 0:
            raise PhpError(rc, self._lib.php_last_error(None).decode())
        self._ctx = ctx
        self._esize = 4 if holder.desc.precision == _abi.PREC["fp32"] else 8

    def planes(self, which: int):
        """The three component planes `which` (php_halo_planes) as torch
        tensors on the slab's device, without copying."""
        import torch
        ptrs = (C.c_void_p * 3)()
        nbytes = C.c_uint64()
        self._ck(self._lib.php_halo_planes(self._ctx, int(which), ptrs, C.byref(nbytes)))
        typestr = "<f4" if self._esize == 4 else "<f8"
        n = nbytes.value // self._esize
        dev = self.holder.desc.device
        return [torch.as_tensor(_DevicePlane(p, n, typestr, dev), device=f"cuda:{dev}") for p in ptrs]

    def half(self, h: int):
        self._ck(self._lib.php_step_half(self._ctx, int(h)))


class LocalSlabs:
    """All slabs of a domain in one process (on one GPU, or one per GPU of
    the process): the halo planes are copied device to device between the
    halves of every step, in slab order."""

    def __init__(self, holder: DescHolder, nslabs: int, devices: Sequence[int] = (0,)):
        self.ranges = slab_ranges(holder.desc.nz, nslabs)
        self.slabs = []
        for r, (z0, n) in enumerate(self.ranges):
            h = DescHolder(_abi.Desc.from_buffer_copy(holder.desc), list(holder.keep))
            h.desc.device = devices[r % len(devices)]
            self.slabs.append(Slab(h, z0, n))
        self._p = [{w: s.planes(w) for w in range(4)} for s in self.slabs]

    def _copy(self, dst, src):
        for d, s in zip(dst, src):
            d.copy_(s)

    def step(self, n: int = 1):
        import torch
        S = self.slabs
        for _ in range(n):
            for s in S:
                s.sync()
            for r in range(len(S) - 1):           # E plane 0 of r+1 -> halo above r
                self._copy(self._p[r][1], self._p[r + 1][0])
            torch.cuda.synchronize()
            for s in S:
                s.half(0)
            for s in S:
                s.sync()
            for r in range(1, len(S)):            # H top plane of r-1 -> halo below r
                self._copy(self._p[r][3], self._p[r - 1][2])
            torch.cuda.synchronize()
            for s in S:
                s.half(1)
        for s in S:
            s.sync()

    def read_volume(self, comp) -> np.ndarray:
        return np.concatenate([s.read_volume(comp) for s in self.slabs], axis=2)

    def close(self):
        for s in self.slabs:
            s.close()


class DistSlab:
    """This rank's slab of a domain decomposed over torch.distributed ranks
    (one process per GPU, NCCL between neighbours)."""

    def __init__(self, holder: DescHolder, rank: int, size: int):
        import torch.distributed as dist
        self.dist = dist
        self.rank, self.size = rank, size
        self.z0, n = slab_ranges(holder.desc.nz, size)[rank]
        self.slab = Slab(holder, self.z0, n)
        self._p = {w: self.slab.planes(w) for w in range(4)}

    def step(self, n: int = 1):
        import torch
        stream = torch.cuda.ExternalStream(self.slab.stream, device=self._p[0][0].device)
        with torch.cuda.stream(stream):
            for _ in range(n):
                exchange_e(self.rank, self.size, self._p[0], self._p[1], self.dist)
                self.slab.half(0)
                exchange_h(self.rank, self.size, self._p[2], self._p[3], self.dist)
                self.slab.half(1)

    def close(self):
        self.slab.close()
