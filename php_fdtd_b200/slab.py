"""z-slab decomposition of one domain over several GPUs.

The reference splits z across MPI ranks (fdtd.c:2761-2771) and exchanges the
boundary planes each half step (fdtd.c:3120, 3235): E plane 0 goes down
before the H sweep, H plane nz-1 goes up before the D/E sweep.  Here a slab
is a device context for its planes (php_create_slab), and each time step
runs in the parts of php_step_part so that the exchanges hide behind the
planes that do not need them:

    side stream   H sweep, lower chunks (1)      E sweep, upper chunks (3)
    main stream   H sweep, top chunk (0)  -> H plane up / H halo from below
                  E sweep, bottom chunk (2) -> E plane 0 down / E halo from above
                  ion pass, probe, DFT (4)

Only plane data crosses between slabs: three planes per neighbour and
exchange (NCCL send/receive between processes, page-locked host staging
over any torch.distributed backend, or device copies between the slabs of
one process).  No collective is on the data path, and nothing waits on the
host between the parts of a step except the host-staged transport.
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

    def part(self, p: int, stream: int = 0):
        """php_step_part on a cudaStream_t handle (0 = the slab's stream)."""
        self._ck(self._lib.php_step_part(self._ctx, int(p), C.c_void_p(stream or None)))


class _StepEvents:
    """The events that order one slab's parts across its two streams."""

    def __init__(self):
        import torch
        self.h0, self.h1, self.e3, self.p4 = (torch.cuda.Event() for _ in range(4))


class LocalSlabs:
    """All slabs of a domain in one process (on one GPU, or one per GPU of
    the process): the halo planes are copied device to device, and every
    dependency between parts, copies and slabs is a CUDA event, so a step is
    enqueued without any host synchronisation."""

    def __init__(self, holder: DescHolder, nslabs: int, devices: Sequence[int] = (0,)):
        import torch
        self.ranges = slab_ranges(holder.desc.nz, nslabs)
        self.slabs = []
        for r, (z0, n) in enumerate(self.ranges):
            h = DescHolder(_abi.Desc.from_buffer_copy(holder.desc), list(holder.keep))
            h.desc.device = devices[r % len(devices)]
            self.slabs.append(Slab(h, z0, n))
        self._p = [{w: s.planes(w) for w in range(4)} for s in self.slabs]
        self._main, self._side, self._ev = [], [], []
        for s in self.slabs:
            dev = torch.device("cuda", s.holder.desc.device)
            self._main.append(torch.cuda.ExternalStream(s.stream, device=dev))
            self._side.append(torch.cuda.Stream(device=dev))
            self._ev.append(_StepEvents())
        n = len(self.slabs)
        self._e2 = [torch.cuda.Event() for _ in range(n)]     # E bottom chunk done (slab r)
        self._cp_e = [torch.cuda.Event() for _ in range(n)]   # E plane 0 of r+1 copied into r
        self._cp_h = [torch.cuda.Event() for _ in range(n)]   # H top plane of r-1 copied into r
        self._copy_e()

    @staticmethod
    def _copy(dst, src):
        for d, s in zip(dst, src):
            d.copy_(s, non_blocking=True)

    def _copy_e(self):
        """E plane 0 of slab r+1 into the halo above slab r, on r's main
        stream once r+1's bottom E chunk is done."""
        import torch
        for r in range(len(self.slabs) - 1):
            m = self._main[r]
            m.wait_event(self._e2[r + 1])
            with torch.cuda.stream(m):
                self._copy(self._p[r][1], self._p[r + 1][0])
            self._cp_e[r].record(m)

    def step(self, n: int = 1):
        import torch
        S, M, Sd, EV = self.slabs, self._main, self._side, self._ev
        R = len(S)
        for _ in range(n):
            for r in range(R):                      # H sweep, chunks below the top (no halo)
                Sd[r].wait_event(EV[r].p4)
                S[r].part(1, Sd[r].cuda_stream)
                EV[r].h1.record(Sd[r])
            for r in range(R):                      # H sweep, top chunk (E halo above)
                if r + 1 < R:
                    M[r].wait_event(self._cp_h[r + 1])   # the last copy of this H plane is done
                S[r].part(0, M[r].cuda_stream)
                EV[r].h0.record(M[r])
            for r in range(R):                      # E sweep, chunks above the bottom (no halo)
                Sd[r].wait_event(EV[r].h0)
                S[r].part(3, Sd[r].cuda_stream)
                EV[r].e3.record(Sd[r])
            for r in range(1, R):                   # H plane nz-1 of r-1 -> halo below r
                M[r].wait_event(EV[r - 1].h0)
                with torch.cuda.stream(M[r]):
                    self._copy(self._p[r][3], self._p[r - 1][2])
                self._cp_h[r].record(M[r])
            for r in range(R):                      # E sweep, bottom chunk (H halo below)
                M[r].wait_event(EV[r].h1)
                if r > 0:
                    M[r].wait_event(self._cp_e[r - 1])   # E plane 0 copied before it is rewritten
                S[r].part(2, M[r].cuda_stream)
                self._e2[r].record(M[r])
            self._copy_e()                          # E halos of the next step
            for r in range(R):                      # ion pass, probe, DFT
                M[r].wait_event(EV[r].e3)
                S[r].part(4, M[r].cuda_stream)
                EV[r].p4.record(M[r])

    def sync(self):
        for s in self.slabs:
            s.sync()

    def read_volume(self, comp) -> np.ndarray:
        self.sync()
        return np.concatenate([s.read_volume(comp) for s in self.slabs], axis=2)

    def close(self):
        self.sync()
        for st in self._side:
            st.synchronize()
        self._p = []
        for s in self.slabs:
            s.close()


class DeviceTransport:
    """Plane exchange of device tensors with torch.distributed point to
    point (NCCL between GPUs), ordered on the current stream."""

    def __init__(self, dist):
        self.dist = dist

    def close(self):
        pass

    def exchange(self, sends, recvs, stream):
        import torch
        ops = [self.dist.P2POp(self.dist.isend, t, peer) for peer, ts in sends for t in ts]
        ops += [self.dist.P2POp(self.dist.irecv, t, peer) for peer, ts in recvs for t in ts]
        if not ops:
            return
        with torch.cuda.stream(stream):
            for w in self.dist.batch_isend_irecv(ops):
                w.wait()


class HostTransport:
    """Plane exchange through page-locked host buffers over any
    torch.distributed backend (gloo included): the device copies run on the
    slab's stream, and the host waits for the copy out before it sends.
    For GPUs without a peer path, and for CPU-side tests of the schedule."""

    def __init__(self, dist):
        self.dist = dist
        self._buf = {}

    def close(self):
        """Frees the page-locked buffers.  Called while the streams they were
        copied on still exist: torch's host allocator records an event on
        each such stream when a buffer is freed."""
        self._buf.clear()

    def _host(self, key, t):
        import torch
        b = self._buf.get(key)
        if b is None:
            b = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
            self._buf[key] = b
        return b

    def exchange(self, sends, recvs, stream):
        import torch
        out = [(peer, [self._host(("s", peer, q), t) for q, t in enumerate(ts)]) for peer, ts in sends]
        inn = [(peer, [self._host(("r", peer, q), t) for q, t in enumerate(ts)]) for peer, ts in recvs]
        with torch.cuda.stream(stream):
            for (_, ts), (_, hs) in zip(sends, out):
                for t, h in zip(ts, hs):
                    h.copy_(t, non_blocking=True)
        ev = torch.cuda.Event()
        ev.record(stream)
        ev.synchronize()
        works = [self.dist.isend(h, peer) for peer, hs in out for h in hs]
        works += [self.dist.irecv(h, peer) for peer, hs in inn for h in hs]
        for w in works:
            w.wait()
        with torch.cuda.stream(stream):
            for (_, ts), (_, hs) in zip(recvs, inn):
                for t, h in zip(ts, hs):
                    t.copy_(h, non_blocking=True)


class DistSlab:
    """This rank's slab of a domain decomposed over torch.distributed ranks
    (one process per GPU).  transport: "device" (NCCL point to point on
    device tensors) or "host" (page-locked host staging, any backend)."""

    def __init__(self, holder: DescHolder, rank: int, size: int, transport: str = "device"):
        import torch
        import torch.distributed as dist
        self.dist = dist
        self.rank, self.size = rank, size
        self.z0, n = slab_ranges(holder.desc.nz, size)[rank]
        self.slab = Slab(holder, self.z0, n)
        self._p = {w: self.slab.planes(w) for w in range(4)}
        dev = torch.device("cuda", holder.desc.device)
        self._main = torch.cuda.ExternalStream(self.slab.stream, device=dev)
        self._side = torch.cuda.Stream(device=dev)
        self._ev = _StepEvents()
        self.transport = HostTransport(dist) if transport == "host" else DeviceTransport(dist)
        self._exchange_e()

    def _exchange_e(self):
        """E plane 0 to rank-1; the halo above from rank+1."""
        r, n = self.rank, self.size
        self.transport.exchange([(r - 1, self._p[0])] if r > 0 else [],
                                [(r + 1, self._p[1])] if r < n - 1 else [], self._main)

    def _exchange_h(self):
        """H plane nz-1 to rank+1; the halo below from rank-1."""
        r, n = self.rank, self.size
        self.transport.exchange([(r + 1, self._p[2])] if r < n - 1 else [],
                                [(r - 1, self._p[3])] if r > 0 else [], self._main)

    def step(self, n: int = 1):
        S, M, Sd, ev = self.slab, self._main, self._side, self._ev
        for _ in range(n):
            Sd.wait_event(ev.p4)
            S.part(1, Sd.cuda_stream)       # H sweep below the top chunk
            ev.h1.record(Sd)
            S.part(0, M.cuda_stream)        # H sweep, top chunk (E halo received)
            ev.h0.record(M)
            Sd.wait_event(ev.h0)
            S.part(3, Sd.cuda_stream)       # E sweep above the bottom chunk, behind both exchanges
            ev.e3.record(Sd)
            self._exchange_h()
            M.wait_event(ev.h1)
            S.part(2, M.cuda_stream)        # E sweep, bottom chunk (H halo received)
            self._exchange_e()              # E halo of the next step
            M.wait_event(ev.e3)
            S.part(4, M.cuda_stream)        # ion pass, probe, DFT
            ev.p4.record(M)

    def sync(self):
        self.slab.sync()

    def close(self):
        """Waits for the slab's work, frees the transport's buffers (their
        streams must still exist) and the planes' views, then the slab."""
        self.slab.sync()
        self._side.synchronize()
        self.transport.close()
        self._p = {}
        self.slab.close()
