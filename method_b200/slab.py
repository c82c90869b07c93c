"""One domain split into x-slabs, one per GPU, with halo exchange.

The counterpart of the reference's ParallelEnv and ParallelOutflow /
ParallelPeriodic / ParallelFlow (Project/CPU/Src/parallelEnv.cc:16-127,
Project/CPU/Src/parallelBoundaryConds.cc:11-725) for a split along x, the
slowest index of METHOD's layout (so a halo of one variable is one contiguous
block of Ng rows).  Each slab is a handle created with ``x_slab`` (its x ghost
rows are filled here, not by the boundary conditions); a time step runs as
the handle's parts (predictor | corrector for RK2, stage 1 | stage 2 |
combination for SSP2) and after every part the Ng-deep x halos of that
part's state are exchanged, as ParallelBcs::apply does after each
finalise through swapGhostBuffers.

Ordering of one exchange, per slab: pack the Ng interior rows beside the low
and the high x face; send the low rows to the left neighbour and the high
rows to the right one; receive into the ghost rows; at a physical outflow x
face fill the ghost rows from the boundary row instead.  Every message
between a pair of ranks is posted in the same order on both (to-left send,
from-right receive, to-right send, from-left receive) and tagged with the
side it fills, so NCCL (which matches in order) and gloo (which matches by
tag) pair them identically, also when both neighbours are the same rank.

Backends: ``DeviceSlab`` (a library handle; halo buffers are device tensors,
copies run on the handle's stream) and ``ArraySlab`` (numpy arrays with the
same row layout, used to test the exchange logic on CPU ranks).
Transports: ``TorchTransport`` (torch.distributed point-to-point over NCCL
between GPUs, or gloo on CPU) and ``LocalTransport`` (several slabs of one
process).
"""
from __future__ import annotations

import contextlib
import ctypes as C

import numpy as np

X_PERIODIC = ("periodic", "flow")  # Flow is periodic in x (boundaryConds.cc:449-588)


def slab_extents(nx: int, parts: int, Ng: int):
    """(offset, count) of each slab's interior columns: an even split with the
    remainder on the first slabs.  Each slab needs at least Ng columns, since
    its halo rows are its own interior rows."""
    if parts < 1:
        raise ValueError("need at least one slab")
    base, extra = divmod(nx, parts)
    out, off = [], 0
    for r in range(parts):
        n = base + (1 if r < extra else 0)
        if n < Ng:
            raise ValueError(f"slab {r} would hold {n} columns, fewer than Ng = {Ng}")
        out.append((off, n))
        off += n
    return out


def neighbours(rank: int, world: int, bcs: str):
    """(left, right) neighbour ranks in x; None at a physical outflow face."""
    periodic = bcs in X_PERIODIC
    left = rank - 1 if rank > 0 else (world - 1 if periodic else None)
    right = rank + 1 if rank < world - 1 else (0 if periodic else None)
    return left, right


# --------------------------------------------------------------------- slabs
class ArraySlab:
    """A slab held as numpy arrays (nvars, Nx, Ny, Nz) with the row layout of
    the library's halo buffers: [cons vars | prims vars | aux vars][Ng rows][Ny*Nz].
    Buffers are float64 CPU tensors (what a gloo process group sends)."""

    def __init__(self, cons, prims, aux, Ng, torch):
        self.arrays = [cons, prims, aux]
        self.Ng = Ng
        self.ie = cons.shape[1] - Ng
        self.torch = torch

    def new_buffer(self):
        n = sum(a.shape[0] for a in self.arrays) * self.Ng * self.arrays[0][0, 0].size
        return self.torch.empty(n, dtype=self.torch.float64)

    def _rows(self, first):
        return slice(first, first + self.Ng)

    def pack(self, part, side, buf):
        rows = self._rows(self.Ng if side == 0 else self.ie - self.Ng)
        buf.numpy()[:] = np.concatenate([a[:, rows].reshape(-1) for a in self.arrays])

    def unpack(self, part, side, buf):
        rows = self._rows(0 if side == 0 else self.ie)
        b = buf.numpy()
        off = 0
        for a in self.arrays:
            blk = a[:, rows]
            a[:, rows] = b[off:off + blk.size].reshape(blk.shape)
            off += blk.size

    def outflow(self, part, side):
        src = self.Ng if side == 0 else self.ie - 1
        first = 0 if side == 0 else self.ie
        for a in self.arrays:
            a[:, first:first + self.Ng] = a[:, src:src + 1]

    def on_stream(self):
        return contextlib.nullcontext()


class DeviceSlab:
    """A slab as a library handle (``Simulation`` created with x_slab).  The
    handle's work, its halo copies and the transport's copies or messages all
    run on `stream`, a non-default torch stream that the slabs of one process
    share, so they are ordered without host synchronisation."""

    def __init__(self, sim, torch, stream):
        self.sim, self.torch = sim, torch
        n = C.c_ulonglong()
        self._check(sim.L.mth_halo_bytes(sim.h, C.byref(n)), "halo_bytes")
        self.nbytes = int(n.value)
        parts = C.c_int()
        self._check(sim.L.mth_step_parts(sim.h, C.byref(parts)), "step_parts")
        self.parts = parts.value
        self.device = torch.device("cuda", sim.cfg.device)
        self.stream = stream
        sim.set_stream(stream.cuda_stream)

    def on_stream(self):
        return self.torch.cuda.stream(self.stream)

    def _check(self, rc, what):
        if rc != 0:
            raise RuntimeError(f"{what}: status {rc}: {self.sim.L.mth_last_error(self.sim.h)}")

    def new_buffer(self):
        return self.torch.empty(self.nbytes, dtype=self.torch.uint8, device=self.device)

    def pack(self, part, side, buf):
        self._check(self.sim.L.mth_halo_pack(self.sim.h, part, side, buf.data_ptr()), "pack")

    def unpack(self, part, side, buf):
        self._check(self.sim.L.mth_halo_unpack(self.sim.h, part, side, buf.data_ptr()), "unpack")

    def outflow(self, part, side):
        self._check(self.sim.L.mth_halo_outflow(self.sim.h, part, side), "outflow")



# ---------------------------------------------------------------- transports
class TorchTransport:
    """One slab per rank; halos travel by torch.distributed point-to-point
    messages (NCCL between GPUs, gloo between CPU processes)."""

    def __init__(self, dist, rank, world, bcs):
        self.dist, self.rank, self.world = dist, rank, world
        self.left, self.right = neighbours(rank, world, bcs)

    def exchange(self, slabs, part, bufs):
        (slab,), (b,) = slabs, bufs
        send, recv = b
        slab.pack(part, 0, send[0])
        slab.pack(part, 1, send[1])
        with slab.on_stream():  # messages and copies ordered after the packs
            if self.world == 1:
                if self.left is not None:  # periodic: the slab is its own neighbour
                    recv[0].copy_(send[1])
                    recv[1].copy_(send[0])
            else:
                ops = []
                P2P = self.dist.P2POp
                if self.left is not None:
                    ops.append(P2P(self.dist.isend, send[0], self.left, tag=1))
                if self.right is not None:
                    ops.append(P2P(self.dist.irecv, recv[1], self.right, tag=1))
                    ops.append(P2P(self.dist.isend, send[1], self.right, tag=0))
                if self.left is not None:
                    ops.append(P2P(self.dist.irecv, recv[0], self.left, tag=0))
                if ops:
                    for req in self.dist.batch_isend_irecv(ops):
                        req.wait()
        for side, nb in ((0, self.left), (1, self.right)):
            if nb is None:
                slab.outflow(part, side)
            else:
                slab.unpack(part, side, recv[side])


class LocalTransport:
    """Every slab of the domain in this process (on one GPU or several):
    halos move by plain copies between the slabs' buffers."""

    def __init__(self, n, bcs):
        self.nb = [neighbours(r, n, bcs) for r in range(n)]

    def exchange(self, slabs, part, bufs):
        for slab, (send, _) in zip(slabs, bufs):
            slab.pack(part, 0, send[0])
            slab.pack(part, 1, send[1])
        for r, (slab, (_, recv)) in enumerate(zip(slabs, bufs)):
            left, right = self.nb[r]
            if left is None:
                slab.outflow(part, 0)
            else:
                with slab.on_stream():
                    recv[0].copy_(bufs[left][0][1])  # the left slab's high rows
                slab.unpack(part, 0, recv[0])
            if right is None:
                slab.outflow(part, 1)
            else:
                with slab.on_stream():
                    recv[1].copy_(bufs[right][0][0])  # the right slab's low rows
                slab.unpack(part, 1, recv[1])


# ------------------------------------------------------------------- domain
class SlabDomain:
    """The slabs of one domain held by this process (one per rank under
    torch.distributed, or all of them with a LocalTransport), stepped
    together: Simulation::updateTime per step, parts separated by halo
    exchanges.  ``cfg`` holds the keywords of ``Simulation`` for the whole
    domain (global nx, xmin, xmax); ``ranks`` lists the slab numbers held here."""

    def __init__(self, cfg, n_slabs, ranks, transport, torch, device=0):
        import method_b200 as mb

        self.cfg = dict(cfg)
        self.Ng = cfg.get("Ng", 4)
        self.extents = slab_extents(cfg["nx"], n_slabs, self.Ng)
        self.ranks = list(ranks)
        self.transport = transport
        self.slabs = []
        self.stream = torch.cuda.Stream(device=device)
        for r in self.ranks:
            off, n = self.extents[r]
            kw = dict(self.cfg, nx=n, x_slab=(off, cfg["nx"]), device=device)
            self.slabs.append(DeviceSlab(mb.Simulation(**kw), torch, self.stream))
        self.bufs = [((s.new_buffer(), s.new_buffer()), (s.new_buffer(), s.new_buffer()))
                     for s in self.slabs]
        self.parts = self.slabs[0].parts

    def exchange(self, part):
        self.transport.exchange(self.slabs, part, self.bufs)

    def set_prims(self, prims):
        """Simulation::set from the whole domain's primitive array (ghosts
        included); each slab takes its columns plus Ng ghost rows a side."""
        for r, s in zip(self.ranks, self.slabs):
            off, n = self.extents[r]
            s.sim.set_prims(np.ascontiguousarray(prims[:, off:off + n + 2 * self.Ng]))
        self.exchange(-1)

    def update_time(self, n=1):
        L = self.slabs[0].sim.L
        for _ in range(n):
            dt = C.c_double()
            L.mth_next_dt(self.slabs[0].sim.h, C.byref(dt))
            for part in range(self.parts):
                for s in self.slabs:
                    s._check(L.mth_step_part(s.sim.h, dt.value, part), "step_part")
                self.exchange(part)
            for s in self.slabs:
                L.mth_advance_time(s.sim.h, dt.value)
        for s in self.slabs:
            s.sim.sync()

    def local_states(self):
        """(cons, prims, aux) of each slab held here, ghost rows included."""
        return [s.sim.state() for s in self.slabs]

    def close(self):
        for s in self.slabs:
            s.sim.close()


def assemble(states, extents, Ng):
    """The whole domain's arrays from every slab's (cons, prims, aux): each
    slab's interior columns, and the outer ghost rows of the end slabs."""
    out = []
    for q in range(3):
        parts = []
        last = len(states) - 1
        for r, st in enumerate(states):
            a = st[q]
            lo = 0 if r == 0 else Ng
            hi = a.shape[1] if r == last else a.shape[1] - Ng
            parts.append(a[:, lo:hi])
        out.append(np.concatenate(parts, axis=1))
    return tuple(out)
