"""The x-slab decomposition's host logic on CPU: slab extents, neighbours,
and the halo pack / exchange / unpack of every slab checked against the
single domain's ghost rows (Periodic or Flow: periodic in x; Outflow: copies
of the boundary row, boundaryConds.cc:5-145, 449-733), both for slabs held by
one process (LocalTransport) and for two gloo ranks exchanging
point-to-point (TorchTransport, the code path NCCL ranks take)."""
import os
import socket

import numpy as np
import pytest

from method_b200 import slab

NG = 4


def _global_state(nx, ny, seed):
    rng = np.random.default_rng(seed)
    return [rng.standard_normal((nv, nx + 2 * NG, ny + 2 * NG, 1)) for nv in (9, 8, 13)]


def _fill_x_ghosts(arrays, nx, bcs):
    """The single domain's x ghost rows after Bcs::apply."""
    out = [a.copy() for a in arrays]
    for a in out:
        if bcs in slab.X_PERIODIC:
            a[:, :NG] = a[:, nx:nx + NG]
            a[:, nx + NG:] = a[:, NG:2 * NG]
        else:
            a[:, :NG] = a[:, NG:NG + 1]
            a[:, nx + NG:] = a[:, nx + NG - 1:nx + NG]
    return out


def _local(arrays, off, n):
    loc = [np.ascontiguousarray(a[:, off:off + n + 2 * NG]) for a in arrays]
    for a in loc:  # the ghost rows must come from the exchange
        a[:, :NG] = np.nan
        a[:, -NG:] = np.nan
    return loc


def test_slab_extents_and_neighbours():
    ext = slab.slab_extents(70, 4, NG)
    assert [n for _, n in ext] == [18, 18, 17, 17]
    assert [o for o, _ in ext] == [0, 18, 36, 53]
    with pytest.raises(ValueError):
        slab.slab_extents(10, 3, NG)  # 3-column slabs cannot supply 4 halo rows
    assert slab.neighbours(0, 3, "periodic") == (2, 1)
    assert slab.neighbours(2, 3, "flow") == (1, 0)
    assert slab.neighbours(0, 3, "outflow") == (None, 1)
    assert slab.neighbours(0, 1, "outflow") == (None, None)
    assert slab.neighbours(0, 1, "periodic") == (0, 0)


@pytest.mark.parametrize("bcs", ["periodic", "flow", "outflow"])
@pytest.mark.parametrize("n_slabs", [1, 2, 3])
def test_local_exchange_matches_single_domain(bcs, n_slabs):
    import torch
    nx, ny = 29, 12
    g = _global_state(nx, ny, seed=n_slabs)
    want = _fill_x_ghosts(g, nx, bcs)
    ext = slab.slab_extents(nx, n_slabs, NG)
    slabs = [slab.ArraySlab(*_local(g, off, n), NG, torch) for off, n in ext]
    bufs = [((s.new_buffer(), s.new_buffer()), (s.new_buffer(), s.new_buffer())) for s in slabs]
    slab.LocalTransport(n_slabs, bcs).exchange(slabs, 0, bufs)
    for s, (off, n) in zip(slabs, ext):
        for got, w in zip(s.arrays, want):
            np.testing.assert_array_equal(got, w[:, off:off + n + 2 * NG])
    # the assembled domain is the single domain's, outer ghost rows included
    asm = slab.assemble([s.arrays for s in slabs], ext, NG)
    for got, w in zip(asm, want):
        np.testing.assert_array_equal(got, w)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, bcs, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=30))
    nx, ny = 21, 10
    g = _global_state(nx, ny, seed=7)
    off, n = slab.slab_extents(nx, world, NG)[rank]
    s = slab.ArraySlab(*_local(g, off, n), NG, torch)
    bufs = [((s.new_buffer(), s.new_buffer()), (s.new_buffer(), s.new_buffer()))]
    t = slab.TorchTransport(dist, rank, world, bcs)
    t.exchange([s], 0, bufs)
    t.exchange([s], 1, bufs)  # a second exchange reuses the buffers
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, [a.copy() for a in s.arrays]))


@pytest.mark.parametrize("bcs", ["periodic", "outflow"])
def test_two_gloo_ranks_exchange_halos(bcs):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    world = 2
    ps = [ctx.Process(target=_worker, args=(r, world, port, bcs, q)) for r in range(world)]
    for p in ps:
        p.start()
    got = dict(q.get(timeout=120) for _ in range(world))
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    nx, ny = 21, 10
    want = _fill_x_ghosts(_global_state(nx, ny, seed=7), nx, bcs)
    for r, (off, n) in enumerate(slab.slab_extents(nx, world, NG)):
        for a, w in zip(got[r], want):
            np.testing.assert_array_equal(a, w[:, off:off + n + 2 * NG])
