"""Multi-rank plumbing on CPU: world_size-2 gloo ranks run the barrier, the
max-over-ranks timing reduction and the ensemble split that bench.py uses
under torchrun, and the split itself is checked for coverage and balance."""
import os
import socket

import pytest

from method_b200.ranks import lpt_partition


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from method_b200 import initial
    from method_b200.ranks import Ranks, lpt_partition as lpt
    r = Ranks("gloo", timeout_s=30)
    r.barrier()
    mx = r.max(10.0 + rank)
    total = r.sum(1.0)
    mem = initial.kh_ensemble(256, seed=2024)
    costs = [c["nx"] * c["ny"] * (2 if c["model"] == "srrmhd" else 1) for c, _ in mem]
    mine = lpt(costs, r.world)[r.rank]
    r.close()
    q.put((rank, mx, total, mine))


def test_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = {}
    for _ in ps:
        rank, mx, total, mine = q.get(timeout=120)
        out[rank] = (mx, total, mine)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0][0] == out[1][0] == 11.0
    assert out[0][1] == out[1][1] == 2.0
    a, b = set(out[0][2]), set(out[1][2])
    assert not (a & b) and a | b == set(range(256))


@pytest.mark.parametrize("parts", [1, 2, 3, 8])
def test_lpt_partition_covers_and_balances(parts):
    import numpy as np
    rng = np.random.default_rng(3)
    costs = [int(x) for x in rng.integers(64, 513, size=256) ** 2 * 2]
    split = lpt_partition(costs, parts)
    flat = sorted(i for p in split for i in p)
    assert flat == list(range(256))
    loads = [sum(costs[i] for i in p) for p in split]
    # LPT bound: max load <= mean + largest item
    assert max(loads) <= sum(costs) / parts + max(costs)
    assert lpt_partition(costs, parts) == split  # deterministic


def test_lpt_partition_rejects_zero_parts():
    with pytest.raises(ValueError):
        lpt_partition([1, 2], 0)
