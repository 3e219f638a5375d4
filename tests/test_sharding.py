"""Multi-process host logic on the CPU (gloo, world size 2): the shift slices and the
Jacobian partition of lhl_gpu.sharding, the column gather in shift order, and bench.py's
max-over-ranks timing.  No GPU is involved."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from lhl_gpu import sharding as SH


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("S", [0, 1, 2, 5, 64, 257])
@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_shift_slices_cover_in_order(S, world):
    got = [SH.shift_slice(S, r, world) for r in range(world)]
    pos = 0
    for s0, cnt in got:
        assert s0 == pos
        pos += cnt
    assert pos == S
    counts = [c for _, c in got]
    assert max(counts) - min(counts) <= 1 and counts == sorted(counts, reverse=True)


def test_jacobian_partition_balances_cost():
    from lhl_gpu import configs
    ns = [int(v) for v in configs.config4(count=512)["ns"]]
    for world in (1, 2, 4, 8):
        parts = SH.jacobian_partition(ns, world)
        assert sorted(i for p in parts for i in p) == list(range(len(ns)))
        loads = [sum(ns[i] ** 3 for i in p) for p in parts]
        # longest-processing-time first: the spread is at most the largest single matrix
        assert max(loads) - min(loads) <= max(n ** 3 for n in ns)


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        n, S, R = 7, 5, 2
        s0, cnt = SH.shift_slice(S, rank, world)
        # the rank's columns hold their global column index in every row
        X = torch.arange(s0 * R, (s0 + cnt) * R, dtype=torch.float64).repeat(n, 1)
        full = SH.gather_columns(X, S, R)
        # complex columns (complex shifts, a complex J): the same gather, imaginary part -index
        Xc = torch.complex(X, -X)
        fullc = SH.gather_columns(Xc, S, R)
        t = bench.max_over_ranks([1.0 + rank, 5.0 - rank], "cpu", dist)
        q.put((rank, full.numpy().tolist(), t, fullc.real.numpy().tolist(), fullc.imag.numpy().tolist(),
               str(fullc.dtype)))
    finally:
        dist.destroy_process_group()


def test_two_ranks_gather_and_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want = np.tile(np.arange(10.0), (7, 1))
    for rank, full, t, cre, cim, cdt in out:
        assert np.array_equal(np.array(full), want), rank
        assert t == [2.0, 5.0]
        assert cdt == "torch.complex128"
        assert np.array_equal(np.array(cre), want) and np.array_equal(np.array(cim), -want), rank
