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


class _FakeWorkspace:
    """A host stand-in for LHLWorkspace: the same fields broadcast_reduction reads, arrays as
    CPU tensors (factors and Ht column-major views), and an import_arrays that keeps copies."""

    def __init__(self, n, complex_j=False, precision=0, seed=None):
        self.n, self.precision, self.device = n, precision, torch.device("cpu")
        self.dtype = torch.complex128 if complex_j else torch.float64
        self.reduced = seed is not None
        if seed is not None:
            g = np.random.default_rng(seed)
            for k in ("factors", "Ht"):
                m = g.standard_normal((n, n)) + (1j * g.standard_normal((n, n)) if complex_j else 0)
                if n:
                    m.flat[0] = np.nan  # payloads travel bit for bit
                setattr(self, k, torch.as_tensor(np.asfortranarray(m)))
            self.ipiv = torch.as_tensor(g.integers(-2**62, 2**62, max(n - 2, 0)))
            self.perm = torch.as_tensor(g.permutation(n) + 1)
            self.iperm = torch.as_tensor(g.permutation(n) + 1)
            self.scale = torch.as_tensor(2.0 ** g.integers(-40, 40, n).astype(float))
            self.iscale = 1.0 / self.scale

    def import_arrays(self, arrays):
        for k, v in arrays.items():
            setattr(self, k, v.clone())
        self.reduced = True


def _bits(t):
    t = torch.view_as_real(t.contiguous()) if t.is_complex() else t.contiguous()
    return t.numpy().view(np.uint8).tobytes(), tuple(t.shape)


@pytest.mark.parametrize("complex_j", [False, True])
@pytest.mark.parametrize("n", [0, 1, 2, 3, 17])
def test_pack_unpack_reduction_round_trip(n, complex_j):
    ws = _FakeWorkspace(n, complex_j, seed=n)
    arrays = {k: getattr(ws, k) for k in SH._REDUCTION_ARRAYS}
    buf = SH.pack_reduction(arrays, n, complex_j)
    assert buf.dtype == torch.float64
    assert buf.numel() == sum(w for _, w in SH.reduction_layout(n, complex_j))
    back = SH.unpack_reduction(buf, n, complex_j)
    for k in SH._REDUCTION_ARRAYS:
        assert back[k].dtype == arrays[k].dtype, k
        assert _bits(back[k]) == _bits(arrays[k]), k
    for k in ("factors", "Ht"):  # column-major with leading dimension n, as lhl_ws_import takes it
        assert back[k].shape == (n, n) and (n < 2 or back[k].stride() == (1, n)), k
    with pytest.raises(ValueError):
        SH.unpack_reduction(torch.cat([buf, torch.zeros(1, dtype=torch.float64)]), n, complex_j)


def _bcast_worker(rank, world, port, q, case):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        n, cj = 9, case == "complex"
        if rank == 1:
            ws = _FakeWorkspace(n, cj, seed=7 if case != "unreduced" else None)
        else:
            ws = _FakeWorkspace(n + (1 if case == "order" else 0), cj)
        try:
            SH.broadcast_reduction(ws, src=1)
            q.put((rank, "ok", {k: _bits(getattr(ws, k)) for k in SH._REDUCTION_ARRAYS}))
        except ValueError as e:
            q.put((rank, "raised", str(e)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("case", ["real", "complex", "order", "unreduced"])
def test_ranks_broadcast_reduction(case, world):
    """Rank 1 holds the reduction; with three ranks a receiver sits on each side of it."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_bcast_worker, args=(r, world, port, q, case)) for r in range(world)]
    for p in procs:
        p.start()
    out = dict((r, (s, v)) for r, s, v in (q.get(timeout=120) for _ in procs))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    if case in ("order", "unreduced"):  # every rank raises, none waits in the data broadcast
        assert all(out[r][0] == "raised" for r in range(world)), out
        return
    assert all(out[r][0] == "ok" for r in range(world))
    assert all(out[r][1] == out[1][1] for r in range(world))
