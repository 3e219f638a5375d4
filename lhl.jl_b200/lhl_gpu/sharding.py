"""Multi-GPU sharding of the path, one process per GPU over torch.distributed.

A single reduction does not shard (every ELMHES step needs a global pivot decision), so each
rank that needs a Jacobian reduces it itself.  What shards (the reference's own units of
independent work are the shift, F:2456-2461, and the Jacobian, F:3179):

* shifts of one J: every rank reduces J (or holds its own copy of the factors), runs the
  shift LUs, solves and refinement for a contiguous slice of the shifts, and the solution
  columns are gathered in shift order (`shift_slice`, `gather_columns`, `sharded_chain`);
* independent Jacobians (batches of matrices of uneven order): a partition balanced by the
  O(n^3) reduction cost (`jacobian_partition`); no exchange at all.

The collectives are plain torch.distributed calls, NCCL over NVLink for CUDA tensors and
gloo for CPU tensors, so the host logic runs the same in CPU tests.
"""
from __future__ import annotations

import heapq

import torch


def shift_slice(S: int, rank: int, world: int):
    """(s0, count) of rank's contiguous slice of S shifts; counts differ by at most one and
    lower ranks take the larger ones."""
    if world < 1 or not 0 <= rank < world or S < 0:
        raise ValueError("bad shard arguments")
    base, extra = divmod(S, world)
    count = base + (1 if rank < extra else 0)
    s0 = rank * base + min(rank, extra)
    return s0, count


def jacobian_partition(ns, world: int):
    """Assign matrices of orders ns to `world` ranks, balancing the sum of n^3 (the reduction's
    cost; the shift and solve work, n^2 per shift, follows it).  Longest-processing-time first:
    matrices in decreasing order, each to the least-loaded rank (ties to the lowest rank).
    Returns one sorted index list per rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    heap = [(0, r) for r in range(world)]
    parts = [[] for _ in range(world)]
    for i in sorted(range(len(ns)), key=lambda i: (-int(ns[i]), i)):
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + int(ns[i]) ** 3, r))
    return [sorted(p) for p in parts]


def gather_columns(X_local: torch.Tensor, S: int, rhs_per_shift: int, group=None) -> torch.Tensor:
    """All ranks' solution columns in shift order: rank r holds the (n, count_r * R) block of
    its shift slice (`shift_slice`).  The blocks are padded to the largest slice for one
    all_gather and trimmed after.  Returns the (n, S * R) block on every rank."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    n = X_local.shape[0]
    R = rhs_per_shift
    cmax = shift_slice(S, 0, world)[1] * R
    buf = torch.zeros((cmax, n), dtype=X_local.dtype, device=X_local.device)
    if X_local.shape[1]:
        buf[: X_local.shape[1]] = X_local.t()
    out = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(out, buf, group=group)
    cols = [out[r][: shift_slice(S, r, world)[1] * R] for r in range(world)]
    return torch.cat(cols, 0).t()


_REDUCTION_ARRAYS = ("factors", "Ht", "ipiv", "perm", "iperm", "scale", "iscale")


def reduction_layout(n: int, complex_j: bool = False):
    """(name, 8-byte words) of each array of a reduction of order n, in the packed order:
    factors and Ht column-major (interleaved re, im for a complex J), ipiv (n-2), perm and
    iperm int64, scale and iscale float64."""
    nn = n * n * (2 if complex_j else 1)
    words = {"factors": nn, "Ht": nn, "ipiv": max(n - 2, 0), "perm": n, "iperm": n, "scale": n, "iscale": n}
    return [(k, words[k]) for k in _REDUCTION_ARRAYS]


def pack_reduction(arrays, n: int, complex_j: bool = False) -> torch.Tensor:
    """One float64 buffer holding the arrays of a reduction (names and shapes as
    LHLWorkspace.import_arrays takes them) in `reduction_layout` order; the int64 arrays are
    carried bit for bit."""
    parts = []
    for k, _ in reduction_layout(n, complex_j):
        t = arrays[k]
        if t.dim() == 2:  # column-major flat: rows of the transpose
            t = t.t().contiguous()
            t = torch.view_as_real(t) if t.is_complex() else t
        parts.append(t.contiguous().reshape(-1).view(torch.float64))
    return torch.cat(parts) if parts else torch.empty(0, dtype=torch.float64)


def unpack_reduction(buf: torch.Tensor, n: int, complex_j: bool = False):
    """The arrays of `pack_reduction`'s buffer as views of it: factors and Ht (n, n)
    column-major (complex128 for a complex J), ipiv, perm, iperm int64, scale, iscale."""
    out, o = {}, 0
    for k, w in reduction_layout(n, complex_j):
        seg = buf[o:o + w]
        o += w
        if k in ("factors", "Ht"):
            m = torch.view_as_complex(seg.view(n, n, 2)) if complex_j else seg.view(n, n)
            out[k] = m.t()
        elif k in ("ipiv", "perm", "iperm"):
            out[k] = seg.view(torch.int64)
        else:
            out[k] = seg
    if o != buf.numel():
        raise ValueError(f"buffer of {buf.numel()} words for a reduction of {o}")
    return out


def broadcast_reduction(ws, src: int = 0, group=None):
    """Share one rank's reduction with every rank of the group, in place of reducing J on
    each: rank `src` (a global rank, as torch.distributed.broadcast takes it) holds the
    reduction; the others' workspaces, of the same order, element type and form, import it
    (lhl_ws_import).  One collective of 8 n^2 (16 n^2 for a complex J) bytes plus small
    arrays.  A header broadcast and a flag reduction first make every rank raise together
    when a workspace differs, so that no rank waits in the data broadcast alone."""
    import torch.distributed as dist
    cj = ws.dtype == torch.complex128
    codes = {torch.float64: 0, torch.float32: 1, torch.complex128: 2}
    dev = ws.device
    me = dist.get_rank()
    mine = torch.tensor([ws.n, int(ws.precision), codes[ws.dtype], int(bool(ws.reduced))],
                        dtype=torch.int64, device=dev)
    head = mine.clone()
    dist.broadcast(head, src, group=group)
    bad = 0
    if me == src:
        bad = 0 if ws.reduced else 1
    elif not torch.equal(head[:3], mine[:3]):
        bad = 2
    flag = torch.tensor([bad], dtype=torch.int64, device=dev)
    dist.all_reduce(flag, op=dist.ReduceOp.MAX, group=group)
    if int(flag.item()) == 1:
        raise ValueError(f"rank {src} holds no reduction to broadcast")
    if int(flag.item()) == 2:
        raise ValueError(f"workspaces differ from rank {src}'s (order, form, element type {head.tolist()[:3]})")
    words = sum(w for _, w in reduction_layout(ws.n, cj))
    if me == src:
        buf = pack_reduction({k: getattr(ws, k) for k in _REDUCTION_ARRAYS}, ws.n, cj)
    else:
        buf = torch.empty(words, dtype=torch.float64, device=dev)
    dist.broadcast(buf, src, group=group)
    if me != src:
        ws.import_arrays(unpack_reduction(buf, ws.n, cj))
    return ws


def sharded_chain(G, ws, J: torch.Tensor, B: torch.Tensor, sigmas: torch.Tensor, taus: torch.Tensor,
                  rhs_per_shift: int = 1, tol: float = 1e-10, refine: str = "gmres", group=None):
    """The per-shift chain on this rank's slice of the shifts of an already reduced workspace:
    shift LUs, solves, refinement to `tol` (GMRES-IR or fixed-point), then the gather.
    B holds all S * R right-hand sides; returns (X with every rank's columns, this rank's
    relative residuals).  Complex shifts (complex sigmas or taus, on a real reduction) and a
    complex J's workspace take a complex shift object and complex right-hand sides."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    S = sigmas.numel()
    R = rhs_per_shift
    s0, cnt = shift_slice(S, rank, world)
    n = ws.n
    if cnt == 0:
        X_local = torch.empty((n, 0), dtype=B.dtype, device=B.device)
        res = torch.empty(0, dtype=torch.float64, device=B.device)
    else:
        cplx = sigmas.is_complex() or taus.is_complex() or getattr(ws, "cj", False)
        sh = G.LHLShift(ws, cnt, complex=cplx)  # the workspace's precision
        G.lhl_shift_batched_(sh, ws, sigmas[s0:s0 + cnt].contiguous(), taus[s0:s0 + cnt].contiguous())
        Bl = B[:, s0 * R:(s0 + cnt) * R]
        X_local = torch.empty((cnt * R, n), dtype=B.dtype, device=B.device).t()
        X_local.copy_(Bl)
        G.lhl_ldiv_(X_local, sh, ws, rhs_per_shift=R)
        Bc = torch.empty_like(X_local)
        Bc.copy_(Bl)
        if refine == "gmres":
            res = G.lhl_refine_gmres_(X_local, J, Bc, sh, ws, tol=tol, rhs_per_shift=R)
        else:
            res = G.lhl_refine_tol_(X_local, J, Bc, sh, ws, tol=tol, rhs_per_shift=R)
    return gather_columns(X_local, S, R, group), res
