"""Autotuner for the launch and refinement choices of the path, by timed trials on the device.

The reference fixes its tile shapes and panel width in code (F:703-706) and has no tuner; on
the GPU three choices per workload are left open, and this module picks them by measurement:

  * the shift LU's launch shape (threads x pending-row elements per thread, rows of H in
    flight): every shape that covers the order gives the same bits (shift.cu, complex.cu), so
    only the time decides;
  * the mixed form's FP32 reduction kernel: rows on chip with a rank-1 update every step
    (the eager kernel) or rows in global memory with rank-16 updates per panel (the
    panel-delayed one); both are similarities to FP32 accuracy, with different roundings;
  * the refinement: fixed-point lhl_refine_tol with a step cap, GMRES-IR with restart m and a
    cycle cap, or a few fixed-point steps followed by GMRES-IR on the columns still above the
    tolerance.  A choice counts only if every solve reaches the tolerance (or, where the
    caller says so, the FP64 floor of its shift).

A workload is keyed by device name, shift kind (real / complex), order bucket (the next power
of two), form and right-hand sides per shift.  Results are kept in a JSON cache
(tuning.json beside this file) that a later run reads instead of tuning again.
"""
from __future__ import annotations

import json
import os
import time

HERE = os.path.dirname(os.path.abspath(__file__))
CACHE = os.path.join(HERE, "tuning.json")

# refinement candidates: ("fixed", max steps), ("gmres", max cycles, restart), or ("hybrid",
# fixed-point steps, then GMRES-IR max cycles, restart) for the columns still above the tolerance
REFINE_CANDIDATES = {
    "mixed": [("fixed", 16), ("gmres", 8, 2), ("gmres", 6, 3), ("gmres", 4, 4), ("gmres", 12, 8),
              ("hybrid", 2, 6, 3), ("hybrid", 3, 6, 2)],
    "plain": [("fixed", 4), ("gmres", 4, 3)],
}


def order_bucket(n: int) -> int:
    b = 16
    while b < n:
        b *= 2
    return b


def workload_key(device: str, is_complex: bool, n: int, form: str, rhs_per_shift: int) -> str:
    return f"{device}|{'complex' if is_complex else 'real'}|n{order_bucket(n)}|{form}|r{rhs_per_shift}"


def load_cache(path: str = CACHE) -> dict:
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def save_cache(cache: dict, path: str = CACHE) -> None:
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(cache, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def lookup(device: str, is_complex: bool, n: int, form: str, rhs_per_shift: int, path: str = CACHE):
    """The cached choice for this workload, or None."""
    return load_cache(path).get(workload_key(device, is_complex, n, form, rhs_per_shift))


def time_ms(torch, fn, reps: int = 3, warmup: int = 1) -> float:
    """Minimum over `reps` runs of fn, timed with CUDA events on the current stream."""
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    best = float("inf")
    st = torch.cuda.current_stream()
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        fn()
        b.record(st)
        torch.cuda.synchronize()
        best = min(best, a.elapsed_time(b))
    return best


def _shift_digest(torch, sh, count: int):
    """Checksum of the shift LU state of the first `count` slots: the bits of rdiag (1 / U[k,k],
    which every elimination step feeds), swap and info."""
    acc = []
    for slot in sorted({0, count // 2, count - 1}):
        r = sh.rdiag(slot)
        r = torch.view_as_real(r) if r.is_complex() else r
        acc.append(int(r.contiguous().view(torch.int64).sum().item()))
        acc.append(int(sh.swap(slot).to(torch.int64).sum().item()))
    acc.append(int(sh.info_all[:count].to(torch.int64).sum().item()))
    return tuple(acc)


def tune_shift_variant(G, torch, ws, sh, sigma, tau, reps: int = 3):
    """Every shift-LU launch shape that covers ws's order, timed on this batch of shifts.
    Returns (best variant, trials); a shape whose shift states differ from the first shape's
    is never chosen (they are the same by construction; this checks it)."""
    count = int(sigma.shape[0])
    cands = G.shift_variants(sh.is_complex, ws.n)
    trials, ref = [], None
    for v in cands:
        ws.set_shift_variant(0 if sh.is_complex else v, v if sh.is_complex else 0)
        ms = time_ms(torch, lambda: G.lhl_shift_batched_(sh, ws, sigma, tau), reps)
        dig = _shift_digest(torch, sh, count)
        if ref is None:
            ref = dig
        trials.append({"variant": v, "ms": ms, "same_bits": dig == ref})
    ws.set_shift_variant(0, 0)
    ok = [t for t in trials if t["same_bits"]]
    return (min(ok, key=lambda t: t["ms"])["variant"] if ok else 0), trials


def tune_mixed_kernel(torch, ws, reduce_fn, reps: int = 2):
    """The mixed form's FP32 reduction kernels (1 eager, 2 panel-delayed), timed on this J.
    Returns (best kernel, trials)."""
    trials = []
    for which in (1, 2):
        ws.set_mixed_kernel(which)
        trials.append({"kernel": which, "ms": time_ms(torch, reduce_fn, reps)})
    best = min(trials, key=lambda t: t["ms"])["kernel"]
    ws.set_mixed_kernel(best)
    return best, trials


def tune_refine(torch, form: str, run_chain, accept, reps: int = 2, candidates=None):
    """Refinement schemes timed through `run_chain(choice)` (the whole per-shift chain: shift
    LUs, solves, refinement), each accepted only if `accept()` says every solve reached its
    target afterwards.  Returns (best choice or None, trials)."""
    trials = []
    for ch in candidates or REFINE_CANDIDATES[form]:
        ms = time_ms(torch, lambda: run_chain(ch), reps)
        ok = bool(accept())
        trials.append({"refine": list(ch), "ms": ms, "ok": ok})
    good = [t for t in trials if t["ok"]]
    return (tuple(min(good, key=lambda t: t["ms"])["refine"]) if good else None), trials


def record(cache: dict, key: str, choice: dict) -> dict:
    """Store `choice` (with its trials and the time it was measured) under `key`."""
    choice = dict(choice)
    choice["measured"] = time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime())
    cache[key] = choice
    return cache
