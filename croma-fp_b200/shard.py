"""Tracer sharding across ranks (one process per GPU).

Tracers are independent in the Fokker-Planck update -- the reference has no
communication inside its per-snapshot loop -- so a multi-GPU run partitions
the tracers and exchanges nothing on the data path.  Two partitions:

* contiguous chunks (``contiguous``), and
* longest-processing-time-first over the tracers' sub-step work
  (``lpt_assign``), the reference's per-thread assignment of
  tracer_fp_batch_execute_parallel (src/tracer_fp_batch.c:905-937): tasks
  sorted by weight nsub x segments (descending, ties by tracer index), each
  given to the currently least-loaded part (lowest index on ties).

The only collective is the optional gather of results to one rank at the end
(``gather_rows``), plus ``max_over_ranks`` for timing.  Collectives go through
torch.distributed (NCCL on GPUs, gloo on CPU); every rank takes the same
collective steps in the same order.
"""
from __future__ import annotations

import numpy as np


def contiguous(ntracer: int, world: int, rank: int) -> np.ndarray:
    """Tracer indices of `rank` when [0, ntracer) is cut into `world`
    contiguous chunks whose sizes differ by at most one."""
    base, extra = divmod(int(ntracer), int(world))
    start = rank * base + min(rank, extra)
    stop = start + base + (1 if rank < extra else 0)
    return np.arange(start, stop, dtype=np.int64)


def coeff_segments(nsub: np.ndarray, max_segments: int = 16, min_steps: int = 4,
                   allow_interp: bool = True) -> np.ndarray:
    """Coefficient segments per tracer (tracer_fp_choose_coeff_interp_segments,
    src/tracer_fp_setup.c:73-95): the largest power of two within
    max_segments and nsub / min_steps."""
    nsub = np.asarray(nsub, dtype=np.int64)
    out = np.ones_like(nsub)
    if not allow_interp or min_steps <= 0:
        return out
    cap = np.minimum(max(1, int(max_segments)), nsub // int(min_steps))
    seg = np.ones_like(nsub)
    while True:
        grow = seg * 2 <= cap
        if not grow.any():
            break
        seg = np.where(grow, seg * 2, seg)
    seg = np.where(nsub <= 1, 1, np.minimum(seg, nsub))
    return np.maximum(seg, 1)


def task_weights(nsub: np.ndarray, nseg: np.ndarray) -> np.ndarray:
    """task_weight of src/tracer_fp_batch.c:113-125 (quantized integration,
    one tracer per task): nsub x segments, each at least 1."""
    return np.maximum(np.asarray(nsub, np.int64), 1) * np.maximum(np.asarray(nseg, np.int64), 1)


def lpt_assign(weights: np.ndarray, nparts: int) -> np.ndarray:
    """Part of every task under longest-processing-time-first."""
    w = np.asarray(weights, dtype=np.int64)
    order = np.lexsort((np.arange(w.size), -w))      # weight desc, index asc
    loads = np.zeros(int(nparts), dtype=np.int64)
    part = np.empty(w.size, dtype=np.int64)
    for i in order:
        best = int(np.argmin(loads))                 # first minimum: lowest index
        part[i] = best
        loads[best] += w[i]
    return part


def lpt_indices(weights: np.ndarray, world: int, rank: int) -> np.ndarray:
    """Tracer indices of `rank` under lpt_assign, in ascending order."""
    return np.flatnonzero(lpt_assign(weights, world) == rank).astype(np.int64)


def imbalance(weights: np.ndarray, part: np.ndarray, nparts: int) -> float:
    """max part load / mean part load."""
    loads = np.bincount(part, weights=np.asarray(weights, np.float64), minlength=nparts)
    mean = loads.mean()
    return float(loads.max() / mean) if mean > 0 else 1.0


def gather_rows(rows: np.ndarray, indices: np.ndarray, ntracer: int, dist, device=None):
    """Reassemble per-tracer rows [n_local][...] from every rank into
    [ntracer][...] on every rank (all-gather; one collective pair).  Ranks
    may hold different counts: rows are padded to the largest count."""
    import torch
    rows = np.ascontiguousarray(rows)
    world = dist.get_world_size()
    n_local = torch.tensor([rows.shape[0]], dtype=torch.int64, device=device)
    counts = [torch.zeros_like(n_local) for _ in range(world)]
    dist.all_gather(counts, n_local)
    counts = [int(c.item()) for c in counts]
    nmax = max(counts)
    tail = rows.shape[1:]
    pad = np.zeros((nmax,) + tail, dtype=rows.dtype)
    pad[:rows.shape[0]] = rows
    ipad = np.full(nmax, -1, dtype=np.int64)
    ipad[:indices.size] = indices
    t_rows = torch.from_numpy(pad).to(device) if device else torch.from_numpy(pad)
    t_idx = torch.from_numpy(ipad).to(device) if device else torch.from_numpy(ipad)
    all_rows = [torch.empty_like(t_rows) for _ in range(world)]
    all_idx = [torch.empty_like(t_idx) for _ in range(world)]
    dist.all_gather(all_rows, t_rows)
    dist.all_gather(all_idx, t_idx)
    out = np.zeros((int(ntracer),) + tail, dtype=rows.dtype)
    for r in range(world):
        idx = all_idx[r].cpu().numpy()[:counts[r]]
        out[idx] = all_rows[r].cpu().numpy()[:counts[r]]
    return out


def max_over_ranks(value: float, dist, device=None) -> float:
    """The maximum of a per-rank scalar (device time of a timed region)."""
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
