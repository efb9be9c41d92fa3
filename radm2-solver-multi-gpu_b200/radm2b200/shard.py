"""Splitting a batch of cells over ranks (one process per GPU) and combining the results.

Cells are independent, so a multi-GPU run has no exchange step inside the solve: each rank
integrates its own cells and the ranks meet only to combine counters (the reference's
IPAR[10..17] statistics, summed) and, when the caller wants one host copy, the states.
This replaces the reference's host-staged two-GPU gather (mgpu.cu:3508-3581).

Two partitions:
  contiguous  rank r takes [lo_r, hi_r), sizes differing by at most one cell.
  balanced    cells sorted by a per-cell cost (the seeding network's predicted step
              count) are dealt to ranks in snake order (0..N-1, N-1..0, ...), so every rank
              gets the same mix of cheap and stiff cells; each rank's cells stay in
              ascending index order for coalesced loads.
"""
import numpy as np

# IPAR slots the library fills with summed per-cell statistics (mgpu.cu:3835-3845).
IPAR_COUNTERS = slice(10, 18)


def contiguous_ranges(ncell, world):
    """[(lo, hi)] per rank."""
    if world < 1 or ncell < 0:
        raise ValueError("bad partition request")
    base, extra = divmod(ncell, world)
    out, lo = [], 0
    for r in range(world):
        hi = lo + base + (1 if r < extra else 0)
        out.append((lo, hi))
        lo = hi
    return out


def balanced_assignment(costs, world):
    """Index arrays per rank: cells sorted by descending cost, dealt in snake order."""
    costs = np.asarray(costs, dtype=np.float64)
    if world < 1:
        raise ValueError("world must be >= 1")
    order = np.argsort(-costs, kind="stable")
    n = len(order)
    rounds = np.arange(n) // world
    pos = np.arange(n) % world
    rank = np.where(rounds % 2 == 0, pos, world - 1 - pos)
    return [np.sort(order[rank == r]) for r in range(world)]


INT_MAX = 2 ** 31 - 1


def reduce_totals(values, dist=None, group=None):
    """Sum 64-bit totals (e.g. radm2_stats' accepted/rejected step counts) over ranks;
    returns a list of Python ints on every rank."""
    vals = [int(v) for v in values]
    if dist is None or not dist.is_initialized() or dist.get_world_size(group) == 1:
        return vals
    import torch
    t = torch.tensor(vals, dtype=torch.int64)
    if dist.get_backend(group) == "nccl":
        t = t.cuda()
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return [int(x) for x in t.cpu().tolist()]


def reduce_counters(ipar, dist=None, group=None):
    """Sum the counter slots of IPAR over ranks (in place), in 64-bit arithmetic, each slot
    saturating at INT_MAX as the library's own update does (int IPAR slots cannot hold the
    sums of large multi-GPU runs; reduce_totals over radm2_stats gives the exact totals).
    Other slots are untouched."""
    if dist is None or not dist.is_initialized() or dist.get_world_size(group) == 1:
        return ipar
    summed = reduce_totals(np.asarray(ipar[IPAR_COUNTERS], dtype=np.int64), dist, group)
    ipar[IPAR_COUNTERS] = np.minimum(np.asarray(summed, dtype=np.int64), INT_MAX).astype(ipar.dtype)
    return ipar


def gather_states(y_local, idx_local, ncell, dist=None, group=None):
    """Every rank's final states [n_r][59] placed at their global cell indices; returns the
    full [ncell][59] array on every rank (a host copy for output)."""
    y_local = np.ascontiguousarray(y_local, dtype=np.float64)
    idx_local = np.asarray(idx_local, dtype=np.int64)
    out = np.empty((ncell, y_local.shape[1]), dtype=np.float64)
    if dist is None or not dist.is_initialized() or dist.get_world_size(group) == 1:
        out[idx_local] = y_local
        return out
    import torch
    world = dist.get_world_size(group)
    sizes = [None] * world
    dist.all_gather_object(sizes, int(len(idx_local)), group=group)
    m = max(sizes)
    ybuf = torch.zeros((m, y_local.shape[1]), dtype=torch.float64)
    ibuf = torch.full((m,), -1, dtype=torch.int64)
    ybuf[:len(idx_local)] = torch.from_numpy(y_local)
    ibuf[:len(idx_local)] = torch.from_numpy(idx_local)
    if dist.get_backend(group) == "nccl":  # NCCL moves device tensors only
        ybuf, ibuf = ybuf.cuda(), ibuf.cuda()
    ys = [torch.empty_like(ybuf) for _ in range(world)]
    iss = [torch.empty_like(ibuf) for _ in range(world)]
    dist.all_gather(ys, ybuf, group=group)
    dist.all_gather(iss, ibuf, group=group)
    for r in range(world):
        k = sizes[r]
        out[iss[r][:k].cpu().numpy()] = ys[r][:k].cpu().numpy()
    return out
