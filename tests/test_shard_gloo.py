"""Multi-rank host logic on CPU (gloo, 2 ranks): each rank integrates its own cells with the
CPU oracle, counters are summed and states gathered, and the result equals one process
integrating every cell.  Also the partitions themselves."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from radm2b200 import inputs, shard


def test_contiguous_ranges_cover_exactly():
    for n, w in [(10, 3), (4096, 8), (5, 8), (0, 2)]:
        r = shard.contiguous_ranges(n, w)
        assert r[0][0] == 0 and r[-1][1] == n
        assert all(a[1] == b[0] for a, b in zip(r, r[1:]))
        sizes = [hi - lo for lo, hi in r]
        assert max(sizes) - min(sizes) <= 1


def test_balanced_assignment_is_a_partition_with_even_cost():
    rng = np.random.default_rng(3)
    costs = np.exp(rng.normal(2.0, 1.5, size=10007))  # heavy-tailed step counts
    for w in (2, 3, 8):
        parts = shard.balanced_assignment(costs, w)
        allidx = np.concatenate(parts)
        assert len(allidx) == len(costs) and len(np.unique(allidx)) == len(costs)
        assert all(np.all(np.diff(p) > 0) for p in parts)
        sums = np.array([costs[p].sum() for p in parts])
        assert sums.max() - sums.min() <= costs.max() + 1e-9
        # contiguous shards of the same heavy-tailed costs are typically far less even
    parts = shard.balanced_assignment(np.arange(8.0), 2)
    assert [list(p) for p in parts] == [[0, 3, 4, 7], [1, 2, 5, 6]]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, ncell, out_path):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import oracle
    import radm2b200
    cells = inputs.make_cells(ncell, 21, "mixed")
    # balanced by a stand-in cost (night cells are cheap, urban ones stiff)
    cost = np.where(cells["cls"] == 3, 1.0, np.where(cells["cls"] == 1, 10.0, 3.0)) + cells["TEMP"] * 1e-3
    idx = shard.balanced_assignment(cost, world)[rank]
    # each rank generates only its own cells: the inputs are a pure function of (seed, cell)
    mine = {k: v[idx] for k, v in cells.items()}
    ipar, rpar = radm2b200.default_params(hstart=6.0)
    ok, p = oracle.params(0.0, 600.0, np.ones(59), np.full(59, 1e-3), rpar, ipar)
    rc = oracle.rconst(mine["JV"], mine["TEMP"], mine["FIX"], mine["RC_N2O5"], 1)
    y, st = oracle.integrate(mine["VAR"], mine["FIX"], rc, p, 1)
    ip = np.zeros(20, dtype=np.int32)
    ip[13] = int(np.sum(st["nacc"]))
    ip[14] = int(np.sum(st["nrej"]))
    shard.reduce_counters(ip, dist)
    full = shard.gather_states(y, idx, ncell, dist)
    if rank == 0:
        np.savez(out_path, y=full, ipar=ip)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_integration_equals_one_process(tmp_path):
    import oracle
    import radm2b200
    ncell, world = 96, 2
    out = str(tmp_path / "r.npz")
    mp.start_processes(_rank_main, args=(world, _free_port(), ncell, out), nprocs=world, start_method="spawn",
                       join=True)
    got = np.load(out)
    cells = inputs.make_cells(ncell, 21, "mixed")
    ipar, rpar = radm2b200.default_params(hstart=6.0)
    ok, p = oracle.params(0.0, 600.0, np.ones(59), np.full(59, 1e-3), rpar, ipar)
    rc = oracle.rconst(cells["JV"], cells["TEMP"], cells["FIX"], cells["RC_N2O5"], 1)
    y, st = oracle.integrate(cells["VAR"], cells["FIX"], rc, p, 1)
    assert np.array_equal(got["y"], y)
    assert int(got["ipar"][13]) == int(np.sum(st["nacc"])) and int(got["ipar"][14]) == int(np.sum(st["nrej"]))


def _counter_rank(rank, world, port, out_path):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    # each rank's counters fit an int; their sum over ranks does not
    ip = np.zeros(20, dtype=np.int32)
    ip[13], ip[14], ip[16] = 1_500_000_000, 40_000_000 + rank, 2_000_000_000
    shard.reduce_counters(ip, dist)
    tot = shard.reduce_totals([1_500_000_000, 40_000_000 + rank], dist)
    if rank == 0:
        np.savez(out_path, ipar=ip, tot=np.array(tot, dtype=np.int64))
    dist.barrier()
    dist.destroy_process_group()


def test_counters_summed_over_ranks_beyond_int32(tmp_path):
    """Two ranks whose summed step counters exceed 2^31: the IPAR slots saturate at INT_MAX
    (as the library's own update does) instead of wrapping, and the 64-bit totals the
    benchmark uses come back exact."""
    out = str(tmp_path / "c.npz")
    mp.start_processes(_counter_rank, args=(2, _free_port(), out), nprocs=2, start_method="spawn", join=True)
    got = np.load(out)
    assert int(got["ipar"][13]) == 2 ** 31 - 1 and int(got["ipar"][16]) == 2 ** 31 - 1
    assert int(got["ipar"][14]) == 80_000_001
    assert list(got["tot"]) == [3_000_000_000, 80_000_001]
