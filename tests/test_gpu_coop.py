"""The cooperative solver kernel (RADM2_SCHED_COOP): 32 cells per block with the LU, state
and stage vectors on chip, every phase of a step attempt split between the block's warps.

Its fast form (reciprocal pivots, contracted multiply-adds) must integrate every cell like
the thread-per-cell fast solver: identical per-cell step counts and states within 1e-10
relative (rounding-level differences of differently contracted multiply-adds, amplified in
the mixed batch's stiff cells).  Its reference-arithmetic form (radm2_opts.parity) must meet the oracle's 1e-10
bar with identical step counts, as the thread-per-cell reference-arithmetic solver does.
"""
import numpy as np
import pytest

import oracle
import radm2b200
from conftest import ATOL, RTOL, rel_err
from radm2b200 import inputs

pytestmark = pytest.mark.gpu
PARITY = 1e-10
COOP = radm2b200.SCHED_COOP


def run(cells, hstart=6.0, max_steps=0, tend=600.0, **opts):
    with radm2b200.Solver(**opts) as s:
        s.set_cells(cells)
        s.update_rconst()
        rc = s.get_rconst()
        ipar, rpar = radm2b200.default_params(hstart=hstart, max_steps=max_steps)
        ierr = s.rosenbrock(0.0, tend, ATOL, RTOL, rpar, ipar)
        return ierr, s.get_state(), s.cell_stats(), rc, ipar, rpar


def oracle_run(cells, rc, hstart=6.0, max_steps=0):
    ipar, rpar = radm2b200.default_params(hstart=hstart, max_steps=max_steps)
    ok, p = oracle.params(0.0, 600.0, ATOL, RTOL, rpar, ipar)
    assert ok == 1
    return oracle.integrate(cells["VAR"], cells["FIX"], rc, p)


@pytest.fixture(scope="module")
def mixed4k():
    return inputs.make_cells(4096, 23, "mixed")


@pytest.fixture(scope="module")
def fast_ref(mixed4k):
    return run(mixed4k, schedule=radm2b200.SCHED_PERSISTENT)


@pytest.mark.parametrize("threads", [128, 256])
def test_coop_matches_thread_per_cell_solver(mixed4k, fast_ref, threads):
    ierr0, y0, st0, _, ipar0, rpar0 = fast_ref
    ierr, y, st, _, ipar, rpar = run(mixed4k, schedule=COOP, block_threads=threads)
    assert ierr == ierr0 == 1
    assert np.array_equal(st["nacc"], st0["nacc"]) and np.array_equal(st["nrej"], st0["nrej"])
    assert (st["status"] == 1).all()
    e = rel_err(y, y0).max()
    print("coop %d threads vs thread-per-cell: max %.2e" % (threads, e))
    # the same expressions contracted differently by the compiler (measured 1.1e-11 on this
    # mixed batch, whose stiff cells amplify rounding differences)
    assert e <= 1e-10
    assert list(ipar[10:17]) == list(ipar0[10:17]) and rpar[10] == rpar0[10] == 600.0


def test_coop_reference_arithmetic_parity(mixed4k):
    """Reference arithmetic on the mixed-regime batch against the oracle: 1e-10, identical
    step counts."""
    ierr, y, st, rc, _, _ = run(mixed4k, schedule=COOP, parity=1)
    assert ierr == 1
    y_o, st_o = oracle_run(mixed4k, rc)
    assert np.array_equal(st["nacc"], st_o["nacc"]) and np.array_equal(st["nrej"], st_o["nrej"])
    e = rel_err(y, y_o).max()
    print("coop reference arithmetic vs oracle: max %.2e" % e)
    assert e <= PARITY


def test_coop_six_split_hour_parity():
    """configs[1]'s hour (6 consecutive 600 s splits, Hstart 0.01 dt) on every 256th cell of
    the 1,048,576-cell workload, reference arithmetic, one CUDA graph; the oracle split by
    split: 1e-10 and identical step counts of the last split."""
    n, seed, wl, night, _ = inputs.WORKLOADS["plain-1m"]
    idx = np.arange(0, n, 256)
    cells = inputs.make_cells(n, seed, wl, night)
    sub = {k: np.ascontiguousarray(v[idx]) for k, v in cells.items()}
    atol, rtol = np.ones(59), np.full(59, 1e-3)
    with radm2b200.Solver(schedule=COOP, parity=1) as s:
        s.set_cells(sub)
        s.update_rconst()
        rc = s.get_rconst()
        ipar, rpar = radm2b200.default_params()
        assert s.run_split(6, 600.0, atol, rtol, rpar, ipar) == 1
        y, st = s.get_state(), s.cell_stats()
    ipar, rpar = radm2b200.default_params(hstart=6.0)
    ok, p = oracle.params(0.0, 600.0, atol, rtol, rpar, ipar)
    y_o = sub["VAR"]
    for _ in range(6):
        y_o, st_o = oracle.integrate(y_o, sub["FIX"], rc, p)
    assert np.array_equal(st["nacc"], st_o["nacc"]) and np.array_equal(st["nrej"], st_o["nrej"])
    e = rel_err(y, y_o).max()
    print("coop 6-split parity: max %.2e" % e)
    assert e <= PARITY


@pytest.mark.parametrize("n", [1, 31, 33, 100])
def test_coop_tiny_and_odd_batches(n):
    """Fewer cells than a block's 32 lanes, or a ragged last block: empty lanes idle."""
    cells = inputs.make_cells(n, 29, "plain", 0.3)
    ierr, y, st, rc, _, _ = run(cells, schedule=COOP, parity=1)
    assert ierr == 1 and (st["status"] == 1).all()
    y_o, st_o = oracle_run(cells, rc)
    assert np.array_equal(st["nacc"], st_o["nacc"])
    assert rel_err(y, y_o).max() <= PARITY


def test_coop_step_cap_and_nonfinite_cell():
    cells = inputs.make_cells(256, 0, "plain")
    ierr, y, st, rc, _, _ = run(cells, max_steps=5, schedule=COOP, parity=1)
    assert ierr == -6 and (st["status"] == -6).all()
    y_o, st_o = oracle_run(cells, rc, max_steps=5)
    assert (st_o["status"] == -6).all() and rel_err(y, y_o).max() <= PARITY
    sub = {k: v[:128].copy() for k, v in cells.items()}
    sub["VAR"][5, 45] = np.nan
    ierr, y, st, _, _, _ = run(sub, max_steps=200, schedule=COOP)
    assert ierr < 0 and st["status"][5] < 0
    good = np.delete(np.arange(128), 5)
    assert (st["status"][good] == 1).all()


def test_coop_wait_limit_selftest_then_normal_run():
    """A warp of every block waits on a flag that nothing sets: the bounded wait runs out,
    the launch ends with RADM2_E_CUDA, the states are untouched, and the same context then
    integrates normally."""
    cells = inputs.make_cells(2048, 3, "plain", 0.3)
    with radm2b200.Solver(schedule=COOP) as s:
        s.set_cells(cells)
        s.coop_selftest_wait_limit()
        assert np.array_equal(s.get_state(), cells["VAR"])
        ipar, rpar = radm2b200.default_params(hstart=6.0)
        assert s.rosenbrock(0.0, 600.0, ATOL, RTOL, rpar, ipar) == 1
        y = s.get_state()
    _, y0, _, _, _, _ = run(cells, schedule=radm2b200.SCHED_PERSISTENT)
    assert rel_err(y, y0).max() <= 1e-10


def test_coop_with_seeding_in_graph_and_host_path():
    """The learned seeding attached to a cooperative context (inside the split graph), and
    the pipelined host-buffer call on the cooperative kernel, match the persistent kernel."""
    from radm2b200 import seeding
    cells = inputs.make_cells(12000, 10, "mixed")
    net = seeding.load_net(seeding.DEFAULT_NET)
    outs = []
    for sched in (radm2b200.SCHED_PERSISTENT, COOP):
        with radm2b200.Solver(schedule=sched) as s:
            s.set_cells(cells)
            s.attach_mlp(net)
            ipar, rpar = radm2b200.default_params()
            assert s.run_split(2, 600.0, ATOL, RTOL, rpar, ipar) == 1
            y_graph, acc = s.get_state(), int(ipar[13])
            y = np.ascontiguousarray(cells["VAR"]).copy()
            ipar, rpar = radm2b200.default_params()
            assert s.rosenbrock_host(y, cells["FIX"], cells["TEMP"], cells["RC_N2O5"], cells["JV"], 0.0, 600.0,
                                     ATOL, RTOL, rpar, ipar, nchunk=3) == 1
            s.attach_mlp(None)
        outs.append((y_graph, acc, y))
    assert outs[0][1] == outs[1][1]
    assert rel_err(outs[1][0], outs[0][0]).max() <= 1e-10
    assert rel_err(outs[1][2], outs[0][2]).max() <= 1e-10


def test_coop_options_validation():
    for bad in ({"precision": radm2b200.PREC_FP32LU}, {"placement": radm2b200.lib.PLACE_LU_SMEM},
                {"min_blocks": 3}):
        with pytest.raises(radm2b200.RadmError):
            radm2b200.Solver(schedule=COOP, **bad)
    with radm2b200.Solver(schedule=COOP, block_threads=64) as s:  # not a built shape
        s.set_cells(inputs.make_cells(64, 0, "plain"))
        ipar, rpar = radm2b200.default_params()
        assert s.rosenbrock(0.0, 600.0, ATOL, RTOL, rpar, ipar) == radm2b200.lib.RADM2_E_ARG
