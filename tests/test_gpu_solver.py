"""The fused ROS-3 solver kernel through the C ABI against the CPU oracle.

Parity bar for the plain FP64 method: max |y_gpu - y_oracle| / max(|y_oracle|, 1)
<= 1e-10 over all species and cells (1 molec/cm^3 = the solver's absolute tolerance),
with the oracle fed the GPU's rate constants so that only the integration is compared.
"""
import numpy as np
import pytest

import oracle
import radm2b200
from conftest import ATOL, RTOL, SAME_ARITH, rel_err
from radm2b200 import inputs

pytestmark = pytest.mark.gpu
PARITY = 1e-10


def run_gpu(cells, tend=600.0, hstart=6.0, max_steps=0, **opts):
    with radm2b200.Solver(**opts) as s:
        s.set_cells(cells)
        s.update_rconst()
        rc = s.get_rconst()
        ipar, rpar = radm2b200.default_params(hstart=hstart, max_steps=max_steps)
        ierr = s.rosenbrock(0.0, tend, ATOL, RTOL, rpar, ipar)
        y = s.get_state()
        st = s.cell_stats()
    return ierr, y, st, rc, ipar, rpar


def run_oracle(cells, rc, tend=600.0, hstart=6.0, rtol=RTOL, max_steps=0):
    ipar, rpar = radm2b200.default_params(hstart=hstart, max_steps=max_steps)
    ok, p = oracle.params(0.0, tend, ATOL, rtol, rpar, ipar)
    assert ok == 1
    return oracle.integrate(cells["VAR"], cells["FIX"], rc, p)


@pytest.fixture(scope="module")
def static_run(cells4k):
    return run_gpu(cells4k)


def test_plain_fp64_parity_4k(cells4k, static_run):
    ierr, y, st, rc, ipar, rpar = static_run
    assert ierr == 1
    y_o, st_o = run_oracle(cells4k, rc)
    assert (st["status"] == 1).all()
    assert np.array_equal(st["nacc"], st_o["nacc"]) and np.array_equal(st["nrej"], st_o["nrej"])
    assert rel_err(y, y_o).max() <= PARITY
    assert ipar[13] == st_o["nacc"].sum() and ipar[14] == st_o["nrej"].sum()
    assert rpar[10] == 600.0


def test_persistent_equals_static(cells4k, static_run):
    _, y_s, st_s, _, _, _ = static_run
    ierr, y_p, st_p, _, _, _ = run_gpu(cells4k, schedule=radm2b200.SCHED_PERSISTENT)
    assert ierr == 1
    assert np.array_equal(st_s["nacc"], st_p["nacc"])
    assert rel_err(y_p, y_s).max() <= SAME_ARITH


@pytest.mark.parametrize("bs", [64, 256])
def test_block_sizes(cells4k, static_run, bs):
    _, y_s, _, _, _, _ = static_run
    ierr, y, _, _, _, _ = run_gpu(cells4k, block_threads=bs, schedule=radm2b200.SCHED_PERSISTENT)
    assert ierr == 1 and rel_err(y, y_s).max() <= SAME_ARITH


def test_cell_order_does_not_change_results(cells4k):
    with radm2b200.Solver(schedule=radm2b200.SCHED_PERSISTENT) as s:
        s.set_cells(cells4k)
        ipar, rpar = radm2b200.default_params(hstart=6.0)
        assert s.rosenbrock(0.0, 600.0, ATOL, RTOL, rpar, ipar) == 1
        y1 = s.get_state()
        s.set_cells(cells4k)
        s.set_cell_order(np.random.default_rng(3).permutation(4096))
        ipar, rpar = radm2b200.default_params(hstart=6.0)
        assert s.rosenbrock(0.0, 600.0, ATOL, RTOL, rpar, ipar) == 1
        y2 = s.get_state()
    assert np.array_equal(y1, y2)


def test_split_graph_matches_loop(cells4k):
    sub = {k: v[:1024] for k, v in cells4k.items()}
    outs = []
    for use_graph in (True, False):
        with radm2b200.Solver(schedule=radm2b200.SCHED_PERSISTENT) as s:
            s.set_cells(sub)
            ipar, rpar = radm2b200.default_params()
            assert s.run_split(3, 600.0, ATOL, RTOL, rpar, ipar, use_graph=use_graph) == 1
            outs.append((s.get_state(), ipar.copy()))
            # replaying the cached graph continues from the new state
            assert s.run_split(3, 600.0, ATOL, RTOL, rpar, ipar, use_graph=use_graph) == 1
            outs.append((s.get_state(), ipar.copy()))
    assert np.array_equal(outs[0][0], outs[2][0]) and np.array_equal(outs[1][0], outs[3][0])
    assert np.array_equal(outs[1][1], outs[3][1])
    # three 600 s splits == three rosenbrock calls with Hstart = 6 s
    with radm2b200.Solver() as s:
        s.set_cells(sub)
        for _ in range(3):
            ipar, rpar = radm2b200.default_params(hstart=6.0)
            assert s.rosenbrock(0.0, 600.0, ATOL, RTOL, rpar, ipar) == 1
        assert rel_err(s.get_state(), outs[0][0]).max() <= SAME_ARITH


def test_parity_full_size_subset():
    """1,048,576-cell workload (30% night) on the GPU, every 256th cell checked against the oracle."""
    n, seed, wl, night, _ = inputs.WORKLOADS["plain-1m"]
    cells = inputs.make_cells(n, seed, wl, night)
    ierr, y, st, rc, _, _ = run_gpu(cells, schedule=radm2b200.SCHED_PERSISTENT)
    assert ierr == 1 and (st["status"] == 1).all()
    idx = np.arange(0, n, 256)
    sub = {k: cells[k][idx] for k in ("VAR", "FIX")}
    y_o, st_o = run_oracle(sub, rc[idx])
    assert rel_err(y[idx], y_o).max() <= PARITY
    assert np.array_equal(st["nacc"][idx], st_o["nacc"])


def test_step_cap_reports_minus6(cells4k):
    sub = {k: v[:256] for k, v in cells4k.items()}
    ierr, y, st, rc, ipar, rpar = run_gpu(sub, max_steps=5)
    assert ierr == -6 and (st["status"] == -6).all()
    y_o, st_o = run_oracle(sub, rc, max_steps=5)
    assert (st_o["status"] == -6).all()
    assert rel_err(y, y_o).max() <= PARITY  # both stop at the same accepted state


def test_bad_parameters_rejected_before_launch(cells4k):
    sub = {k: v[:64] for k, v in cells4k.items()}
    with radm2b200.Solver() as s:
        s.set_cells(sub)
        for field, value, code in (("i2", -1, -1), ("i3", 7, -2), ("i3", 1, -2), ("r0", -1.0, -3),
                                   ("r3", -0.5, -4)):
            ipar, rpar = radm2b200.default_params()
            (ipar if field[0] == "i" else rpar)[int(field[1:])] = value
            assert s.rosenbrock(0.0, 600.0, ATOL, RTOL, rpar, ipar) == code
        ipar, rpar = radm2b200.default_params()
        assert s.rosenbrock(0.0, 600.0, ATOL, np.full(59, 2.0), rpar, ipar) == -5
        assert np.array_equal(s.get_state(), sub["VAR"])  # nothing ran


def test_nonfinite_cell_is_isolated(cells4k):
    sub = {k: v[:128].copy() for k, v in cells4k.items()}
    sub["VAR"][5, 45] = np.nan
    ierr, y, st, _, _, _ = run_gpu(sub, max_steps=200)
    assert ierr < 0 and st["status"][5] < 0
    good = np.delete(np.arange(128), 5)
    assert (st["status"][good] == 1).all()


def test_hstart_override(cells4k):
    sub = {k: v[:512] for k, v in cells4k.items()}
    with radm2b200.Solver(schedule=radm2b200.SCHED_PERSISTENT) as s:
        s.set_cells(sub)
        ipar, rpar = radm2b200.default_params(hstart=6.0)
        s.rosenbrock(0.0, 600.0, ATOL, RTOL, rpar, ipar)
        y_def, st_def = s.get_state(), s.cell_stats()
        # invalid overrides fall back to the default start step
        s.set_cells(sub)
        s.set_cell_hstart(np.full(512, np.nan))
        ipar, rpar = radm2b200.default_params(hstart=6.0)
        s.rosenbrock(0.0, 600.0, ATOL, RTOL, rpar, ipar)
        assert np.array_equal(s.get_state(), y_def)
        # a valid override changes the first step and stays within tolerance
        s.set_cells(sub)
        s.set_cell_hstart(np.full(512, 0.5))
        ipar, rpar = radm2b200.default_params(hstart=6.0)
        assert s.rosenbrock(0.0, 600.0, ATOL, RTOL, rpar, ipar) == 1
        st = s.cell_stats()
        assert (st["hfirst"] <= 0.5).all()
        assert rel_err(s.get_state(), y_def).max() < 1e-1


def test_fp32_lu_accuracy(cells4k):
    """FP32 Jacobian/LU + one FP64 refinement sweep per stage solve.

    Gate: against the plain FP64 solver at the same rtol (1e-3), max relative error on
    species above atol <= 1e-3 (measured ~1e-10).  Reported: both against an FP64
    oracle run at rtol 1e-8; the mixed-precision solver may not be less accurate than
    the FP64 method itself (whose own error at rtol 1e-3 reaches a few 1e-2 on NO3/N2O5).
    """
    sub = {k: v[:1024] for k, v in cells4k.items()}
    ierr, y64, _, rc, _, _ = run_gpu(sub, schedule=radm2b200.SCHED_PERSISTENT)
    assert ierr == 1
    ierr, y32, st, _, _, _ = run_gpu(sub, precision=radm2b200.PREC_FP32LU, refine_sweeps=1,
                                     schedule=radm2b200.SCHED_PERSISTENT)
    assert ierr == 1
    above = np.abs(y64) > 1.0
    gate = np.abs(y32 - y64)[above] / np.abs(y64)[above]
    assert gate.max() <= 1e-3 and np.median(gate) <= 1e-12
    y_tight, _ = run_oracle(sub, rc, rtol=np.full(59, 1e-8))
    above = np.abs(y_tight) > 1.0
    e32 = np.abs(y32 - y_tight)[above] / np.abs(y_tight)[above]
    e64 = np.abs(y64 - y_tight)[above] / np.abs(y_tight)[above]
    assert e32.max() <= e64.max() * 1.01 + 1e-9


@pytest.mark.parametrize("schedule", [radm2b200.SCHED_STATIC, radm2b200.SCHED_PERSISTENT])
def test_fp32_lu_without_refinement(cells4k, schedule):
    """FP32 Jacobian/LU with no refinement sweep (refine_sweeps = 0, the kernels built
    without the refinement code).  Gate against the plain FP64 solver at the same rtol:
    max relative error on species above atol <= 1e-3; against an FP64 oracle at rtol 1e-8
    it may not be less accurate than the FP64 method by more than that margin."""
    sub = {k: v[:1024] for k, v in cells4k.items()}
    ierr, y64, _, rc, _, _ = run_gpu(sub, schedule=schedule)
    assert ierr == 1
    ierr, y32, st, _, ipar, _ = run_gpu(sub, precision=radm2b200.PREC_FP32LU, refine_sweeps=0, schedule=schedule)
    assert ierr == 1 and (st["status"] == 1).all()
    above = np.abs(y64) > 1.0
    gate = np.abs(y32 - y64)[above] / np.abs(y64)[above]
    assert gate.max() <= 1e-3
    # no refinement: the float solves leave differences well above FP64 round-off
    assert gate.max() > 1e-9
    y_tight, _ = run_oracle(sub, rc, rtol=np.full(59, 1e-8))
    above = np.abs(y_tight) > 1.0
    e32 = np.abs(y32 - y_tight)[above] / np.abs(y_tight)[above]
    e64 = np.abs(y64 - y_tight)[above] / np.abs(y_tight)[above]
    assert e32.max() <= e64.max() + 1e-3
    # one refinement sweep brings it back to FP64 round-off
    _, y32r, _, _, _, _ = run_gpu(sub, precision=radm2b200.PREC_FP32LU, refine_sweeps=1, schedule=schedule)
    g1 = np.abs(y32r - y64)[above] / np.maximum(np.abs(y64)[above], 1.0)
    assert np.median(g1) <= 1e-12


def test_kernel_timing_with_and_without_graph():
    """Solver-kernel timing works for host-driven splits and inside the split graph."""
    cells = inputs.make_cells(2048, 4, "plain", 0.3)
    for use_graph in (False, True):
        with radm2b200.Solver(schedule=radm2b200.SCHED_PERSISTENT) as s:
            s.set_cells(cells)
            s.set_kernel_timing(True)
            ipar, rpar = radm2b200.default_params()
            assert s.run_split(2, 600.0, np.ones(59), np.full(59, 1e-3), rpar, ipar, use_graph=use_graph) == 1
            ms, n = s.kernel_time()
            assert n == 2 and ms > 0.0, (use_graph, ms, n)



def test_autotune_picks_fastest_and_keeps_results():
    """The autotuner times every built variant of the context's precision on a sample of its
    cells, keeps the fastest, leaves the cells untouched, and the tuned context integrates
    to the same answer as the untuned one."""
    cells = inputs.make_cells(65536, 6, "mixed")
    atol, rtol = np.ones(59), np.full(59, 1e-3)
    with radm2b200.Solver() as s:
        s.set_cells(cells)
        ipar, rpar = radm2b200.default_params()
        assert s.run_split(1, 600.0, atol, rtol, rpar, ipar) == 1
        y_before, acc_before = s.get_state(), int(ipar[13])
        s.set_cells(cells)
        table = s.autotune(600.0, atol, rtol, sample_cells=32768)
        # 2 cooperative shapes, 2 x 2 two-cells-per-thread, 10 FP64 variants x 2 schedules, and the
        # persistent-only wide tensor-memory shape
        assert len(table) == 27
        ran = [t for t in table if t["ms"] > 0]
        assert len(ran) >= 10 and len({t["attempts"] for t in ran}) == 1
        best = min(ran, key=lambda t: t["ms"])
        o = s.opts()
        assert (o["schedule"], o["block_threads"], o["placement"], o["min_blocks"], o["cells_per_thread"]) == \
            (best["schedule"], best["block_threads"], best["placement"], best["min_blocks"], best["cells_per_thread"])
        assert np.array_equal(s.get_state(), cells["VAR"])  # the sample ran in a scratch context
        ipar, rpar = radm2b200.default_params()
        assert s.run_split(1, 600.0, atol, rtol, rpar, ipar) == 1
        assert int(ipar[13]) == acc_before
        # the tuned kernel may have another code shape (cooperative, two cells per thread):
        # differently contracted multiply-adds, amplified in this mixed batch's stiff cells
        assert rel_err(s.get_state(), y_before).max() <= 1e-10


@pytest.mark.parametrize("nchunk", [1, 5])
def test_pipelined_host_integration_matches_separate_calls(nchunk):
    """radm2_rosenbrock_host (chunked, copies overlapped with the solve) gives exactly what
    set_inputs + rosenbrock + get_state give, counters included."""
    cells = inputs.make_cells(20000, 9, "mixed")
    atol, rtol = np.ones(59), np.full(59, 1e-3)
    with radm2b200.Solver(schedule=radm2b200.SCHED_PERSISTENT) as s:
        s.set_cells(cells)
        ipar0, rpar0 = radm2b200.default_params(hstart=6.0)
        assert s.rosenbrock(0.0, 600.0, atol, rtol, rpar0, ipar0) == 1
        y0 = s.get_state()
    with radm2b200.Solver(schedule=radm2b200.SCHED_PERSISTENT) as s:
        y = np.ascontiguousarray(cells["VAR"]).copy()
        ipar, rpar = radm2b200.default_params(hstart=6.0)
        ierr = s.rosenbrock_host(y, cells["FIX"], cells["TEMP"], cells["RC_N2O5"], cells["JV"], 0.0, 600.0, atol,
                                 rtol, rpar, ipar, nchunk=nchunk)
        assert ierr == 1
    assert np.array_equal(y, y0)
    assert list(ipar[10:17]) == list(ipar0[10:17])
    assert rpar[10] == rpar0[10] and rpar[11] == rpar0[11]


@pytest.mark.parametrize("threads", [32, 256])
def test_pipelined_host_many_chunks(threads):
    """Many small chunks of stiff mixed cells (48 launches, each with its own queue counter,
    copies and transposes in flight on the copy streams): states and counters equal one
    whole-batch call bit for bit, and a second call on the same context gives the same
    again."""
    cells = inputs.make_cells(100000, 12, "mixed")
    atol, rtol = np.ones(59), np.full(59, 1e-3)
    opts = dict(schedule=radm2b200.SCHED_PERSISTENT, block_threads=threads)
    with radm2b200.Solver(**opts) as s:
        s.set_cells(cells)
        ipar0, rpar0 = radm2b200.default_params(hstart=6.0)
        assert s.rosenbrock(0.0, 600.0, atol, rtol, rpar0, ipar0) == 1
        y0 = s.get_state()
    with radm2b200.Solver(**opts) as s:
        for _ in range(2):
            y = np.ascontiguousarray(cells["VAR"]).copy()
            ipar, rpar = radm2b200.default_params(hstart=6.0)
            assert s.rosenbrock_host(y, cells["FIX"], cells["TEMP"], cells["RC_N2O5"], cells["JV"], 0.0, 600.0,
                                     atol, rtol, rpar, ipar, nchunk=48) == 1
            assert np.array_equal(y, y0)
            assert list(ipar[10:17]) == list(ipar0[10:17])


def test_pipelined_host_integration_with_seeding():
    from radm2b200 import seeding
    cells = inputs.make_cells(12000, 10, "mixed")
    net = seeding.load_net(seeding.DEFAULT_NET)
    outs = []
    for chunked in (False, True):
        with radm2b200.Solver(schedule=radm2b200.SCHED_PERSISTENT) as s:
            s.set_cells(cells)
            s.attach_mlp(net)
            ipar, rpar = radm2b200.default_params()
            if chunked:
                y = np.ascontiguousarray(cells["VAR"]).copy()
                assert s.rosenbrock_host(y, cells["FIX"], cells["TEMP"], cells["RC_N2O5"], cells["JV"], 0.0, 600.0,
                                         seeding.ATOL, seeding.RTOL, rpar, ipar, nchunk=4) == 1
            else:
                assert s.rosenbrock(0.0, 600.0, seeding.ATOL, seeding.RTOL, rpar, ipar) == 1
                y = s.get_state()
            s.attach_mlp(None)
        outs.append((y, int(ipar[13]), int(ipar[14])))
    assert outs[0][1:] == outs[1][1:]
    assert np.array_equal(outs[0][0], outs[1][0])


@pytest.mark.parametrize("n", [1, 31, 33])
def test_tiny_and_odd_batches_match_oracle(n):
    """Batches smaller than a warp or just over it (padding of the leading dimension):
    static and persistent schedules agree with each other and with the oracle."""
    cells = inputs.make_cells(n, 23, "plain", 0.3)
    atol, rtol = np.ones(59), np.full(59, 1e-3)
    ys = []
    for sched in (radm2b200.SCHED_STATIC, radm2b200.SCHED_PERSISTENT):
        with radm2b200.Solver(schedule=sched) as s:
            s.set_cells(cells)
            s.update_rconst()
            rc = s.get_rconst()
            ipar, rpar = radm2b200.default_params(hstart=6.0)
            assert s.rosenbrock(0.0, 600.0, atol, rtol, rpar, ipar) == 1
            ys.append(s.get_state())
    assert rel_err(ys[1], ys[0]).max() <= SAME_ARITH
    ipar, rpar = radm2b200.default_params(hstart=6.0)
    ok, p = oracle.params(0.0, 600.0, atol, rtol, rpar, ipar)
    y_o, _ = oracle.integrate(cells["VAR"], cells["FIX"], rc, p)
    assert rel_err(ys[0], y_o).max() <= PARITY


def _mixed_case(**opts):
    """The 4,096-cell mixed-regime batch (urban NOx, 220 K) on the GPU and the oracle, both
    fed the GPU's rate constants: per-element errors and both sets of cell statistics."""
    cells = inputs.make_cells(4096, 23, "mixed")
    atol, rtol = np.ones(59), np.full(59, 1e-3)
    with radm2b200.Solver(schedule=radm2b200.SCHED_PERSISTENT, **opts) as s:
        s.set_cells(cells)
        s.update_rconst()
        rc = s.get_rconst()
        ipar, rpar = radm2b200.default_params(hstart=6.0)
        assert s.rosenbrock(0.0, 600.0, atol, rtol, rpar, ipar) == 1
        y = s.get_state()
        st = s.cell_stats()
    ipar, rpar = radm2b200.default_params(hstart=6.0)
    ok, p = oracle.params(0.0, 600.0, atol, rtol, rpar, ipar)
    y_o, st_o = oracle.integrate(cells["VAR"], cells["FIX"], rc, p)
    return rel_err(y, y_o), st, st_o


def test_mixed_regime_parity():
    """Reference arithmetic (radm2_opts.parity: pivot divisions kept, no multiply-add
    contraction) on the mixed-regime batch: within 1e-10 of the oracle, identical step counts."""
    e, st, st_o = _mixed_case(parity=1)
    print("mixed parity (reference arithmetic): max %.2e" % e.max())
    assert np.array_equal(st["nacc"], st_o["nacc"]) and np.array_equal(st["nrej"], st_o["nrej"])
    assert e.max() <= PARITY


def test_mixed_regime_fast_solver_deviation():
    """The fast solver (reciprocal pivots, contracted multiply-adds) on the same batch: its
    deviation from the oracle is reported; step counts stay identical.  Measured 2.0e-10 on
    B200 (a few stiff cells' species near atol)."""
    e, st, st_o = _mixed_case()
    print("mixed parity (fast solver): max %.2e, cells above 1e-10: %d, above 1e-12: %d"
          % (e.max(), int((e.max(1) > 1e-10).sum()), int((e.max(1) > 1e-12).sum())))
    assert np.array_equal(st["nacc"], st_o["nacc"]) and np.array_equal(st["nrej"], st_o["nrej"])
    assert e.max() <= 1e-9


def _six_splits(parity):
    """configs[1]'s hour as 6 consecutive 600 s operator splits (Hstart 0.01 dt, the state
    carried over) on every 256th cell of the 1,048,576-cell, 30%-night workload (4,096
    cells): the GPU one split at a time, the oracle likewise, compared after every split."""
    n, seed, wl, night, _ = inputs.WORKLOADS["plain-1m"]
    idx = np.arange(0, n, 256)
    cells = inputs.make_cells(n, seed, wl, night)
    sub = {k: np.ascontiguousarray(v[idx]) for k, v in cells.items()}
    atol, rtol = np.ones(59), np.full(59, 1e-3)
    worst, per_split = 0.0, []
    with radm2b200.Solver(schedule=radm2b200.SCHED_PERSISTENT, parity=parity) as s:
        s.set_cells(sub)
        s.update_rconst()
        rc = s.get_rconst()
        ipar, rpar = radm2b200.default_params(hstart=6.0)
        ok, p = oracle.params(0.0, 600.0, atol, rtol, rpar, ipar)
        y_o = sub["VAR"]
        for k in range(6):
            ipar, rpar = radm2b200.default_params()
            assert s.run_split(1, 600.0, atol, rtol, rpar, ipar) == 1
            y, st = s.get_state(), s.cell_stats()
            y_o, st_o = oracle.integrate(y_o, sub["FIX"], rc, p)
            same_steps = np.array_equal(st["nacc"], st_o["nacc"]) and np.array_equal(st["nrej"], st_o["nrej"])
            e = rel_err(y, y_o).max()
            worst = max(worst, e)
            per_split.append((k, e, same_steps))
        y_seq = s.get_state()
    # the same hour as one 6-split graph from the initial state ends in the same state
    with radm2b200.Solver(schedule=radm2b200.SCHED_PERSISTENT, parity=parity) as s:
        s.set_cells(sub)
        ipar, rpar = radm2b200.default_params()
        assert s.run_split(6, 600.0, atol, rtol, rpar, ipar) == 1
        assert np.array_equal(s.get_state(), y_seq)
    return worst, per_split


def test_six_split_hour_parity():
    """Reference arithmetic over 6 consecutive splits: within 1e-10 of the oracle after every
    split, with identical per-cell accepted and rejected step counts in every split."""
    worst, per_split = _six_splits(1)
    print("6-split parity (reference arithmetic):", ["%d: %.2e" % (k, e) for k, e, _ in per_split])
    assert all(same for _, _, same in per_split), per_split
    assert worst <= PARITY


def test_six_split_hour_fast_solver_deviation():
    """The fast solver over the same 6 splits: its largest deviation from the oracle is
    reported (the states and the step counts are compared after every split)."""
    worst, per_split = _six_splits(0)
    print("6-split deviation (fast solver):", ["%d: %.2e steps %s" % x for x in per_split])
    assert worst <= 1e-8


def test_parity_option_validation():
    """The reference-arithmetic solver exists for FP64 with global placement only."""
    with pytest.raises(radm2b200.RadmError):
        radm2b200.Solver(parity=1, precision=radm2b200.PREC_FP32LU)
    with pytest.raises(radm2b200.RadmError):
        radm2b200.Solver(parity=1, placement=radm2b200.lib.PLACE_LU_SMEM)
    with radm2b200.Solver(parity=1) as s:
        assert s.opts()["parity"] == 1


def _parity_case(sub, tstart, tend, atol, rtol, ipar, rpar):
    """GPU (persistent schedule) and oracle on the same cells, rate constants and
    parameters; returns both results and both sets of statistics."""
    with radm2b200.Solver(schedule=radm2b200.SCHED_PERSISTENT) as s:
        s.set_cells(sub)
        s.update_rconst()
        rc = s.get_rconst()
        ip, rp = ipar.copy(), rpar.copy()
        ierr = s.rosenbrock(tstart, tend, atol, rtol, rp, ip)
        y, st = s.get_state(), s.cell_stats()
    ok, p = oracle.params(tstart, tend, atol, rtol, rpar, ipar)
    assert ok == 1
    y_o, st_o = oracle.integrate(sub["VAR"], sub["FIX"], rc, p)
    return ierr, y, st, ip, rp, y_o, st_o


def test_species_tolerances_and_control_parameters(cells4k):
    """Per-species AbsTol/RelTol (IPAR[1] = 0), every step-control parameter away from its
    default (Hmin, Hmax, Hstart, FacMin, FacMax, FacRej, FacSafe) and a window that does
    not start at 0: the same steps and states as the oracle (mgpu.cu:3734-3791)."""
    sub = {k: v[:1024] for k, v in cells4k.items()}
    rng = np.random.default_rng(11)
    atol = 10.0 ** rng.uniform(-1.0, 1.0, 59)
    rtol = 10.0 ** rng.uniform(-4.0, -2.0, 59)
    ipar, rpar = radm2b200.default_params(hstart=2.0)
    rpar[0], rpar[1], rpar[3], rpar[4], rpar[5], rpar[6] = 1e-3, 240.0, 0.3, 4.0, 0.2, 0.85
    ierr, y, st, ip, rp, y_o, st_o = _parity_case(sub, 3600.0, 4200.0, atol, rtol, ipar, rpar)
    assert ierr == 1 and (st_o["status"] == 1).all()
    assert np.array_equal(st["nacc"], st_o["nacc"]) and np.array_equal(st["nrej"], st_o["nrej"])
    assert rel_err(y, y_o).max() <= PARITY
    assert ip[13] == st_o["nacc"].sum() and ip[14] == st_o["nrej"].sum()
    assert rp[10] == 4200.0


def test_scalar_tolerances_use_first_entry(cells4k):
    """IPAR[1] != 0: AbsTol[0] and RelTol[0] apply to every species (the rest of the arrays
    is ignored), as in the oracle."""
    sub = {k: v[:512] for k, v in cells4k.items()}
    atol = np.concatenate([[0.5], np.full(58, 1e6)])
    rtol = np.concatenate([[3e-4], np.full(58, 0.5)])
    ipar, rpar = radm2b200.default_params(hstart=6.0)
    ipar[1] = 1
    ierr, y, st, _, _, y_o, st_o = _parity_case(sub, 0.0, 600.0, atol, rtol, ipar, rpar)
    assert ierr == 1
    assert np.array_equal(st["nacc"], st_o["nacc"]) and np.array_equal(st["nrej"], st_o["nrej"])
    assert rel_err(y, y_o).max() <= PARITY
    # and it equals the run with uniform arrays of those values
    ipar[1] = 0
    _, y_u, st_u, _, _, _, _ = _parity_case(sub, 0.0, 600.0, np.full(59, 0.5), np.full(59, 3e-4), ipar, rpar)
    assert np.array_equal(y, y_u) and np.array_equal(st["nacc"], st_u["nacc"])


def test_backward_window_reports_minus7_like_the_oracle(cells4k):
    """Tend < Tstart integrates backwards (direction -1, mgpu.cu:3475-3477 and the mirrored
    time-loop test).  The stiff chemistry is unstable backwards: the oracle ends every cell
    with status -7 (step size too small); the GPU must report the same per cell and IERR -7."""
    sub = {k: v[:256] for k, v in cells4k.items()}
    ipar, rpar = radm2b200.default_params(hstart=1.0)
    ierr, y, st, ip, rp, y_o, st_o = _parity_case(sub, 600.0, 540.0, ATOL, RTOL, ipar, rpar)
    assert (st_o["status"] == -7).all()
    assert ierr == -7 and np.array_equal(st["status"], st_o["status"])


@pytest.mark.parametrize("schedule", [radm2b200.SCHED_STATIC, radm2b200.SCHED_PERSISTENT])
@pytest.mark.parametrize("bs", [64, 128])
def test_two_cells_per_thread(cells4k, static_run, schedule, bs):
    """Every thread integrating two cells side by side gives the thread-per-cell results:
    the same arithmetic, the same per-cell step counts."""
    _, y_s, st_s, _, ipar_s, _ = static_run
    ierr, y, st, _, ipar, _ = run_gpu(cells4k, schedule=schedule, block_threads=bs, cells_per_thread=2)
    assert ierr == 1 and (st["status"] == 1).all()
    assert np.array_equal(st["nacc"], st_s["nacc"]) and np.array_equal(st["nrej"], st_s["nrej"])
    # the same expressions in another code shape: differently contracted multiply-adds
    assert rel_err(y, y_s).max() <= 1e-12
    assert list(ipar[10:17]) == list(ipar_s[10:17])


def test_two_cells_per_thread_odd_batch_and_options():
    cells = inputs.make_cells(301, 17, "mixed")
    _, y0, st0, _, _, _ = run_gpu(cells)
    ierr, y, st, _, _, _ = run_gpu(cells, schedule=radm2b200.SCHED_PERSISTENT, cells_per_thread=2)
    # a mixed batch: its stiff cells amplify the rounding-level differences
    assert ierr == 1 and np.array_equal(st["nacc"], st0["nacc"]) and rel_err(y, y0).max() <= 1e-10
    for bad in ({"precision": radm2b200.PREC_FP32LU}, {"schedule": radm2b200.SCHED_COOP}, {"parity": 1},
                {"cells_per_thread": 3}):
        with pytest.raises(radm2b200.RadmError):
            radm2b200.Solver(**dict({"cells_per_thread": 2}, **bad))
