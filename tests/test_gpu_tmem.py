"""Tensor-memory LU slots: the thread-per-cell solver with its 128 most used LU slots in tensor
memory (RADM2_PLACE_LU_TMEM), or with its 256 most used slots in tensor memory and its rate
constants and state in shared memory, one 128-thread CTA per SM (RADM2_PLACE_LU_TMEM_WIDE).

The arithmetic is that of the global-scratch kernel of the same block size and schedule, so
both must take identical steps and agree to rounding (SAME_ARITH).  Lanes without an attempt
(finished, failed or never given a cell) run the warp-collective phases alongside the others:
ragged batches, the step cap and a non-finite cell check that they neither disturb their
neighbours nor are disturbed.
"""
import numpy as np
import pytest

import oracle
import radm2b200
from conftest import ATOL, RTOL, SAME_ARITH, rel_err
from radm2b200 import inputs

pytestmark = pytest.mark.gpu
TMEM = radm2b200.lib.PLACE_LU_TMEM
WIDE = radm2b200.lib.PLACE_LU_TMEM_WIDE
PERS = radm2b200.SCHED_PERSISTENT
PARITY = 1e-10
# (placement, schedules it is built for)
PLACES = [(TMEM, (radm2b200.SCHED_STATIC, PERS)), (WIDE, (PERS,))]


def run(cells, hstart=6.0, max_steps=0, **opts):
    with radm2b200.Solver(**opts) as s:
        s.set_cells(cells)
        s.update_rconst()
        rc = s.get_rconst()
        ipar, rpar = radm2b200.default_params(hstart=hstart, max_steps=max_steps)
        ierr = s.rosenbrock(0.0, 600.0, ATOL, RTOL, rpar, ipar)
        return ierr, s.get_state(), s.cell_stats(), rc, ipar


@pytest.fixture(scope="module")
def mixed4k():
    return inputs.make_cells(4096, 23, "mixed")


@pytest.mark.parametrize("schedule", [radm2b200.SCHED_STATIC, radm2b200.SCHED_PERSISTENT])
@pytest.mark.parametrize("bs", [128, 256])
def test_tmem_equals_global_scratch(mixed4k, schedule, bs):
    ierr0, y0, st0, _, ipar0 = run(mixed4k, schedule=schedule, block_threads=bs)
    ierr, y, st, _, ipar = run(mixed4k, schedule=schedule, block_threads=bs, placement=TMEM)
    assert ierr == ierr0 == 1
    assert np.array_equal(st["nacc"], st0["nacc"]) and np.array_equal(st["nrej"], st0["nrej"])
    assert (st["status"] == 1).all()
    e = rel_err(y, y0).max()
    print("tensor-memory LU slots vs global scratch (bs %d, schedule %d): max %.2e" % (bs, schedule, e))
    assert e <= SAME_ARITH
    assert list(ipar[10:17]) == list(ipar0[10:17])


def test_tmem_wide_equals_global_scratch(mixed4k):
    """The 256-slot map with rate constants and state in shared memory: the same arithmetic
    as the global-scratch kernel of the same shape, identical steps."""
    ierr0, y0, st0, _, ipar0 = run(mixed4k, schedule=PERS, block_threads=128)
    ierr, y, st, _, ipar = run(mixed4k, schedule=PERS, placement=WIDE)
    assert ierr == ierr0 == 1
    assert np.array_equal(st["nacc"], st0["nacc"]) and np.array_equal(st["nrej"], st0["nrej"])
    assert (st["status"] == 1).all()
    e = rel_err(y, y0).max()
    print("wide tensor-memory map vs global scratch: max %.2e" % e)
    assert e <= SAME_ARITH
    assert list(ipar[10:17]) == list(ipar0[10:17])


@pytest.mark.parametrize("place,schedules", PLACES)
@pytest.mark.parametrize("n", [1, 31, 33, 100, 300])
def test_tmem_ragged_batches_match_oracle(n, place, schedules):
    """Warps with idle lanes (fewer cells than lanes, ragged last warps): within the fast
    solver's bar of the oracle, identical step counts."""
    cells = inputs.make_cells(n, 29, "plain", 0.3)
    for schedule in schedules:
        ierr, y, st, rc, _ = run(cells, schedule=schedule, placement=place)
        assert ierr == 1 and (st["status"] == 1).all()
        ipar, rpar = radm2b200.default_params(hstart=6.0)
        ok, p = oracle.params(0.0, 600.0, ATOL, RTOL, rpar, ipar)
        y_o, st_o = oracle.integrate(cells["VAR"], cells["FIX"], rc, p)
        assert np.array_equal(st["nacc"], st_o["nacc"])
        assert rel_err(y, y_o).max() <= PARITY


@pytest.mark.parametrize("place", [TMEM, WIDE])
def test_tmem_step_cap_and_nonfinite_cell(place):
    """Lanes that stop (step cap, a non-finite cell) keep running the collective phases on
    their own scratch; the other cells finish exactly as on the global-scratch kernel."""
    cells = inputs.make_cells(512, 0, "plain")
    ierr, y, st, _, _ = run(cells, max_steps=5, schedule=radm2b200.SCHED_PERSISTENT, placement=place)
    assert ierr == -6 and (st["status"] == -6).all()
    _, y0, _, _, _ = run(cells, max_steps=5, schedule=radm2b200.SCHED_PERSISTENT, block_threads=128)
    assert rel_err(y, y0).max() <= SAME_ARITH
    sub = {k: v[:256].copy() for k, v in cells.items()}
    sub["VAR"][5, 45] = np.nan
    sub["VAR"][200, 3] = np.inf
    ierr, y, st, _, _ = run(sub, max_steps=300, schedule=radm2b200.SCHED_PERSISTENT, placement=place)
    _, y0, st0, _, _ = run(sub, max_steps=300, schedule=radm2b200.SCHED_PERSISTENT, block_threads=128)
    # each cell ends as on the global-scratch kernel (the NaN cell fails; an infinite
    # background species need not)
    assert ierr < 0 and st["status"][5] < 0
    assert np.array_equal(st["status"], st0["status"])
    good = np.flatnonzero(st0["status"] == 1)
    assert len(good) >= 254
    assert np.array_equal(st["nacc"][good], st0["nacc"][good])
    fin = np.isfinite(y0[good]).all(axis=1)
    assert np.array_equal(y[good][~fin], y0[good][~fin], equal_nan=True)
    assert rel_err(y[good][fin], y0[good][fin]).max() <= SAME_ARITH


def test_tmem_split_graph_and_host_pipeline():
    """The split graph and the chunked host-buffer call on the tensor-memory kernel give
    the same states as on the global-scratch kernel."""
    cells = inputs.make_cells(20000, 9, "mixed")
    outs = []
    for place in (radm2b200.lib.PLACE_GLOBAL, TMEM, WIDE):
        with radm2b200.Solver(schedule=radm2b200.SCHED_PERSISTENT, block_threads=128, placement=place) as s:
            s.set_cells(cells)
            ipar, rpar = radm2b200.default_params()
            assert s.run_split(2, 600.0, ATOL, RTOL, rpar, ipar) == 1
            y_graph = s.get_state()
            y = np.ascontiguousarray(cells["VAR"]).copy()
            ipar, rpar = radm2b200.default_params(hstart=6.0)
            assert s.rosenbrock_host(y, cells["FIX"], cells["TEMP"], cells["RC_N2O5"], cells["JV"], 0.0, 600.0,
                                     ATOL, RTOL, rpar, ipar, nchunk=5) == 1
        outs.append((y_graph, y))
    # the stiffest cells of this mixed batch amplify the two builds' rounding-level
    # differences (multiply-adds contracted differently): measured 1.1e-13 over two splits
    # and 1.5e-13 for the host call
    for out in outs[1:]:
        assert rel_err(out[0], outs[0][0]).max() <= 1e-12
        assert rel_err(out[1], outs[0][1]).max() <= 1e-12


@pytest.mark.parametrize("place,bs", [(TMEM, 256), (WIDE, 128)])
def test_tmem_reference_arithmetic(mixed4k, place, bs):
    """Reference arithmetic (radm2_opts.parity: pivot divisions, no multiply-add contraction)
    with tensor-memory slots (128 per thread, or 256 with the rate constants and state in
    shared memory): the division-form fragments give the global-scratch parity kernel's
    results bit for bit, and the oracle's within 1e-10 with identical step counts."""
    opts = dict(schedule=radm2b200.SCHED_PERSISTENT, block_threads=bs, parity=1)
    ierr0, y0, st0, rc, _ = run(mixed4k, **opts)
    ierr, y, st, _, _ = run(mixed4k, placement=place, **opts)
    assert ierr == ierr0 == 1
    assert np.array_equal(y, y0) and np.array_equal(st["nacc"], st0["nacc"])
    ipar, rpar = radm2b200.default_params(hstart=6.0)
    ok, p = oracle.params(0.0, 600.0, ATOL, RTOL, rpar, ipar)
    y_o, st_o = oracle.integrate(mixed4k["VAR"], mixed4k["FIX"], rc, p)
    assert np.array_equal(st["nacc"], st_o["nacc"]) and np.array_equal(st["nrej"], st_o["nrej"])
    e = rel_err(y, y_o).max()
    print("reference arithmetic, tensor-memory LU slots (placement %d), vs oracle: max %.2e" % (place, e))
    assert e <= PARITY


def test_tmem_options():
    """Tensor-memory slots exist for the FP64 solvers with 128 or 256 threads per block (256
    for reference arithmetic)."""
    for bad in ({"precision": radm2b200.PREC_FP32LU}, {"schedule": radm2b200.SCHED_COOP},
                {"cells_per_thread": 2}):
        with pytest.raises(radm2b200.RadmError):
            radm2b200.Solver(**dict({"placement": TMEM}, **bad))
    cells = inputs.make_cells(64, 1, "plain")
    for shape in ({"block_threads": 64}, {"block_threads": 128, "parity": 1}):  # not built
        with radm2b200.Solver(placement=TMEM, **shape) as s:
            s.set_cells(cells)
            ipar, rpar = radm2b200.default_params()
            assert s.rosenbrock(0.0, 600.0, ATOL, RTOL, rpar, ipar) == radm2b200.lib.RADM2_E_ARG
    with radm2b200.Solver(placement=TMEM) as s:
        assert s.opts()["block_threads"] in (0, 128) and s.opts()["placement"] == TMEM
    # the wide map: FP64, persistent, 128 threads per block
    for bad in ({"precision": radm2b200.PREC_FP32LU}, {"schedule": radm2b200.SCHED_STATIC},
                {"schedule": radm2b200.SCHED_COOP}, {"cells_per_thread": 2}):
        with pytest.raises(radm2b200.RadmError):
            radm2b200.Solver(**dict({"placement": WIDE, "schedule": PERS}, **bad))
    with radm2b200.Solver(placement=WIDE, schedule=PERS, block_threads=256) as s:  # not built
        s.set_cells(cells)
        ipar, rpar = radm2b200.default_params()
        assert s.rosenbrock(0.0, 600.0, ATOL, RTOL, rpar, ipar) == radm2b200.lib.RADM2_E_ARG
