"""Learned step seeding: traces from the solver, training on the GPU, use.

The network (radm2_mlp_* in the C ABI) maps each cell's state features to two
standardised targets: log10 of a good starting step h0 and log10(accepted steps + 1).
Labels come from the plain FP64 solver itself: for every cell and operator split, the
first accepted step size (the h0 that would have avoided the initial rejections) and the
number of accepted steps of that split.  At use, the predictions seed per-cell starting
steps (the Rosenbrock error controller still judges every step; invalid predictions fall
back to the default Hstart) and, optionally, order cells by descending predicted cost
for the persistent schedule.  Attached to a solver (Solver.attach_mlp), the seeding
kernels run in front of every split inside the split loop's CUDA graph.
"""
import os

import numpy as np

from . import inputs
from .lib import PREC_FP64, SCHED_PERSISTENT, Mlp, Solver, default_params

ATOL = np.ones(59)
RTOL = np.full(59, 1.0e-3)


def generate_traces(ncell, nsplit, seed, dt=600.0, workload="mixed", night_frac=0.4, probe_h0=None):
    """(X, Y): features of the state before each split and its (h0, accepted) labels.

    The h0 label is the first accepted step of a split started from probe_h0 (default:
    the whole split, dt): the largest first step the error controller accepts from that
    state, after its own rejections shrink the trial step."""
    cells = inputs.make_cells(ncell, seed, workload, night_frac)
    xs, ys = [], []
    probe = dt if probe_h0 is None else probe_h0
    with Solver(precision=PREC_FP64, schedule=SCHED_PERSISTENT) as s:
        s.set_cells(cells)
        for _ in range(nsplit):
            x = s.features(dt)
            ipar, rpar = default_params(hstart=probe)
            ierr = s.run_split(1, dt, ATOL, RTOL, rpar, ipar, use_graph=False)
            if ierr != 1:
                raise RuntimeError("trace generation: IERR %d" % ierr)
            st = s.cell_stats()
            ok = (st["status"] == 1) & (st["hfirst"] > 0)
            y = np.stack([np.log10(np.where(ok, st["hfirst"], 1.0)), np.log10(st["nacc"] + 1.0)], axis=1)
            xs.append(x[ok])
            ys.append(y[ok].astype(np.float32))
    return np.concatenate(xs), np.concatenate(ys)


def normalisation(X, Y):
    xm, xs = X.mean(0), X.std(0)
    xs = np.where(xs > 1e-6, xs, 1.0)
    ym, ys = Y.mean(0), Y.std(0)
    return xm.astype(np.float32), xs.astype(np.float32), ym.astype(np.float32), ys.astype(np.float32)


def fit(X, Y, epochs=6, batch=4096, lr=2e-3, seed=0, device=0, log=None):
    """Train a fresh network on the GPU (own forward/backward/Adam kernels).  Returns it."""
    import torch  # device buffers for the training set (plumbing)
    xm, xs, ym, ys = normalisation(X, Y)
    net = Mlp(seed=seed, device=device)
    net.set_norm(xm, xs, ym, ys)
    Yn = ((Y - ym) / ys).astype(np.float32)
    dev = torch.device("cuda", device)
    xt = torch.from_numpy(np.ascontiguousarray(X, dtype=np.float32)).to(dev)
    yt = torch.from_numpy(np.ascontiguousarray(Yn)).to(dev)
    n = X.shape[0]
    g = torch.Generator(device="cpu").manual_seed(seed)
    history = []
    step = 0
    nsteps = epochs * (n // batch)
    for ep in range(epochs):
        perm = torch.randperm(n, generator=g).to(dev)
        xe, ye = xt[perm].contiguous(), yt[perm].contiguous()
        torch.cuda.synchronize(dev)
        last = None
        for b in range(n // batch):
            # cosine decay of the learning rate
            lr_t = lr * 0.5 * (1.0 + np.cos(np.pi * step / max(nsteps, 1)))
            want = b == (n // batch) - 1
            lo = b * batch
            l = net.train_step(batch, xe.data_ptr() + lo * 84 * 4, ye.data_ptr() + lo * 2 * 4, lr_t, want_loss=want)
            if want:
                last = l
            step += 1
        history.append(last)
        if log:
            log("epoch %d loss %.4f" % (ep, last))
    net.synchronize()
    return net, history


# The training recipe: traces of 262,144 cells x 8 splits (2.1 M state/label pairs) of the
# mixed-regime distribution under a seed disjoint from every evaluation batch, labels from
# splits started at h0 = dt, 6 epochs; seeded steps are half the predicted step.
TRAIN_CELLS, TRAIN_SPLITS, TRAIN_SEED, TRAIN_EPOCHS, H0_SAFETY = 262144, 8, 100, 6, 0.5


def train_default(device=0, dt=600.0, log=None):
    """Generate traces with the solver and train the seeding network on the GPU.
    Returns (net, info) with the pair count and the final training loss."""
    X, Y = generate_traces(TRAIN_CELLS, TRAIN_SPLITS, TRAIN_SEED, dt=dt, workload="mixed")
    net, hist = fit(X, Y, epochs=TRAIN_EPOCHS, seed=0, device=device, log=log)
    net.set_h0_scale(H0_SAFETY)
    return net, {"pairs": int(X.shape[0]), "loss": float(hist[-1]), "epochs": TRAIN_EPOCHS,
                 "trace_cells": TRAIN_CELLS, "trace_splits": TRAIN_SPLITS, "trace_seed": TRAIN_SEED,
                 "h0_safety": H0_SAFETY}


# A network trained by train_default (regenerate: python bench.py --save-weights PATH, or
# save_net(train_default()[0], PATH)), shipped for seeding without training first.
DEFAULT_NET = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "seed_net_mixed.npz")


def save_net(net, path, h0_scale=H0_SAFETY):
    """Store a trained network (parameters, normalisation, seeding scale) as .npz."""
    xm, xs, ym, ys = net.norm
    np.savez(path, params=net.params(), xmean=xm, xstd=xs, ymean=ym, ystd=ys, h0_scale=np.float32(h0_scale))


def load_net(path, device=0):
    """A network stored by save_net, ready to seed."""
    d = np.load(path)
    net = Mlp(seed=0, device=device)
    net.set_params(d["params"])
    net.set_norm(d["xmean"], d["xstd"], d["ymean"], d["ystd"])
    net.set_h0_scale(float(d["h0_scale"]))
    return net


def evaluate_split_loop(cells, nsplit, dt=600.0, net=None, precision=PREC_FP64, schedule=SCHED_PERSISTENT,
                        use_h0=True, use_order=True, timer=None, safety=None, carry=False, attach=False):
    """Integrate nsplit consecutive splits; with a network, seed every split from it
    (h0 = safety * predicted step) -- host-driven per split, or with attach=True inside one
    CUDA graph of all nsplit splits; with carry, start each split from the step size the
    previous split ended with.  Returns (final state, totals, seconds, solver-kernel ms)."""
    tot = {"acc": 0, "rej": 0}
    with Solver(precision=precision, schedule=schedule) as s:
        s.set_cells(cells)
        s.update_rconst()
        s.set_kernel_timing(True)
        s.synchronize()
        if net is not None and safety is not None:
            net.set_h0_scale(safety)
        if attach and net is not None:
            s.attach_mlp(net, order=use_order and schedule == SCHED_PERSISTENT)
            ipar, rpar = default_params()
            t0 = timer() if timer else None
            ierr = s.run_split(nsplit, dt, ATOL, RTOL, rpar, ipar, use_graph=True)
            if ierr != 1:
                raise RuntimeError("IERR %d" % ierr)
            tot["acc"] += int(ipar[13])
            tot["rej"] += int(ipar[14])
            s.synchronize()
            el = (timer() - t0) if timer else None
            kms, _ = s.kernel_time()
            y = s.get_state()
            s.attach_mlp(None)
            return y, tot, el, kms
        t0 = timer() if timer else None
        for k in range(nsplit):
            if net is not None:
                s.seed_cells(net, dt, h0=use_h0, order=use_order and schedule == SCHED_PERSISTENT)
            elif carry and k > 0:
                s.set_cell_hstart(s.cell_stats()["hexit"])
            ipar, rpar = default_params()
            ierr = s.run_split(1, dt, ATOL, RTOL, rpar, ipar, use_graph=True)
            if ierr != 1:
                raise RuntimeError("IERR %d" % ierr)
            tot["acc"] += int(ipar[13])
            tot["rej"] += int(ipar[14])
        s.synchronize()
        el = (timer() - t0) if timer else None
        kms, _ = s.kernel_time()
        y = s.get_state()
    return y, tot, el, kms
