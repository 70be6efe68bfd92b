"""Learned two-level preconditioner: training data, training, evaluation and
weight files around the C ABI (pg_net / pg_learned, include/plategpu.h).

The reference solves with block-Jacobi PCG only; its preconditioner apply
(src/lib/plate/gpu/shaders/index.ts:214-262, once per iteration of
runGPUPCG, src/lib/plate/gpu/solver.ts:190-553) is where this library's
flexible PCG adds the network's coarse correction.  The network is trained
on residual/error pairs that the plain solver produces for seeded
random-field loads of the plate (pairs (F, x*) and (F - K x_k, x* - x_k)
with x_k an early iterate of plain block-Jacobi PCG); everything here runs
on the GPU through the library (torch provides the device buffers).

Command line (trains the plate_q4_141 network and writes its weight file):
    python -m plategpu.learned train --out <file.npz> [--loads 8192] [--epochs 40]
Timing (and profiling) entry points:
    python -m plategpu.learned forward --batch 32     the network's forward pass
    python -m plategpu.learned solve --count 4        learned solves of plate_q4_141
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import _lib, workloads

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS_DIR = os.path.join(HERE, "weights")
DEFAULT_WEIGHTS = os.path.join(WEIGHTS_DIR, "unet_plate_q4_141.npz")
TRAIN_SEED = 1000        # training loads: random_field_loads(wl, count, TRAIN_SEED)
HELD_OUT_SEED = 2000     # held-out evaluation loads


# the network's layers as the library builds them (csrc/learned.cu):
# (name, input channels, output channels, pyramid level); input and output
# layers have 3 channels, stored padded to 16
LAYERS = (("e0a", 3, 16, 0), ("e0b", 16, 16, 0), ("e1a", 16, 32, 1), ("e1b", 32, 32, 1),
          ("e2a", 32, 64, 2), ("e2b", 64, 64, 2), ("e3a", 64, 128, 3), ("e3b", 128, 128, 3),
          ("d2a", 192, 64, 2), ("d2b", 64, 64, 2), ("d1a", 96, 32, 1), ("d1b", 32, 32, 1),
          ("d0a", 48, 16, 0), ("d0b", 16, 16, 0), ("out", 16, 3, 0))


def flops_per_image(height, width):
    """Tensor-core FLOPs of one forward pass (2 x 9 x cin x cout per pixel of
    each convolution, with the channels as stored, i.e. padded to 16)."""
    tot = 0
    for _n, ci, co, lv in LAYERS:
        pci, pco = (ci + 15) // 16 * 16, (co + 15) // 16 * 16
        tot += 2 * 9 * pci * pco * (height >> lv) * (width >> lv)
    return tot


def net_grid(mesh):
    """(height, width) of the network grid for a mesh on a regular node
    grid: the node rows / columns plus at least one pixel of zero border on
    each side, rounded up to multiples of 8 (142 x 142 nodes -> 144 x 144)."""
    xy = mesh.nodes.reshape(-1, 2).astype(np.float64)
    nx = len(np.unique(np.round(xy[:, 0], 5)))
    ny = len(np.unique(np.round(xy[:, 1], 5)))
    return (ny + 2 + 7) // 8 * 8, (nx + 2 + 7) // 8 * 8


def grid_node_pixel(mesh, height, width):
    """node -> pixel (y * width + x) for a mesh whose nodes sit on a regular
    grid, centred in a height x width image."""
    xy = mesh.nodes.reshape(-1, 2).astype(np.float64)
    xs = np.unique(np.round(xy[:, 0], 5))
    ys = np.unique(np.round(xy[:, 1], 5))
    if len(xs) * len(ys) != mesh.nodeCount:
        raise ValueError("the mesh's nodes are not on a regular grid")
    if len(xs) > width or len(ys) > height:
        raise ValueError("the node grid does not fit the network grid")
    ix = np.searchsorted(xs, np.round(xy[:, 0], 5))
    iy = np.searchsorted(ys, np.round(xy[:, 1], 5))
    ox, oy = (width - len(xs)) // 2, (height - len(ys)) // 2
    return ((iy + oy) * width + ix + ox).astype(np.int32)


def solve_options(tolerance=1e-6, max_iterations=5000):
    """Options of the learned flexible PCG: relative stop on the FP64 true
    residual."""
    return _lib.make_options(tolerance=tolerance, max_iterations=max_iterations,
                             stop_rule=_lib.PG_STOP_RELATIVE)


class LearnedSolver:
    """The plan, the network and the learned solver of one structured plate."""

    def __init__(self, ctx: _lib.Context, wl: workloads.Workload, seed: int = 1, weights=None):
        self.ctx, self.wl = ctx, wl
        self.prob = _lib.Problem(wl.mesh, wl.material, wl.coloring, wl.F, wl.cons_mask)
        self.plan = ctx.plan(self.prob, _lib.make_options())
        H, W = net_grid(wl.mesh)
        self.net = _lib.Net(ctx, H, W, seed=seed)
        if weights is not None:
            load_weights(self.net, weights)
        self.node_pixel = grid_node_pixel(wl.mesh, H, W)
        self.learned = _lib.Learned(self.plan, self.net, self.node_pixel)

    def close(self):
        for o in (self.learned, self.net, self.plan):
            o.close()


def save_weights(net: _lib.Net, path, meta=None):
    p, s = net.get_params()
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    np.savez_compressed(path, params=p, scales=s, height=net.height, width=net.width,
                        meta=json.dumps(meta or {}))


def load_weights(net: _lib.Net, path):
    d = np.load(path)
    if int(d["height"]) != net.height or int(d["width"]) != net.width:
        raise ValueError(f"{path}: grid {int(d['height'])}x{int(d['width'])}, network "
                         f"{net.height}x{net.width}")
    net.set_params(d["params"], d["scales"])
    return json.loads(str(d["meta"])) if "meta" in d.files else {}


def generate_pairs(torch, ctx, ls: LearnedSolver, loads, k_max=300, seed=0, x_tol=1e-9):
    """Residual/error pairs on the device for `loads` [count, n] (float32):
    x* by the fast plain solver (mixed-precision two-level Chebyshev PCG to
    ||r||/||b|| < x_tol), x_k by k steps of plain FP64 block-Jacobi PCG with
    k uniform in [0, k_max] (k = 0: x_k = 0, the pair (F, x*)).  Returns
    (R, E) float32 device tensors [count, n]."""
    dev = torch.device("cuda", torch.cuda.current_device())
    count, n = loads.shape
    rng = np.random.default_rng(seed)
    fast = _lib.make_options(tolerance=x_tol, max_iterations=20000, stop_rule=_lib.PG_STOP_RELATIVE,
                             precision=_lib.PG_PREC_MIXED, preconditioner=_lib.PG_PRECOND_TWO_LEVEL,
                             smoother=_lib.PG_SMOOTHER_CHEBYSHEV)
    plan_fast = ctx.plan(ls.prob, fast)
    F = torch.from_numpy(np.ascontiguousarray(loads, np.float32)).to(dev)
    XS = torch.empty((count, n), dtype=torch.float64, device=dev)
    XK = torch.zeros((count, n), dtype=torch.float64, device=dev)
    ks = rng.integers(0, k_max + 1, size=count)
    torch.cuda.synchronize()
    for i in range(count):
        plan_fast.solve_device(fast, F[i].data_ptr(), XS[i].data_ptr())
        if ks[i] > 0:
            o = _lib.make_options(tolerance=0.0, max_iterations=int(ks[i]), stop_rule=_lib.PG_STOP_RELATIVE)
            ls.plan.solve_device(o, F[i].data_ptr(), XK[i].data_ptr())
    plan_fast.close()
    R = torch.empty((count, n), dtype=torch.float32, device=dev)
    E = torch.empty_like(R)
    ls.learned.make_pairs(count, F.data_ptr(), XS.data_ptr(), XK.data_ptr(), R.data_ptr(), E.data_ptr())
    return R, E, ks


def evaluate(torch, ls: LearnedSolver, loads, tolerance=1e-6, mode=_lib.LEARNED_NETWORK, truth=None):
    """Learned (or, by mode, network-free) solves of `loads`; per load the
    iterations, device ms and, when truth [count, n] is given, the FP64
    relative error."""
    dev = torch.device("cuda", torch.cuda.current_device())
    n = loads.shape[1]
    F = torch.from_numpy(np.ascontiguousarray(loads, np.float32)).to(dev)
    x = torch.zeros(n, dtype=torch.float64, device=dev)
    opts = solve_options(tolerance)
    rows = []
    for i in range(loads.shape[0]):
        info, st = ls.learned.solve_device(opts, F[i].data_ptr(), x.data_ptr(), mode)
        row = {"iterations": int(info.iterations), "ms": float(info.solve_ms), "pdl": int(st.pdl),
               "converged": int(info.converged), "network_iterations": int(st.network_iterations),
               "network_off_at": int(st.network_off_at)}
        if truth is not None:
            xt = truth[i]
            row["rel_l2"] = float(np.linalg.norm(x.cpu().numpy() - xt) / np.linalg.norm(xt))
        rows.append(row)
    return rows


def tight_solutions(torch, ctx, ls: LearnedSolver, loads, tol=1e-12):
    """FP64 two-level PCG solutions to ||r||/||b|| < tol (the reference
    solutions of evaluations too large for the sparse-LU oracle)."""
    dev = torch.device("cuda", torch.cuda.current_device())
    o = _lib.make_options(tolerance=tol, max_iterations=50000, stop_rule=_lib.PG_STOP_RELATIVE,
                          preconditioner=_lib.PG_PRECOND_TWO_LEVEL)
    plan = ctx.plan(ls.prob, o)
    F = torch.from_numpy(np.ascontiguousarray(loads, np.float32)).to(dev)
    x = torch.zeros(loads.shape[1], dtype=torch.float64, device=dev)
    out = np.zeros(loads.shape, np.float64)
    for i in range(loads.shape[0]):
        plan.solve_device(o, F[i].data_ptr(), x.data_ptr())
        out[i] = x.cpu().numpy()
    plan.close()
    return out


def train_net(ls: LearnedSolver, count, R, E, epochs=40, energy_epochs=None, batch=32, lr=3e-3, val=256,
              seed=TRAIN_SEED):
    """Trains ls's network on `count` pairs (device tensors R, E): first
    with the scaled-L2 loss of the error (well-conditioned gradients: the
    network learns the smooth bulk of the error), then `energy_epochs`
    (default a quarter of `epochs`) with the energy-norm loss of the error
    after the correction and the solve's smoothing sweeps, the quantity the
    preconditioner depends on.  Returns one info dict for the run."""
    if energy_epochs is None:
        energy_epochs = epochs // 4
    stages = [(_lib.PG_LOSS_SCALED_L2, epochs - energy_epochs), (_lib.PG_LOSS_SMOOTHED_ENERGY, energy_epochs)]
    out = {"stages": [], "epoch_loss": [], "epoch_val_loss": [], "train_ms": 0.0, "steps": 0}
    first = True
    for loss, ep in stages:
        if ep <= 0:
            continue
        opts = _lib.train_options(epochs=ep, batch=batch, lr=lr, seed=seed, val_count=val,
                                  set_scales=first, loss=loss)
        info = ls.learned.train(count, R.data_ptr(), E.data_ptr(), opts)
        if first:
            out["val_loss_before"] = info.val_loss_before
            out["loss_first_step"] = info.loss_first_step
            out["batch"] = int(info.batch)
        first = False
        out["stages"].append({"loss": "scaled_l2" if loss == _lib.PG_LOSS_SCALED_L2 else "smoothed_energy",
                              "epochs": ep, "steps": int(info.steps), "val_loss": info.val_loss,
                              "loss_last_step": info.loss_last_step})
        out["epoch_loss"] += list(info.epoch_loss)[:ep]
        out["epoch_val_loss"] += list(info.epoch_val_loss)[:ep]
        out["train_ms"] += info.train_ms
        out["steps"] += int(info.steps)
        out["val_loss"] = info.val_loss
        out["loss_last_step"] = info.loss_last_step
    return out


def train_plate(torch, ctx, wl, loads=8192, epochs=40, energy_epochs=None, batch=32, lr=3e-3, k_max=300,
                val=256, seed=TRAIN_SEED, log=print):
    """The full pipeline for one plate: seeded random-field loads, plain
    solves, pairs, training (train_net).  Returns (LearnedSolver, info
    dict); the validation losses are energy-norm losses (1 = no gain)."""
    t0 = time.time()
    ls = LearnedSolver(ctx, wl, seed=seed)
    F = workloads.random_field_loads(wl, loads, seed)
    t1 = time.time()
    R, E, ks = generate_pairs(torch, ctx, ls, F, k_max=k_max, seed=seed)
    torch.cuda.synchronize()
    t2 = time.time()
    log(f"pairs: {loads} loads in {t1 - t0:.1f} s (host), solved in {t2 - t1:.1f} s")
    tr = train_net(ls, loads, R, E, epochs=epochs, energy_epochs=energy_epochs, batch=batch, lr=lr, val=val,
                   seed=seed)
    del R, E
    torch.cuda.synchronize()
    out = {"loads": loads, "epochs": epochs, "lr": lr, "k_max": k_max, "val_pairs": val, "seed": seed,
           "load_gen_s": t1 - t0, "pair_solve_s": t2 - t1, "params": ls.net.param_count}
    out.update(tr)
    log(f"trained {out['steps']} steps in {out['train_ms'] / 1e3:.1f} s: validation energy loss "
        f"{out['val_loss_before']:.4f} -> {out['val_loss']:.4f}")
    return ls, out


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m plategpu.learned")
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train", help="train the plate_q4_141 network and write its weight file")
    t.add_argument("--out", default=DEFAULT_WEIGHTS)
    t.add_argument("--loads", type=int, default=8192)
    t.add_argument("--epochs", type=int, default=40)
    t.add_argument("--energy-epochs", type=int, default=None,
                   help="final epochs with the energy-norm loss (default a quarter of --epochs)")
    t.add_argument("--batch", type=int, default=32)
    t.add_argument("--lr", type=float, default=3e-3)
    t.add_argument("--k-max", type=int, default=300)
    t.add_argument("--eval", type=int, default=64, help="held-out loads evaluated after training")
    t.add_argument("--json", default=None, help="write the training record here too")
    f = sub.add_parser("forward", help="time the network's forward pass (random weights and input)")
    f.add_argument("--batch", type=int, default=32)
    f.add_argument("--size", type=int, default=144, help="grid height = width (multiple of 8)")
    f.add_argument("--reps", type=int, default=20)
    v = sub.add_parser("solve", help="learned solves of plate_q4_141 held-out loads")
    v.add_argument("--weights", default=DEFAULT_WEIGHTS)
    v.add_argument("--count", type=int, default=4)
    v.add_argument("--mode", type=int, default=_lib.LEARNED_NETWORK)
    v.add_argument("--tolerance", type=float, default=1e-6)
    v.add_argument("--phase-timing", action="store_true",
                   help="run without the graph and print the average device time per iteration of each "
                        "kernel group")
    v.add_argument("--workload", default="plate_q4_141")
    a = ap.parse_args(argv)
    import torch

    if a.cmd == "solve":
        ctx = _lib.Context(0)
        wl = workloads.WORKLOADS[a.workload]()
        ls = LearnedSolver(ctx, wl, weights=a.weights if a.mode == _lib.LEARNED_NETWORK else None)
        H = workloads.random_field_loads(wl, a.count, HELD_OUT_SEED)
        if a.phase_timing:
            opts = solve_options(a.tolerance)
            opts.phase_timing = 1
            F = torch.from_numpy(np.ascontiguousarray(H, np.float32)).cuda()
            x = torch.zeros(wl.n_dof, dtype=torch.float64, device="cuda")
            names = ("update", "true_residual", "smoothing_input", "network", "Ky_sweeps", "preconditioner",
                     "direction_Kp", "tick")
            for i in range(a.count):
                info, st = ls.learned.solve_device(opts, F[i].data_ptr(), x.data_ptr(), a.mode)
                print(json.dumps({"iterations": int(info.iterations),
                                  "us_per_iteration": dict(zip(names, [round(v, 2) for v in info.phase_us]))}))
        else:
            for r in evaluate(torch, ls, H, tolerance=a.tolerance, mode=a.mode):
                print(json.dumps(r))
        ls.close()
        ctx.close()
        return

    if a.cmd == "forward":
        ctx = _lib.Context(0)
        net = _lib.Net(ctx, a.size, a.size, seed=1)
        x = torch.randn(a.batch, a.size, a.size, 3, device="cuda")
        y = torch.empty_like(x)
        for _ in range(3):
            net.forward(a.batch, x.data_ptr(), y.data_ptr())
        torch.cuda.synchronize()
        s_, e_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s_.record()
        for _ in range(a.reps):
            net.forward(a.batch, x.data_ptr(), y.data_ptr())
        e_.record()
        torch.cuda.synchronize()
        ms = s_.elapsed_time(e_) / a.reps
        fl = flops_per_image(a.size, a.size) * a.batch
        print(json.dumps({"batch": a.batch, "size": a.size, "ms": ms, "tflops": fl / (ms * 1e-3) / 1e12}))
        net.close()
        ctx.close()
        return

    wl = workloads.plate_q4_141()
    ctx = _lib.Context(0)
    ls, info = train_plate(torch, ctx, wl, loads=a.loads, epochs=a.epochs, energy_epochs=a.energy_epochs,
                           batch=a.batch, lr=a.lr, k_max=a.k_max)
    if a.eval:
        H = workloads.random_field_loads(wl, a.eval, HELD_OUT_SEED)
        xt = tight_solutions(torch, ctx, ls, H)
        rows = evaluate(torch, ls, H, truth=xt)
        rows0 = evaluate(torch, ls, H[: min(8, a.eval)], mode=_lib.LEARNED_SMOOTHING_ONLY)
        its = [r["iterations"] for r in rows]
        info["held_out"] = {"loads": a.eval, "iterations_p50": float(np.median(its)),
                            "iterations_max": int(max(its)),
                            "ms_p50": float(np.median([r["ms"] for r in rows])),
                            "rel_l2_max": max(r["rel_l2"] for r in rows),
                            "smoothing_only_iterations_p50": float(np.median([r["iterations"] for r in rows0]))}
        print(json.dumps(info["held_out"]))
    save_weights(ls.net, a.out, meta=info)
    if a.json:
        with open(a.json, "w") as f:
            json.dump(info, f, indent=1)
    ls.close()
    ctx.close()


if __name__ == "__main__":
    main()
