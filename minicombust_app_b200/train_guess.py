"""Train the learned pressure-correction guess on snapshots of the plain solver.

    python -m minicombust_app_b200.train_guess --m 32 --seeds 20 --snapshots 250 \\
        --steps 2000 --batch 8 --out minicombust_app_b200/data/pressure_guess.f32

1. Data: for each seed, the plain FP64 solver (simple mode, AMG-PCG) runs
   `snapshots` SIMPLE passes on the 2m x m x m box from seeded noisy initial
   fields and seeded source blobs, and its snapshot writer records every
   pressure solve (right-hand side, diagonal, previous correction, converged
   correction).
2. Split by seed: the last 20 % of the seeds are held out.
3. Training: Adam on random batches of training records through the
   library's forward/backward kernels; cosine learning-rate decay.
4. Output: the FP32 parameters (raw little-endian float32) and a JSON record
   of the run next to them.
"""
import argparse
import json
import math
import os
import tempfile
import time

import numpy as np

from . import flow, gnn
from .workload import gaussian_blobs, noisy_fields

LENGTHS = (0.2, 0.1, 0.1)
BLOBS_PER_CELL = 1000 / 4194304  # the 2 x 128^3 benchmark's source density


def box(m):
    return (2 * m, m, m)


def make_solver(m, seed, guess=flow.GUESS_ZERO, precision=flow.PRECISION_FP64, params=None):
    dims = box(m)
    mesh = flow.Mesh.box(*dims, *LENGTHS)
    s = flow.FlowSolver(mesh, params=flow.default_params(flow.MODE_SIMPLE, pressure_solver=flow.PSOLVER_PCG_AMG,
                                                         initial_guess=guess, precision=precision))
    for name, vals in noisy_fields(s.N, seed).items():
        a = s.field(name)
        a[:s.N] = vals
        s.set_field(name, a)
    k = max(1, int(round(BLOBS_PER_CELL * s.N)))
    s.set_sources(gaussian_blobs(dims, LENGTHS, k, seed))
    if params is not None:
        s.set_guess_params(params)
    return s


def generate(m, seeds, snapshots, workdir, log=print):
    paths = []
    for seed in seeds:
        path = os.path.join(workdir, f"snap_m{m}_seed{seed}.bin")
        s = make_solver(m, seed)
        s.snapshot_open(path, snapshots)
        t = time.perf_counter()
        for _ in range(snapshots):
            s.simple_iteration()
        s.snapshot_close()
        s.close()
        log(f"seed {seed}: {snapshots} passes in {time.perf_counter() - t:.1f} s -> {path}")
        paths.append(path)
    return paths


def load(paths):
    import torch
    return [torch.from_numpy(np.array(flow.read_snapshots(p))).cuda() for p in paths]


def samples_of(data, picks):
    return [(data[f][r, 0], data[f][r, 1], data[f][r, 2], data[f][r, 3]) for f, r in picks]


def prev_baseline_loss(data, picks):
    """Held-out loss of the plain previous-correction guess (y = prev / s_x),
    in the network's loss units, for comparison."""
    tot = 0.0
    for f, r in picks:
        rec = data[f][r].double()
        b, diag, prev, x = rec[0], rec[1], rec[2], rec[3]
        sb = float(b.pow(2).mean().sqrt())
        sd = float(diag.mean())
        sx = sb / sd if sd > 0 and sb > 0 else 0.0
        if sx == 0.0:
            continue
        d = (prev - x) / sx
        d = d - d.mean()
        tot += float(d.pow(2).mean())
    return tot / max(len(picks), 1)


def train(net, graph, data, train_files, held_files, steps, batch, lr, seed, log=print):
    rng = np.random.default_rng(seed)
    recs = lambda files: [(f, r) for f in files for r in range(data[f].shape[0])]
    train_recs, held_recs = recs(train_files), recs(held_files)
    held_eval = [held_recs[i] for i in rng.choice(len(held_recs), size=min(32, len(held_recs)), replace=False)]
    history = []
    t0 = time.perf_counter()
    for step in range(steps):
        lr_t = 0.5 * lr * (1.0 + math.cos(math.pi * step / steps)) + 0.02 * lr
        picks = [train_recs[i] for i in rng.choice(len(train_recs), size=batch, replace=False)]
        loss = net.train_step(graph, samples_of(data, picks), lr_t)
        if step % 100 == 0 or step == steps - 1:
            held = net.loss_grad(graph, samples_of(data, held_eval), want_grad=False)[0]
            history.append({"step": step, "train_loss": loss, "held_out_loss": held, "lr": lr_t})
            log(f"step {step:5d}  train {loss:.4e}  held-out {held:.4e}  lr {lr_t:.2e}")
    return {"history": history, "train_seconds": time.perf_counter() - t0,
            "held_out_loss": history[-1]["held_out_loss"],
            "held_out_prev_guess_loss": prev_baseline_loss(data, held_eval)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--m", type=int, default=32, help="training box 2m x m x m")
    ap.add_argument("--seeds", type=int, default=20)
    ap.add_argument("--snapshots", type=int, default=250, help="SIMPLE passes recorded per seed")
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=0, help="initialisation and batch sampling")
    ap.add_argument("--out", default=os.path.join(os.path.dirname(os.path.abspath(__file__)), "data",
                                                  "pressure_guess.f32"))
    ap.add_argument("--workdir", default=None, help="snapshot files (default: a temporary directory)")
    args = ap.parse_args()
    workdir = args.workdir or tempfile.mkdtemp(prefix="mc_snapshots_")
    os.makedirs(workdir, exist_ok=True)
    seeds = list(range(args.seeds))
    n_held = max(1, args.seeds // 5)
    t = time.perf_counter()
    paths = generate(args.m, seeds, args.snapshots, workdir)
    gen_s = time.perf_counter() - t
    data = load(paths)
    net = gnn.GuessNet(seed=args.seed)
    graph = net.graph(flow.Mesh.box(*box(args.m), *LENGTHS))
    files = list(range(len(paths)))
    rep = train(net, graph, data, files[:-n_held], files[-n_held:], args.steps, args.batch, args.lr, args.seed)
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    net.params().astype("<f4").tofile(args.out)
    rep.update({"mesh": list(box(args.m)), "seeds": args.seeds, "held_out_seeds": seeds[-n_held:],
                "snapshots_per_seed": args.snapshots, "records": int(sum(d.shape[0] for d in data)),
                "steps": args.steps, "batch": args.batch, "lr": args.lr, "init_seed": args.seed,
                "generate_seconds": gen_s, "params": int(net.nparam)})
    with open(args.out + ".json", "w") as f:
        json.dump(rep, f, indent=1)
    print(json.dumps({k: v for k, v in rep.items() if k != "history"}))


def load_params(path=None):
    """The committed trained parameters (float32)."""
    path = path or os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "pressure_guess.f32")
    p = np.fromfile(path, dtype="<f4")
    if len(p) != gnn.param_count():
        raise ValueError(f"{path}: {len(p)} parameters, the network has {gnn.param_count()}")
    return p


if __name__ == "__main__":
    main()
