"""Training of the learned preconditioner on (source, solution) pairs that the
plain solver generates.

Each synthetic problem (the batched-magnetostatics distribution: coils,
permeability-1000 rectangles, Dirichlet boundary) is solved to 1e-10 with the
plain FP64 solver, giving (b, x*).  Looser plain solves of the same problem
(relative tolerances 1e-1 ... 1e-5) give iterates x_k and with them further
exact pairs (b - A x_k, x* - x_k): residuals of the kind the preconditioner
meets inside a Krylov solve, each with its exact error.  Training runs on the
GPU through the library's own forward / backward kernels and Adam step.

    python -m similie_b200.train_precond --problems 512 --steps 3000 --out precond_2d.npy
"""
import argparse
import json
import math
import time

import numpy as np

from . import magnetostatics as mag
from .precond import LearnedPreconditioner

SNAPSHOT_TOLS = (1e-1, 1e-2, 1e-3, 1e-5)


def generate_pairs(seed, count, sizes=(256, 384, 512, 768, 1024), snapshot_tols=SNAPSHOT_TOLS, batch=64,
                   min_cores=0):
    """Pairs grouped by grid size: {n: [(nu, b, x), ...]} as flat FP32 CUDA tensors
    (nu shared by the pairs of one problem).  min_cores > 0 draws the number
    of permeability-1000 rectangles from min_cores..3 instead of 0..3."""
    import torch
    rng = np.random.default_rng(seed)
    pairs = {}
    for start in range(0, count, batch):
        probs = [mag.synthetic_problem(rng, int(rng.choice(sizes)),
                                       cores=int(rng.integers(min_cores, 4)) if min_cores > 0 else None)
                 for _ in range(min(batch, count - start))]
        shapes = [(p.nx, p.ny) for p in probs]
        mus = [torch.from_numpy(p.node_mu()).cuda() for p in probs]
        rhss = [torch.from_numpy(p.rhs()).cuda() for p in probs]
        sols = [torch.zeros_like(r) for r in rhss]
        mag.solve_batch(mus, rhss, sols, shapes, solver="cg", tol=1e-10)
        nus = [(1.0 / m).float() for m in mus]
        for k, p in enumerate(probs):
            pairs.setdefault(p.nx, []).append((nus[k], rhss[k].float(), sols[k].float()))
        for t in snapshot_tols:
            xk = [torch.zeros_like(r) for r in rhss]
            mag.solve_batch(mus, rhss, xk, shapes, solver="cg", tol=t)
            for k, p in enumerate(probs):
                ax = torch.zeros_like(xk[k])
                mag.apply(mus[k], xk[k], ax, p.nx, p.ny)
                pairs[p.nx].append((nus[k], (rhss[k] - ax).float(), (sols[k] - xk[k]).float()))
        del mus, rhss, sols
    return pairs


def train(net, pairs, steps, batch=8, lr=1e-3, seed=0, log_every=100, log=None, start=0, checkpoint=None,
          checkpoint_every=500):
    """Adam with a cosine learning-rate schedule; each step draws `batch` pairs
    of one grid size (sizes drawn in proportion to their pair counts).
    start: the step to resume from (the schedule and the draws continue
    there); checkpoint: a path written every `checkpoint_every` steps."""
    import torch
    rng = np.random.default_rng(seed)
    sizes = sorted(pairs)
    weights = np.array([len(pairs[n]) for n in sizes], dtype=np.float64)
    weights /= weights.sum()
    history = []
    t0 = time.perf_counter()
    for _ in range(start):                      # replay the draws of the steps already taken
        n = sizes[int(rng.choice(len(sizes), p=weights))]
        rng.integers(0, len(pairs[n]), batch)
    for step in range(start, steps):
        n = sizes[int(rng.choice(len(sizes), p=weights))]
        idx = rng.integers(0, len(pairs[n]), batch)
        nu = torch.cat([pairs[n][i][0] for i in idx])
        b = torch.cat([pairs[n][i][1] for i in idx])
        x = torch.cat([pairs[n][i][2] for i in idx])
        lr_t = lr * 0.5 * (1.0 + math.cos(math.pi * step / max(1, steps)))
        loss = net.train_step([(n, n)] * batch, nu, b, x, max(lr_t, 1e-6))
        history.append(loss)
        if log is not None and (step % log_every == 0 or step == steps - 1):
            log(json.dumps({"step": step, "size": n, "loss": round(float(np.mean(history[-log_every:])), 5),
                            "seconds": round(time.perf_counter() - t0, 2)}))
        if checkpoint is not None and ((step + 1) % checkpoint_every == 0 or step == steps - 1):
            net.save_checkpoint(checkpoint, step + 1, seed, {"steps": steps, "batch": batch, "lr": lr})
    if torch.cuda.is_available():
        torch.cuda.synchronize()
    return history, time.perf_counter() - t0


def check_resume(path, seed, steps, batch, lr):
    """Raises ValueError when the run's seed, step count, batch or learning
    rate differ from those the checkpoint was written with: the pair set and
    the batch draws follow the seed and the cosine schedule follows the step
    count, so a resumed run continues the original one only with the same
    settings."""
    from .precond import read_checkpoint
    _, step, ck_seed, extra = read_checkpoint(path)
    want = {"seed": ck_seed, "steps": extra.get("steps"), "batch": extra.get("batch"), "lr": extra.get("lr")}
    have = {"seed": seed, "steps": steps, "batch": batch, "lr": lr}
    bad = {k: (want[k], have[k]) for k in want if want[k] is not None and want[k] != have[k]}
    if bad:
        raise ValueError("--resume: settings differ from the checkpoint's (checkpoint, run): "
                         + ", ".join(f"{k} {a!r} vs {b!r}" for k, (a, b) in sorted(bad.items())))
    return step


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--problems", type=int, default=256)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--init", default=None, help="start from these parameters (.npy)")
    ap.add_argument("--sizes", default="256,384,512,768,1024", help="grid sizes of the generated problems")
    ap.add_argument("--min-cores", type=int, default=0,
                    help="draw min..3 permeability-1000 rectangles per problem instead of 0..3")
    ap.add_argument("--out", default="precond_2d.npy")
    ap.add_argument("--checkpoint", default=None, help="write a resumable checkpoint here while training")
    ap.add_argument("--resume", default=None,
                    help="continue from this checkpoint: parameters, step and (version-2 checkpoints) the Adam "
                         "moments; a version-1 checkpoint restarts the Adam moments.  The seed, --steps, --batch "
                         "and --lr must be the checkpoint's (the pair set, the batch draws and the schedule depend "
                         "on them); a mismatch is an error.  Not combinable with --init")
    args = ap.parse_args()
    if args.init and args.resume:
        ap.error("--init and --resume are exclusive: a resumed run takes its parameters from the checkpoint")
    if args.resume:
        check_resume(args.resume, args.seed, args.steps, args.batch, args.lr)
    import torch
    torch.cuda.init()
    t0 = time.perf_counter()
    pairs = generate_pairs(args.seed, args.problems, sizes=tuple(int(v) for v in args.sizes.split(",")),
                           min_cores=args.min_cores)
    npairs = sum(len(v) for v in pairs.values())
    print(json.dumps({"pairs": npairs, "by_size": {int(k): len(v) for k, v in pairs.items()},
                      "generate_seconds": round(time.perf_counter() - t0, 2)}), flush=True)
    net = LearnedPreconditioner(seed=args.seed)
    if args.init:
        net.load(args.init)
    start = 0
    if args.resume:
        start, _, _ = net.load_checkpoint(args.resume)
    hist, t_train = train(net, pairs, args.steps, args.batch, args.lr, args.seed, log=lambda s: print(s, flush=True),
                          start=start, checkpoint=args.checkpoint)
    net.save(args.out)
    print(json.dumps({"train_seconds": round(t_train, 2), "final_loss": float(np.mean(hist[-100:]))}), flush=True)


if __name__ == "__main__":
    main()
