#!/usr/bin/env python3
"""Training and held-out evaluation of the learned preconditioner on the pile
configuration: 3 message-passing layers of width 32 (BF16 weights, FP32
accumulation) emitting a factor on the matrix's own lower pattern, trained
on the Newton systems the simulator produces for pile seeds 0-49 and
evaluated on seeds 50-59 against block-Jacobi and the exact FSAI factor of
the same pattern, at PCG relative residual 1e-6 (the FP64 true residual).

Training streams the systems through the network as they arise: each train
seed's pile runs --train-steps steps in mixed precision with the learned
factor, and from step --train-from on every Newton system, at the
linear-solve seam, takes --adam-iters Adam steps of the loss before it is
solved (the systems stay on the GPU; nothing is written to disk).  The
weights carry over from seed to seed; --init-weights starts from a previous
run's.

Evaluation: each test seed's pile settles --settle steps in FP64, then the
same state is restored into every variant (FP64 block-Jacobi, mixed
block-Jacobi, mixed learned with the frozen weights, mixed FSAI), which each
run --eval-steps device-timed steps.

    python cpu-ipc_b200/train_precond.py --weights w.bin --report r.json
"""
import argparse
import json
import os
import sys
import time

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import cipc  # noqa: E402

VARIANTS = (("fp64", "jacobi"), ("mixed", "jacobi"), ("mixed", "learned"), ("mixed", "fsai"))


def seeds(spec):
    a, b = spec.split(":")
    return list(range(int(a), int(b)))


def parse(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--cubes", type=int, default=64)
    ap.add_argument("--cells", type=int, default=12)
    ap.add_argument("--train-seeds", default="0:50")
    ap.add_argument("--test-seeds", default="50:60")
    ap.add_argument("--train-steps", type=int, default=25)
    ap.add_argument("--train-from", type=int, default=0, help="steps of each train seed run before its systems train the network")
    ap.add_argument("--adam-iters", type=int, default=4)
    ap.add_argument("--probes", type=int, default=4)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--settle", type=int, default=30)
    ap.add_argument("--eval-steps", type=int, default=5)
    ap.add_argument("--weights", default=None, help="write the trained weights here (raw float32)")
    ap.add_argument("--init-weights", default=None, help="start from these weights (raw float32) instead of the initial factor")
    ap.add_argument("--skip-training", action="store_true")
    ap.add_argument("--report", default=None)
    return ap.parse_args(argv)


def train(args, log):
    w = np.fromfile(args.init_weights, np.float32) if args.init_weights else None
    systems = 0
    t0 = time.time()
    for seed in seeds(args.train_seeds):
        sim = cipc.Simulator(cipc.scene_pile(args.cubes, args.cells, seed=seed), precision="mixed", precond="learned")
        if w is not None:
            sim.set_precond_weights(w)
        for k in range(args.train_steps):
            if k == args.train_from:
                sim.set_online_training(args.adam_iters, args.probes, args.lr, 7919 * seed + 1)
            sim.step()
        n = sim.hook_systems()
        systems += n
        w = sim.precond_weights()
        sim.close()
        log(f"train seed {seed}: {n} systems ({systems} in all), {time.time() - t0:.0f} s")
    return w, systems, time.time() - t0


def restore(sim, state):
    for k in ("x", "vel", "vprev", "xtilde"):
        sim.set(k, state[k])
    sim.set_kappa(state["kappa"])
    sim.collision_sets()


def evaluate(args, w, log):
    rows = []
    for seed in seeds(args.test_seeds):
        sc = cipc.scene_pile(args.cubes, args.cells, seed=seed)
        base = cipc.Simulator(sc, precision="fp64", precond="jacobi")
        for _ in range(args.settle):
            base.step()
        state = {k: base.get(k) for k in ("x", "vel", "vprev", "xtilde")}
        state["kappa"] = base.scalars()["kappa"]
        base.close()
        for prec, pre in VARIANTS:
            sim = cipc.Simulator(sc, precision=prec, precond=pre)
            if pre == "learned":
                sim.set_precond_weights(w)
            restore(sim, state)
            ms = 0.0
            newton = pcg = 0
            for _ in range(args.eval_steps):
                m, st = sim.timed_steps(1)
                ms += m
                newton += st["newtonIterations"]
                pcg += st["pcgIterations"]
            fb = sim.precond_stats()["fallbacks"] if pre != "jacobi" else 0
            sim.close()
            rows.append(dict(seed=seed, precision=prec, precond=pre, steps=args.eval_steps, ms=ms, newton=newton, pcg=pcg, fallbacks=fb))
            log(f"test seed {seed} {prec}/{pre}: {args.eval_steps / (ms / 1000):.2f} steps/s, {pcg / max(1, newton):.1f} PCG it. per Newton, "
                f"{fb} fallbacks")
    return rows


def summarise(rows):
    out = {}
    for prec, pre in VARIANTS:
        r = [x for x in rows if x["precision"] == prec and x["precond"] == pre]
        if not r:
            continue
        steps = sum(x["steps"] for x in r)
        ms = sum(x["ms"] for x in r)
        out[f"{prec}/{pre}"] = dict(steps_per_s=steps / (ms / 1000), pcg_per_newton=sum(x["pcg"] for x in r) / max(1, sum(x["newton"] for x in r)),
                                    newton_per_step=sum(x["newton"] for x in r) / steps, fallbacks=sum(x["fallbacks"] for x in r))
    return out


def main(argv=None):
    args = parse(argv)
    log = lambda m: print(m, flush=True)  # noqa: E731
    import torch
    torch.cuda.set_device(0)
    report = dict(config=vars(args))
    if args.skip_training:
        w = np.fromfile(args.init_weights, np.float32)
        report["training"] = None
    else:
        w, systems, secs = train(args, log)
        report["training"] = dict(systems=systems, seconds=secs)
        if args.weights:
            w.tofile(args.weights)
    rows = evaluate(args, w, log)
    report["runs"] = rows
    report["summary"] = summarise(rows)
    log(json.dumps(report["summary"], indent=1))
    if args.report:
        with open(args.report, "w") as f:
            json.dump(report, f, indent=1)
    return report


if __name__ == "__main__":
    main()
