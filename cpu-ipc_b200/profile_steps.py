#!/usr/bin/env python3
"""Profiling driver for ncu: a bench scene restored from the oracle's saved
contact-phase state (oracle/states/), one untimed step, then --steps steps
inside cudaProfilerStart/Stop, so that

    ncu --profile-from-start off --clock-control none ... python cpu-ipc_b200/profile_steps.py

captures only contact-phase launches.  Prints each step's Newton and PCG
counts and host stage timers.

    python cpu-ipc_b200/profile_steps.py --scene pile --precision mixed --precond learned --steps 2
"""
import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import cipc  # noqa: E402

STATES = {"pile": ("pile_64x12_frame35.npz", lambda: cipc.scene_pile(64, 12)),
          "cloth_drape": ("cloth_drape_128_frame40.npz", lambda: cipc.scene_cloth_drape(128, 10))}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--scene", default="pile", choices=list(STATES))
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--precond", default="learned", choices=["jacobi", "learned", "fsai"])
    ap.add_argument("--weights", default=None, help="network weights (raw float32)")
    ap.add_argument("--steps", type=int, default=2)
    args = ap.parse_args()
    import torch
    torch.cuda.set_device(0)
    fname, make = STATES[args.scene]
    sc = make()
    sim = cipc.Simulator(sc, precision=args.precision, precond=args.precond)
    if args.weights:
        sim.set_precond_weights(np.fromfile(args.weights, np.float32))
    s = np.load(os.path.join(HERE, "..", "oracle", "states", fname))
    dt = sc["params"]["dt"]
    x, vel = s["x"], s["vel"]
    sim.set("x", x); sim.set("vprev", x); sim.set("vel", vel)
    sim.set("xtilde", x + vel * dt + np.array([0.0, float(s["gravity"]) * dt * dt, 0.0]))
    sim.set_kappa(float(s["kappa"]))
    sim.collision_sets()
    sim.step()  # untimed: buffers reach their sizes
    torch.cuda.synchronize()
    torch.cuda.cudart().cudaProfilerStart()
    t0 = time.time()
    for k in range(args.steps):
        st = sim.step()
        print(k, "newton", st["newtonIterations"], "pcg", st["pcgIterations"], "contacts", st["selfContacts"],
              {kk: round(st[kk], 1) for kk in ("stepMilliseconds", "assemblyMilliseconds", "linearSolveMilliseconds", "ccdMilliseconds",
                                               "lineSearchMilliseconds")}, flush=True)
    torch.cuda.synchronize()
    torch.cuda.cudart().cudaProfilerStop()
    print("done", round(time.time() - t0, 3), "s", flush=True)
    sim.close()


if __name__ == "__main__":
    main()
