"""Contact-phase starting state of the cloth-drape scene for bench.py's CPU legs.

The oracle (test infrastructure: the FP64 CPU restatement of the reference's
time step) runs the cloth-drape scene, a 128x128-vertex cloth over the fixed
10^3-cell tetrahedral cube at dt 0.005, for as many steps as bench.py's GPU
arm runs untimed before its warm-up (40: the cloth has reached the cube).  It
writes the state the next step starts from (positions, velocities, kappa).
bench.py's CPU legs restore it, so they time the same contact frames as the
GPU arm rather than the cheaper free-fall frames at the start of the scene.

    python oracle/states/make_contact_state.py [--steps 40] [--threads N]

takes about four minutes on 8 host cores and writes
oracle/states/cloth_drape_128_frame40.npz.
"""
import argparse
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "cpu-ipc_b200"))


def state_path(cloth, frame):
    return os.path.join(HERE, f"cloth_drape_{cloth}_frame{frame}.npz")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--cloth", type=int, default=128)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    args = ap.parse_args()
    import cipc
    import oracle
    o = oracle.Oracle(cipc.scene_cloth_drape(args.cloth, 10), linear="pcg", threads=args.threads)
    t0 = time.time()
    for k in range(args.steps):
        st = o.step()
        print(f"step {k + 1}: {st['newton']} Newton, {st['pcgIterations']} PCG, {st['selfContacts']} self contacts, "
              f"{time.time() - t0:.1f} s", flush=True)
    path = state_path(args.cloth, args.steps)
    o.save_state(path, args.steps)
    print("wrote", path)


if __name__ == "__main__":
    main()
