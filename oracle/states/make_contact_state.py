"""Contact-phase starting states of the bench scenes for bench.py's CPU legs
and the full-size parity tests.

The oracle (test infrastructure: the FP64 CPU restatement of the reference's
time step) runs a scene from frame 0 for as many steps as bench.py's GPU arm
runs before its timed steps, and writes the state the next step starts from
(positions, velocities, kappa).  bench.py's CPU legs restore it, so they time
the same contact frames as the GPU arm rather than the cheaper free-fall
frames at the start of the scene; the parity tests restore it to compare the
GPU and the oracle in contact at the configurations' own sizes.

    python oracle/states/make_contact_state.py --scene cloth_drape --steps 40
        128x128 cloth over the 10^3-cell cube, dt 0.005 (about four minutes on
        8 host cores) -> cloth_drape_128_frame40.npz
    python oracle/states/make_contact_state.py --scene pile --cubes 64 --cells 12 --steps 35 --linear multifrontal
        64 cubes of 12^3 cells in the open box, dt 0.01 (40-100 s per step
        on 8 host cores) -> pile_64x12_frame35.npz
    python oracle/states/make_contact_state.py --scene pile --cubes 8 --cells 12 --steps 60 --linear multifrontal
        -> pile_8x12_frame60.npz
"""
import argparse
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "cpu-ipc_b200"))


def state_path(scene_name, frame):
    return os.path.join(HERE, f"{scene_name}_frame{frame}.npz")


def make_scene(args):
    import cipc
    if args.scene == "pile":
        return cipc.scene_pile(args.cubes, args.cells)
    return cipc.scene_cloth_drape(args.cloth, 10)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--scene", default="cloth_drape", choices=["cloth_drape", "pile"])
    ap.add_argument("--cloth", type=int, default=128)
    ap.add_argument("--cubes", type=int, default=64)
    ap.add_argument("--cells", type=int, default=12)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--linear", default="pcg", choices=["pcg", "multifrontal", "direct"])
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--save-every", type=int, default=0, help="also write the state every N steps")
    args = ap.parse_args()
    import oracle
    scene = make_scene(args)
    o = oracle.Oracle(scene, linear=args.linear, threads=args.threads)
    t0 = time.time()
    for k in range(args.steps):
        st = o.step()
        print(f"step {k + 1}: {st['newton']} Newton, {st['linearSolves']} solves, {st['selfContacts']} self / "
              f"{st['groundContacts']} ground contacts, {time.time() - t0:.1f} s", flush=True)
        if args.save_every and (k + 1) % args.save_every == 0 and k + 1 < args.steps:
            o.save_state(state_path(scene["name"], k + 1), k + 1)
    path = state_path(scene["name"], args.steps)
    o.save_state(path, args.steps)
    print("wrote", path)


if __name__ == "__main__":
    main()
