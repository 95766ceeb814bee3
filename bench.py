"""Benchmark of the GPU IPC time step (one JSON line on rank 0).

A "step" is one solveIPCStep of the pile scene: 64 cubes of 0.2 m (12^3
cells, 6 tets per cell: 663,552 tets, 140,608 vertices) at seeded random
rotations and positions in a 1.5 m box, dropped into a static open box,
Neo-Hookean E ~ U[5e4, 5e5], nu 0.4, friction 0.2, dt = 0.01 s, relative dhat
1e-3, Newton threshold 1e-2 (the reference's parameterSetting.txt value).
Inputs are synthetic (the reference's benchmark scenes are not in its
repository); the meshes are generated here with the sizes the configuration
states.

  value    steps/s over all ranks, device time from CUDA events on the
           library's stream, state resident in HBM; L2 is flushed (256 MiB
           write) before every timed step.
  e2e      same metric through the C ABI with host buffers, on the same
           frames (the simulator returns to its state at the first timed
           frame, kept in pinned host memory): every step uploads x, v,
           V_prev, x_tilde from pinned host memory and reads x and v back;
           wall clock around the calls.
  roofline achieved bandwidth of the dominant kernel, the persistent PCG
           solve: algorithmic bytes per launch (iterations x bytes per
           iteration) / launch time, both from the timed region (CUDA events
           on the library's stream around every launch).
The learned preconditioner is trained online on the Newton systems of the
first --train-steps steps (Adam on the GPU, not timed), then frozen.  Timing
starts after --settle-steps untimed steps and the warm-up (pile: 30, the
lower layers of cubes rest on the box and on each other; cloth: 40, the
cloth has reached the cube), so the timed steps are in contact.  The same
run also times the plain FP64 block-Jacobi GPU path on the same frames, from
the same state (restored from pinned host memory).
Multi-GPU: replicas only (one independent simulation per rank, weak scaling).

--scene twist measures the large twist (configuration 5: 1,011,840 tets,
both caps rotated through animated Dirichlet conditions) from its first step.
--scene cloth_drape measures the cloth-drape configuration instead: a
128x128-vertex 1 m cloth (32,258 triangles, Baraff-Witkin membrane +
quadratic bending, friction 0.3) 0.1 m above a fixed 0.5 m tetrahedral cube
(10^3 cells), dt = 0.005 s.

--impl reference times the reference's CPU path on the host cores.  The
reference itself cannot be compiled here (Eigen, oneTBB, oneMKL and
SuiteSparse are absent), so its FP64 restatement (oracle/) stands in, with
the reference's default linear solver, PARDISO, restated as a parallel
multifrontal Cholesky under a nested-dissection ordering.  Both CPU legs
start from the oracle's own state at the first timed frame of the GPU arm
(oracle/states/, settle + warm-up steps; or at the last settle step, then the
warm-up), so they time the same frames as the GPU arm.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "cpu-ipc_b200"))

METRIC = "sim steps/s mixed+learned-PCG vs plain FP64 GPU at same residual; ms/Newton it"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scene", default="pile", choices=["cloth_drape", "pile", "twist"])
    ap.add_argument("--cloth", type=int, default=128)
    ap.add_argument("--pile-cubes", type=int, default=64)
    ap.add_argument("--pile-cells", type=int, default=12)
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--precond", default="learned", choices=["jacobi", "learned", "fsai"])
    ap.add_argument("--settle-steps", type=int, default=None, help="untimed steps before warm-up (pile 30, cloth 40: in contact)")
    ap.add_argument("--train-steps", type=int, default=None, help="settle steps whose last Newton system trains the network (default: all)")
    ap.add_argument("--train-iters", type=int, default=60)
    ap.add_argument("--no-plain", action="store_true", help="skip timing the plain FP64 block-Jacobi path")
    ap.add_argument("--roofline-kernel", default="pcg")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-timed", action="store_true",
                    help="bracket the device-timed steps with cudaProfilerStart/Stop (for ncu --profile-from-start off)")
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    a = ap.parse_args()
    if a.settle_steps is None:
        a.settle_steps = {"pile": 30, "cloth_drape": 40, "twist": 0}[a.scene]
    if a.train_steps is None:
        a.train_steps = a.settle_steps
    return a


def make_scene(args, cipc):
    if args.scene == "pile":
        return cipc.scene_pile(args.pile_cubes, args.pile_cells)
    if args.scene == "twist":
        return cipc.scene_twist(16, 64, 170)
    return cipc.scene_cloth_drape(args.cloth, 10)


def workload(args):
    """Name of the measured workload (the same string on both arms)."""
    if args.scene == "pile":
        return f"pile_{args.pile_cubes}x{args.pile_cells}"
    if args.scene == "twist":
        return "twist_16x64x170"
    return f"cloth_drape_{args.cloth}"


def describe(args):
    if args.scene == "twist":
        return ("cylinder of radius 0.1 m and length 1 m, 16 radial x 64 angular x 170 axial layers, wedge-split (1,011,840 tets, "
                "175,275 vertices), both end caps Dirichlet-rotated opposite ways at 2 pi rad/s, no gravity; Neo-Hookean E=1e5, nu=0.45, "
                "friction 0.1, dt=0.01, relative dhat 1e-3")
    if args.scene == "pile":
        n, c = args.pile_cubes, args.pile_cells
        return (f"{n} cubes of 0.2 m ({c}^3 cells x 6 tets each, {n * 6 * c ** 3} tets, {n * (c + 1) ** 3} vertices) "
                "at seeded random rotations and positions in a 1.5 m box, dropped into a static open box; "
                "Neo-Hookean E ~ U[5e4, 5e5], nu=0.4, friction 0.2, dt=0.01, relative dhat 1e-3")
    return (f"{args.cloth}x{args.cloth}-vertex 1 m cloth ({2 * (args.cloth - 1) ** 2} tris, BW membrane E=1e4, "
            "quadratic bending k_b=1e-3, friction 0.3) 0.1 m above a fixed 0.5 m tet cube (10^3 cells x 6 tets), dt=0.005, relative dhat 1e-3")


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            out, _ = self.p.communicate(timeout=5)
        except Exception:
            self.p.kill()
            out, _ = self.p.communicate()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1])); mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(workload_name):
    """DRAM bytes (read + write) of one launch of the PCG kernel on this
    workload from an ncu capture (profiles/roofline_traffic.json), or None."""
    p = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    if os.path.exists(p):
        d = json.load(open(p)).get(workload_name)
        if d:
            return d.get("bytes_per_launch")
    return None


def spmv_bytes(counts, mixed):
    """Algorithmic bytes of one SpMV launch: every static and contact block and
    its column index once, row pointers, the diagonal extras, x and y once."""
    nv, nnzb, ndyn = counts[0], counts[7], counts[8]
    blk = 36 if mixed else 72
    return nnzb * (blk + 4) + (nv + 1) * 4 + ndyn * (blk + 4) + 2 * nv * 4 + nv * (72 + 24 + 24)


def pcg_iteration_bytes(counts, mixed, factor):
    """Algorithmic bytes of one PCG iteration, as the survey's measurement
    section defines them: every static and contact block of A with its
    column index once (full symmetric storage: 36 B FP32 or 72 B FP64 + 4),
    the row pointers, eight vectors of 3 FP32 per vertex, and the 3x3
    preconditioner block per vertex (block-Jacobi inverse, or the factor's
    scaling S).  A factor adds its blocks once: the static part as stored for
    the streaming kernel (FP16, both the lower and the transposed part, 18 B
    + 4 B column; the diagonal in both) and the contact part (FP32, 36 + 4)."""
    nv, nnzb, ndyn = counts[0], counts[7], counts[8]
    blk = 36 if mixed else 72
    b = (nnzb + ndyn) * (blk + 4) + (nv + 1) * 4 + 8 * nv * 12 + nv * 36
    if factor:
        b += (nnzb + nv) * (18 + 4) + ndyn * (36 + 4)
    return b


# grid barriers per PCG iteration of the pipelined kernel
BARRIERS_PER_ITERATION = {False: 1, True: 3}


def host_threads():
    """Host cores this process may run on (the affinity mask, which a
    container's CPU set narrows; the machine's count where there is none)."""
    try:
        return max(1, len(os.sched_getaffinity(0)))
    except AttributeError:
        return os.cpu_count() or 1


def oracle_at_frame(args, scene, threads, frame):
    """The FP64 oracle on the bench scene, restored from the oracle's own saved
    state (oracle/states/, written by make_contact_state.py) at `frame`, the
    latest saved frame at or before it, or frame 0 when none is saved.
    Returns (oracle, index of the next step)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    o = oracle.Oracle(scene, linear="multifrontal", threads=threads)
    for f in range(frame, 0, -1):
        path = os.path.join(ROOT, "oracle", "states", f"{scene['name']}_frame{f}.npz")
        if os.path.exists(path):
            try:
                return o, o.restore_state(path)
            except ValueError:  # saved from another version of the scene
                break
    return o, 0


def frames(first, n, restored):
    return f"frames {first}-{first + n - 1}" + (" (from the restored contact-phase state)" if restored else " (from the start of the scene)")


def first_timed_frame(args):
    """Index of the GPU arm's first timed step (settle + warm-up steps)."""
    return args.settle_steps + max(3, args.warmup)


def cpu_baseline(args, scene, seconds, steps_cap=50):
    """The FP64 oracle on the same scene and frames, all host cores, bounded
    by time (at least one step)."""
    threads = host_threads()
    o, f0 = oracle_at_frame(args, scene, threads, first_timed_frame(args))
    t0 = time.time()
    n = 0
    while n < steps_cap:
        o.step()
        n += 1
        if time.time() - t0 >= seconds:
            break
    dt = time.time() - t0
    return {"value": n / dt, "unit": "steps/s", "cores": threads, "kind": "port",
            "sample": f"{frames(f0, n, f0 > 0)} of the same scene ({dt:.1f} s, multifrontal Cholesky under nested dissection, {threads} threads)"}


def run_reference(args, world, rank):
    if rank != 0:
        return
    import cipc
    scene = make_scene(args, cipc)
    threads = host_threads()
    first = first_timed_frame(args)
    o, f0 = oracle_at_frame(args, scene, threads, first)
    budget = 150.0
    w = n = 0
    t1 = time.time()
    try:
        # steps from the restored frame up to the GPU arm's first timed frame
        # (none when the state of that frame is saved)
        while f0 + w < first:
            o.step(); w += 1
        t1 = time.time()
        while n < args.steps and (n == 0 or time.time() - t1 < budget):
            o.step(); n += 1
    except RuntimeError as e:
        # the restated reference algorithm itself gave up (its own error message)
        print(json.dumps({"impl": "reference", "unavailable": f"the reference pipeline failed at frame {f0 + w + n}: {e}"}),
              flush=True)
        return
    dt = time.time() - t1
    v = n / dt
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "steps/s", "n_gpus": args.gpus, "steps": n, "warmup": args.warmup,
            "ms_per_step": 1000 * dt / n, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": workload(args), "description": describe(args),
                                            "newton_threshold": scene["params"]["newtonThr"],
                                            "solver": "FP64 CPU restatement of the reference pipeline; linear solve by a parallel multifrontal "
                                                      "Cholesky under nested dissection (the PARDISO algorithm class)",
                                            "timed_frames": f"{f0 + w}-{f0 + w + n - 1}",
                                            "warm_start": (f"restored the oracle's saved state at frame {f0}" if f0 else "frame 0") +
                                                          (f", then {w} untimed steps" if w else "")},
            "cpu_baseline": {"value": v, "unit": "steps/s", "cores": threads, "kind": "port",
                             "sample": f"{frames(f0 + w, n, f0 > 0)}, bounded to {budget:.0f} s; the reference itself does not compile here"},
            "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# host-clock stage timers of IPCStepStats (IPCSolver.cpp:1286-1315), per step
STAGES = ("assemblyMilliseconds", "linearSolveMilliseconds", "ccdMilliseconds", "lineSearchMilliseconds", "postLineSearchMilliseconds")


def max_over_ranks(value, pg, device):
    """The slowest rank's time (all ranks take part; pg None means one rank)."""
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    if pg:
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(steps_per_rank, world, max_ms):
    """Steps per second of the whole job: every rank ran `steps_per_rank`
    independent replica steps; the job took as long as its slowest rank."""
    return world * steps_per_rank / (max_ms / 1000.0)


def mark(what):
    """With CIPC_DEBUG_ALLOC=1 (the library then reports every buffer
    reallocation on stderr), mark the bench's phases on stderr too."""
    if os.environ.get("CIPC_DEBUG_ALLOC") == "1":
        print(f"[bench] {what}", file=sys.stderr, flush=True)


def device_timed(sim, steps, flush, kind, cipc, torch):
    """Device time of `steps` single steps (CUDA events on the library's
    stream), L2 flushed before each; profile of one kernel family."""
    if kind:
        sim.profile(kind, capacity=200000)
    launches0 = cipc.kernel_launches()
    syncs0 = sim.host_syncs()
    total_ms = 0.0
    newton = pcg = 0
    stages = {k: 0.0 for k in STAGES}
    ndyn = []
    step_ms = []
    step_newton = []
    for _ in range(steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        ms, st = sim.timed_steps(1)
        total_ms += ms
        step_ms.append(round(ms, 3))
        step_newton.append(st["newtonIterations"])
        mark(f"step {ms:.1f} ms")
        newton += st["newtonIterations"]
        pcg += st["pcgIterations"]
        for k in STAGES:
            stages[k] += st[k]
        ndyn.append(sim.counts()[8])
    launches = cipc.kernel_launches() - launches0
    syncs = sim.host_syncs() - syncs0
    nprof, prof_ms = sim.profile_read() if kind else (0, 0.0)
    if kind:
        sim.profile(0)
    return dict(ms=total_ms, step_ms=step_ms, step_newton=step_newton, newton=newton, pcg=pcg, ndyn=ndyn, nprof=nprof, prof_ms=prof_ms, launches=launches, syncs=syncs,
                stages={k: v / max(1, steps) for k, v in stages.items()})


def main():
    args = parse()
    world, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference(args, world, rank)
        return
    import torch
    import cipc
    pg = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
        pg = dist
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()
    scene = make_scene(args, cipc)
    learned = args.precond == "learned"
    sim = cipc.Simulator(scene, precision=args.precision, precond=args.precond)
    is_plain = args.precision == "fp64" and args.precond == "jacobi"
    plain = None if (args.no_plain or is_plain) else cipc.Simulator(scene, precision="fp64", precond="jacobi")
    nv = sim.nv
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MiB > 126 MB L2

    # ---- settle into the contact phase (not timed); the learned
    # preconditioner trains online on the Newton systems of these steps
    # (free fall and first contact), then its weights are frozen ----
    train = None
    t0 = time.perf_counter()
    first = last = None
    for k in range(args.settle_steps):
        sim.step()
        if learned and k < args.train_steps:
            a, b = sim.precond_train(args.train_iters, probes=4, lr=2e-3, seed=1000 + k)
            first = a if first is None else first
            last = b
        if plain is not None:
            plain.step()
    torch.cuda.synchronize()
    if learned:
        train = {"steps": min(args.train_steps, args.settle_steps), "adam_iterations_per_step": args.train_iters, "probes": 4, "lr": 2e-3,
                 "loss_first": first, "loss_last": last, "seconds_with_settle_steps": time.perf_counter() - t0}
    for _ in range(max(3, args.warmup)):
        sim.step()
        if plain is not None:
            plain.step()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()

    # the state the timed frames start from, kept in pinned host memory for
    # the end-to-end leg below
    pins = {k: torch.empty((nv, 3), dtype=torch.float64, pin_memory=True).numpy() for k in ("x", "vel", "vprev", "xtilde")}
    for k in pins:
        pins[k][:] = sim.get(k)
    kappa0 = sim.scalars()["kappa"]
    torch.cuda.synchronize()

    # ---- device-timed steps ----
    sampler = ClockSampler(dev)
    sampler.start()
    if args.profile_timed:
        torch.cuda.cudart().cudaProfilerStart()
    fb0 = sim.precond_stats()["fallbacks"]
    mark("timed steps")
    r = device_timed(sim, args.steps, flush, args.roofline_kernel, cipc, torch)
    mark("timed steps done")
    fb_timed = sim.precond_stats()["fallbacks"] - fb0
    if args.profile_timed:
        torch.cuda.cudart().cudaProfilerStop()
    clocks = sampler.stop()
    rp = None
    if plain is not None:
        # the plain path times the same frames from the same state
        for k in ("x", "vel", "vprev", "xtilde"):
            plain.set(k, pins[k])
        plain.set_kappa(kappa0)
        plain.collision_sets()
        mark("plain steps")
        rp = device_timed(plain, args.steps, flush, None, cipc, torch)
        mark("plain steps done")
    max_ms = max_over_ranks(r["ms"], pg, "cuda")
    value = whole_job_rate(args.steps, world, max_ms)

    # ---- end to end through the C ABI with pinned host buffers, on the same
    # frames as the device-timed steps: the simulator goes back to the state
    # it had at the first timed frame (kept in pinned host memory), and the
    # timed frames run again through the host-buffer calls: every step
    # uploads x, v, V_prev and x_tilde and reads x and v back ----
    for k in ("x", "vel", "vprev", "xtilde"):
        sim.set(k, pins[k])
    sim.set_kappa(kappa0)
    sim.collision_sets()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    e2e_steps = args.steps
    dt = scene["params"]["dt"]
    gdt2 = np.array([0.0, -9.8 * dt * dt, 0.0]) if scene["params"].get("apply_gravity", 1) else np.zeros(3)
    t0 = time.perf_counter()
    lib_ms = 0.0
    for _ in range(e2e_steps):
        for k in ("x", "vel", "vprev", "xtilde"):
            sim.set(k, pins[k])
        lib_ms += sim.step()["stepMilliseconds"]
        pins["x"][:] = sim.get("x")
        pins["vel"][:] = sim.get("vel")
        # host-side state of the next step (updateInertialTarget)
        pins["vprev"][:] = pins["x"]
        pins["xtilde"][:] = pins["x"] + pins["vel"] * dt + gdt2
    e2e_s = time.perf_counter() - t0
    e2e_value = whole_job_rate(e2e_steps, world, 1000.0 * max_over_ranks(e2e_s, pg, "cuda"))

    if rank == 0:
        counts = sim.counts()
        counts[8] = int(np.mean(r["ndyn"])) if r["ndyn"] else counts[8]
        peak, peak_kind = measured_peak()
        roof = None
        if r["nprof"] > 0 and args.roofline_kernel == "pcg":
            per_it = pcg_iteration_bytes(counts, args.precision == "mixed", args.precond != "jacobi")
            bytes_ = per_it * r["pcg"] / r["nprof"]
            avg_ms = r["prof_ms"] / r["nprof"]
            achieved = bytes_ / (avg_ms / 1000.0) / 1e9
            iters_per_launch = r["pcg"] / r["nprof"]
            roof = {"kernel": "pcgPipelinedKernel (whole PCG solve, one cooperative launch)", "bound": "hbm", "achieved": achieved,
                    "peak": peak, "peak_source": peak_kind, "unit": "GB/s", "frac": achieved / peak, "traffic": ncu_traffic(workload(args)),
                    "algorithmic_bytes_per_launch": bytes_, "bytes_per_iteration": per_it, "launches": r["nprof"],
                    "mean_launch_us": 1000 * avg_ms, "us_per_iteration": 1000 * avg_ms / max(1e-9, iters_per_launch),
                    "barriers_per_iteration": BARRIERS_PER_ITERATION[args.precond != "jacobi"],
                    "share_of_step_time": r["prof_ms"] / r["ms"]}
        cfg = {"workload": workload(args), "description": describe(args), "newton_threshold": scene["params"]["newtonThr"],
               "precision": args.precision, "preconditioner": args.precond, "pcg_rel_tol": 1e-6,
               "newton_iterations": r["newton"], "pcg_iterations": r["pcg"],
               "ms_per_newton_iteration": max_ms / max(1, r["newton"]), "step_ms": r["step_ms"],
               "step_newton_iterations": r["step_newton"],
               "host_syncs_per_newton_iteration": r["syncs"] / max(1, r["newton"]),
               "kernel_launches_per_newton_iteration": r["launches"] / max(1, r["newton"]),
               "parallelism": f"replicas x{world}", "l2": "flushed (256 MiB write) before every timed step",
               "vertices": nv, "static_blocks": counts[7], "contact_blocks_mean": counts[8]}
        cfg["stage_ms_per_step"] = {k.replace("Milliseconds", ""): round(v, 3) for k, v in r["stages"].items()}
        cfg["timed_frames"] = f"{args.settle_steps + max(3, args.warmup)}-{args.settle_steps + max(3, args.warmup) + args.steps - 1}"
        if train:
            cfg["training"] = train
        if args.precond != "jacobi":
            cfg["factor_fallbacks_timed"] = fb_timed
            cfg["factor_fallbacks_total"] = sim.precond_stats()["fallbacks"]
        if rp is not None:
            plain_v = args.steps / (rp["ms"] / 1000.0)
            cfg["plain_fp64_gpu"] = {"steps_per_s": plain_v, "ms_per_newton_iteration": rp["ms"] / max(1, rp["newton"]),
                                     "newton_iterations": rp["newton"], "pcg_iterations": rp["pcg"], "step_ms": rp["step_ms"],
                                     "step_newton_iterations": rp["step_newton"],
                                     "speedup_of_this_config": (value / world) / plain_v}
        line = {
            "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": max_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 blocks+SpMV / f64 barrier, CCD, energy" if args.precision == "mixed" else "f64",
            "data": "synthetic",
            "config": cfg,
            "roofline": roof,
            "e2e": {"value": e2e_value, "unit": "steps/s", "h2d_bytes_per_step": 4 * 24 * nv, "d2h_bytes_per_step": 2 * 24 * nv,
                    "steps": e2e_steps, "library_step_ms": lib_ms / e2e_steps, "wall_ms_per_step": 1000 * e2e_s / e2e_steps},
            "gpu_launches": int(r["launches"]),
            "clocks": clocks,
        }
        if not args.no_cpu_baseline and world == 1:
            try:
                line["cpu_baseline"] = cpu_baseline(args, scene, args.cpu_seconds)
            except Exception as e:
                line["cpu_baseline"] = {"error": str(e)}
        print(json.dumps(line), flush=True)
    sim.close()
    if plain is not None:
        plain.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
