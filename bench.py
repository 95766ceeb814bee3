"""Benchmark of the GPU IPC time step (one JSON line on rank 0).

A "step" is one solveIPCStep of the cloth-drape scene: a 128x128-vertex 1 m
cloth (32,258 triangles, Baraff-Witkin membrane + quadratic bending,
self-contact, friction 0.3) 0.1 m above a fixed 0.5 m tetrahedral cube
(10^3 cells, 6 tets per cell), dt = 0.005 s.  Inputs are synthetic (the
reference's benchmark scenes are not in its repository); the mesh is
generated here with the sizes the configuration states.

  value    steps/s over all ranks, device time from CUDA events on the
           library's stream, state resident in HBM; L2 is flushed (256 MiB
           write) before every timed step.
  e2e      same metric through the C ABI with host buffers: every step
           uploads x, v, V_prev, x_tilde from pinned host memory and reads x
           and v back; wall clock around the calls.
  roofline achieved HBM bandwidth of the dominant kernel (PCG SpMV):
           algorithmic bytes per launch / mean launch time, both measured
           in the timed region.
Multi-GPU: replicas only (one independent simulation per rank, weak scaling).

--impl reference times the reference's CPU path on the host cores.  The
reference itself cannot be compiled here (Eigen, oneTBB, oneMKL and
SuiteSparse are absent), so its FP64 restatement (oracle/) stands in.
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
    ap.add_argument("--cloth", type=int, default=128)
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--precond", default="jacobi", choices=["jacobi", "learned"])
    ap.add_argument("--roofline-kernel", default="spmv")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    return ap.parse_args()


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


def ncu_traffic(kernel):
    p = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    if os.path.exists(p):
        d = json.load(open(p)).get(kernel)
        if d:
            return d.get("bytes_per_launch")
    return None


def spmv_bytes(counts, mixed):
    """Algorithmic bytes of one SpMV launch: every static and contact block and
    its column index once, row pointers, the diagonal extras, x and y once."""
    nv, nnzb, ndyn = counts[0], counts[7], counts[8]
    blk = 36 if mixed else 72
    return nnzb * (blk + 4) + (nv + 1) * 4 + ndyn * (blk + 4) + 2 * nv * 4 + nv * (72 + 24 + 24)


def cpu_baseline(scene, seconds, steps_cap=50):
    """The FP64 oracle on the same scene, all host cores, bounded by time."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    threads = os.cpu_count() or 1
    o = oracle.Oracle(scene, linear="pcg", threads=threads)
    t0 = time.time()
    n = 0
    while n < steps_cap:
        o.step()
        n += 1
        if time.time() - t0 >= seconds:
            break
    dt = time.time() - t0
    return {"value": n / dt, "unit": "steps/s", "cores": threads, "kind": "port",
            "sample": f"first {n} steps of the same scene ({dt:.1f} s, block-Jacobi PCG at 1e-6, {threads} threads)"}


def run_reference(args, world, rank):
    if rank != 0:
        return
    import cipc
    scene = cipc.scene_cloth_drape(args.cloth, 10)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    threads = os.cpu_count() or 1
    o = oracle.Oracle(scene, linear="pcg", threads=threads)
    budget = 150.0
    t0 = time.time()
    w = 0
    while w < args.warmup and time.time() - t0 < budget / 4:
        o.step(); w += 1
    t1 = time.time()
    n = 0
    while n < args.steps and (n == 0 or time.time() - t1 < budget):
        o.step(); n += 1
    dt = time.time() - t1
    v = n / dt
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "steps/s", "n_gpus": args.gpus, "steps": n, "warmup": w,
            "ms_per_step": 1000 * dt / n, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": f"cloth_drape_{args.cloth} (cloth {args.cloth}x{args.cloth} + 10^3-cell tet cube)",
                                            "solver": "FP64 CPU restatement of the reference pipeline, block-Jacobi PCG 1e-6"},
            "cpu_baseline": {"value": v, "unit": "steps/s", "cores": threads, "kind": "port",
                             "sample": f"{n} steps after {w} warm-up steps; the reference itself does not compile here"},
            "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


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
    scene = cipc.scene_cloth_drape(args.cloth, 10)
    sim = cipc.Simulator(scene, precision=args.precision, precond=args.precond)
    nv = sim.nv
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MiB > 126 MB L2

    for _ in range(max(3, args.warmup)):
        sim.step()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()

    # ---- device-timed steps ----
    sampler = ClockSampler(dev)
    sampler.start()
    sim.profile(args.roofline_kernel, capacity=200000)
    launches0 = cipc.kernel_launches()
    total_ms = 0.0
    newton = pcg = 0
    ndyn = []
    for _ in range(args.steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        ms, st = sim.timed_steps(1)
        total_ms += ms
        newton += st["newtonIterations"]
        pcg += st["pcgIterations"]
        ndyn.append(sim.counts()[8])
    launches = cipc.kernel_launches() - launches0
    nprof, prof_ms = sim.profile_read()
    sim.profile(0)
    clocks = sampler.stop()
    t = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
    if pg:
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
    max_ms = float(t.item())
    value = world * args.steps / (max_ms / 1000.0)

    # ---- end to end through the C ABI with pinned host buffers ----
    pins = {k: torch.empty((nv, 3), dtype=torch.float64, pin_memory=True).numpy() for k in ("x", "vel", "vprev", "xtilde")}
    for k in pins:
        pins[k][:] = sim.get(k)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    e2e_steps = max(3, min(args.steps, 10))
    dt = scene["params"]["dt"]
    gdt2 = np.array([0.0, -9.8 * dt * dt, 0.0])
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        for k in ("x", "vel", "vprev", "xtilde"):
            sim.set(k, pins[k])
        sim.step()
        pins["x"][:] = sim.get("x")
        pins["vel"][:] = sim.get("vel")
        # host-side state of the next step (updateInertialTarget)
        pins["vprev"][:] = pins["x"]
        pins["xtilde"][:] = pins["x"] + pins["vel"] * dt + gdt2
    e2e_s = time.perf_counter() - t0
    te = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
    if pg:
        pg.all_reduce(te, op=pg.ReduceOp.MAX)
    e2e_value = world * e2e_steps / float(te.item())

    if rank == 0:
        counts = sim.counts()
        counts[8] = int(np.mean(ndyn)) if ndyn else counts[8]
        peak, peak_kind = measured_peak()
        roof = None
        if nprof > 0 and args.roofline_kernel == "spmv":
            avg_ms = prof_ms / nprof
            bytes_ = spmv_bytes(counts, args.precision == "mixed")
            achieved = bytes_ / (avg_ms / 1000.0) / 1e9
            roof = {"kernel": "spmvKernel (PCG SpMV)", "bound": "hbm", "achieved": achieved, "peak": peak, "peak_source": peak_kind,
                    "unit": "GB/s", "frac": achieved / peak, "traffic": ncu_traffic("spmv"), "algorithmic_bytes_per_launch": bytes_,
                    "launches": nprof, "mean_launch_us": 1000 * avg_ms}
        line = {
            "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": max_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 blocks+SpMV / f64 barrier, CCD, energy" if args.precision == "mixed" else "f64",
            "data": "synthetic",
            "config": {"workload": f"cloth_drape_{args.cloth}: {args.cloth}x{args.cloth}-vertex 1 m cloth "
                                   f"({2 * (args.cloth - 1) ** 2} tris, BW membrane E=1e4, quadratic bending k_b=1e-3, mu=0.3) "
                                   "0.1 m above a fixed 0.5 m tet cube (10^3 cells x 6 tets), dt=0.005, dhat=1e-3",
                       "precision": args.precision, "preconditioner": args.precond, "pcg_rel_tol": 1e-6,
                       "newton_iterations": newton, "pcg_iterations": pcg,
                       "ms_per_newton_iteration": max_ms / max(1, newton),
                       "parallelism": f"replicas x{world}", "l2": "flushed (256 MiB write) before every timed step",
                       "vertices": nv, "static_blocks": counts[7], "contact_blocks_mean": counts[8]},
            "roofline": roof,
            "e2e": {"value": e2e_value, "unit": "steps/s", "h2d_bytes_per_step": 4 * 24 * nv, "d2h_bytes_per_step": 2 * 24 * nv},
            "gpu_launches": int(launches),
            "clocks": clocks,
        }
        if not args.no_cpu_baseline and world == 1:
            try:
                line["cpu_baseline"] = cpu_baseline(scene, args.cpu_seconds)
            except Exception as e:
                line["cpu_baseline"] = {"error": str(e)}
        print(json.dumps(line), flush=True)
    sim.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
