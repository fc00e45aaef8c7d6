#!/usr/bin/env python3
"""Benchmark of the B200-native FLIP step (betajippity/Ariel's FlipSim::Step).

Workload (the headline configuration): the 128^3 synthetic dam break -- liquid block
x in [0,.4], y in [0,.6], z in [0,1] seeded at 8 particles per cell with seeded in-sub-cell
jitter (4,021,248 particles), gravity -9.8 y, dt = 1/240, FLIP/PIC 0.95, reference
preconditioner, MIXED-precision pressure solve (fp32 inner PCG inside fp64 iterative
refinement) to a 1e-5 relative residual.  One "step" is one full FLIP step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Our arm prints one JSON line: device throughput (`value`, inputs resident in HBM, CUDA events
around exactly K graph-replayed steps, max over ranks), the same metric end to end through
the C ABI with host buffers (`e2e`), per-stage device times, PCG ms/solve beside the plain
FP64 GPU path, p50/p99 step latency, the solve kernel's roofline, clocks, and the CPU
oracle's throughput on a bounded sample (`cpu_baseline`).  `--impl reference` times the CPU
restatement of the reference step (the reference itself cannot be built here) on the same
workload.  Multi-GPU runs are independent replicas (one scene per GPU, no data-path
collective); only timing scalars cross ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# Algorithmic bytes of the persistent pressure-solve kernel per FLUID cell (unique bytes each
# phase must move; see the solve section of the design notes).
PCG_BYTES_PER_CELL_ITER = {"fp64": 113.0, "mixed": 65.0, "ref32": 61.0}
PCG_BYTES_PER_CELL_OUTER = {"fp64": 69.0 + 16.0, "mixed": 89.0, "ref32": 35.0}
STAGE_NAMES = ["begin", "sort", "density", "forces", "p2g", "classify", "boundary_div", "solve",
               "gradient", "extrapolate", "g2p_advect", "resample"]


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def pin_device(local_rank, world):
    """One GPU per rank: restrict this process to its GPU before the CUDA library loads."""
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if world > 1:
        ids = vis.split(",") if vis else [str(i) for i in range(64)]
        os.environ["CUDA_VISIBLE_DEVICES"] = ids[local_rank]
    return os.environ.get("CUDA_VISIBLE_DEVICES", "0").split(",")[0]


class ClockSampler:
    """nvidia-smi clock / throttle-reason sampling while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.path = os.path.join("/tmp", "ariel_clocks_%d_%s.csv" % (os.getpid(), gpu))

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), parts[5:9]))
            except ValueError:
                continue
        try:
            os.remove(self.path)
        except OSError:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, r in rows for i, v in enumerate(r) if v.lower().startswith("active")})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def load_traffic(workload):
    """DRAM bytes per launch of the solve kernel from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as f:
            return json.load(f).get(workload)
    except Exception:
        return None


def make_params(A, precision, tol, timing=1, graph=1):
    p = A.params_default()
    p.precision = precision
    p.precond = A.PRECOND_REF
    p.stop_rule = A.STOP_REL
    p.tol = tol
    p.use_graph = graph
    p.timing = timing
    return p


def run_gpu_pass(A, Batch, desc, prm, steps, warmup, sampler=None, barrier=None):
    b = Batch([desc], prm)
    b.init()
    b.step(warmup)
    b.synchronize()
    b.timing_reset()
    launches0 = b.L.ariel_kernel_launches()
    if barrier:
        barrier()
    if sampler:
        sampler.start()
    b.timer_begin()
    b.step(steps)
    ms = b.timer_end()
    if sampler:
        clocks = sampler.stop()
    else:
        clocks = None
    launches = b.L.ariel_kernel_launches() - launches0
    tim = b.timing(max_steps=steps)
    tot = b.solver_totals()
    st = b.stats()
    return b, dict(ms=ms, timing=tim, totals=tot, stats=st, clocks=clocks, launches=launches,
                   np=b.count())


def run_e2e(b, steps):
    """Same metric through the public API with host buffers: every step uploads the particle
    state from pinned host memory, steps, and reads the new state back."""
    import numpy as np
    n = b.count()
    try:
        import torch
        pos_t = torch.empty((n, 3), dtype=torch.float32, pin_memory=True)
        vel_t = torch.empty((n, 3), dtype=torch.float32, pin_memory=True)
        pos, vel = pos_t.numpy(), vel_t.numpy()
        pinned = True
    except Exception:
        pos = np.empty((n, 3), np.float32)
        vel = np.empty((n, 3), np.float32)
        pinned = False
    b.download_state(pos, vel)
    b.synchronize()
    b.timer_begin()
    for _ in range(steps):
        b.upload_state(pos, vel)
        b.step(1)
        b.download_state(pos, vel)
    ms = b.timer_end()
    return ms, 24 * n, 24 * n, pinned


def cpu_baseline_sample(A, desc, tol, faithful=True, max_steps=1):
    """The CPU restatement of the reference step (oracle/, reference-faithful parallel
    granularity) on the same workload: one step from Init, wall clock on this host's cores."""
    from oracle.pyoracle import RefSim, lib as olib
    prm = make_params(A, A.PREC_REF32, tol, timing=0, graph=0)
    r = RefSim(desc, prm, faithful=faithful)
    r.init()
    n = r.count()
    t0 = time.perf_counter()
    r.step(max_steps)
    dt = time.perf_counter() - t0
    cores = olib().ariel_ref_max_threads()
    st = r.stats()
    r.close()
    return n, dt, cores, st


def reference_arm(args, A, ws, rank):
    if rank != 0:
        return 0
    desc = A.scene_dambreak(args.n, seed=1)
    from oracle.pyoracle import RefSim, lib as olib
    prm = make_params(A, A.PREC_REF32, args.tol, timing=0, graph=0)
    r = RefSim(desc, prm, faithful=True)
    r.init()
    n = r.count()
    budget = args.ref_budget_s
    done, t_total = 0, 0.0
    # the CPU needs no warm-up; each timed step is a full FLIP step of the workload, run until
    # K steps or the time budget, whichever comes first
    while done < args.steps:
        t0 = time.perf_counter()
        r.step(1)
        t_total += time.perf_counter() - t0
        done += 1
        if t_total >= budget:
            break
    cores = olib().ariel_ref_max_threads()
    value = n * done / t_total
    sample = ("%d of %d FLIP steps of the %d^3 dam break (%d particles) from Init, reference-faithful "
              "OpenMP granularity, %.1f s" % (done, args.steps, args.n, n, t_total))
    line = {
        "impl": "reference", "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s",
        "n_gpus": ws, "steps": done, "warmup": 0, "ms_per_step": 1000.0 * t_total / done,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": config_dict(args, n, ws),
        "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": cores, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def config_dict(args, n_particles, ws):
    return {"workload": "dam break %d^3, %d particles per scene, mixed-precision PCG to %g relative residual"
            % (args.n, n_particles, args.tol),
            "grid": args.n, "particles_per_scene": n_particles, "scenes": ws, "precision": args.precision,
            "preconditioner": "reference (solver.inl:104-135)", "tolerance": args.tol, "dt": 1.0 / 240.0,
            "parallelism": "replicas" if ws > 1 else "single",
            "l2": "inputs larger than L2 (particle state %.0f MB)" % (n_particles * 64 / 1e6)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=128, help="grid size (the headline workload is 128)")
    ap.add_argument("--precision", choices=["mixed", "fp64", "ref32"], default="mixed")
    ap.add_argument("--tol", type=float, default=1e-5)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-fp64-compare", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-budget-s", type=float, default=150.0)
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3

    ws, rank, local = dist_env()
    gpu_index = pin_device(local, ws)
    from ariel_b200 import _abi as A
    from ariel_b200.flipsim import Batch
    from ariel_b200.replicas import aggregate, replica_seed

    pg = None
    if ws > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
        pg = dist
    if args.impl == "reference":
        rc = reference_arm(args, A, ws, rank)
        if pg:
            pg.destroy_process_group()
        return rc

    prec = {"mixed": A.PREC_MIXED, "fp64": A.PREC_FP64, "ref32": A.PREC_REF32}[args.precision]
    desc = A.scene_dambreak(args.n, seed=replica_seed(rank))
    barrier = (lambda: pg.barrier()) if pg else None
    sampler = ClockSampler(gpu_index)
    b, res = run_gpu_pass(A, Batch, desc, make_params(A, prec, args.tol), args.steps, args.warmup, sampler, barrier)

    n_local = res["np"]
    ms, total_particles = aggregate(res["ms"], n_local, pg)
    value = total_particles * args.steps / (ms / 1000.0)

    tim = res["timing"]
    tot = res["totals"]
    nsteps = max(tim["steps"], 1)
    stage_ms = {STAGE_NAMES[i]: tim["stage_ms"][i] / nsteps for i in range(len(STAGE_NAMES))}
    step_list = sorted(tim["step_ms"])
    p50 = statistics.median(step_list) if step_list else None
    p99 = step_list[min(len(step_list) - 1, int(round(0.99 * (len(step_list) - 1))))] if step_list else None
    solve_ms = tim["solve_kernel_ms"] / max(tot.solves, 1)
    key = args.precision
    alg_bytes = (tot.cell_iterations * PCG_BYTES_PER_CELL_ITER[key] +
                 tot.cell_outer * PCG_BYTES_PER_CELL_OUTER[key]) / max(tot.solves, 1)
    peak, peak_kind = load_peaks()
    achieved = alg_bytes / (solve_ms / 1000.0) / 1e9 if solve_ms > 0 else None
    workload_key = "pcg_%s_%d" % (args.precision, args.n)
    traffic = load_traffic(workload_key)
    roofline = {"kernel": "k_pcg<%s> (persistent pressure solve)" % args.precision, "bound": "hbm",
                "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None, "peak_source": peak_kind,
                "traffic": traffic, "algorithmic_bytes_per_launch": alg_bytes,
                "avg_launch_ms": solve_ms,
                "note": "frac of %s HBM copy bandwidth; working set is L2-resident at this size" % peak_kind}

    out = {
        "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": config_dict(args, n_local, ws),
        "stage_ms": stage_ms, "step_ms_p50": p50, "step_ms_p99": p99,
        "pcg": {"ms_per_solve": solve_ms, "iterations_per_solve": tot.iterations / max(tot.solves, 1),
                "outer_per_solve": tot.outer / max(tot.solves, 1), "not_converged": tot.not_converged,
                "final_rel_residual": res["stats"].pcg_rel_residual},
        "roofline": roofline, "clocks": res["clocks"], "gpu_launches": res["launches"],
    }

    if not args.no_e2e:
        e2e_ms, h2d, d2h, pinned = run_e2e(b, args.steps)
        e_ms, _ = aggregate(e2e_ms, n_local, pg)
        out["e2e"] = {"value": total_particles * args.steps / (e_ms / 1000.0), "unit": "particle-steps/s",
                      "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "pinned": pinned,
                      "api": "ariel_upload_state + ariel_step + ariel_download_state"}
    b.close()

    if not args.no_fp64_compare and args.precision != "fp64":
        b64, r64 = run_gpu_pass(A, Batch, desc, make_params(A, A.PREC_FP64, args.tol), args.steps, args.warmup)
        b64.close()
        t64 = r64["totals"]
        solve64 = r64["timing"]["solve_kernel_ms"] / max(t64.solves, 1)
        out["pcg"]["fp64_plain"] = {"ms_per_solve": solve64, "iterations_per_solve": t64.iterations / max(t64.solves, 1),
                                    "particle_steps_per_s": r64["np"] * args.steps / (r64["ms"] / 1000.0)}
        out["pcg"]["speedup_vs_fp64"] = solve64 / solve_ms if solve_ms > 0 else None
        # per-GPU ratio of this rank's mixed pass to its plain FP64 pass
        out["throughput_vs_fp64"] = r64["ms"] / res["ms"] if res["ms"] > 0 else None

    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        n, dt, cores, st = cpu_baseline_sample(A, desc, args.tol)
        out["cpu_baseline"] = {"value": n / dt, "unit": "particle-steps/s", "cores": cores, "kind": "port",
                               "sample": "1 FLIP step (from Init) of the same %d^3 dam break, %d particles, "
                                         "reference-faithful OpenMP granularity, fp32 PCG to %g relative "
                                         "(%d iterations), %.1f s" % (args.n, n, args.tol, st.pcg_iterations, dt)}
    if rank == 0:
        print(json.dumps(out), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
