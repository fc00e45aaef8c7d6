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
the C ABI with host buffers (`e2e`), per-stage device times and their HBM fractions, PCG
ms/solve beside the plain FP64 GPU path, p50/p99 step latency, the solve kernel's roofline,
clocks, the batched 64-scene workload beside the plain FP64 path (`batch`), and the reference
CPU step's throughput on a bounded sample (`cpu_baseline`).  `--impl reference` times the
reference's own FlipSim::Step, compiled from its sources into oracle/_ref with TBB's parallel_for
spread over the host's threads, on the same workload in the reference's own configuration (the
oracle's restatement when that build is absent).  Multi-GPU runs are independent replicas (one scene per GPU, no data-path
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

# Algorithmic bytes of the persistent pressure-solve kernel per FLUID cell: the unique bytes each
# phase must move (a neighbour's value is its owner's bytes, counted once; the cell records of
# the bench workloads' first chunks stay in shared memory).
#   inner CG iteration (single-reduction path): read packed Av (r, w, s, pc) and packed Bv
#   (p, x), write both: MIXED 16 + 8 + 16 + 8 = 48, FP64 32 + 16 + 32 + 16 = 96.
#   refinement sweep: residual (read P64, D; write r: 8 + 4 + 8), setup (read r, pc; write Av,
#   Bv) and fold (read Bv [, P64]; write P64): MIXED 20 + 36 + 24 = 80, FP64 20 + 64 + 24 = 108.
#   REF32 (the reference's two-reduction PCG): 61 per iteration, 35 per solve.
PCG_BYTES_PER_CELL_ITER = {"fp64": 96.0, "mixed": 48.0, "ref32": 61.0}
PCG_BYTES_PER_CELL_OUTER = {"fp64": 108.0, "mixed": 80.0, "ref32": 35.0}
# The fixed per-unit figures the roofline is reported on (bytes per FLUID cell per CG iteration of
# a two-reduction PCG: SpMV 21 + two axpys 48 + diagonal preconditioner 20 + s-update 24 = 113 in
# fp64, 61 with fp32 vectors); refinement sweeps as above.
PCG_SPEC_BYTES_PER_CELL_ITER = {"fp64": 113.0, "mixed": 61.0, "ref32": 61.0}
# Per-stage algorithmic bytes per particle and per cell (fp32 state): sort 64/p + 8/c (offsets);
# density 16/p; forces 32/p; P2G 24/p + 24/c (current and previous faces); classify 5/c;
# boundary + divergence 16/c; gradient 33/c; extrapolate 25/c + the FLIP delta 36/c; G2P + blend +
# advect 48/p; resampling 48/p plus its own sort.
STAGE_BYTES = {"sort": (64.0, 8.0), "density": (16.0, 0.0), "forces": (32.0, 0.0), "p2g": (24.0, 24.0),
               "classify": (0.0, 5.0), "boundary_div": (0.0, 16.0), "gradient": (0.0, 33.0),
               "extrapolate": (0.0, 61.0), "g2p_advect": (48.0, 0.0), "resample": (112.0, 8.0)}
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
    path = os.path.join(ROOT, "profiles", "traffic.txt")
    try:
        with open(path) as f:
            for line in f:
                parts = line.split()
                if len(parts) >= 2 and not line.startswith("#") and parts[0] == workload:
                    return int(parts[1])
    except Exception:
        pass
    return None


PRECOND = "ref"
INNER_TOL = 0.0


def make_params(A, precision, tol, timing=1, graph=1, resample_every=1, reseed_every=0):
    p = A.params_default()
    p.precision = precision
    p.precond = A.PRECOND_MIC0 if PRECOND == "mic0" else A.PRECOND_REF
    p.stop_rule = A.STOP_REL
    p.tol = tol
    p.use_graph = graph
    p.timing = timing
    p.resample_every = resample_every
    p.reseed_every = reseed_every  # bounds: the library's defaults, 6 and 10 particles per cell
    if INNER_TOL > 0:
        p.inner_tol = INNER_TOL
    return p


def run_gpu_pass(A, Batch, desc, prm, steps, warmup, sampler=None, barrier=None):
    descs = desc if isinstance(desc, list) else [desc]
    b = Batch(descs, prm)
    b.init()
    if sampler:
        # nvidia-smi needs a moment to start; the warm-up steps keep the GPU loaded meanwhile
        sampler.start()
    b.step(warmup)
    b.synchronize()
    b.timing_reset()
    launches0 = b.L.ariel_kernel_launches()
    if barrier:
        barrier()
    b.timer_begin()
    b.step(steps)
    ms = b.timer_end()
    if sampler:
        clocks = sampler.stop()
    else:
        clocks = None
    launches = b.L.ariel_kernel_launches() - launches0
    tim = b.timing(max_steps=steps)
    tots = [b.solver_totals(i) for i in range(b.k)]
    tot = tots[0]
    if b.k > 1:
        # batch totals: solves are simultaneous, so count one solve per step
        for name in ("iterations", "outer", "cell_iterations", "cell_outer", "not_converged"):
            setattr(tot, name, sum(getattr(t, name) for t in tots))
        tot.solves = tots[0].solves
    st = b.stats()
    return b, dict(ms=ms, timing=tim, totals=tot, stats=st, clocks=clocks, launches=launches,
                   np=sum(b.count(i) for i in range(b.k)))


def run_e2e(b, steps):
    """Same metric through the public API with host buffers: every step uploads the particle
    state of every scene from pinned host memory, steps, and reads the new state back."""
    import numpy as np
    bufs, pinned, total = [], True, 0
    for i in range(b.k):
        n = b.count(i)
        total += n
        try:
            import torch
            pos = torch.empty((n, 3), dtype=torch.float32, pin_memory=True).numpy()
            vel = torch.empty((n, 3), dtype=torch.float32, pin_memory=True).numpy()
        except Exception:
            pos = np.empty((n, 3), np.float32)
            vel = np.empty((n, 3), np.float32)
            pinned = False
        b.download_state(pos, vel, i)
        bufs.append((pos, vel))
    b.synchronize()
    b.timer_begin()
    for _ in range(steps):
        for i, (pos, vel) in enumerate(bufs):
            b.upload_state(pos, vel, i)
        b.step(1)
        for i, (pos, vel) in enumerate(bufs):
            b.download_state(pos, vel, i)
    ms = b.timer_end()
    return ms, 24 * total, 24 * total, pinned


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


def fp64_oracle_error(A, Batch, b, desc, tols=(1e-5, 1e-7)):
    """Error of the MIXED solve against a tight FP64 CPU solve (the oracle, as the checker) on the
    bench's own last pressure system (flags, liquid SDF and divergence of its final step), each
    tolerance solved from a zero start: |P - P*| / |P*| over FLUID cells."""
    import numpy as np
    from oracle.pyoracle import solve_fp64
    n = desc.dim
    flags, L, D = b.get_grid(A.GRID_A), b.get_grid(A.GRID_L), b.get_grid(A.GRID_D)
    fl = flags == A.FLUID
    t0 = time.perf_counter()
    xstar, it, rel = solve_fp64(n, flags, L, D.astype(np.float64).ravel(), tol=1e-12)
    out = {"oracle": {"tol": 1e-12, "iterations": it, "rel_residual": rel, "seconds": time.perf_counter() - t0},
           "fluid_cells": int(fl.sum())}
    p = b.get_particles()
    zeros = np.zeros((n, n, n), np.float32)
    for tol in tols:
        g = Batch([desc], make_params(A, A.PREC_MIXED, tol, timing=0, graph=0))
        g.set_particles(p["pos"], p["vel"], p["mass"], p["type"])
        for w, arr in ((A.GRID_A, flags), (A.GRID_L, L), (A.GRID_D, D), (A.GRID_P, zeros)):
            g.set_grid(w, arr)
        g.set_grid(A.GRID_P64, zeros.astype(np.float64))
        g.stage(A.STAGE_SOLVE)
        x = g.get_grid(A.GRID_P64)
        st = g.stats()
        err = float(np.linalg.norm((x - xstar)[fl]) / max(np.linalg.norm(xstar[fl]), 1e-300))
        out["tol_%g" % tol] = {"rel_error": err, "iterations": st.pcg_iterations, "sweeps": st.pcg_outer,
                               "rel_residual": st.pcg_rel_residual}
        g.close()
    return out


def reference_sim(A, desc, rng_seed=0x5EED):
    """The reference's own FlipSim (oracle/_ref, compiled from its sources; TBB's parallel_for on
    all host threads) when that build is present, else None.  Seeded with the oracle's restatement
    of Scene::GenerateParticles (scene.cpp needs meshes and OpenVDB)."""
    try:
        from oracle import pyref
        if not pyref.available("omp"):
            return None
        from oracle.pyoracle import RefSim
        seed = RefSim(desc, pyref.reference_params())
        seed.init()
        st = seed.get_particles()
        seed.close()
        r = pyref.ReferenceSim(desc, rng_seed, variant="omp")
        r.init_with(st)
        return r, len(st["mass"]), pyref.threads("omp")
    except Exception:
        return None


REFERENCE_CONFIG = ("the reference's own configuration: fp32 PCG with its preconditioner to its absolute stop "
                    "rule r.r <= 1e-2 n^3 (solver.inl:289-354), resampling every step")


def reference_arm(args, A, ws, rank):
    if rank != 0:
        return 0
    desc = A.scene_dambreak(args.n, seed=1)
    ref = reference_sim(A, desc)
    budget = args.ref_budget_s
    done, t_total = 0, 0.0
    if ref is not None:
        r, n, cores = ref
        kind = "reference"
        what = "the reference's own FlipSim::Step compiled from its sources (oracle/_ref), " + REFERENCE_CONFIG
    else:
        from oracle.pyoracle import RefSim, lib as olib
        r = RefSim(desc, make_params(A, A.PREC_REF32, args.tol, timing=0, graph=0), faithful=True)
        r.init()
        n = r.count()
        cores = olib().ariel_ref_max_threads()
        kind = "port"
        what = "the oracle's restatement of the reference step, reference-faithful OpenMP granularity"
    # the CPU needs no warm-up; each timed step is a full FLIP step of the workload, run until
    # K steps or the time budget, whichever comes first
    while done < args.steps:
        t0 = time.perf_counter()
        r.step(1)
        t_total += time.perf_counter() - t0
        done += 1
        if t_total >= budget:
            break
    r.close()
    value = n * done / t_total
    sample = ("frames 1-%d (of %d asked) of the %d^3 dam break (%d particles) from Init: %s; %d threads, %.1f s"
              % (done, args.steps, args.n, n, what, cores, t_total))
    cfg = config_dict(args, n, ws)
    cfg["precision"] = "fp32 (the reference's)" if kind == "reference" else "ref32"
    cfg["stop_rule"] = "absolute r.r <= 1e-2 n^3 (solver.inl:322)" if kind == "reference" else "relative %g" % args.tol
    cfg["workload"] = "dam break %d^3, %d particles, %s" % (args.n, n, REFERENCE_CONFIG if kind == "reference"
                                                              else "fp32 PCG to %g relative residual" % args.tol)
    cfg["frames"] = [1, done]
    if kind == "reference":
        cfg["tolerance"] = None
    line = {
        "impl": "reference", "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s",
        "n_gpus": ws, "steps": done, "warmup": 0, "ms_per_step": 1000.0 * t_total / done,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": cfg,
        "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": cores, "kind": kind,
                         "sample": sample},
        "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def mic0_subresult(A, Batch, desc, args):
    """The same workload with the MIC(0) preconditioner (tau 0.97, FP64 factorisation, brick
    wavefront sweeps) in MIXED precision: a few graph-replayed steps."""
    prm = make_params(A, A.PREC_MIXED, args.tol)
    prm.precond = A.PRECOND_MIC0
    b, r = run_gpu_pass(A, Batch, desc, prm, args.mic0_steps, 3)
    t = r["totals"]
    b.close()
    return {"ms_per_solve": r["timing"]["solve_kernel_ms"] / max(t.solves, 1),
            "iterations_per_solve": t.iterations / max(t.solves, 1), "outer_per_solve": t.outer / max(t.solves, 1),
            "not_converged": t.not_converged, "frames": [4, 3 + args.mic0_steps]}


def batch_subresult(A, Batch, args):
    """The batched workload beside the headline: 64 uneven dam-break scenes (grids drawn from
    {32,48,64,96,128}^3), MIXED against the plain FP64 path, a few graph-replayed steps each (step
    and solve ratios)."""
    from ariel_b200 import workloads as W
    descs = W.uneven_batch(args.batch_sub, seed=args.seed)
    res = {}
    for name, prec in (("mixed", A.PREC_MIXED), ("fp64", A.PREC_FP64)):
        b, r = run_gpu_pass(A, Batch, descs, make_params(A, prec, args.tol), args.batch_steps, 3)
        t = r["totals"]
        res[name] = {"ms_per_step": r["ms"] / args.batch_steps,
                     "solve_ms": r["timing"]["solve_kernel_ms"] / max(t.solves, 1),
                     "particle_steps_per_s": r["np"] * args.batch_steps / (r["ms"] / 1000.0)}
        n = r["np"]
        b.close()
    return {"workload": "%d dam-break scenes, grids drawn from {32,48,64,96,128}^3 (seed %d), blocks filling "
                        "20-50%%, %d particles, PCG to %g relative, frames 4-%d"
                        % (args.batch_sub, args.seed, n, args.tol, 3 + args.batch_steps),
            "mixed": res["mixed"], "fp64": res["fp64"],
            "step_speedup_vs_fp64": res["fp64"]["ms_per_step"] / res["mixed"]["ms_per_step"],
            "solve_speedup_vs_fp64": res["fp64"]["solve_ms"] / res["mixed"]["solve_ms"]}


def config_dict(args, n_particles, ws):
    if args.workload == "batch":
        return {"workload": "batched: %d dam-break scenes, grids drawn from {32,48,64,96,128}^3 (seed %d), "
                            "blocks filling 20-50%% of each domain, %d particles in all, %s PCG to %g relative "
                            "residual, one launch per stage over all scenes" % (args.scenes, args.seed, n_particles,
                                                                               args.precision, args.tol),
                "scenes": args.scenes, "seed": args.seed, "particles": n_particles, "precision": args.precision,
                "tolerance": args.tol, "parallelism": "replicas" if ws > 1 else "single",
                "l2": "inputs larger than L2 (particle state %.0f MB)" % (n_particles * 64 / 1e6)}
    if args.workload == "sphere":
        return {"workload": "dam break %d^3 with a static solid sphere (c=(.6,.3,.5), r=.15), %d particles, "
                            "dt 1/480, resampling and reseeding to 6-10 particles per cell every 5 steps, "
                            "%s PCG to %g relative residual"
                            % (args.n, n_particles, args.precision, args.tol),
                "grid": args.n, "particles_per_scene": n_particles, "precision": args.precision,
                "tolerance": args.tol, "parallelism": "replicas" if ws > 1 else "single",
                "l2": "inputs larger than L2 (particle state %.0f MB)" % (n_particles * 64 / 1e6)}
    pname = {"mixed": "mixed-precision", "fp64": "fp64", "ref32": "fp32"}[args.precision]
    return {"workload": "dam break %d^3, %d particles per scene, %s PCG to %g relative residual"
            % (args.n, n_particles, pname, args.tol),
            "grid": args.n, "particles_per_scene": n_particles, "scenes": ws, "precision": args.precision,
            "preconditioner": ("MIC(0), tau 0.97" if args.precond == "mic0" else "reference (solver.inl:104-135)"),
            "tolerance": args.tol, "dt": 1.0 / 240.0,
            "parallelism": "replicas" if ws > 1 else "single",
            "l2": "inputs larger than L2 (particle state %.0f MB)" % (n_particles * 64 / 1e6)}


def serve_arm(args, A, prec, ws, rank, pg, gpu_index):
    """Poisson arrivals through the request server for `duration` seconds.  `value` is the
    particle-steps the server ran in that window divided by its length; the step latency
    percentiles are device times of the batch steps."""
    from ariel_b200 import workloads as W
    from ariel_b200.flipsim import Server
    stream = W.arrival_stream(args.rate, args.duration, seed=args.seed + 1000 * rank)
    prm = make_params(A, prec, args.tol)
    srv = Server(prm, max_live=args.max_live, keep_results=0, reserve_budget=1)
    sampler = ClockSampler(gpu_index)
    if pg:
        pg.barrier()
    sampler.start()
    t0 = time.perf_counter()
    launches0 = srv.L.ariel_kernel_launches()
    st0 = srv.stats()
    for ta, d in stream:
        dt = t0 + ta - time.perf_counter()
        if dt > 0:
            time.sleep(dt)
        srv.submit(d, args.serve_steps)
    dt = t0 + args.duration - time.perf_counter()
    if dt > 0:
        time.sleep(dt)
    st = srv.stats()
    wall = time.perf_counter() - t0
    clocks = sampler.stop()
    launches = srv.L.ariel_kernel_launches() - launches0
    srv.shutdown()
    ps = st.particle_steps - st0.particle_steps
    from ariel_b200.replicas import aggregate
    # replicas: every rank serves its own stream; the job's window is the longest rank's
    ms, ps_all = aggregate(wall * 1000.0, ps, pg)
    value = ps_all / (ms / 1000.0)
    out = {
        "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": ws,
        "steps": int(st.batch_steps), "warmup": 0, "ms_per_step": st.step_ms_p50,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "serving: Poisson arrivals (mean %g/s) of dam-break scenes with grids uniform "
                               "in 48^3-192^3 and blocks filling 20-50%%, %d steps each, %s PCG to %g, admitted "
                               "by device-byte budget, at most %d live, over %.0f s"
                               % (args.rate, args.serve_steps, args.precision, args.tol, args.max_live, args.duration),
                   "rate": args.rate, "duration_s": args.duration, "steps_per_request": args.serve_steps,
                   "max_live": args.max_live, "precision": args.precision,
                   "parallelism": "replicas" if ws > 1 else "single",
                   "l2": "inputs larger than L2"},
        "serving": {"submitted": len(stream), "admitted": st.admitted, "finished": st.finished,
                    "failed": st.failed, "live_at_end": st.live, "waiting_at_end": st.waiting,
                    "batch_steps": st.batch_steps, "particle_steps": ps, "busy_frac": st.busy_ms / (wall * 1000.0),
                    "step_ms_p50": st.step_ms_p50, "step_ms_p99": st.step_ms_p99, "step_ms_max": st.step_ms_max,
                    "request_latency_ms_p50": st.latency_ms_p50 if st.finished else None,
                    "request_latency_ms_p99": st.latency_ms_p99 if st.finished else None,
                    "relayouts": st.relayouts, "relayout_ms": st.relayout_ms,
                    "relayout_wait_ms": st.relayout_wait_ms, "relayout_build_ms": st.relayout_build_ms,
                    "graph_build_ms": st.graph_build_ms,
                    "staged": st.staged,
                    "hbm_budget_gb": st.hbm_budget_bytes / 1e9, "hbm_peak_gb": st.hbm_peak_bytes / 1e9,
                    "max_live_seen": st.max_live_seen},
        "step_ms_p50": st.step_ms_p50, "step_ms_p99": st.step_ms_p99,
        "clocks": clocks, "gpu_launches": launches,
        "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": None, "d2h_bytes_per_step": None,
                "api": "ariel_server_submit (host-seeded scenes, results copied out at retirement)",
                "note": "the server path is end to end by construction: scenes enter from the host and leave "
                        "to host memory; inputs are uploaded once per request, not per step"},
    }
    if rank == 0:
        print(json.dumps(out), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=128, help="grid size (the headline workload is 128)")
    ap.add_argument("--precision", choices=["mixed", "fp64", "ref32"], default="mixed")
    ap.add_argument("--tol", type=float, default=1e-5)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-fp64-compare", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-budget-s", type=float, default=150.0)
    ap.add_argument("--workload", choices=["dambreak", "sphere", "batch", "serve"], default="dambreak",
                    help="dambreak: the headline 128^3 scene; sphere: 256^3 with a solid sphere; batch: 64 "
                         "uneven scenes stepped together; serve: Poisson arrivals through the request server")
    ap.add_argument("--scenes", type=int, default=64)
    ap.add_argument("--batch-sub", type=int, default=64,
                    help="dambreak: also time this many uneven scenes batched, MIXED and FP64; 0: off")
    ap.add_argument("--batch-steps", type=int, default=6)
    ap.add_argument("--mic0-steps", type=int, default=3,
                    help="dambreak: also time this many steps with the MIC(0) preconditioner; 0: off")
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--rate", type=float, default=20.0, help="serve: mean arrivals per second")
    ap.add_argument("--duration", type=float, default=120.0, help="serve: seconds of arrivals")
    ap.add_argument("--serve-steps", type=int, default=200)
    ap.add_argument("--max-live", type=int, default=32)
    ap.add_argument("--autotune", action="store_true",
                    help="time the solve's launch-shape candidates on this workload first and run the fastest")
    ap.add_argument("--precond", choices=["ref", "mic0"], default="ref",
                    help="ref: the reference's preconditioner (solver.inl:104-135); mic0: MIC(0), tau .97")
    ap.add_argument("--inner-tol", type=float, default=0.0,
                    help="MIXED: relative reduction asked of each fp32 correction solve (0: library default)")
    args = ap.parse_args()
    global PRECOND, INNER_TOL
    PRECOND = args.precond
    INNER_TOL = args.inner_tol
    if args.workload == "sphere" and args.n == 128:
        args.n = 256
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
    from ariel_b200 import workloads as W
    resample_every = 1
    reseed_every = 0
    if args.workload == "serve":
        rc = serve_arm(args, A, prec, ws, rank, pg, gpu_index)
        if pg:
            pg.barrier()
            pg.destroy_process_group()
        return rc
    if args.workload == "batch":
        desc = W.uneven_batch(args.scenes, seed=args.seed + 1000 * rank)
    elif args.workload == "sphere":
        desc = W.sphere_dambreak(args.n, seed=replica_seed(rank))
        resample_every = 5
        reseed_every = 5
    else:
        desc = A.scene_dambreak(args.n, seed=replica_seed(rank))
    barrier = (lambda: pg.barrier()) if pg else None
    sampler = ClockSampler(gpu_index)
    prm = make_params(A, prec, args.tol, resample_every=resample_every, reseed_every=reseed_every)
    tune_report = None
    if args.autotune:
        from ariel_b200 import autotune
        prm, tune_report = autotune.tune(desc if isinstance(desc, list) else [desc], prm)
        prm.timing = 1
    b, res = run_gpu_pass(A, Batch, desc, prm, args.steps, args.warmup, sampler, barrier)

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
    alg_bytes = (tot.cell_iterations * PCG_SPEC_BYTES_PER_CELL_ITER[key] +
                 tot.cell_outer * PCG_BYTES_PER_CELL_OUTER[key]) / max(tot.solves, 1)
    own_bytes = (tot.cell_iterations * PCG_BYTES_PER_CELL_ITER[key] +
                 tot.cell_outer * PCG_BYTES_PER_CELL_OUTER[key]) / max(tot.solves, 1)
    peak, peak_kind = load_peaks()
    achieved = alg_bytes / (solve_ms / 1000.0) / 1e9 if solve_ms > 0 else None
    # DRAM traffic per launch from a committed capture of this very workload, if there is one
    if args.workload == "batch":
        workload_key = "pcg_%s_batch%d" % (args.precision, args.scenes)
    else:
        workload_key = "pcg_%s_%s%d" % (args.precision, args.workload, args.n)
    traffic = load_traffic(workload_key)
    # the solve's packed state (Av twice, Bv) of the FLUID cells fits the 126 MB L2 or not;
    # FLUID cells of all scenes from the per-scene sweep totals (cell_outer = sum nf * sweeps)
    fluid_cells = tot.cell_outer * b.k / max(tot.outer, 1)
    in_l2 = fluid_cells * (2 * 4 + 2) * (8 if args.precision == "fp64" else 4) < 100e6
    roofline = {"kernel": "k_pcg_fast<%s> (persistent pressure solve)" % args.precision, "bound": "hbm",
                "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None, "peak_source": peak_kind,
                "traffic": traffic,
                "traffic_source": ("committed ncu capture of this workload (profiles/traffic.txt), not measured "
                                   "by this run" if traffic is not None else None),
                "algorithmic_bytes_per_launch": alg_bytes,
                "bytes_model": "%g B per FLUID cell per CG iteration (two-reduction PCG, fp%s vectors) + %g B per "
                               "cell per refinement sweep" % (PCG_SPEC_BYTES_PER_CELL_ITER[key],
                                                              "64" if key == "fp64" else "32",
                                                              PCG_BYTES_PER_CELL_OUTER[key]),
                "achieved_own_model": own_bytes / (solve_ms / 1000.0) / 1e9 if solve_ms > 0 else None,
                "own_model": "%g B per cell-iteration: the single-reduction algorithm's own traffic"
                             % PCG_BYTES_PER_CELL_ITER[key],
                "avg_launch_ms": solve_ms,
                "note": "frac of %s HBM copy bandwidth; " % peak_kind +
                        ("the solve's working set stays in L2 at this size, so DRAM traffic is far below "
                         "the algorithmic bytes" if in_l2 else
                         "the solve's working set exceeds L2: DRAM traffic includes the streamed "
                         "16-byte cell records (about 16 B per FLUID cell per iteration)")}

    # every stage against HBM with its per-particle and per-cell bytes, from the same CUDA-event
    # stage times (stages with several kernels are timed as one)
    n_cells = sum(d.dim ** 3 for d in (desc if isinstance(desc, list) else [desc]))
    stage_roof = {}
    for name, (bp, bc) in STAGE_BYTES.items():
        t = stage_ms.get(name)
        if not t:
            continue
        if name == "resample" and resample_every > 1:
            t = t * resample_every  # the stage runs on one step in resample_every
        nbytes = bp * n_local + bc * n_cells
        gbs = nbytes / (t / 1000.0) / 1e9
        stage_roof[name] = {"ms": t, "bytes": nbytes, "achieved_gbs": gbs, "frac": gbs / peak}
    cfg = config_dict(args, n_local, ws)
    cfg["frames"] = [args.warmup + 1, args.warmup + args.steps]
    out = {
        "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "config": cfg,
        "stage_ms": stage_ms, "stage_roofline": stage_roof, "step_ms_p50": p50, "step_ms_p99": p99,
        "pcg": {"ms_per_solve": solve_ms, "iterations_per_solve": tot.iterations / max(tot.solves, 1),
                "outer_per_solve": tot.outer / max(tot.solves, 1), "not_converged": tot.not_converged,
                "final_rel_residual": res["stats"].pcg_rel_residual},
        "roofline": roofline, "clocks": res["clocks"], "gpu_launches": res["launches"],
    }
    if tune_report is not None:
        out["autotune"] = tune_report

    if rank == 0 and ws == 1 and not args.no_cpu_baseline and args.workload == "dambreak":
        out["pcg"]["fp64_oracle_error"] = fp64_oracle_error(A, Batch, b, desc)

    if not args.no_e2e:
        e2e_ms, h2d, d2h, pinned = run_e2e(b, args.steps)
        e_ms, _ = aggregate(e2e_ms, n_local, pg)
        out["e2e"] = {"value": total_particles * args.steps / (e_ms / 1000.0), "unit": "particle-steps/s",
                      "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "pinned": pinned,
                      "api": "ariel_upload_state + ariel_step + ariel_download_state"}
    b.close()

    if not args.no_fp64_compare and args.precision != "fp64":
        b64, r64 = run_gpu_pass(A, Batch, desc, make_params(A, A.PREC_FP64, args.tol, resample_every=resample_every,
                                                                reseed_every=reseed_every),
                                args.steps, args.warmup)
        b64.close()
        t64 = r64["totals"]
        solve64 = r64["timing"]["solve_kernel_ms"] / max(t64.solves, 1)
        out["pcg"]["fp64_plain"] = {"ms_per_solve": solve64, "iterations_per_solve": t64.iterations / max(t64.solves, 1),
                                    "particle_steps_per_s": r64["np"] * args.steps / (r64["ms"] / 1000.0)}
        out["pcg"]["speedup_vs_fp64"] = solve64 / solve_ms if solve_ms > 0 else None
        # per-GPU ratio of this rank's mixed pass to its plain FP64 pass
        out["throughput_vs_fp64"] = r64["ms"] / res["ms"] if res["ms"] > 0 else None

    if rank == 0 and ws == 1 and not args.no_cpu_baseline and args.workload == "dambreak":
        ref = reference_sim(A, desc)
        if ref is not None:
            r, n, cores = ref
            t0 = time.perf_counter()
            r.step(1)
            dt = time.perf_counter() - t0
            r.close()
            out["cpu_baseline"] = {"value": n / dt, "unit": "particle-steps/s", "cores": cores, "kind": "reference",
                                   "sample": "frame 1 (from Init) of the same %d^3 dam break, %d particles: the "
                                             "reference's own FlipSim::Step compiled from its sources (oracle/_ref), "
                                             "%s; %.1f s" % (args.n, n, REFERENCE_CONFIG, dt)}
        else:
            n, dt, cores, st = cpu_baseline_sample(A, desc, args.tol)
            out["cpu_baseline"] = {"value": n / dt, "unit": "particle-steps/s", "cores": cores, "kind": "port",
                                   "sample": "1 FLIP step (from Init) of the same %d^3 dam break, %d particles, "
                                             "reference-faithful OpenMP granularity, fp32 PCG to %g relative "
                                             "(%d iterations), %.1f s" % (args.n, n, args.tol, st.pcg_iterations, dt)}
    if rank == 0 and ws == 1 and args.batch_sub > 0 and args.workload == "dambreak":
        out["batch"] = batch_subresult(A, Batch, args)
    if rank == 0 and ws == 1 and args.mic0_steps > 0 and args.workload == "dambreak" and PRECOND != "mic0":
        out["pcg"]["mic0"] = mic0_subresult(A, Batch, desc, args)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
