"""Benchmark: ALI iterations and wall-clock to 1e-4 populations on one B200.

Workload (default): the 64^3 jittered spherical wind (262,144 cells, 10-level
linear rotor, 9 lines x 31 bins = 279 bins, 48 HEALPix rays = 24 pairs),
seeded synthetic data.  One step is one complete solve of the hot path:
trace every ray, set the starting populations (learned warm start by
default, LTE with --start lte), and iterate formal solve + Jeff +
statistical equilibrium (+ an Ng step after every three normal iterations
from the learned start, four -- the reference's cadence -- from LTE;
--ng-every overrides) until the max relative population change over all
(cell, level) with n > 1e-10 n_tot drops below 1e-4.  The headline arm is learned start + mixed precision; the plain FP64
solve from LTE is measured in the same run and reported beside it.

    value  seconds per converged solve, device-timed (CUDA events on the
           library's stream), model already resident in HBM
    e2e    the same through the C ABI from host buffers: model upload,
           set-up, trace, ALI, download of the populations, all timed
    roofline  the formal-solve kernel: algorithmic bytes (44 B per
           ray-point-frequency update in FP64, 24 B in mixed) / its average
           launch time, against the measured HBM copy bandwidth
    cpu_baseline  the reference's compiled CPU path (oracle/_ref; the C
           oracle where that binary is absent) on this host's cores: the
           per-origin work of one formal solve on a sample of origins,
           extrapolated, plus the full rate-equation step, times the
           iteration count of the solve

``--impl reference`` times the reference's own C++ (Magritte's CPU path
compiled from its sources into oracle/_ref; the CPU oracle, the same
algorithm restated in C, where that binary is absent) with OpenMP on every
host core, and prints one line with "impl": "reference".

Multi-GPU (torchrun): the ranks partition the origins of the one model
(``magritte_b200.partition``: each rank solves its own origins and cells,
then one NCCL all-gather of the population blocks per iteration), so the
scaling is strong and value is the max over ranks of the time per
converged solve.  ``--replicas`` solves an independent replica per GPU
instead (weak scaling); ``--partition`` runs the partitioned driver on one
GPU.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "ALI iters & wall-clock to 1e-4 pops on 1 B200: learned+FP32 vs plain FP64"
TOL = 1.0e-4
MAX_ITER = 400
FALLBACK_HBM_GBS = 6650.0
STAGED_DRAM_BYTES_PER_UPDATE = 0.685
# thread instructions (warp instructions x 32) per update of the same kernel
# in the same capture: the issue-bound ceiling is 148 SMs x 4 schedulers x
# the SM clock x 32 lanes / this
STAGED_THREAD_INST_PER_UPDATE = 34.2
B200_SMS = 148


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--start", default="learned", choices=["learned", "lte"])
    ap.add_argument("--weights", default=None,
                    help="warm-start network (default: the workload's trained network)")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain FP64 comparison")
    ap.add_argument("--workload", default="wind64", choices=sorted(WORKLOADS),
                    help="wind32 (the same wind at 32^3) is the small case for ncu captures")
    ap.add_argument("--no-graph", action="store_true", help="launch iterations without CUDA graphs")
    ap.add_argument("--ng-every", type=int, default=0,
                    help="normal iterations before each Ng step of the headline arm (default: 3 "
                         "after the learned start, 4 = the reference's cadence after LTE); the "
                         "plain FP64 arm always uses 4"),
    ap.add_argument("--no-autotune", action="store_true", help="default solve kernel shapes")
    ap.add_argument("--no-e2e", action="store_true",
                    help="skip the end-to-end repeat (for workloads whose solve takes minutes)")
    ap.add_argument("--max-iter", type=int, default=MAX_ITER,
                    help="ALI iteration cap (a batch stops when every model converged or at the cap)")
    ap.add_argument("--plain-max-iter", type=int, default=None,
                    help="iteration cap of the plain FP64 solve (default: --max-iter); a plain "
                         "solve stopped by the cap reports converged: false and a lower bound")
    ap.add_argument("--partition", action="store_true",
                    help="run the partitioned driver (one shard per rank, NCCL all-gather of "
                         "the populations every iteration) even on one GPU")
    ap.add_argument("--replicas", action="store_true",
                    help="with several GPUs, solve an independent replica per GPU instead of "
                         "partitioning one model")
    ap.add_argument("--cpu-sample-s", type=float, default=15.0)
    ap.add_argument("--ref-sample-s", type=float, default=3.0,
                    help="seconds of the reference's formal-solve sample per step (reference arm)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


WEIGHTS_DIR = os.path.join(ROOT, "magritte_b200", "weights")
# name: (description, builder, trained warm-start network or None)
WORKLOADS = {
    "wind64": ("64^3 spherical wind, 10-level rotor", "config2", "wind_rotor10.npz"),
    "wind32": ("32^3 spherical wind, 10-level rotor", "wind32", "wind_rotor10.npz"),
    "lattice16": ("16^3 lattice cloud, 2-level line", "config1", None),
    "lattice16_dense": ("16^3 lattice cloud at 1e3 x density (line-centre tau ~1e4), "
                        "2-level line", "config3", None),
    "batch256": ("256 independent spherical winds of 2k-60k points, 20-level rotor, 24 rays",
                 "config4", None),
    "turb128": ("128^3 turbulent cloud, 21-level rotor, 96 rays, 41 bins/line", "config5",
                "turb_rotor21.npz"),
}


def make_model(name):
    import magritte_b200.model as M
    b = WORKLOADS[name][1]
    if b == "wind32":
        return M.wind_model(32, seed=2, nlev=10, nside=2, name="wind32")
    return getattr(M, b)()


def weights_for(name, override=None):
    w = override or WORKLOADS[name][2]
    if w is None:
        return None
    p = w if os.path.isabs(w) else os.path.join(WEIGHTS_DIR, w)
    return p if os.path.exists(p) else None


def workload_config(name, model, prec, start="LTE"):
    cfg = {"workload": WORKLOADS[name][0],
           "cells": model.ncells, "levels": model.linedata.nlev, "lines": model.nlines,
           "bins_per_line": model.nquads, "rays": model.nrays,
           "start": start, "tol_max_rel": TOL, "ng": True, "precision": prec,
           "l2": "inputs larger than L2 (ray traces of several GB re-read every iteration)"}
    seg = model.meta.get("segments")
    if seg:
        cfg["models"] = len(seg) - 1
    return cfg


def max_over_ranks(values):
    """Element-wise max of `values` over the ranks of the default process
    group (NCCL: through a device tensor; gloo: on the host)."""
    import torch
    import torch.distributed as tdist
    dev = "cuda" if tdist.get_backend() == "nccl" else "cpu"
    t = torch.tensor(list(values), dtype=torch.float64, device=dev)
    tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
    return [float(x) for x in t.cpu()]


def free_port():
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class Clocks:
    """nvidia-smi samples, started ahead of the timed region (its start-up
    is kept out of the timed steps) and summarised over the timed window
    only (`mark_start` / `mark_end`)."""

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.t0 = self.t1 = None

    def mark_start(self):
        import datetime
        self.t0 = datetime.datetime.now()

    def mark_end(self):
        import datetime
        self.t1 = datetime.datetime.now()

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}",
                 "--query-gpu=timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        import datetime
        rows = []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in (self.out or "").strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm, mx = float(f[1]), float(f[2])
            except ValueError:
                continue
            try:
                ts = datetime.datetime.strptime(f[0], "%Y/%m/%d %H:%M:%S.%f")
                inside = self.t0 is None or self.t1 is None or self.t0 <= ts <= self.t1
            except ValueError:
                inside = True
            rows.append((inside, sm, mx, [n for n, v in zip(names, f[5:9]) if v.lower() == "active"]))
        sel = [r for r in rows if r[0]] or rows   # every sample if none carries a usable time
        if not sel:
            return None
        return {"sm_mhz": statistics.median(r[1] for r in sel), "sm_max_mhz": max(r[2] for r in sel),
                "reasons": sorted({n for r in sel for n in r[3]}), "samples": len(sel)}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


# ------------------------------------------------------------------ CPU arm

class CpuOracle:
    """The CPU oracle on this host's cores (OpenMP over origins, as the
    reference): one formal solve over a seeded sample of origins (all ray
    pairs) scaled to all origins, plus one full rate-equation step, times
    the iteration count of the solve."""

    def __init__(self, model, nthreads=None):
        import oracle
        self.model = model
        self.nthreads = nthreads or os.cpu_count() or 1
        self.o = oracle.Oracle(model).setup()

    def time(self, iterations, sample_s, seed=0, ng_steps=0):
        """`iterations` formal solves (each with Jeff and the rate
        equations) and `ng_steps` Ng steps."""
        import numpy as np
        m, o = self.model, self.o
        rng = np.random.default_rng(seed)
        n = 64
        while True:
            origins = np.sort(rng.choice(m.ncells, size=min(n, m.ncells), replace=False))
            t0 = time.perf_counter()
            o.compute_radiation_field(origins=origins, nthreads=self.nthreads)
            dt = time.perf_counter() - t0
            if dt > 0.25 * sample_s or n >= m.ncells:
                t_solve = dt * m.ncells / len(origins)
                break
            n = min(m.ncells, int(n * max(2.0, 0.3 * sample_s / max(dt, 1e-3))))
        t0 = time.perf_counter()
        o.compute_Jeff()
        o.compute_level_populations_from_stateq()
        t_stateq = time.perf_counter() - t0
        t_ng = 0.0
        if ng_steps:
            t0 = time.perf_counter()
            o.ng_acceleration()
            t_ng = time.perf_counter() - t0
        per_iter = t_solve + t_stateq
        return {"seconds": per_iter * iterations + t_ng * ng_steps, "per_iteration_s": per_iter,
                "formal_solve_s": t_solve, "stateq_s": t_stateq, "ng_s": t_ng,
                "sample_origins": int(len(origins)), "cores": self.nthreads}


REF_BIN = os.path.join(ROOT, "oracle", "_ref", "magritte_ref")


class ReferenceCpu:
    """The reference's own C++ (Magritte's CPU path compiled from its
    sources into oracle/_ref, OpenMP on all host cores), fed the workload
    as a model folder in its text layout.  A step times the reference's
    per-origin work of compute_radiation_field (trace, setup, solve,
    update_Lambda, J; sim_radiation.tpp:150-264) on a seeded sample of
    origins over all ray pairs, scaled to every origin, times the number of
    formal solves, plus the whole model's Jeff + rate-equation step per
    formal solve and Ng step per Ng iteration (those two timed once per
    run, on the full model)."""

    def __init__(self, model, name, nthreads=None):
        import tempfile
        from magritte_b200 import io_text
        self.model = model
        self.nthreads = nthreads or os.cpu_count() or 1
        self.dir = tempfile.mkdtemp(prefix=f"mgr_ref_{name}_")
        self.folder = os.path.join(self.dir, "model") + "/"
        io_text.write_model(model, self.folder)

    def run(self, samples):
        path = os.path.join(self.dir, "samples.txt")
        with open(path, "w") as f:
            for o in samples:
                f.write(" ".join(str(int(x)) for x in o) + "\n")
        env = dict(os.environ, OMP_NUM_THREADS=str(self.nthreads))
        r = subprocess.run([REF_BIN, self.folder, self.dir, "sample", path], capture_output=True,
                           text=True, env=env, cwd=self.dir)
        if r.returncode != 0:
            raise RuntimeError(r.stderr[-2000:])
        return [json.loads(l) for l in r.stdout.splitlines() if l.startswith('{"origins"')]

    def time_steps(self, n_solve, n_ng, sample_s, steps, seed0=0):
        import numpy as np
        N = self.model.ncells
        rng = np.random.default_rng(seed0)
        probe = self.run([np.sort(rng.choice(N, size=min(256, N), replace=False))])[0]
        per_origin = probe["formal_solve_s"] / probe["origins"]
        n = int(min(N, max(64, sample_s / max(per_origin, 1e-9))))
        samples = [np.sort(rng.choice(N, size=n, replace=False)) for _ in range(steps)]
        out = self.run(samples)
        t_stateq, t_ng = probe["stateq_s"], probe["ng_s"]
        secs = [o["formal_solve_s"] * N / o["origins"] * n_solve + t_stateq * n_solve + t_ng * n_ng
                for o in out]
        info = {"sample_origins": n, "cores": self.nthreads, "stateq_s": t_stateq, "ng_s": t_ng,
                "formal_solve_s": statistics.mean(o["formal_solve_s"] * N / o["origins"] for o in out)}
        return secs, info


def cpu_oracle_time(model, iterations, sample_s, nthreads=None, ng_every=4):
    """The oracle's time for `iterations` iterations of the ALI loop, Ng
    steps (after every ng_every normal iterations) charged as Ng steps, not
    formal solves."""
    from oracle.measure_iterations import step_kinds
    k = step_kinds(iterations, ng_every=ng_every)
    info = CpuOracle(model, nthreads).time(k.count("solve"), sample_s, ng_steps=k.count("ng"))
    info["formal_solves"], info["ng_steps"] = k.count("solve"), k.count("ng")
    return info


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def reference_counts(name, model):
    """(formal solves, Ng steps, source) of the reference's ALI (LTE start,
    FP64) on this workload: from the record of a full oracle run
    (oracle/measure_iterations.py), else -- for workloads small enough --
    from running the oracle's ALI here."""
    from oracle.measure_iterations import step_kinds
    rec = os.path.join(ROOT, "oracle", f"iterations_{name}.json")
    if os.path.exists(rec):
        d = json.load(open(rec))
        return d["formal_solves"], d["ng_steps"], f"measured full oracle ALI ({d['iterations']} iterations, oracle/iterations_{name}.json)"
    if model.ncells <= 40 ** 3:
        import oracle
        it, _ = oracle.Oracle(model).setup().compute_level_populations(True, MAX_ITER, TOL)
        k = step_kinds(it)
        return k.count("solve"), k.count("ng"), f"oracle ALI run here ({it} iterations)"
    return None, None, None


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    model = make_model(args.workload)
    n_solve, n_ng, source = reference_counts(args.workload, model)
    if n_solve is None:
        print(json.dumps({"impl": "reference", "unavailable":
                          f"no measured iteration count of the oracle for {args.workload}"}))
        return
    if os.path.exists(REF_BIN):
        # the reference's own compiled C++; warm-up samples lead the run
        ref = ReferenceCpu(model, args.workload)
        secs, info = ref.time_steps(n_solve, n_ng, args.ref_sample_s,
                                    args.warmup + max(1, args.steps))
        steps = secs[args.warmup:]
        kind = "reference"
        sample = (f"the reference's compiled per-origin work of compute_radiation_field over "
                  f"{info['sample_origins']} seeded origins x all ray pairs per step, scaled to "
                  f"{model.ncells} origins, x {n_solve} formal solves; plus its full-model Jeff + "
                  f"rate-equation step ({info['stateq_s']:.2f} s, x {n_solve}) and Ng step "
                  f"({info['ng_s']:.2f} s, x {n_ng}), timed once")
    else:
        cpu = CpuOracle(model)
        for w in range(args.warmup):
            cpu.time(n_solve, min(2.0, args.cpu_sample_s), seed=100 + w, ng_steps=n_ng)
        steps = []
        info = None
        for k in range(max(1, args.steps)):
            info = cpu.time(n_solve, args.cpu_sample_s, seed=k, ng_steps=n_ng)
            steps.append(info["seconds"])
        kind = "port"
        sample = (f"one formal solve over {info['sample_origins']} seeded origins x all ray pairs "
                  f"scaled to {model.ncells} origins, plus one full Jeff + rate-equation step, x "
                  f"{n_solve} formal solves; plus {n_ng} full Ng step(s)")
    value = statistics.mean(steps)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": value * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": workload_config(args.workload, model, "fp64"),
        "ali_iterations": n_solve + n_ng, "formal_solves": n_solve, "ng_steps": n_ng,
        "iteration_source": source,
        "cpu_baseline": {"value": value, "unit": "s", "cores": info["cores"], "kind": kind,
                         "cpu_model": cpu_model(), "sample": sample},
        "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ GPU arm

def _max_rel(a, b, mask=None):
    import numpy as np
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    with np.errstate(invalid="ignore", divide="ignore"):
        r = np.abs(a - b) / np.abs(b)
    r[a == b] = 0.0
    if mask is not None:
        r = r[mask]
    return float(np.nanmax(r)) if r.size else 0.0


def precision_errors(sim, model, pop_head, prec):
    """The headline arm's error against the plain FP64 arm of the same run,
    which sits on the simulation when this is called: (1) its converged
    populations against the FP64-converged ones (max relative difference
    over levels with n > 1e-10 n_tot; both stop at a max relative change
    below the tolerance, so this includes the convergence tolerance), and
    (2) with the FP64-converged populations fixed, J (when it fits), Jlin and
    the ALO of one formal solve in the headline precision against one in FP64
    (the precision error alone)."""
    import numpy as np
    pop64 = sim.population
    mask = pop64 > 1e-10 * model.population_tot[:, None]
    out = {"pop_max_rel": _max_rel(pop_head, pop64, mask),
           "pop_note": "converged populations of the headline arm vs the plain FP64 arm "
                       "(levels with n > 1e-10 n_tot)"}
    if prec == "fp64":
        return out
    keep_J = model.ncells * model.nfreqs <= 200_000_000
    sim.compute_radiation_field(prec, keep_J=keep_J)
    J_m = sim.J if keep_J else None
    Jlin_m, L_m = sim.Jlin, sim.Lambda
    sim.compute_radiation_field("fp64", keep_J=keep_J)
    if keep_J:
        out["J_max_rel"] = _max_rel(J_m, sim.J)
    out["Jlin_max_rel"] = _max_rel(Jlin_m, sim.Jlin)
    out["lambda_max_rel"] = _max_rel(L_m, sim.Lambda)
    out["J_note"] = (f"one {prec} formal solve vs one FP64 formal solve on the FP64-converged "
                     f"populations, all cells" + ("" if keep_J else " (J per bin not kept at this size)"))
    sim.compute_radiation_field(prec, keep_J=False)
    return out


def run_b200(args):
    import numpy as np
    from magritte_b200 import Simulation
    rank, world, local = dist_env()
    dist = world > 1
    partitioned = (dist and not args.replicas) or args.partition
    if dist or partitioned:
        import datetime
        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(local)
        if dist:
            # a rank that loses its peers ends its next collective with an
            # error within 5 minutes (a formal solve here takes seconds)
            tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        else:
            tdist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{free_port()}",
                                     rank=0, world_size=1,
                                     timeout=datetime.timedelta(seconds=300))
    model = make_model(args.workload)
    prec = args.precision
    net = None
    start_name = "LTE"
    if args.start == "learned":
        from magritte_b200.learned import WarmStartNet
        wp = weights_for(args.workload, args.weights)
        if wp is not None:
            net = WarmStartNet.load(wp)
            if net.nlev != model.linedata.nlev:
                net = None
        start_name = "learned" if net is not None else "LTE (no trained network for this species)"
    graph = not args.no_graph
    # Ng cadence of the headline arm: after the learned start the iteration
    # is in its geometric regime from the first step, so the extrapolation
    # can come after three normal iterations; from LTE the reference's four
    ng_head = args.ng_every or (3 if net is not None else 4)

    def start(sim, learned):
        if learned:
            sim.warm_start(net)
        else:
            sim.compute_LTE_level_populations()

    shards = {}

    def one_solve(sim, learned=net is not None, precision=prec, max_iter=None, ng=None):
        ng = ng_head if ng is None else ng
        sim.trace()
        start(sim, learned)
        if not partitioned:
            return sim.compute_level_populations(True, max_iter or args.max_iter, precision,
                                                 tol_max_rel=TOL, use_graph=graph, ng_every=ng)
        # this rank's shard of the origins; one all-gather per iteration
        from magritte_b200.partition import DeviceShard, partitioned_level_populations
        key = (id(sim), precision)
        if key not in shards:
            shards[key] = DeviceShard(sim, rank, world, precision)
        it, hist, conv = partitioned_level_populations(shards[key], None, True,
                                                       max_iter or args.max_iter, TOL, ng_every=ng)
        sim.error_max, sim.converged = hist, conv
        return it

    # ---- device-resident solve
    sim = Simulation(model, device=local if dist else 0)
    if not args.no_autotune:
        sim.set_autotune(True)
    sim.compute_spectral_discretisation()
    sim.compute_boundary_intensities()
    for _ in range(max(0, args.warmup - 1)):
        one_solve(sim)
    if not args.no_plain and not dist and not args.no_autotune:
        # tune the FP64 kernel before the plain solve is timed
        sim.trace()
        start(sim, False)
        for _ in range(3):
            sim.compute_radiation_field("fp64")
    if dist:
        tdist.barrier()
    times, iters, solve_ms, solve_upd, trace_ms = [], [], [], [], []
    with Clocks(local) as clk:
        time.sleep(2.0)          # sampler start-up outside the timed steps
        if args.warmup > 0:
            one_solve(sim)       # the last warm-up step, with the sampler running
        if dist:
            tdist.barrier()
        launches0 = sim.launch_count()
        clk.mark_start()
        for _ in range(args.steps):
            sim.timer_start()
            it = one_solve(sim)
            times.append(sim.timer_stop() / 1e3)
            iters.append(it)
            ms, up = sim.solve_stats()
            solve_ms.append(ms)
            solve_upd.append(up)
            trace_ms.append(sim.solve_trace_ms())
        clk.mark_end()
    launches = (sim.launch_count() - launches0) // max(1, args.steps)
    converged = bool(getattr(sim, "converged", False))
    pop_head = sim.population          # converged populations of the headline arm
    model_iters = None
    if model.meta.get("segments"):
        import numpy as np
        _, mit = sim.segment_results()
        mst, _ = sim.segment_results()
        model_iters = {"min": int(mit.min()), "median": float(np.median(mit)),
                       "max": int(mit.max()), "sum": int(mit.sum()),
                       "not_converged": [int(i) for i in np.nonzero(~(mst[:, 2] < TOL))[0]]}
    tuning = sim.tuning(prec)   # the kernel that ran (and, with the autotuner, its timings)
    err_hist = list(sim.error_max)
    t_step = statistics.mean(times)

    # ---- end to end through the C ABI from host buffers
    e2e = []
    h2d = model.nbytes() + (int(net.params.nbytes) if net is not None else 0)
    d2h = model.ncells * model.linedata.nlev * 8
    for _ in range(0 if args.no_e2e else max(1, args.steps)):
        t0 = time.perf_counter()
        s2 = Simulation(model, device=local if dist else 0)
        s2.compute_spectral_discretisation()
        s2.compute_boundary_intensities()
        start(s2, net is not None)
        if not args.no_autotune:
            s2.set_autotune(True)
        if partitioned:
            from magritte_b200.partition import DeviceShard, partitioned_level_populations
            partitioned_level_populations(DeviceShard(s2, rank, world, prec), None, True,
                                          args.max_iter, TOL, ng_every=ng_head)
        else:
            s2.compute_level_populations(True, args.max_iter, prec, tol_max_rel=TOL,
                                         use_graph=graph, ng_every=ng_head)
        pop = s2.population
        e2e.append(time.perf_counter() - t0)
        s2.close()
    if e2e:
        assert np.all(np.isfinite(pop))

    # ---- the plain method: FP64 from the LTE start (north-star comparison)
    plain = None
    errors = None
    if not args.no_plain and not dist:
        print(json.dumps({"progress": "headline step done", "seconds": times, "iterations": iters,
                          "converged": converged, "history": err_hist}), file=sys.stderr,
              flush=True)
        sim.timer_start()
        it_p = one_solve(sim, learned=False, precision="fp64", max_iter=args.plain_max_iter, ng=4)
        t_p = sim.timer_stop() / 1e3
        plain = {"start": "LTE", "precision": "fp64", "ng_every": 4, "ali_iterations": it_p,
                 "seconds": t_p,
                 "converged": bool(getattr(sim, "converged", False)),
                 "final_max_rel_change": sim.error_max[-1] if sim.error_max else None}
        if model.meta.get("segments"):
            import numpy as np
            _, mit = sim.segment_results()
            plain["model_iterations"] = {"min": int(mit.min()), "median": float(np.median(mit)),
                                         "max": int(mit.max()), "sum": int(mit.sum())}
        plain["iterations_ratio"] = it_p / max(1, iters[-1])
        plain["wallclock_ratio"] = t_p / max(1e-12, statistics.mean(times))
        plain["wallclock_ratio_median"] = t_p / max(1e-12, statistics.median(times))
        errors = precision_errors(sim, model, pop_head, prec)
    sim.close()

    # ---- multi-GPU: max over ranks
    if dist:
        t_step, e2e_t = max_over_ranks([t_step, statistics.mean(e2e) if e2e else 0.0])
        tdist.barrier()
    else:
        e2e_t = statistics.mean(e2e) if e2e else None
    if dist or partitioned:
        tdist.destroy_process_group()
    if rank != 0:
        return

    hbm, kind = peaks()
    bpu = 44.0 if prec == "fp64" else 24.0
    avg_ms = statistics.mean(solve_ms)
    achieved = solve_upd[-1] * bpu / (avg_ms / 1e3) / 1e9
    # DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per update of
    # the staged mixed kernel from one ncu capture of a launch on the wind,
    # scaled to this launch by its update count
    traffic = (solve_upd[-1] * STAGED_DRAM_BYTES_PER_UPDATE
               if prec == "mixed" and tuning and tuning.get("kernel") == "staged" else None)
    line = {
        "metric": METRIC, "value": t_step if partitioned else t_step / world, "unit": "s",
        "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_step * 1e3,
        "higher_is_better": False, "scaling": "strong" if partitioned else "weak",
        "vs_baseline": None,
        "dtype": "f64" if prec == "fp64" else "f32+f64",
        "data": "synthetic (seeded)",
        "config": dict(workload_config(args.workload, model, prec, start_name),
                       ng_every=ng_head,
                       parallelism=(f"origins partitioned over {world} GPU(s), populations "
                                    f"all-gathered over NCCL every iteration" if partitioned
                                    else ("one replica per GPU" if dist else "1 GPU"))),
        "step_s": {"mean": statistics.mean(times), "median": statistics.median(times),
                   "min": min(times), "max": max(times)},
        "ali_iterations": iters[-1], "converged": converged,
        "errors_vs_fp64": errors,
        "model_iterations": model_iters,
        "solve_kernel": tuning,
        "plain_fp64_lte": plain,
        "final_max_rel_change": err_hist[-1] if err_hist else None,
        "formal_solve": {"ms": avg_ms, "updates": solve_upd[-1],
                         "updates_per_s": solve_upd[-1] / (avg_ms / 1e3),
                         "trace_rebuild_ms": statistics.mean(trace_ms),
                         "note": "ms of the last formal solve of each step; trace_rebuild_ms: of "
                                 "it, rebuilding the traces batch by batch of origins when they "
                                 "exceed the trace budget (0: traces stored)"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": traffic,
                     "note": f"formal-solve kernel; effective operand bytes {bpu:.0f} B/update "
                             f"(what an unstaged kernel reads); peak = {kind} copy bandwidth. The "
                             f"staged kernel reads each point once per 32 bins: DRAM traffic is "
                             f"`traffic` bytes per launch, and the kernel is bound by instruction "
                             f"issue and the XU pipe, not HBM"},
        "e2e": None if not e2e else {"value": e2e_t if partitioned else e2e_t / world, "unit": "s",
                "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    if traffic is not None:
        # the bound that holds: instruction issue at the measured clock
        mhz = (line["clocks"] or {}).get("sm_mhz") or 1965.0
        ceiling = B200_SMS * 4 * mhz * 1e6 * 32 / STAGED_THREAD_INST_PER_UPDATE
        ups = solve_upd[-1] / (avg_ms / 1e3)
        line["roofline"]["issue"] = {
            "thread_instructions_per_update": STAGED_THREAD_INST_PER_UPDATE,
            "ceiling_updates_per_s": ceiling, "achieved_updates_per_s": ups,
            "frac": ups / ceiling,
            "note": "instructions per update from ncu on the 32^3 wind (same kernel); ceiling = "
                    "148 SMs x 4 schedulers x SM clock x 32 lanes / instructions per update"}
    if not args.no_cpu_baseline and world == 1:
        from oracle.measure_iterations import step_kinds
        k = step_kinds(iters[-1], ng_every=ng_head)
        n_solve, n_ng = k.count("solve"), k.count("ng")
        if os.path.exists(REF_BIN):
            secs, info = ReferenceCpu(model, args.workload).time_steps(n_solve, n_ng,
                                                                     args.cpu_sample_s, 1)
            line["cpu_baseline"] = {
                "value": secs[0], "unit": "s", "cores": info["cores"], "kind": "reference",
                "cpu_model": cpu_model(),
                "sample": f"the reference's compiled per-origin work of compute_radiation_field "
                          f"over {info['sample_origins']} seeded origins x all ray pairs, scaled "
                          f"to {model.ncells} origins, x {n_solve} formal solves, plus its "
                          f"full-model Jeff + rate-equation step per solve and {n_ng} Ng "
                          f"step(s) ({iters[-1]} iterations of the headline arm)"}
        else:
            info = cpu_oracle_time(model, iters[-1], args.cpu_sample_s, ng_every=ng_head)
            line["cpu_baseline"] = {
                "value": info["seconds"], "unit": "s", "cores": info["cores"], "kind": "port",
                "cpu_model": cpu_model(),
                "sample": f"one formal solve over {info['sample_origins']} seeded origins x all "
                          f"ray pairs scaled to {model.ncells} origins, plus one full Jeff + "
                          f"rate-equation step, x {info['formal_solves']} formal solves, plus "
                          f"{info['ng_steps']} full Ng step(s) ({iters[-1]} iterations)"}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
