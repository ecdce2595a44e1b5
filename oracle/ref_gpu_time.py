"""One formal solve of the reference (its CPU path and its own GPU solver)
timed beside this library's formal solve on the same model and GPU (TEST
INFRASTRUCTURE ONLY: a measurement of the reference, never part of the
product).

``oracle/ref_build.sh`` builds ``oracle/_ref/magritte_ref_gpu`` from the
reference's unmodified sources with its GPU path compiled in (nvcc with the
reference's own flags).  This script writes a seeded model (the 16^3
lattice cloud, its x1e3-density variant, or a jittered wind) in Magritte's
text layout and runs, on that folder:

* the reference's CPU path, ``Simulation::compute_radiation_field`` +
  ``compute_Jeff`` (``oracle/_ref/magritte_ref ... radiation``, OpenMP over
  all host cores), as the values the other two are compared with;
* the reference's GPU path, ``Simulation::gpu_compute_radiation_field``
  (``src/Simulation/simulation.cu:512-726``: ray pairs traced on the host,
  queued by depth, each block of equal-depth pairs solved by
  ``feautrierKernel`` (``src/Simulation/Solver/gpu/gpu_solver.cu:204-240``)
  in managed memory with a device synchronisation per block), with one
  OpenMP thread: the GPU thread alone.  With more threads the reference
  starts CPU solver threads beside it that share one ``Timer`` object
  without a lock (``simulation.cu:673-694``), a data race on its vectors;
  one thread measures the GPU solver without it;
* this library's ``compute_radiation_field`` in FP64 and in mixed
  precision, through the C ABI (device time of the formal solve, and the
  wall time of the call with the trace stored).

It prints one JSON line: wall times, updates per second (updates = the
ray-point-bin triples of one formal solve), the max relative differences of
J, Jlin and the diagonal ALO against the reference's CPU path (bins with J
below 1e-12 of its maximum left out; NaNs counted) and, for the lattice
models, the line-centre optical depth across the cube.

    python -m oracle.ref_gpu_time --model wind --n 32 [--block 128 --nblocks 1184 --reps 2]
    python -m oracle.ref_gpu_time --model config3
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_CPU = os.path.join(ROOT, "oracle", "_ref", "magritte_ref")
REF_GPU = os.path.join(ROOT, "oracle", "_ref", "magritte_ref_gpu")


def rel_stats(a, b, floor=1e-12):
    """Max relative difference of a from b over entries with |b| above
    floor * max|b|, and the count of non-finite entries of a."""
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    bad = int(np.count_nonzero(~np.isfinite(a)))
    keep = np.isfinite(a) & (np.abs(b) > floor * np.abs(b).max())
    r = np.abs(a[keep] - b[keep]) / np.abs(b[keep])
    return {"max_rel": float(r.max()) if r.size else 0.0,
            "median_rel": float(np.median(r)) if r.size else 0.0, "nonfinite": bad}


def run(cmd, out, threads, timeout):
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    t = time.perf_counter()
    r = subprocess.run(cmd, capture_output=True, text=True, env=env, cwd=out, timeout=timeout)
    wall = time.perf_counter() - t
    if r.returncode != 0:
        raise RuntimeError(f"{cmd[0]} exited {r.returncode}: {r.stderr[-1500:]}{r.stdout[-1500:]}")
    return r.stdout, wall


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--model", choices=("wind", "config1", "config3"), default="wind",
                    help="jittered wind of --n^3 cells, the 16^3 lattice cloud, or the "
                         "lattice at 1e3 x density")
    ap.add_argument("--n", type=int, default=32, help="wind lattice size n (n^3 cells)")
    ap.add_argument("--no-ref-gpu", action="store_true", help="skip the reference's GPU solver")
    ap.add_argument("--block", type=int, default=128, help="gpuBlockSize of the reference")
    ap.add_argument("--nblocks", type=int, default=1184, help="gpuNumBlocks of the reference")
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--timeout", type=float, default=1500.0)
    ap.add_argument("--out", default=None, help="write the JSON line here as well")
    args = ap.parse_args(argv)
    for b in (REF_CPU,) + (() if args.no_ref_gpu else (REF_GPU,)):
        if not os.path.exists(b):
            sys.exit(f"{b} not built (oracle/ref_build.sh)")

    import magritte_b200.model as M
    from magritte_b200 import io_text
    from magritte_b200.simulation import Simulation

    if args.model == "wind":
        model = M.wind_model(args.n, seed=2, nlev=10, nside=2, name=f"wind{args.n}")
    else:
        model = getattr(M, args.model)()
    tmp = tempfile.mkdtemp(prefix="refgpu_")
    folder = os.path.join(tmp, "model") + "/"
    io_text.write_model(model, folder)
    N, nf = model.ncells, None

    # the reference's CPU path; its own Timer gives compute_radiation_field
    out_cpu = os.path.join(tmp, "cpu")
    os.makedirs(out_cpu)
    threads = os.cpu_count() or 1
    text, cpu_wall = run([REF_CPU, folder, out_cpu, "radiation"], out_cpu, threads, args.timeout)
    cpu_rf = [float(l.split(":")[-1].split()[0]) for l in text.splitlines()
              if l.startswith("T ") and "compute radiation field" in l]
    J_cpu = np.fromfile(os.path.join(out_cpu, "J.bin"))
    nf = J_cpu.size // N
    Jl_cpu = np.fromfile(os.path.join(out_cpu, "Jlin.bin"))
    L_cpu = np.fromfile(os.path.join(out_cpu, "Lambda.bin"))

    # this library, both precisions; a first call traces and tunes
    ours = {}
    updates = None
    with Simulation(model) as sim:
        sim.compute_spectral_discretisation()
        sim.compute_boundary_intensities()
        sim.compute_LTE_level_populations()
        kap = sim.emissivity_opacity()[1]
        for prec in ("fp64", "mixed"):
            sim.compute_radiation_field(prec, keep_J=True)
            walls, devs = [], []
            for _ in range(3):
                t = time.perf_counter()
                sim.compute_radiation_field(prec, keep_J=True)
                walls.append(time.perf_counter() - t)
                ms, updates = sim.solve_stats()
                devs.append(ms * 1e-3)
            sim.compute_Jeff()
            ours[prec] = {"solve_device_s": min(devs), "call_wall_s": min(walls),
                          "J": rel_stats(sim.J, J_cpu), "Jlin": rel_stats(sim.Jlin, Jl_cpu),
                          "Lambda": rel_stats(sim.Lambda, L_cpu)}
    for v in ours.values():
        v["updates_per_s"] = updates / v["solve_device_s"]
    line = {
        "model": model.name, "cells": N, "ray_pairs": model.nrays // 2, "bins": nf,
        "updates_per_solve": updates,
        "reference_cpu": {"compute_radiation_field_s": cpu_rf[-1] if cpu_rf else None,
                          "updates_per_s": updates / cpu_rf[-1] if cpu_rf else None,
                          "program_wall_s": cpu_wall, "threads": threads,
                          "cpu": cpu_model(),
                          "what": "the reference's Timer around compute_radiation_field "
                                  "(magritte_ref radiation, OpenMP over all host cores); the "
                                  "program's wall time adds reading, set-up, Jeff and writing"},
        "ours": ours,
    }
    if model.meta.get("kind") == "lattice_cloud":
        # line-centre optical depth across the cube along a lattice axis:
        # chi(nu_line) = kappa nu phi = kappa / (sqrt(pi) pw), uniform cells
        pw = np.sqrt(2.0 * 1.38064852e-23 / (1.66053904e-27 * 2.99792458e8 ** 2)
                     * model.linedata.inverse_mass * model.temperature + model.vturb2)
        chi0 = kap / (np.sqrt(np.pi) * pw[:, None])
        line["line_centre_tau_across"] = float(chi0.max() * model.meta["L"])

    if not args.no_ref_gpu:
        # the reference's GPU path, one OpenMP thread
        out_gpu = os.path.join(tmp, "gpu")
        os.makedirs(out_gpu)
        text, _ = run([REF_GPU, folder, out_gpu, "gpu", str(args.block), str(args.nblocks),
                       str(args.reps)], out_gpu, 1, args.timeout)
        reps = [json.loads(l) for l in text.splitlines() if l.startswith("{\"rep\"")]
        # the reference's own Timer around each call ("-- overall"; its
        # "-- compute" line prints the last block's interval only)
        overall = [float(l.split(":")[-1].split()[0]) for l in text.splitlines()
                   if l.startswith("T ") and "GPU compute radiation field -- overall" in l]
        J_gpu = np.fromfile(os.path.join(out_gpu, "J.bin"))
        Jl_gpu = np.fromfile(os.path.join(out_gpu, "Jlin.bin"))
        L_gpu = np.fromfile(os.path.join(out_gpu, "Lambda.bin"))
        warm = reps[-1]["seconds"]
        line["reference_gpu"] = {
            "seconds_per_call": [r["seconds"] for r in reps], "reference_timer_overall_s": overall,
            "threads": 1, "block": args.block, "nblocks": args.nblocks,
            "max_npoints_on_rays": reps[-1]["max_npoints_on_rays"],
            "updates_per_s": updates / warm if updates else None,
            "J": rel_stats(J_gpu, J_cpu), "Jlin": rel_stats(Jl_gpu, Jl_cpu),
            "Lambda": rel_stats(L_gpu, L_cpu)}
        line["speedup_vs_reference_gpu"] = {k: warm / v["call_wall_s"] for k, v in ours.items()}
    s = json.dumps(line)
    print(s)
    if args.out:
        with open(args.out, "w") as f:
            f.write(s + "\n")


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for l in f:
                if l.startswith("model name"):
                    return l.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


if __name__ == "__main__":
    main()
