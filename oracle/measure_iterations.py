"""Runs the CPU oracle's full ALI + Ng iteration on a benchmark workload and
records its iteration history (TEST AND BENCHMARK INFRASTRUCTURE ONLY).

The record says how many formal solves and how many Ng steps the
reference's algorithm (LTE start, FP64, Ng after every four normal
iterations as in Simulation::compute_level_populations,
src/Simulation/sim_lines.tpp:101-129) needs to reach a max relative
population change below the tolerance.  ``bench.py --impl reference``
multiplies its sampled per-step CPU times by these counts.

    python oracle/measure_iterations.py wind64      # writes oracle/iterations_wind64.json
"""
from __future__ import annotations

import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)

TOL = 1.0e-4


def step_kinds(iterations: int, use_ng: bool = True, ng_every: int = 4):
    """Kinds of the iterations of the reference's loop: 'solve' (formal
    solve + Jeff + statistical equilibrium) or 'ng' (sim_lines.tpp:110-118:
    an Ng step after every four normal iterations, counted as an
    iteration; ng_every normal iterations where the loop was run so)."""
    kinds, normal = [], 0
    for _ in range(iterations):
        if use_ng and normal == ng_every:
            kinds.append("ng")
            normal = 0
        else:
            kinds.append("solve")
            normal += 1
    return kinds


def main():
    import oracle
    import magritte_b200.model as M
    name = sys.argv[1] if len(sys.argv) > 1 else "wind64"
    builders = {"wind64": M.config2, "wind32": lambda: M.wind_model(32, seed=2, nlev=10, nside=2,
                                                                      name="wind32")}
    model = builders[name]()
    t0 = time.perf_counter()
    orc = oracle.Oracle(model).setup()
    it, hist = orc.compute_level_populations(True, 400, TOL, nthreads=os.cpu_count() or 1)
    dt = time.perf_counter() - t0
    kinds = step_kinds(it)
    rec = {"workload": name, "tol_max_rel": TOL, "start": "LTE", "precision": "fp64",
           "iterations": it, "formal_solves": kinds.count("solve"), "ng_steps": kinds.count("ng"),
           "history": [float(x) for x in hist], "seconds": dt, "threads": os.cpu_count(),
           "converged": bool(hist[-1] < TOL)}
    out = os.path.join(HERE, f"iterations_{name}.json")
    with open(out, "w") as f:
        json.dump(rec, f, indent=1)
    print(json.dumps(rec))


if __name__ == "__main__":
    main()
