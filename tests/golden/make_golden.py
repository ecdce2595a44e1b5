"""Writes the golden fixtures of tests/golden/ from the CPU oracle.

Run from the repository root:  python tests/golden/make_golden.py
Each fixture holds a small seeded model's formal-solve outputs (J, Jlin, the
diagonal ALO) with LTE populations, and the populations after three ALI
iterations.  The GPU tests compare the device path with these files without
running the oracle; the CPU tests check the oracle still reproduces them.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import magritte_b200.model as M  # noqa: E402
import oracle  # noqa: E402

CASES = {
    "lattice6": lambda: M.lattice_cloud(6, name="lattice6"),
    "wind6": lambda: M.wind_model(6, seed=21, nlev=5, nside=1, name="wind6"),
    "thick6": lambda: M.lattice_cloud(6, n_h2=1.0e15, name="thick6"),
    # turbulent cloud: 41 bins per line, k^-4 velocity field (Doppler sub-points)
    "turb6": lambda: M.turbulent_cloud(6, seed=31, nlev=6, npairs=6, nquads=41, name="turb6"),
}


def compute(name):
    model = CASES[name]()
    o = oracle.Oracle(model).setup()
    o.compute_radiation_field()
    o.compute_Jeff()
    out = dict(J=o.J.copy(), Jlin=o.Jlin.copy(), Ls=o.Ls.copy(), pop_lte=o.pop.copy())
    it, hist = o.compute_level_populations(use_ng=True, max_iter=3, tol_max_rel=1e-30)
    out.update(pop_it3=o.pop.copy(), err_max_it3=hist)
    return out


def main():
    for name in CASES:
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **compute(name))
        print("wrote", name)


if __name__ == "__main__":
    main()
