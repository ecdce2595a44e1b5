"""Magritte's own Simulation routed to the B200 library through the C++
binding (magritte_b200/integration/magritte_b200_binding.cpp).

``oracle/_ref/magritte_ref_b200`` is the reference's C++ (its model reader,
set-up and Simulation object, compiled here by oracle/ref_build.sh) calling
``compute_level_populations_b200`` / ``compute_radiation_field_b200``;
``oracle/_ref/magritte_ref`` is the same reference running its own CPU
``compute_level_populations`` / ``compute_radiation_field``.  On the same
model folder they must agree: FP64 populations to 1e-6 (levels above 1e-6
of the total) after the same number of iterations of the reference's own
stop test, J to 1e-6.  Both binaries are built where the reference's
sources are; elsewhere the test skips.
"""
import os
import subprocess

import numpy as np
import pytest

import magritte_b200.model as M
from magritte_b200 import io_text

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "magritte_ref")
REF_B200 = os.path.join(ROOT, "oracle", "_ref", "magritte_ref_b200")

needs = pytest.mark.skipif(not (os.path.exists(REF) and os.path.exists(REF_B200)),
                           reason="reference binaries not built (needs the reference's sources)")


def run(binary, folder, out, *args):
    os.makedirs(out, exist_ok=True)
    env = dict(os.environ, OMP_NUM_THREADS=str(min(16, os.cpu_count() or 1)))
    r = subprocess.run([binary, folder, out, *args], capture_output=True, text=True, env=env,
                       cwd=out, timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]


def rel(a, b):
    with np.errstate(invalid="ignore", divide="ignore"):
        r = np.abs(a - b) / np.abs(b)
    r[a == b] = 0.0
    return float(np.nanmax(r))


@needs
@pytest.mark.parametrize("make,max_iter", [
    (M.config1, 12),
    (lambda: M.wind_model(8, seed=7, nlev=5, nside=1, name="wind8"), 9),
])
def test_binding_reproduces_reference_ali(gpu, tmp_path, make, max_iter):
    model = make()
    folder = str(tmp_path / "model") + "/"
    io_text.write_model(model, folder)
    run(REF_B200, folder, str(tmp_path / "b200"), "ali", str(max_iter))
    run(REF, folder, str(tmp_path / "ref"), "ali", str(max_iter))
    it_b = int(np.fromfile(tmp_path / "b200" / "iterations.bin")[0])
    it_r = int(np.fromfile(tmp_path / "ref" / "iterations.bin", dtype=np.int64)[0])
    assert it_b == it_r
    pb = np.fromfile(tmp_path / "b200" / "population.bin").reshape(model.ncells, -1)
    pr = np.fromfile(tmp_path / "ref" / "population.bin").reshape(model.ncells, -1)
    big = pr > 1e-6 * model.population_tot[:, None]
    assert rel(pb[big], pr[big]) < 1e-6


@needs
def test_binding_reproduces_reference_radiation_field(gpu, tmp_path):
    model = M.wind_model(8, seed=7, nlev=5, nside=1, name="wind8")
    folder = str(tmp_path / "model") + "/"
    io_text.write_model(model, folder)
    run(REF_B200, folder, str(tmp_path / "b200"), "radiation")
    run(REF, folder, str(tmp_path / "ref"), "radiation")
    Jb = np.fromfile(tmp_path / "b200" / "J.bin")
    Jr = np.fromfile(tmp_path / "ref" / "J.bin")
    assert rel(Jb, Jr) < 1e-6
