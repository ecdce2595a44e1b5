"""Non-local ALO (parameters.n_off_diag) in the oracle (CPU; test
infrastructure).

* The origin's row of a ray pair's Lambda operator from the non-local branch
  of RayPair::solve (raypair_solver.tpp:336-388) equals the row of the
  inverse of the pair's Feautrier matrix.
* n_off_diag = 1 adds no off-diagonal element (raypair_lambda.tpp:129 starts
  at m = 1) and gives the local ALO's results; the reference's compiled C++
  with n_off_diag = 1 agrees with the oracle.
* With 2 <= n_off_diag the ALI iteration converges to the local ALO's fixed
  point: the ALO changes how the iteration gets there, not where it ends.
"""
import os
import subprocess

import numpy as np
import pytest

import magritte_b200.model as M
from magritte_b200 import io_text

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "magritte_ref")
THREADS = min(8, os.cpu_count() or 1)


def feautrier_matrix(dtau):
    """The ray pair's matrix with the reference's coefficients
    (raypair_solver.tpp:200-260): boundary rows 1 + 2/dtau + 2/dtau^2 and
    -2/dtau^2, interior rows -A, 1 + A + C, -C."""
    n = dtau.shape[0] + 1
    T = np.zeros((n, n))
    T[0, 0] = 1 + 2 / dtau[0] + 2 / dtau[0] ** 2
    T[0, 1] = -2 / dtau[0] ** 2
    for i in range(1, n - 1):
        da = 0.5 * (dtau[i - 1] + dtau[i])
        A, C = 1 / (da * dtau[i - 1]), 1 / (da * dtau[i])
        T[i, i - 1], T[i, i], T[i, i + 1] = -A, 1 + A + C, -C
    T[n - 1, n - 1] = 1 + 2 / dtau[-1] + 2 / dtau[-1] ** 2
    T[n - 1, n - 2] = -2 / dtau[-1] ** 2
    return T


@pytest.mark.parametrize("ndep,n_ar", [(2, 1), (7, 1), (9, 4), (9, 8), (12, 3), (40, 20)])
def test_lambda_row_is_the_inverse_row(ndep, n_ar):
    rng = np.random.default_rng(ndep * 100 + n_ar)
    dtau = 10 ** rng.uniform(-3, 2, ndep - 1)
    term1 = rng.uniform(0.1, 1.0, ndep)
    M_ = 5
    diag, lo, up = oracle.raypair_lambda_row(n_ar, term1, dtau, M_)
    L = np.linalg.inv(feautrier_matrix(dtau))
    assert diag == pytest.approx(L[n_ar, n_ar], rel=1e-12)
    for d in range(1, M_):
        ref_lo = L[n_ar, n_ar - d] if n_ar - d >= 0 else 0.0
        ref_up = L[n_ar, n_ar + d] if n_ar + d <= ndep - 1 else 0.0
        assert lo[d - 1] == pytest.approx(ref_lo, rel=1e-11, abs=1e-300)
        assert up[d - 1] == pytest.approx(ref_up, rel=1e-11, abs=1e-300)


def small_wind():
    return M.wind_model(8, seed=7, nlev=5, nside=1, name="wind8")


def test_n_off_diag_one_is_the_local_alo():
    m = small_wind()
    a = oracle.Oracle(m).setup()
    b = oracle.Oracle(m).setup().set_n_off_diag(1)
    it_a, h_a = a.compute_level_populations(True, 20, 1e-8)
    it_b, h_b = b.compute_level_populations(True, 20, 1e-8)
    assert it_a == it_b
    np.testing.assert_allclose(b.pop, a.pop, rtol=1e-12)
    np.testing.assert_allclose(b.Ls, a.Ls, rtol=1e-12)


@pytest.mark.parametrize("noff", [2, 3])
def test_nonlocal_ali_keeps_the_fixed_point(noff):
    m = small_wind()
    loc = oracle.Oracle(m).setup()
    loc.compute_level_populations(True, 40, 1e-9)
    nl = oracle.Oracle(m).setup().set_n_off_diag(noff)
    it, hist = nl.compute_level_populations(True, 40, 1e-9)
    assert hist[-1] < 1e-9 and nl.lu_errors == 0
    # every point of each pair that exists has its cell; the rest are -1
    assert (nl.Loff_nr >= -1).all() and (nl.Loff_nr >= 0).mean() > 0.8
    assert np.isfinite(nl.Loff).all() and (nl.Loff[nl.Loff_nr[:, None].repeat(m.nlines, 1) < 0] == 0).all()
    sel = loc.pop > 1e-10 * m.population_tot[:, None]
    rel = np.abs(nl.pop - loc.pop)[sel] / loc.pop[sel]
    assert rel.max() < 1e-7


@pytest.mark.skipif(not os.path.exists(REF), reason="oracle/_ref not built (needs the reference's sources)")
def test_reference_with_n_off_diag_one_matches(tmp_path):
    """The reference's compiled C++ with n_off_diag = 1 (its non-local solve
    branch, no off-diagonal element) against the oracle with the same
    setting: J, Jlin and the ALO after one formal solve."""
    m = small_wind()
    folder = str(tmp_path / "model") + "/"
    out = tmp_path / "out"
    out.mkdir()
    io_text.write_model(m, folder)
    env = dict(os.environ, OMP_NUM_THREADS=str(THREADS), MGR_REF_N_OFF_DIAG="1")
    r = subprocess.run([REF, folder, str(out), "radiation"], capture_output=True, text=True,
                       env=env, cwd=str(out), timeout=600)
    assert r.returncode == 0, r.stderr[-2000:] + r.stdout[-2000:]
    orc = oracle.Oracle(m).setup().set_n_off_diag(1)
    orc.compute_radiation_field(nthreads=THREADS)
    orc.compute_Jeff()
    N, K = m.ncells, m.nlines
    J = np.fromfile(out / "J.bin").reshape(orc.J.shape)
    Jlin = np.fromfile(out / "Jlin.bin").reshape(N, K)
    Lam = np.fromfile(out / "Lambda.bin").reshape(N, K)
    np.testing.assert_allclose(orc.J, J, rtol=1e-12, atol=0)
    np.testing.assert_allclose(orc.Jlin, Jlin, rtol=1e-12, atol=0)
    np.testing.assert_allclose(orc.Ls, Lam, rtol=1e-12, atol=0)
