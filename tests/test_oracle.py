"""Pins of the CPU oracle against the reference's own known answers.

Each test restates one of the reference's tests or analytic checks:
* Doppler shifts: tests/unit/Model/Geometry/test_geometry.cpp:46-59;
* T L = I on a ray pair: tests/unit/Simulation/Raypair/test_raypair.cpp:83-163;
* constant slab J: tests/integration/test_0_1D_all_constant.py:240-244;
* statistical-equilibrium balance: tests/unit/Model/Lines/test_lineProducingSpecies.cpp:157-160;
* detailed balance and Einstein relations: magritte/setup/setup.py:452, :488-489.
Plus a pure-Python restatement of the tracer on small grids, and the
two-sided Feautrier sweep the device uses against the reference's
elimination + back substitution.
"""
import math

import numpy as np
import pytest

import magritte_b200.model as M
import oracle


def _doppler_model():
    pos, offs, nbr, b2c = M.chain_grid(4, 1.0)
    m = M._assemble(pos, offs, nbr, b2c, np.zeros((4, 3)), 20.0, 150.0, np.full(4, 1e12), 1e-4,
                    M.two_level_species(), np.array([[1.0, 0, 0], [-1.0, 0, 0]]),
                    np.array([0.5, 0.5]), 5, "doppler", {})
    m.velocity[:, 0] = [0.2, 0.3, 0.1, -0.1]
    return m


def test_doppler_shift_kat():
    o = oracle.Oracle(_doppler_model())
    assert [o.doppler_shift(0, 0, c) for c in range(4)] == [1.0, 0.9, 1.1, 1.3]
    assert [o.doppler_shift(0, 0, c, rest=True) for c in range(4)] == [0.8, 0.7, 0.9, 1.1]


def _feautrier_matrix(term1, dtau, I0, In):
    """T and S of test_raypair.cpp:83-118 (boundary rows with the 2/dtau
    and 2/dtau^2 terms, interior 1 + A + C)."""
    n = term1.shape[0]
    T = np.zeros((n, n))
    S = term1.copy()
    for d in range(1, n - 1):
        A = 2.0 / ((dtau[d - 1] + dtau[d]) * dtau[d - 1])
        C = 2.0 / ((dtau[d - 1] + dtau[d]) * dtau[d])
        T[d, d - 1] = -A
        T[d, d + 1] = -C
        T[d, d] = 1.0 + A + C
    T[0, 0] = 1 + 2.0 / dtau[0] + 2.0 / dtau[0] ** 2
    T[0, 1] = -2.0 / dtau[0] ** 2
    T[-1, -1] = 1 + 2.0 / dtau[-1] + 2.0 / dtau[-1] ** 2
    T[-1, -2] = -2.0 / dtau[-1] ** 2
    S[0] += 2.0 * I0 / dtau[0]
    S[-1] += 2.0 * In / dtau[-1]
    return T, S


def two_sided_sweep(n_ar, term1, dtau, I0, In):
    """The device's elimination (magritte_b200/csrc/solve.cu, Chain and
    ProjChain): the front half is eliminated from its far end toward the
    origin and the back half from its far end toward the origin, on half
    optical depths dh = dtau/2 in projective form F~ = a/b, S~ = c/b with a
    power-of-two rescaling after each step, and the halves meet in the
    origin's row."""
    import math
    last = term1.shape[0] - 1
    o = n_ar

    def half(idx_far_to_origin, dh_list, I):
        # idx: point indices from the far end to the point next to the origin
        t_far = term1[idx_far_to_origin[0]]
        dh = dh_list[0]
        a = dh * (dh + 1.0)
        b = 2.0 * a + 1.0
        c = dh * (t_far * dh + I)
        dp = dh
        for k in range(1, len(dh_list)):
            dh = dh_list[k]
            t = term1[idx_far_to_origin[k]]
            H = dp + dh
            P, Q = H * dp, H * dh
            Pb = P * b
            a = Q * (Pb + a)
            c = Q * (t * Pb + c)
            b = 2.0 * a + Pb
            sc = 2.0 ** -(math.frexp(b)[1] - 1)
            a, b, c = a * sc, b * sc, c * sc
            dp = dh
        return a, b, c, dp

    # front: points 0 .. o-1, segment n between n and n+1
    af, bf, cf, df = half(list(range(0, o)), [0.5 * dtau[n] for n in range(0, o)], I0)
    to = term1[o]
    if o == last:
        D = 1.0 / (df * (df + 1.0) * bf + af)
        return (df * (to * df + In) * bf + cf) * D, df * df * bf * D
    ab, bb, cb, db = half(list(range(last, o, -1)),
                          [0.5 * dtau[n] for n in range(last - 1, o - 1, -1)], In)
    H = df + db
    P, Q = H * df, H * db
    PQB = P * Q * (bf * bb)
    D = 1.0 / (af * bb * Q + ab * bf * P + PQB)
    return (to * PQB + cf * bb * Q + cb * bf * P) * D, PQB * D


@pytest.mark.parametrize("n_ar,n_r", [(5, 5), (1, 0), (1, 1), (2, 1), (7, 0), (12, 3), (30, 29)])
@pytest.mark.parametrize("scale", [1e-3, 1.0, 1e3])
def test_raypair_T_L_identity(n_ar, n_r, scale):
    rng = np.random.default_rng(n_ar * 100 + n_r)
    ndep = n_ar + n_r + 1
    term1 = rng.uniform(0.5, 2.0, ndep)
    dtau = scale * rng.uniform(0.1, 3.0, ndep - 1)
    I0, In = rng.uniform(0, 1, 2)
    T, S = _feautrier_matrix(term1, dtau, I0, In)
    Tinv = np.linalg.inv(T)
    u_ref = (Tinv @ S)[n_ar]
    L_ref = Tinv[n_ar, n_ar]
    u, L = oracle.solve_raypair(n_ar, term1, dtau, I0, In)
    assert abs(u - u_ref) <= 1e-9 * abs(u_ref)
    assert abs(L - L_ref) <= 1e-9 * abs(L_ref)
    u2, L2 = two_sided_sweep(n_ar, term1, dtau, I0, In)
    assert abs(u2 - u) <= 1e-12 * abs(u)
    assert abs(L2 - L) <= 1e-12 * abs(L)


def test_two_sided_sweep_extreme_depths():
    """Optically thin (dtau ~ 1e-12) and thick (dtau ~ 1e4) segments."""
    rng = np.random.default_rng(3)
    for scale in (1e-12, 1e-6, 1e4):
        for n_ar, n_r in ((40, 39), (60, 0)):
            ndep = n_ar + n_r + 1
            term1 = rng.uniform(0.5, 2.0, ndep)
            dtau = scale * rng.uniform(0.1, 3.0, ndep - 1)
            u, L = oracle.solve_raypair(n_ar, term1, dtau, 0.3, 0.7)
            u2, L2 = two_sided_sweep(n_ar, term1, dtau, 0.3, 0.7)
            assert abs(u2 - u) <= 1e-10 * abs(u), scale
            assert abs(L2 - L) <= 1e-10 * abs(L), scale


def _slab_error(n, x_abund):
    m = M.slab_1d(n, x_abund=x_abund)
    o = oracle.Oracle(m).setup()
    o.compute_radiation_field()
    ld = m.linedata
    eps, kap = o.emissivity[0, 0], o.opacity[0, 0]
    pw = math.sqrt(2 * M.KB / (M.AMU * M.C_SQUARED) * ld.inverse_mass * m.temperature[0]
                   + m.vturb2[0])
    nu0 = ld.frequency[0]
    dnu = nu0 * pw
    x = m.position[:, 0]
    L = x[-1]
    nu = o.nu[0]
    phi = 1 / (math.sqrt(math.pi) * dnu) * np.exp(-((nu - nu0) / dnu) ** 2)
    chi = kap * nu * phi + 1e-26
    S = eps * nu * phi / chi
    B = o.I_bdy[0]
    J = S[None, :] + 0.5 * (B - S)[None, :] * (np.exp(-chi[None, :] * x[:, None])
                                             + np.exp(-chi[None, :] * (L - x)[:, None]))
    return float(np.max(np.abs(o.J - J) / J))


def _gradient_slab_error(n, vmax, x_abund=1e-4):
    """The slab with velocity rising linearly to vmax along x against the
    closed form of tests/integration/test_1_1D_velocity_gradient.py: with
    a = vmax/c, tau_nu(l) = kappa L nu / (a nu) * 1/2
    (erf((nu - nu0)/dnu) + erf(a nu/dnu l/L - (nu - nu0)/dnu)) in each
    direction, J = S + (B - S)/2 (e^-tau(x) + e^-tau(L - x))."""
    from scipy.special import erf
    m = M.slab_1d(n, x_abund=x_abund, vmax=vmax)
    o = oracle.Oracle(m).setup()
    o.compute_radiation_field()
    ld = m.linedata
    eps, kap = o.emissivity[0, 0], o.opacity[0, 0]
    pw = math.sqrt(2 * M.KB / (M.AMU * M.C_SQUARED) * ld.inverse_mass * m.temperature[0]
                   + m.vturb2[0])
    nu0 = ld.frequency[0]
    dnu = nu0 * pw
    x = m.position[:, 0]
    L = x[-1]
    nu = o.nu[0][None, :]
    fct = vmax / M.CC * nu / dnu
    arg = (nu - nu0) / dnu

    def tau(l):
        return kap * L * nu / (fct * dnu) * 0.5 * (erf(arg) + erf(fct * l / L - arg))

    S = eps / kap
    B = o.I_bdy[0][None, :]
    J = S + 0.5 * (B - S) * (np.exp(-tau(x[:, None])) + np.exp(-tau((L - x)[:, None])))
    return float(np.max(np.abs(o.J - J) / J))


def test_velocity_gradient_slab_analytic():
    """J of the velocity-gradient slab (2 Doppler widths across) against the
    closed form; second-order convergence as for the constant slab."""
    e50 = _gradient_slab_error(50, 980.0)
    e200 = _gradient_slab_error(200, 980.0)
    assert e50 < 2e-3
    assert e200 < e50 / 8.0


@pytest.mark.parametrize("x_abund,tol50", [(1e-6, 1e-8), (1e-4, 1e-4), (1e-3, 1e-2)])
def test_constant_slab_analytic(x_abund, tol50):
    """J of a constant slab against the closed form; the error falls as
    1/n^2 (second-order Feautrier)."""
    e50 = _slab_error(50, x_abund)
    e200 = _slab_error(200, x_abund)
    assert e50 < tol50
    assert e200 < e50 / 8.0


def _rate_matrix(model, Jeff, Ls, pop_prev, p):
    """Independent numpy assembly of one cell's block of RT
    (lineProducingSpecies.tpp:282-389)."""
    ld = model.linedata
    nl = ld.nlev
    last = nl - 1
    Mx = np.zeros((nl, nl))
    for k in range(ld.nrad):
        I, J = ld.irad[k], ld.jrad[k]
        vIJ = ld.A[k] + ld.Bs[k] * Jeff[p, k]
        vJI = ld.Ba[k] * Jeff[p, k]
        if J != last:
            Mx[J, I] += vIJ
            Mx[J, J] -= vJI
        if I != last:
            Mx[I, J] += vJI
            Mx[I, I] -= vIJ
    for k in range(ld.nrad):
        I, J = ld.irad[k], ld.jrad[k]
        opac = M.HH / (4 * math.pi) * (pop_prev[p, J] * ld.Ba[k] - pop_prev[p, I] * ld.Bs[k])
        v = -Ls[p, k] * opac
        if J != last:
            Mx[J, I] += v
        if I != last:
            Mx[I, I] -= v
    T = model.temperature[p]
    for cp in ld.colpar:
        abn = model.abundance[p, cp.num_col_partner]
        tmp = cp.tmp
        if T >= tmp[-1]:
            t = len(tmp) - 1
        elif T <= tmp[0]:
            t = 0
        else:
            t = int(np.searchsorted(tmp, T))
        if t == 0:
            Cd, Ce = cp.Cd[0], cp.Ce[0]
        else:
            s = (T - tmp[t - 1]) / (tmp[t] - tmp[t - 1])
            Cd = cp.Cd[t - 1] + (cp.Cd[t] - cp.Cd[t - 1]) * s
            Ce = cp.Ce[t - 1] + (cp.Ce[t] - cp.Ce[t - 1]) * s
        for k in range(len(cp.icol)):
            I, J = cp.icol[k], cp.jcol[k]
            vIJ, vJI = Cd[k] * abn, Ce[k] * abn
            if J != last:
                Mx[J, I] += vIJ
                Mx[J, J] -= vJI
            if I != last:
                Mx[I, J] += vJI
                Mx[I, I] -= vIJ
    Mx[last, :] += 1.0
    y = np.zeros(nl)
    y[last] = model.population_tot[p]
    return Mx, y


def test_statistical_equilibrium_balance():
    model = M.wind_model(6, seed=5, nlev=6, nside=1, name="wind6")
    o = oracle.Oracle(model).setup()
    o.compute_radiation_field()
    o.compute_Jeff()
    prev = o.pop.copy()
    assert o.compute_level_populations_from_stateq() == 0
    for p in range(0, model.ncells, 7):
        Mx, y = _rate_matrix(model, o.Jeff, o.Ls, prev, p)
        r = Mx @ o.pop[p] - y
        scale = np.abs(Mx).max(1) * np.abs(o.pop[p]).max()
        assert np.all(np.abs(r) <= 1e-10 * scale + 1e-300)
        assert abs(o.pop[p].sum() - model.population_tot[p]) <= 1e-12 * model.population_tot[p]


def test_detailed_balance_gives_lte():
    """With Jeff = B_nu(T) at every line and no ALO term, the rate equations
    (radiative Einstein relations + collisional detailed balance) return
    the Boltzmann populations at T.  T is set to a temperature of the rate
    table, where the interpolated Ce/Cd ratio is exactly the detailed-balance
    one (between table points the reference interpolates Ce and Cd linearly,
    collisionPartner.tpp:15-47, and the balance holds only approximately)."""
    model = M.wind_model(5, seed=9, nlev=8, nside=1, name="wind5")
    model.temperature[:] = 200.0
    o = oracle.Oracle(model).setup()
    lte = o.pop.copy()
    ld = model.linedata
    nu = ld.frequency
    for p in range(model.ncells):
        T = model.temperature[p]
        o.Jeff[p] = 2 * M.HH / M.C_SQUARED * nu ** 3 / np.expm1(M.HH / M.KB / T * nu)
    o.Ls[:] = 0.0
    o.pop[:] = model.population_tot[:, None] / ld.nlev
    o.compute_level_populations_from_stateq()
    floor = 1e-12 * model.population_tot[:, None]
    assert np.all(np.abs(o.pop - lte) <= 1e-8 * np.abs(lte) + floor)


def _py_trace(model, o, r):
    """Pure-Python restatement of Geometry::trace_ray<CoMoving>
    (geometry.tpp:21-207) for small grids."""
    pos, vel, ray = model.position, model.velocity, model.rays[r]
    bmask = model.boundary_mask()
    pw = math.sqrt(2.0 * M.KB / (M.AMU * M.C_SQUARED) * model.linedata.inverse_mass
                   * model.temperature[o] + model.vturb2[o])
    dsm = model.max_width_fraction * pw

    def dot(a, b):
        return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]

    def shift(c):
        dv = [vel[c][i] - vel[o][i] for i in range(3)]
        return 1.0 - dot(dv, ray)

    def nxt(cur, Z, dZ):
        dmin, best = float("inf"), -1
        for nb in model.nbr_list[model.nbr_offsets[cur]:model.nbr_offsets[cur + 1]]:
            R = [pos[nb][i] - pos[o][i] for i in range(3)]
            Zn = dot(R, ray)
            if Zn > Z:
                d2 = dot(R, R) - Zn * Zn
                if d2 < dmin:
                    dmin, best, dZ = d2, int(nb), Zn - Z
        return best, Z + dZ, dZ

    out = []

    def set_data(crt, nx, sc, sn, dz):
        ds = sn - sc
        if abs(ds) > dsm:
            n = int(abs(ds) / dsm + 1)
            half = int(0.5 * n)
            dzi, dsi = dz / n, ds / n
            for k in range(1, half):
                out.append((crt, sc + k * dsi, dzi))
            for k in range(half, n + 1):
                out.append((nx, sc + k * dsi, dzi))
        else:
            out.append((nx, sn, dz))

    nx, Z, dZ = nxt(o, 0.0, 0.0)
    if nx == -1:
        return out
    crt = o
    sc, sn = shift(crt), shift(nx)
    set_data(crt, nx, sc, sn, dZ)
    while not bmask[nx]:
        sc, crt = sn, nx
        nx, Z, dZ = nxt(nx, Z, dZ)
        assert nx >= 0
        sn = shift(nx)
        set_data(crt, nx, sc, sn, dZ)
    return out


def test_tracer_python_restatement():
    model = M.wind_model(5, seed=13, nlev=3, nside=1, vmax=60e3, name="wind5v")
    o = oracle.Oracle(model)
    n_interp = 0
    for org in range(model.ncells):
        for r in range(model.nrays):
            ref = _py_trace(model, org, r)
            c, s, z = o.trace_ray(org, r)
            assert [x[0] for x in ref] == list(c)
            assert [x[1] for x in ref] == list(s)
            assert [x[2] for x in ref] == list(z)
            n_interp += int(np.sum(c[:-1] == c[1:]))
    assert n_interp > 0   # the velocity field forces interpolation points


def test_spectral_grid_is_identity_sorted():
    for model in (M.config1(), M.wind_model(6, nlev=10, nside=1)):
        o = oracle.Oracle(model)
        o.compute_spectral_discretisation()
        assert o.identity_sort
        assert np.all(np.diff(o.nu, axis=1) > 0)
        nq = model.nquads
        expect = np.arange(model.nfreqs).reshape(model.nlines, nq)
        assert np.array_equal(o.nr_line[0], expect)


def test_ng_matches_formula():
    model = M.lattice_cloud(4, name="l4")
    o = oracle.Oracle(model).setup()
    rng = np.random.default_rng(2)
    base = o.pop.copy()
    hist = [base * (1 + 0.1 * rng.uniform(-1, 1, base.shape)) for _ in range(4)]
    o.pop[:], o.prev1[:], o.prev2[:], o.prev3[:] = hist
    P, p1, p2, p3 = (h.ravel() for h in hist)
    Q1, Q2, Q3 = P - 2 * p1 + p2, P - p1 - p2 + p3, P - p1
    A1, A2, B2, C1, C2 = Q1 @ Q1, Q1 @ Q2, Q2 @ Q2, Q1 @ Q3, Q2 @ Q3
    den = A1 * B2 - A2 * A2
    a, b = (C1 * B2 - C2 * A2) / den, (C2 * A1 - C1 * A2) / den
    expect = (1 - a - b) * P + a * p1 + b * p2
    o.ng_acceleration()
    assert np.allclose(o.pop.ravel(), expect, rtol=1e-10)
    assert np.array_equal(o.prev1.ravel(), P)


def test_ng_cadence_keeps_the_fixed_point():
    """ALI + Ng with three normal iterations before each Ng step (instead of
    the reference's four): the Ng step falls on the 4th iteration, and the
    iteration converges to the same populations."""
    pops = {}
    for ng in (4, 3):
        orc = oracle.Oracle(M.config1()).setup()
        it, hist = orc.compute_level_populations(True, 40, 1e-9, ng_every=ng)
        assert hist[-1] < 1e-9
        pops[ng] = orc.pop.copy()
    p4, p3 = pops[4], pops[3]
    mask = p4 > 1e-10 * p4.sum(1, keepdims=True)
    assert np.max(np.abs(p3 - p4)[mask] / p4[mask]) < 1e-7
    # the cadence itself: the first three iterations are the same normal
    # ones; the 4th is the Ng step with ng_every = 3 and a normal one with 4
    h = {}
    for ng in (4, 3):
        orc = oracle.Oracle(M.config1()).setup()
        _, h[ng] = orc.compute_level_populations(True, 5, 1e-30, ng_every=ng)
    assert np.array_equal(h[3][:3], h[4][:3]) and h[3][3] != h[4][3]


def test_step_kinds_follow_the_cadence():
    """The iteration kinds the CPU baseline charges: an Ng step after every
    four normal iterations (the reference), or after every three."""
    from oracle.measure_iterations import step_kinds
    assert step_kinds(5) == ["solve"] * 4 + ["ng"]
    assert step_kinds(9) == (["solve"] * 4 + ["ng"]) + ["solve"] * 4
    assert step_kinds(4, ng_every=3) == ["solve"] * 3 + ["ng"]
    assert step_kinds(8, ng_every=3) == (["solve"] * 3 + ["ng"]) * 2
    assert step_kinds(6, use_ng=False) == ["solve"] * 6


def test_ali_oracle_converges_and_is_stationary():
    model = M.lattice_cloud(6, name="l6")
    o = oracle.Oracle(model).setup()
    it, hist = o.compute_level_populations(True, 300, 1e-8)
    assert hist[-1] < 1e-8
    assert it < 300
    # a further plain iteration changes nothing beyond the tolerance
    pop = o.pop.copy()
    o.compute_radiation_field()
    o.compute_Jeff()
    o.compute_level_populations_from_stateq()
    assert np.max(np.abs(o.pop - pop) / pop) < 1e-7


def test_concat_models_keeps_each_member():
    """A batch renumbers cells, neighbours and boundary cells; every member's
    rays trace exactly as in the member alone (graphs stay disjoint)."""
    ms = [M.wind_model(n, seed=40 + i, nlev=4, npairs=3, name=f"m{i}", species_seed=40,
                       ray_seed=40) for i, n in enumerate((4, 5))]
    b = M.concat_models(ms)
    seg = b.meta["segments"]
    assert seg == [0, 64, 64 + 125]
    assert b.ncells == 189 and b.nboundary == ms[0].nboundary + ms[1].nboundary
    ob = oracle.Oracle(b).setup()
    for s, m in enumerate(ms):
        om = oracle.Oracle(m).setup()
        for o in (0, m.ncells // 2, m.ncells - 1):
            for r in range(m.nrays):
                cm, shm, dzm = om.trace_ray(o, r)
                cb, shb, dzb = ob.trace_ray(o + seg[s], r)
                assert np.array_equal(cb, cm + seg[s])
                assert np.array_equal(shb, shm) and np.array_equal(dzb, dzm)
    with pytest.raises(ValueError):
        M.concat_models([ms[0], M.wind_model(4, seed=9, nlev=4, npairs=3)])


def test_two_sided_sweep_with_inverted_segments():
    """Masing segments (negative optical depth, allowed by the reference's
    iteration): the device's elimination still solves the reference's
    system."""
    rng = np.random.default_rng(11)
    for _ in range(300):
        n_ar, n_r = int(rng.integers(1, 30)), int(rng.integers(0, 30))
        ndep = n_ar + n_r + 1
        term1 = rng.uniform(-2.0, 2.0, ndep)
        sign = np.where(rng.random(ndep - 1) < 0.2, -1.0, 1.0)
        dtau = sign * rng.uniform(0.1, 3.0, ndep - 1) * 10 ** rng.uniform(-3, 2)
        I0, In = rng.uniform(0, 1, 2)
        u, L = oracle.solve_raypair(n_ar, term1, dtau, I0, In)
        u2, L2 = two_sided_sweep(n_ar, term1, dtau, I0, In)
        assert abs(u2 - u) <= 1e-9 * abs(u) + 1e-300
        assert abs(L2 - L) <= 1e-9 * abs(L) + 1e-300
