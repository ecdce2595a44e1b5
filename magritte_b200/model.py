"""Model description for the radiation hot path, plus seeded synthetic models.

A :class:`Model` carries exactly the data that Magritte's ``Simulation`` reads
for the ALI path (``src/Model/model.hpp:23-44``):

* geometry: cell positions, velocities (fractions of c), neighbour lists,
  boundary cells and ray directions (``src/Model/Geometry/geometry.hpp:31-54``,
  ``Rays/rays.hpp:59-127``, ``Boundary/boundary.hpp:16-30``);
* thermodynamics: gas temperature and squared turbulent speed over c^2
  (``src/Model/Thermodynamics/thermodynamics.tpp:52-69``);
* one line-producing species with its LAMDA-style line data, collision
  partners and frequency quadrature
  (``src/Model/Lines/LineProducingSpecies/Linedata/linedata.hpp``,
  ``magritte/setup/setup.py:370-506``).

Units are SI, as in the reference (``src/Tools/constants.hpp:25-31``).
Velocities are stored as fractions of the speed of light, like ``cells.velocity``.

The generators below build the seeded synthetic inputs that stand in for the
reference's model folders: a regular lattice cloud, a jittered spherical wind,
a high-optical-depth variant, a batch of uneven wind models and a turbulent
cloud. None of them reproduces a published benchmark's data.
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional

import numpy as np

# Physical constants with the exact values the reference uses
# (src/Tools/constants.hpp:25-46).
CC = 2.99792458e8
HH = 6.62607004e-34
KB = 1.38064852e-23
AMU = 1.66053904e-27
T_CMB = 2.7254800
C_SQUARED = 8.98755179e16
DEBYE = 3.33564095198152e-30  # C m
EPS0 = 8.8541878128e-12


@dataclasses.dataclass
class CollisionPartner:
    """Collisional rate table of one partner (``collisionPartner.hpp``).

    ``icol`` is the upper and ``jcol`` the lower level of each transition;
    ``Cd[t, k]`` is the downward and ``Ce[t, k]`` the upward rate coefficient
    [m^3 s^-1] at temperature ``tmp[t]``.
    """
    num_col_partner: int
    orth_or_para_H2: str
    icol: np.ndarray
    jcol: np.ndarray
    tmp: np.ndarray
    Cd: np.ndarray
    Ce: np.ndarray


@dataclasses.dataclass
class Linedata:
    """Line data of one species (``linedata.hpp``; derived quantities as in
    ``magritte/setup/setup.py:476-490``)."""
    num: int
    inverse_mass: float
    energy: np.ndarray
    weight: np.ndarray
    irad: np.ndarray
    jrad: np.ndarray
    A: np.ndarray
    colpar: List[CollisionPartner]

    @property
    def nlev(self) -> int:
        return int(self.energy.shape[0])

    @property
    def nrad(self) -> int:
        return int(self.irad.shape[0])

    @property
    def frequency(self) -> np.ndarray:
        return (self.energy[self.irad] - self.energy[self.jrad]) / HH

    @property
    def Bs(self) -> np.ndarray:
        nu = self.frequency
        return self.A * CC ** 2 / (2.0 * HH * nu ** 3)

    @property
    def Ba(self) -> np.ndarray:
        return self.weight[self.irad] / self.weight[self.jrad] * self.Bs


@dataclasses.dataclass
class Model:
    """Everything the radiation hot path reads, as contiguous numpy arrays."""
    position: np.ndarray          # [N, 3] m
    velocity: np.ndarray          # [N, 3] fraction of c
    nbr_offsets: np.ndarray       # [N+1] int64, CSR over nbr_list
    nbr_list: np.ndarray          # int64 neighbour cell numbers
    boundary2cell: np.ndarray     # [nb] int64
    boundary_temperature: np.ndarray  # [nb] K
    rays: np.ndarray              # [nrays, 3]
    ray_weights: np.ndarray       # [nrays]
    temperature: np.ndarray       # [N] K
    vturb2: np.ndarray            # [N] (v_turb / c)^2
    abundance: np.ndarray         # [N, nspec] m^-3
    linedata: Linedata
    quad_roots: np.ndarray        # [nquads]
    quad_weights: np.ndarray      # [nquads]
    pop_prec: float = 1.0e-6
    max_width_fraction: float = 0.5
    name: str = "model"
    meta: dict = dataclasses.field(default_factory=dict)

    # ----------------------------------------------------------------- sizes
    @property
    def ncells(self) -> int:
        return int(self.position.shape[0])

    @property
    def nrays(self) -> int:
        return int(self.rays.shape[0])

    @property
    def nboundary(self) -> int:
        return int(self.boundary2cell.shape[0])

    @property
    def nquads(self) -> int:
        return int(self.quad_roots.shape[0])

    @property
    def nlines(self) -> int:
        return self.linedata.nrad

    @property
    def nfreqs(self) -> int:
        return self.nlines * self.nquads

    @property
    def population_tot(self) -> np.ndarray:
        return np.ascontiguousarray(self.abundance[:, self.linedata.num])

    def antipod(self) -> np.ndarray:
        """Antipodal ray numbers, found as in ``Rays::setup_antipodal_rays``
        (``src/Model/Geometry/Rays/rays.cpp:90-102``): the last ray whose sum
        with ray r has squared norm below 1e-9."""
        r = self.rays
        s = r[:, None, :] + r[None, :, :]
        n2 = (s * s).sum(-1)
        out = np.full(self.nrays, -1, dtype=np.int64)
        for r1 in range(self.nrays):
            hits = np.nonzero(n2[r1] < 1.0e-9)[0]
            if hits.size:
                out[r1] = hits[-1]
        return out

    def boundary_mask(self) -> np.ndarray:
        m = np.zeros(self.ncells, dtype=np.uint8)
        m[self.boundary2cell] = 1
        return m

    def nbytes(self) -> int:
        return sum(int(getattr(self, f).nbytes) for f in (
            "position", "velocity", "nbr_offsets", "nbr_list", "boundary2cell",
            "boundary_temperature", "rays", "ray_weights", "temperature",
            "vturb2", "abundance", "quad_roots", "quad_weights"))

    def contiguous(self) -> "Model":
        for f in ("position", "velocity", "rays", "ray_weights", "temperature",
                  "vturb2", "abundance", "quad_roots", "quad_weights",
                  "boundary_temperature"):
            setattr(self, f, np.ascontiguousarray(getattr(self, f), dtype=np.float64))
        for f in ("nbr_offsets", "nbr_list", "boundary2cell"):
            setattr(self, f, np.ascontiguousarray(getattr(self, f), dtype=np.int64))
        return self


# ===================================================================== rays

_JRLL = (2, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 4)
_JPLL = (1, 3, 5, 7, 0, 2, 4, 6, 1, 3, 5, 7)


def _deinterleave(v: int) -> int:
    out, bit = 0, 0
    while v:
        out |= (v & 1) << bit
        v >>= 2
        bit += 1
    return out


def healpix_nest_vectors(nside: int) -> np.ndarray:
    """Pixel-centre unit vectors of the HEALPix NESTED scheme (Gorski et al.
    2005, ApJ 622, 759), the directions the reference draws its rays from
    (``src/Model/Geometry/healpix.hpp:218-232``, ``pix2vec_nest``)."""
    npface = nside * nside
    npix = 12 * npface
    nl4 = 4 * nside
    out = np.empty((npix, 3))
    for pix in range(npix):
        face, ipf = divmod(pix, npface)
        ix = _deinterleave(ipf)
        iy = _deinterleave(ipf >> 1)
        jrt = ix + iy
        jpt = ix - iy
        jr = _JRLL[face] * nside - jrt - 1
        if jr < nside:
            nr = jr
            z = 1.0 - nr * nr / (3.0 * npface)
            kshift = 0
        elif jr > 3 * nside:
            nr = nl4 - jr
            z = nr * nr / (3.0 * npface) - 1.0
            kshift = 0
        else:
            nr = nside
            z = (2 * nside - jr) * 2.0 / (3.0 * nside)
            kshift = (jr - nside) & 1
        jp = (_JPLL[face] * nr + jpt + 1 + kshift) // 2
        if jp > nl4:
            jp -= nl4
        if jp < 1:
            jp += nl4
        phi = (jp - (kshift + 1) * 0.5) * (0.5 * math.pi / nr)
        st = math.sqrt(max(0.0, (1.0 - z) * (1.0 + z)))
        out[pix] = (st * math.cos(phi), st * math.sin(phi), z)
    return out


def antipodal_ray_set(npairs: int, seed: int) -> np.ndarray:
    """``2*npairs`` directions: a near-uniform Fibonacci half-sphere, randomly
    rotated, followed by the antipode of each, so that rays r and r+npairs
    form a pair. Used where no HEALPix set has the required size."""
    rng = np.random.default_rng(seed)
    i = np.arange(npairs) + 0.5
    z = 1.0 - i / npairs
    phi = math.pi * (3.0 - 5.0 ** 0.5) * i
    st = np.sqrt(1.0 - z * z)
    half = np.stack([st * np.cos(phi), st * np.sin(phi), z], 1)
    q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
    half = half @ q.T
    half /= np.linalg.norm(half, axis=1, keepdims=True)
    return np.concatenate([half, -half], 0)


# ================================================================== species


def _detailed_balance_Ce(weight, energy, icol, jcol, tmp, Cd):
    Ce = np.empty_like(Cd)
    for t in range(tmp.shape[0]):
        gi = weight[icol]
        gj = weight[jcol]
        Ce[t] = Cd[t] * gi / gj * np.exp(-(energy[icol] - energy[jcol]) / (KB * tmp[t]))
    return Ce


def two_level_species(freq=115.27e9, A=7.2e-8, g=(1.0, 3.0), mass=28.0,
                      Cd=3.0e-17, tmp=(10.0, 1000.0)) -> Linedata:
    """Two-level species of the lattice-cloud set-up: E1 = h*nu, one H2
    partner with a constant downward rate and Ce by detailed balance
    (as ``magritte/setup/setup.py:452`` derives it)."""
    energy = np.array([0.0, HH * freq])
    weight = np.array(g, dtype=np.float64)
    icol = np.array([1], dtype=np.int64)
    jcol = np.array([0], dtype=np.int64)
    tmp = np.array(tmp, dtype=np.float64)
    Cdt = np.full((tmp.shape[0], 1), Cd)
    Ce = _detailed_balance_Ce(weight, energy, icol, jcol, tmp, Cdt)
    cp = CollisionPartner(0, "n", icol, jcol, tmp, Cdt, Ce)
    return Linedata(num=1, inverse_mass=1.0 / mass, energy=energy, weight=weight,
                    irad=np.array([1], dtype=np.int64), jrad=np.array([0], dtype=np.int64),
                    A=np.array([A]), colpar=[cp])


def linear_rotor_species(nlev: int, B: float = 57.6e9, mu_debye: float = 0.11,
                         mass: float = 28.0, seed: int = 0,
                         tmp=None) -> Linedata:
    """Rigid linear rotor: E_J = h B J (J+1), g = 2J+1, lines J -> J-1 at
    nu = 2 B J with dipole Einstein A; collisional rates from a seeded
    power law Cd(J->J') = C0 (dJ)^-alpha (T/100 K)^beta, Ce by detailed
    balance.  C0 (2e-17..6e-17 m^3/s) and alpha (2..2.6) follow the size and
    the dJ fall-off of CO-H2 rate tables: weaker coupling or a flatter
    fall-off lets collisional pumping and the radiative cascade invert the
    lowest levels at the wind's densities, and the reference's local-ALO
    iteration does not settle in such masing cells."""
    rng = np.random.default_rng(seed)
    J = np.arange(nlev, dtype=np.float64)
    energy = HH * B * J * (J + 1.0)
    weight = 2.0 * J + 1.0
    up = np.arange(1, nlev, dtype=np.int64)
    irad = up
    jrad = up - 1
    nu = 2.0 * B * up
    mu = mu_debye * DEBYE
    A = 16.0 * math.pi ** 3 * nu ** 3 * mu ** 2 / (3.0 * EPS0 * HH * CC ** 3) * up / (2.0 * up + 1.0)
    if tmp is None:
        tmp = np.array([10.0, 20.0, 50.0, 100.0, 200.0, 500.0, 1000.0, 2000.0, 3000.0])
    tmp = np.asarray(tmp, dtype=np.float64)
    C0 = 10 ** rng.uniform(-16.7, -16.2)
    alpha = rng.uniform(2.0, 2.6)
    beta = rng.uniform(0.1, 0.4)
    ic, jc = [], []
    for i in range(1, nlev):
        for j in range(i):
            ic.append(i)
            jc.append(j)
    icol = np.array(ic, dtype=np.int64)
    jcol = np.array(jc, dtype=np.int64)
    dJ = (icol - jcol).astype(np.float64)
    Cd = np.stack([C0 * dJ ** (-alpha) * (t / 100.0) ** beta for t in tmp], 0)
    Ce = _detailed_balance_Ce(weight, energy, icol, jcol, tmp, Cd)
    cp = CollisionPartner(0, "n", icol, jcol, tmp, Cd, Ce)
    return Linedata(num=1, inverse_mass=1.0 / mass, energy=energy, weight=weight,
                    irad=irad, jrad=jrad, A=A, colpar=[cp])


def linspace_quadrature(nquads: int, span: float = 5.0):
    """Roots evenly spaced over +-span Doppler widths with weights
    proportional to exp(-x^2), normalised to one."""
    roots = np.linspace(-span, span, nquads)
    w = np.exp(-roots ** 2)
    return roots, w / w.sum()


# =================================================================== grids


def lattice_grid(n: int, L: float, jitter: float = 0.0, seed: int = 0):
    """n^3 lattice x_i = i L/(n-1), cell p = (iz n + iy) n + ix; 26-point
    neighbour lists in fixed (dz, dy, dx) order; boundary = face cells.
    ``jitter`` displaces interior coordinates by U(-jitter, +jitter) spacings
    (faces stay planar)."""
    idx = np.arange(n)
    iz, iy, ix = np.meshgrid(idx, idx, idx, indexing="ij")
    ix = ix.ravel(); iy = iy.ravel(); iz = iz.ravel()
    d = L / (n - 1)
    pos = np.stack([ix, iy, iz], 1).astype(np.float64) * d
    if jitter > 0.0:
        rng = np.random.default_rng(seed)
        disp = rng.uniform(-jitter, jitter, size=pos.shape) * d
        onface = np.stack([ix, iy, iz], 1)
        disp[(onface == 0) | (onface == n - 1)] = 0.0
        pos = pos + disp
    offs = [(dz, dy, dx) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1)
            if (dz, dy, dx) != (0, 0, 0)]
    N = n ** 3
    lists = []
    counts = np.zeros(N, dtype=np.int64)
    cand = []
    for (dz, dy, dx) in offs:
        jx, jy, jz = ix + dx, iy + dy, iz + dz
        ok = (jx >= 0) & (jx < n) & (jy >= 0) & (jy < n) & (jz >= 0) & (jz < n)
        cand.append(np.where(ok, (jz * n + jy) * n + jx, -1))
    cand = np.stack(cand, 1)  # [N, 26] in (dz, dy, dx) order
    valid = cand >= 0
    counts = valid.sum(1)
    offsets = np.zeros(N + 1, dtype=np.int64)
    offsets[1:] = np.cumsum(counts)
    nbr = cand[valid].astype(np.int64)  # row-major keeps per-cell order
    face = (ix == 0) | (ix == n - 1) | (iy == 0) | (iy == n - 1) | (iz == 0) | (iz == n - 1)
    b2c = np.nonzero(face)[0].astype(np.int64)
    return pos, offsets, nbr, b2c


def chain_grid(n: int, L: float):
    """1D chain of n points on the x axis, neighbours i-1 and i+1, boundary
    at both ends (the constant-slab set-up of the reference's analytic test,
    ``tests/integration/test_0_1D_all_constant.py``)."""
    pos = np.zeros((n, 3))
    pos[:, 0] = np.arange(n) * (L / (n - 1))
    lists = [[i - 1, i + 1] for i in range(n)]
    lists[0] = [1]
    lists[-1] = [n - 2]
    offsets = np.zeros(n + 1, dtype=np.int64)
    offsets[1:] = np.cumsum([len(x) for x in lists])
    nbr = np.array([j for x in lists for j in x], dtype=np.int64)
    return pos, offsets, nbr, np.array([0, n - 1], dtype=np.int64)


# ================================================================== models


def _assemble(pos, offsets, nbr, b2c, vel_c, T, vturb, n_h2, x_abund, species,
              rays, weights, nquads, name, meta, pop_prec=1.0e-6) -> Model:
    N = pos.shape[0]
    roots, qw = linspace_quadrature(nquads)
    abund = np.stack([n_h2, n_h2 * x_abund], 1)
    return Model(position=pos, velocity=vel_c, nbr_offsets=offsets, nbr_list=nbr,
                 boundary2cell=b2c, boundary_temperature=np.full(b2c.shape[0], T_CMB),
                 rays=rays, ray_weights=weights, temperature=np.broadcast_to(T, (N,)).copy(),
                 vturb2=np.broadcast_to((vturb / CC) ** 2, (N,)).copy(), abundance=abund,
                 linedata=species, quad_roots=roots, quad_weights=qw, pop_prec=pop_prec,
                 name=name, meta=meta).contiguous()


def lattice_cloud(n: int = 16, L: float = 1.0e13, n_h2: float = 1.0e12, x_abund: float = 1.0e-4,
                  T: float = 20.0, vturb: float = 150.0, nside: int = 1, nquads: int = 31,
                  name: Optional[str] = None) -> Model:
    """Uniform static lattice cloud with the two-level species (the 16^3,
    12-ray, 31-bin CPU set-up at its defaults)."""
    pos, offs, nbr, b2c = lattice_grid(n, L)
    N = pos.shape[0]
    rays = healpix_nest_vectors(nside)
    w = np.full(rays.shape[0], 1.0 / rays.shape[0])
    return _assemble(pos, offs, nbr, b2c, np.zeros((N, 3)), T, vturb, np.full(N, n_h2),
                     x_abund, two_level_species(), rays, w, nquads,
                     name or f"lattice_cloud_{n}",
                     dict(kind="lattice_cloud", n=n, L=L, n_h2=n_h2, x_abund=x_abund,
                          T=T, vturb=vturb, nside=nside))


def wind_model(n: int = 64, L: float = 1.0e13, seed: int = 2, nlev: int = 10,
               rho0: float = 1.0e14, T0: float = 1000.0, vmax: float = 15.0e3,
               x_abund: float = 1.0e-4, vturb: float = 150.0, nside: int = 2,
               npairs: Optional[int] = None, nquads: int = 31, jitter: float = 0.3,
               name: Optional[str] = None, species_seed: Optional[int] = None,
               ray_seed: Optional[int] = None) -> Model:
    """Jittered n^3 grid shaped as a spherical wind: n(H2) = rho0 (r/0.05L)^-2,
    T = T0 (r/0.05L)^-0.7 (both held at their r = 0.05L value inside), radial
    velocity rising linearly to vmax at the half-diagonal; linear rotor with
    ``nlev`` levels. HEALPix rays (``nside``) unless ``npairs`` is given.
    The species' collision rates and the antipodal ray set are drawn with
    ``species_seed`` / ``ray_seed`` (default: ``seed``)."""
    pos, offs, nbr, b2c = lattice_grid(n, L, jitter=jitter, seed=seed)
    c = 0.5 * L
    d = pos - c
    r = np.sqrt((d * d).sum(1))
    r0 = 0.05 * L
    rr = np.maximum(r, r0) / r0
    n_h2 = rho0 * rr ** -2.0
    T = T0 * rr ** -0.7
    rmax = math.sqrt(3.0) * 0.5 * L
    with np.errstate(invalid="ignore", divide="ignore"):
        rhat = np.where(r[:, None] > 0, d / np.maximum(r, 1e-300)[:, None], 0.0)
    vel = rhat * (vmax * r / rmax)[:, None] / CC
    if npairs is None:
        rays = healpix_nest_vectors(nside)
    else:
        rays = antipodal_ray_set(npairs, seed if ray_seed is None else ray_seed)
    w = np.full(rays.shape[0], 1.0 / rays.shape[0])
    return _assemble(pos, offs, nbr, b2c, vel, T, vturb, n_h2, x_abund,
                     linear_rotor_species(nlev, seed=seed if species_seed is None else species_seed),
                     rays, w, nquads, name or f"wind_{n}",
                     dict(kind="wind", n=n, L=L, seed=seed, nlev=nlev, rho0=rho0, T0=T0,
                          vmax=vmax, x_abund=x_abund, vturb=vturb, nside=nside,
                          npairs=npairs, jitter=jitter))


def _grf_velocity(n: int, rms: float, slope: float, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    k = np.fft.fftfreq(n)
    kx, ky, kz = np.meshgrid(k, k, k, indexing="ij")
    kk = np.sqrt(kx ** 2 + ky ** 2 + kz ** 2)
    kk[0, 0, 0] = 1.0
    amp = kk ** (slope / 2.0)
    amp[0, 0, 0] = 0.0
    comps = []
    for _ in range(3):
        f = (rng.normal(size=kk.shape) + 1j * rng.normal(size=kk.shape)) * amp
        comps.append(np.real(np.fft.ifftn(f)))
    v = np.stack(comps, -1)
    v *= rms / np.sqrt((v ** 2).sum(-1).mean())
    # grid order (iz, iy, ix) to match lattice_grid
    return v.reshape(-1, 3)


def turbulent_cloud(n: int = 128, L: float = 1.0e14, seed: int = 5, nlev: int = 21,
                    mean_h2: float = 1.0e11, sigma_ln: float = 1.5, vrms: float = 2.0e3,
                    x_abund: float = 1.0e-4, vturb: float = 150.0, npairs: int = 48,
                    nquads: int = 41, name: Optional[str] = None) -> Model:
    """Jittered n^3 turbulent cloud: lognormal n(H2) (sigma_ln, mean),
    Gaussian-random-field velocity with P(k) ~ k^-4 and the given rms,
    T ~ U(15, 40) K, linear rotor with ``nlev`` levels."""
    rng = np.random.default_rng(seed)
    pos, offs, nbr, b2c = lattice_grid(n, L, jitter=0.3, seed=seed)
    N = pos.shape[0]
    g = rng.normal(size=N)
    n_h2 = mean_h2 * np.exp(sigma_ln * g - 0.5 * sigma_ln ** 2)
    T = rng.uniform(15.0, 40.0, size=N)
    vel = _grf_velocity(n, vrms, -4.0, seed + 1000) / CC
    rays = antipodal_ray_set(npairs, seed)
    w = np.full(rays.shape[0], 1.0 / rays.shape[0])
    return _assemble(pos, offs, nbr, b2c, vel, T, vturb, n_h2, x_abund,
                     linear_rotor_species(nlev, seed=seed), rays, w, nquads,
                     name or f"turbulent_{n}",
                     dict(kind="turbulent", n=n, L=L, seed=seed, nlev=nlev, mean_h2=mean_h2,
                          sigma_ln=sigma_ln, vrms=vrms, npairs=npairs))


def slab_1d(n: int = 50, L: float = 1.0e13, n_h2: float = 1.0e12, x_abund: float = 1.0e-6,
            T: float = 250.0, vturb: float = 250.0, nquads: int = 31,
            vmax: float = 0.0) -> Model:
    """Constant 1D slab with rays +x and -x (weights 1/2), the set-up whose
    mean intensity has the closed form J = S + (B-S)/2 (e^-tau(x) + e^-tau(L-x))
    (``tests/integration/test_0_1D_all_constant.py:240-244``).  With vmax
    (m/s) the velocity rises linearly along x from 0 to vmax, the set-up of
    ``tests/integration/test_1_1D_velocity_gradient.py``, where tau follows
    from the shifted profile as a difference of error functions."""
    pos, offs, nbr, b2c = chain_grid(n, L)
    rays = np.array([[1.0, 0.0, 0.0], [-1.0, 0.0, 0.0]])
    w = np.array([0.5, 0.5])
    vel = np.zeros((n, 3))
    vel[:, 0] = vmax * pos[:, 0] / L / CC
    return _assemble(pos, offs, nbr, b2c, vel, T, vturb, np.full(n, n_h2),
                     x_abund, two_level_species(), rays, w, nquads,
                     f"slab_{n}" if vmax == 0.0 else f"slab_{n}_gradient",
                     dict(kind="slab", n=n, L=L, vmax=vmax))


# ----------------------------------------------------------- named configs

def config1() -> Model:
    """16^3 lattice cloud, 2-level line, 12 HEALPix rays, 31 bins (CPU case)."""
    return lattice_cloud(16, name="cfg1_lattice16")


def config2() -> Model:
    """64^3 jittered spherical wind, 10-level rotor, 48 rays, 31 bins/line."""
    return wind_model(64, seed=2, nlev=10, nside=2, name="cfg2_wind64")


def config3() -> Model:
    """Config-1 lattice with n(H2) x 1e3 (line-centre optical depth ~1e4)."""
    return lattice_cloud(16, n_h2=1.0e15, name="cfg3_lattice16_thick")


def config4_member(m: int) -> Model:
    """Member m of the 256-model batch: 2k..60k points, random density scale,
    T0 and vmax, 20-level rotor, 24 rays (12 antipodal pairs).  Species and
    ray set are common to the batch (drawn with seed 4)."""
    rng = np.random.default_rng(4 + m)
    u = rng.uniform()
    N = min(int(2.0e3 * 30.0 ** u), 60000)
    n = max(4, int(math.ceil(N ** (1.0 / 3.0))))
    rho0 = 10 ** rng.uniform(12.0, 15.0)
    T0 = rng.uniform(100.0, 2000.0)
    vmax = rng.uniform(5.0e3, 30.0e3)
    return wind_model(n, seed=4 + m, nlev=20, rho0=rho0, T0=T0, vmax=vmax, npairs=12,
                      name=f"cfg4_m{m}", species_seed=4, ray_seed=4)


def concat_models(models: List[Model], name: str = "batch") -> Model:
    """One point cloud holding independent models side by side: cells,
    neighbour lists and boundary cells are renumbered, the graphs stay
    disjoint, and ``meta["segments"]`` holds each model's first cell (plus
    the total), which the library uses to iterate every model to its own
    convergence.  The models must share species, rays, quadrature and
    population precision."""
    m0 = models[0]
    for m in models[1:]:
        if not (np.array_equal(m.rays, m0.rays) and np.array_equal(m.ray_weights, m0.ray_weights)
                and np.array_equal(m.quad_roots, m0.quad_roots)
                and np.array_equal(m.quad_weights, m0.quad_weights)
                and m.pop_prec == m0.pop_prec and m.max_width_fraction == m0.max_width_fraction
                and _same_species(m.linedata, m0.linedata)):
            raise ValueError(f"model {m.name} does not share species/rays/quadrature with {m0.name}")
    seg = np.zeros(len(models) + 1, dtype=np.int64)
    seg[1:] = np.cumsum([m.ncells for m in models])
    offs, nbrs, b2c = [np.zeros(1, dtype=np.int64)], [], []
    for m, c0 in zip(models, seg[:-1]):
        offs.append(m.nbr_offsets[1:] + offs[-1][-1])
        nbrs.append(m.nbr_list + c0)
        b2c.append(m.boundary2cell + c0)
    cat = lambda f: np.concatenate([getattr(m, f) for m in models])
    return Model(position=cat("position"), velocity=cat("velocity"),
                 nbr_offsets=np.concatenate(offs), nbr_list=np.concatenate(nbrs),
                 boundary2cell=np.concatenate(b2c), boundary_temperature=cat("boundary_temperature"),
                 rays=m0.rays, ray_weights=m0.ray_weights, temperature=cat("temperature"),
                 vturb2=cat("vturb2"), abundance=cat("abundance"), linedata=m0.linedata,
                 quad_roots=m0.quad_roots, quad_weights=m0.quad_weights, pop_prec=m0.pop_prec,
                 max_width_fraction=m0.max_width_fraction, name=name,
                 meta=dict(kind="batch", members=[m.name for m in models],
                           segments=seg.tolist())).contiguous()


def _same_species(a: Linedata, b: Linedata) -> bool:
    if not (a.num == b.num and a.inverse_mass == b.inverse_mass and len(a.colpar) == len(b.colpar)):
        return False
    for f in ("energy", "weight", "irad", "jrad", "A"):
        if not np.array_equal(getattr(a, f), getattr(b, f)):
            return False
    for ca, cb in zip(a.colpar, b.colpar):
        for f in dataclasses.fields(ca):
            va, vb = getattr(ca, f.name), getattr(cb, f.name)
            if isinstance(va, np.ndarray):
                if not np.array_equal(va, vb):
                    return False
            elif va != vb:
                return False
    return True


def config4(nmodels: int = 256) -> Model:
    """The 256-model batch as one point cloud of independent models."""
    return concat_models([config4_member(m) for m in range(nmodels)], name=f"cfg4_batch{nmodels}")


def config5() -> Model:
    """128^3 turbulent cloud, 21-level rotor, 96 rays, 41 bins/line."""
    return turbulent_cloud(128, seed=5, nlev=21, npairs=48, nquads=41, name="cfg5_turb128")
