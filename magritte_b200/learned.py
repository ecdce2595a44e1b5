"""Learned warm start of the level populations.

A 3 x 128 tanh MLP maps ten per-cell features (densities, temperature, line
width, velocity-gradient length, column densities along the traced rays) to a
correction of the LTE log level fractions; the populations
n = n_tot softmax(log x_LTE + MLP(f)) replace the LTE start, and the plain
ALI + Ng iteration then runs to the same tolerance, so it is both the
fallback and the check on the network's error.  The network is trained on
converged populations produced by this solver, with the library's own
forward, backward and Adam kernels (``mgr_mlp_train``).

    python -m magritte_b200.learned train --n 32 --models 12 --epochs 600 \
        --out magritte_b200/weights/wind_rotor10.npz
    python -m magritte_b200.learned train --family turb --n 64 --models 8 --nlev 21 \
        --epochs 600 --subsample 0.5 --out magritte_b200/weights/turb_rotor21.npz
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import time

import numpy as np

from . import _capi
from . import model as M

FEATURES = _capi.MLP_FEATURES
HIDDEN = _capi.MLP_HIDDEN
LOG_FLOOR = float(np.log(1e-30))


class WarmStartNet:
    """Parameters of the network in the layout of ``mgr_mlp``."""

    def __init__(self, nlev: int, params=None, feat_mean=None, feat_istd=None, meta=None):
        self.nlev = int(nlev)
        n = C.c_int64()
        st = _capi.load().mgr_mlp_param_count(self.nlev, C.byref(n))
        if st != 0:
            raise _capi.MagritteError(st, "bad level count")
        self.nparams = n.value
        self.params = (np.zeros(self.nparams, np.float32) if params is None
                       else np.ascontiguousarray(params, np.float32))
        self.feat_mean = (np.zeros(FEATURES, np.float32) if feat_mean is None
                          else np.ascontiguousarray(feat_mean, np.float32))
        self.feat_istd = (np.ones(FEATURES, np.float32) if feat_istd is None
                          else np.ascontiguousarray(feat_istd, np.float32))
        self.meta = dict(meta or {})

    def init(self, seed: int = 0):
        """Glorot-uniform hidden layers, zero output layer: the untrained
        network reproduces the LTE start exactly."""
        rng = np.random.default_rng(seed)
        shapes = [(HIDDEN, FEATURES), (HIDDEN, HIDDEN), (HIDDEN, HIDDEN), (self.nlev, HIDDEN)]
        parts = []
        for l, (o, i) in enumerate(shapes):
            lim = np.sqrt(6.0 / (o + i))
            W = rng.uniform(-lim, lim, size=(o, i)) if l < 3 else np.zeros((o, i))
            parts += [W.ravel(), np.zeros(o)]
        self.params = np.concatenate(parts).astype(np.float32)
        return self

    def desc(self):
        d = _capi.MlpDesc()
        d.nin = FEATURES
        d.nout = self.nlev
        d.params = self.params.ctypes.data
        d.feat_mean = self.feat_mean.ctypes.data
        d.feat_istd = self.feat_istd.ctypes.data
        return d

    def save(self, path: str):
        os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
        np.savez_compressed(path, params=self.params, feat_mean=self.feat_mean,
                            feat_istd=self.feat_istd, nlev=self.nlev,
                            meta=json.dumps(self.meta))

    @classmethod
    def load(cls, path: str) -> "WarmStartNet":
        d = np.load(path)
        meta = json.loads(str(d["meta"])) if "meta" in d else {}
        return cls(int(d["nlev"]), d["params"], d["feat_mean"], d["feat_istd"], meta)

    # ------------------------------------------------------------ device
    def forward(self, X: np.ndarray, device: int = 0) -> np.ndarray:
        X = np.ascontiguousarray(X, np.float32)
        out = np.zeros((X.shape[0], self.nlev), np.float32)
        d = self.desc()
        st = _capi.load().mgr_mlp_forward(device, C.byref(d), X.ctypes.data, X.shape[0],
                                          out.ctypes.data)
        if st != 0:
            raise _capi.MagritteError(st, "mgr_mlp_forward")
        return out

    def loss_grad(self, X, lte, tgt, device: int = 0):
        X = np.ascontiguousarray(X, np.float32)
        lte = np.ascontiguousarray(lte, np.float32)
        tgt = np.ascontiguousarray(tgt, np.float32)
        loss = np.zeros(1, np.float32)
        grad = np.zeros(self.nparams, np.float32)
        d = self.desc()
        st = _capi.load().mgr_mlp_loss_grad(device, C.byref(d), X.ctypes.data, lte.ctypes.data,
                                            tgt.ctypes.data, X.shape[0], loss.ctypes.data,
                                            grad.ctypes.data)
        if st != 0:
            raise _capi.MagritteError(st, "mgr_mlp_loss_grad")
        return float(loss[0]), grad

    def train(self, X, lte, tgt, epochs=200, batch=4096, lr=2e-3, weight_decay=0.0, seed=0,
              device: int = 0):
        X = np.ascontiguousarray(X, np.float32)
        lte = np.ascontiguousarray(lte, np.float32)
        tgt = np.ascontiguousarray(tgt, np.float32)
        self.feat_mean = X.mean(0).astype(np.float32)
        self.feat_istd = (1.0 / np.maximum(X.std(0), 1e-6)).astype(np.float32)
        o = _capi.TrainOpts()
        o.epochs, o.batch, o.lr, o.weight_decay, o.seed = epochs, batch, lr, weight_decay, seed
        hist = np.zeros(epochs, np.float32)
        d = self.desc()
        st = _capi.load().mgr_mlp_train(device, C.byref(d), X.ctypes.data, lte.ctypes.data,
                                        tgt.ctypes.data, X.shape[0], C.byref(o), hist.ctypes.data)
        if st != 0:
            raise _capi.MagritteError(st, "mgr_mlp_train")
        return hist


def samples_from(sim, pop=None):
    """Features, LTE log fractions and (if pop) target log fractions of a
    Simulation's model."""
    X = sim.features()
    L = sim.lte_logfrac()
    if pop is None:
        return X, L, None
    frac = pop / sim.model.population_tot[:, None]
    T = np.log(np.maximum(frac, 1e-30)).astype(np.float32)
    return X, L, T


def converged_samples(model, precision="mixed", tol=1e-6, max_iter=400, device=0):
    """Solve one model to convergence from LTE and return its samples and
    the iteration count."""
    from .simulation import Simulation
    sim = Simulation(model, device=device)
    sim.set_autotune(True)
    sim.compute_spectral_discretisation()
    sim.compute_boundary_intensities()
    sim.compute_LTE_level_populations()
    it = sim.compute_level_populations(True, max_iter, precision, tol_max_rel=tol, use_graph=True)
    X, L, T = samples_from(sim, sim.population)
    sim.close()
    return X, L, T, it


def wind_family(n: int, count: int, seed0: int, nlev: int = 10, nside: int = 2):
    """Seeded members of the spherical-wind family: density scale, central
    temperature and terminal speed drawn around the 64^3 wind's values."""
    out = []
    for i in range(count):
        rng = np.random.default_rng(seed0 + i)
        out.append(M.wind_model(n, seed=seed0 + i, nlev=nlev, nside=nside,
                                rho0=10 ** rng.uniform(13.5, 15.0),
                                T0=rng.uniform(300.0, 3000.0),
                                vmax=rng.uniform(5.0e3, 30.0e3),
                                name=f"wind{n}_s{seed0 + i}"))
    return out


def turb_family(n: int, count: int, seed0: int, nlev: int = 21):
    """Seeded members of the turbulent-cloud family (lognormal density,
    k^-4 velocity field): mean density and velocity dispersion drawn around
    the 128^3 cloud's 1e11 m^-3 and 2 km/s, new random fields per seed."""
    out = []
    for i in range(count):
        rng = np.random.default_rng(seed0 + i)
        out.append(M.turbulent_cloud(n, seed=seed0 + i, nlev=nlev, npairs=48, nquads=41,
                                     mean_h2=10 ** rng.uniform(10.6, 11.4),
                                     vrms=rng.uniform(1.5e3, 2.5e3),
                                     name=f"turb{n}_s{seed0 + i}"))
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("cmd", choices=["train"])
    ap.add_argument("--family", choices=["wind", "turb"], default="wind")
    ap.add_argument("--subsample", type=float, default=1.0,
                    help="fraction of each model's cells used for training")
    ap.add_argument("--n", type=int, default=32)
    ap.add_argument("--models", type=int, default=12)
    ap.add_argument("--seed0", type=int, default=100)
    ap.add_argument("--nlev", type=int, default=10)
    ap.add_argument("--epochs", type=int, default=600)
    ap.add_argument("--max-iter", type=int, default=400,
                    help="ALI cap of each training model; models that do not converge by it "
                         "are left out of the training set")
    ap.add_argument("--out", default=os.path.join(os.path.dirname(__file__), "weights",
                                                  "wind_rotor10.npz"))
    a = ap.parse_args(argv)
    t0 = time.time()
    Xs, Ls, Ts, its = [], [], [], []
    fam = wind_family if a.family == "wind" else turb_family
    rng = np.random.default_rng(a.seed0)
    for m in fam(a.n, a.models, a.seed0, a.nlev):
        t_m = time.time()
        X, L, T, it = converged_samples(m, max_iter=a.max_iter)
        if it >= a.max_iter:
            print(f"{m.name}: not converged in {it} iterations, left out", flush=True)
            its.append(it)
            continue
        if a.subsample < 1.0:
            keep = rng.random(X.shape[0]) < a.subsample
            X, L, T = X[keep], L[keep], T[keep]
        Xs.append(X); Ls.append(L); Ts.append(T); its.append(it)
        print(f"{m.name}: {it} iterations, {time.time() - t_m:.1f} s", flush=True)
    X, L, T = np.concatenate(Xs), np.concatenate(Ls), np.concatenate(Ts)
    t1 = time.time()
    net = WarmStartNet(a.nlev).init(0)
    hist = net.train(X, L, T, epochs=a.epochs)
    t2 = time.time()
    net.meta = dict(family=a.family, n=a.n, subsample=a.subsample, models=a.models, seed0=a.seed0, nlev=a.nlev,
                    epochs=a.epochs, max_iter=a.max_iter, samples=int(X.shape[0]),
                    final_loss=float(hist[-1]),
                    first_loss=float(hist[0]), ali_iterations=its,
                    data_s=round(t1 - t0, 1), train_s=round(t2 - t1, 1))
    net.save(a.out)
    print(json.dumps(net.meta))


if __name__ == "__main__":
    main()
