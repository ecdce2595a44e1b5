"""Model folders in Magritte's text layout, and checkpoints of an ALI run.

Magritte's ``IoText`` (``src/Io/cpp/io_cpp_text.cpp``) stores a model as a
folder of text files, one per field: ``<folder>/<path>.txt``, where a list
holds one value per line, an array one row per line with tab-separated
columns, and numbers are written in scientific notation with 17
significant digits (``std::setprecision(16)``), which reproduces every
double exactly.  The paths are the ones the reference's readers use:

    .ncells .nrays .nrays_red .order_min .order_max .nboundary .nfreqs
    .nfreqs_red .nspecs .nlspecs .nlines .nquads .pop_prec .use_scattering
    .use_Ng_acceleration .spherical_symmetry .adaptive_ray_tracing
                                            (Model/parameters.cpp:15-57)
    Geometry/Cells/{position,velocity,n_neighbors,neighbors}
                                            (Geometry/Cells/cells.cpp:20-90)
    Geometry/Rays/{rays,weights}           (Geometry/Rays/rays.cpp:20-50)
    Geometry/Boundary/{boundary2cell_nr,boundary_temperature,boundary_condition}
                                            (Geometry/Boundary/boundary.cpp:20-75)
    Thermodynamics/Temperature/gas, Thermodynamics/Turbulence/vturb2
    Chemistry/Species/{species,abundance}  (Chemistry/Species/species.cpp:20-50)
    Lines/LineProducingSpecies_0/Linedata/{.num,.sym,.inverse_mass,.nlev,.nrad,
        irad,jrad,energy,weight,frequency,A,Bs,Ba}
                                            (LineProducingSpecies/Linedata/linedata.cpp:25-80)
    Lines/LineProducingSpecies_0/Linedata/CollisionPartner_<c>/{.num_col_partner,
        .orth_or_para_H2,tmp,icol,jcol,Ce,Cd}
                                            (Linedata/CollisionPartner/collisionPartner.cpp:20-60)
    Lines/LineProducingSpecies_0/Quadrature/{weights,roots}
    Lines/LineProducingSpecies_0/{population_tot,population<tag>,
        population_prev1,population_prev2,population_prev3,J_lin<tag>,J_eff<tag>}
                                            (LineProducingSpecies/lineProducingSpecies.cpp:60-200)

A folder written here is read by the reference's own ``IoText`` reader
(the tests build the reference's C++ and load such folders), and
``read_model`` reads folders in that layout back into a
:class:`magritte_b200.model.Model`.  One line-producing species; the
boundary condition is written as ``cmb`` and the temperature of every
boundary cell is stored, so the reference's
``compute_boundary_intensities(temperatures)`` and this library's
``compute_boundary_intensities`` see the same boundary.

Checkpoints: :func:`write_populations` writes the current populations and
the three previous iterates that Ng acceleration needs, under the names
the reference uses for its per-iteration output
(``Simulation::compute_level_populations``, ``sim_lines.tpp:77-83``, and
``LineProducingSpecies::write``); :func:`read_populations` reads them back,
so an ALI run can stop and resume exactly where it was.
"""
from __future__ import annotations

import os
from typing import Dict, Optional

import numpy as np

from . import model as M

LSPEC = "Lines/LineProducingSpecies_0/"


# ------------------------------------------------------------ primitives

def _path(folder: str, name: str) -> str:
    return os.path.join(folder, name + ".txt")


def _mkdir_for(path: str):
    d = os.path.dirname(path)
    if d:
        os.makedirs(d, exist_ok=True)


def _fmt(x) -> str:
    if isinstance(x, (bool, np.bool_)):
        return "true" if x else "false"
    if isinstance(x, (int, np.integer)):
        return str(int(x))
    return "%.16e" % float(x)


def write_number(folder: str, name: str, x):
    p = _path(folder, name)
    _mkdir_for(p)
    with open(p, "w") as f:
        f.write(_fmt(x))


def write_word(folder: str, name: str, w: str):
    p = _path(folder, name)
    _mkdir_for(p)
    with open(p, "w") as f:
        f.write(w)


def write_list(folder: str, name: str, a):
    p = _path(folder, name)
    _mkdir_for(p)
    a = np.asarray(a)
    with open(p, "w") as f:
        if a.dtype.kind in "iu":
            f.write("".join("%d\n" % v for v in a.tolist()))
        elif a.dtype.kind in "US":
            f.write("".join("%s\n" % v for v in a.tolist()))
        else:
            f.write("".join("%.16e\n" % v for v in a.astype(np.float64).tolist()))


def write_array(folder: str, name: str, a):
    """Rows on lines, columns separated (and terminated) by tabs, as
    ``IoText::write_array`` writes them."""
    p = _path(folder, name)
    _mkdir_for(p)
    a = np.asarray(a)
    if a.ndim == 1:
        a = a[:, None]
    fmt = "%d\t" if a.dtype.kind in "iu" else "%.16e\t"
    with open(p, "w") as f:
        for row in a.tolist():
            f.write("".join(fmt % v for v in row) + "\n")


def exists(folder: str, name: str) -> bool:
    return os.path.exists(_path(folder, name))


def read_number(folder: str, name: str, kind=float):
    with open(_path(folder, name)) as f:
        tok = f.read().split()
    v = float(tok[0])
    return int(v) if kind is int else v


def read_word(folder: str, name: str) -> str:
    with open(_path(folder, name)) as f:
        return f.read().split()[0]


def read_list(folder: str, name: str, dtype=np.float64) -> np.ndarray:
    with open(_path(folder, name)) as f:
        tok = f.read().split()
    if dtype is str:
        return np.array(tok)
    if np.dtype(dtype).kind in "iu":
        return np.array([int(float(t)) for t in tok], dtype=dtype)
    return np.array([float(t) for t in tok], dtype=dtype)


def read_array(folder: str, name: str, dtype=np.float64) -> np.ndarray:
    rows = []
    with open(_path(folder, name)) as f:
        for line in f:
            tok = line.split()
            if tok:
                rows.append([float(t) for t in tok])
    return np.array(rows, dtype=dtype)


def count_indexed(folder: str, prefix: str) -> int:
    """``IoText::read_length`` on a name without a .txt file: the number of
    paths prefix0, prefix1, ... that exist."""
    n = 0
    while os.path.exists(os.path.join(folder, prefix + str(n))):
        n += 1
    return n


# ------------------------------------------------------------ the model

def write_model(model: "M.Model", folder: str, species_names=None):
    """Writes ``model`` as a Magritte text model folder."""
    os.makedirs(folder, exist_ok=True)
    m = model
    ld = m.linedata
    N, R = m.ncells, m.nrays
    nspec = m.abundance.shape[1]
    w = lambda name, x: write_number(folder, name, x)
    w(".ncells", N)
    w(".nrays", R)
    w(".nrays_red", R // 2)
    w(".order_min", 0)
    w(".order_max", 0)
    w(".nboundary", m.nboundary)
    w(".nfreqs", m.nfreqs)
    w(".nfreqs_red", m.nfreqs)
    w(".nspecs", nspec)
    w(".nlspecs", 1)
    w(".nlines", m.nlines)
    w(".nquads", m.nquads)
    w(".pop_prec", float(m.pop_prec))
    for b, v in ((".use_scattering", False), (".use_Ng_acceleration", True),
                 (".spherical_symmetry", False), (".adaptive_ray_tracing", False)):
        w(b, v)
    g = "Geometry/"
    write_array(folder, g + "Cells/position", m.position)
    write_array(folder, g + "Cells/velocity", m.velocity)
    write_list(folder, g + "Cells/n_neighbors", np.diff(m.nbr_offsets).astype(np.int64))
    write_list(folder, g + "Cells/neighbors", m.nbr_list.astype(np.int64))
    write_array(folder, g + "Rays/rays", m.rays)
    write_list(folder, g + "Rays/weights", m.ray_weights)
    write_list(folder, g + "Boundary/boundary2cell_nr", m.boundary2cell.astype(np.int64))
    write_list(folder, g + "Boundary/boundary_temperature", m.boundary_temperature)
    write_list(folder, g + "Boundary/boundary_condition", np.array(["cmb"] * m.nboundary))
    write_list(folder, "Thermodynamics/Temperature/gas", m.temperature)
    write_list(folder, "Thermodynamics/Turbulence/vturb2", m.vturb2)
    names = species_names or [f"species_{i}" for i in range(nspec)]
    write_list(folder, "Chemistry/Species/species", np.array(names))
    write_array(folder, "Chemistry/Species/abundance", m.abundance)
    L = LSPEC + "Linedata/"
    w(L + ".num", int(ld.num))
    write_word(folder, L + ".sym", str(m.meta.get("species_sym", "rotor")))
    w(L + ".inverse_mass", float(ld.inverse_mass))
    w(L + ".nlev", ld.nlev)
    w(L + ".nrad", ld.nrad)
    write_list(folder, L + "irad", ld.irad.astype(np.int64))
    write_list(folder, L + "jrad", ld.jrad.astype(np.int64))
    write_list(folder, L + "energy", ld.energy)
    write_list(folder, L + "weight", ld.weight)
    write_list(folder, L + "frequency", ld.frequency)
    write_list(folder, L + "A", ld.A)
    write_list(folder, L + "Bs", ld.Bs)
    write_list(folder, L + "Ba", ld.Ba)
    for c, cp in enumerate(ld.colpar):
        C = L + f"CollisionPartner_{c}/"
        w(C + ".num_col_partner", int(cp.num_col_partner))
        write_word(folder, C + ".orth_or_para_H2", cp.orth_or_para_H2)
        write_list(folder, C + "tmp", cp.tmp)
        write_list(folder, C + "icol", cp.icol.astype(np.int64))
        write_list(folder, C + "jcol", cp.jcol.astype(np.int64))
        write_array(folder, C + "Ce", cp.Ce)
        write_array(folder, C + "Cd", cp.Cd)
    write_list(folder, LSPEC + "Quadrature/weights", m.quad_weights)
    write_list(folder, LSPEC + "Quadrature/roots", m.quad_roots)
    write_list(folder, LSPEC + "population_tot", m.population_tot)
    # what this library adds beyond the reference's fields
    w(".max_width_fraction", float(m.max_width_fraction))


def read_model(folder: str, name: Optional[str] = None) -> "M.Model":
    """Reads a Magritte text model folder (one line-producing species)."""
    g = "Geometry/"
    pos = read_array(folder, g + "Cells/position")
    vel = read_array(folder, g + "Cells/velocity")
    nn = read_list(folder, g + "Cells/n_neighbors", np.int64)
    nbr = read_list(folder, g + "Cells/neighbors", np.int64)
    offs = np.zeros(nn.shape[0] + 1, dtype=np.int64)
    offs[1:] = np.cumsum(nn)
    rays = read_array(folder, g + "Rays/rays")
    rw = read_list(folder, g + "Rays/weights")
    b2c = read_list(folder, g + "Boundary/boundary2cell_nr", np.int64)
    if exists(folder, g + "Boundary/boundary_temperature"):
        bT = read_list(folder, g + "Boundary/boundary_temperature")
    else:
        bT = np.full(b2c.shape[0], 2.72548)
    T = read_list(folder, "Thermodynamics/Temperature/gas")
    vt2 = read_list(folder, "Thermodynamics/Turbulence/vturb2")
    abn = read_array(folder, "Chemistry/Species/abundance")
    nlspecs = count_indexed(folder, "Lines/LineProducingSpecies_")
    if nlspecs != 1:
        raise ValueError(f"{folder}: {nlspecs} line-producing species; one is supported")
    L = LSPEC + "Linedata/"
    colpar = []
    for c in range(count_indexed(folder, L + "CollisionPartner_")):
        C = L + f"CollisionPartner_{c}/"
        colpar.append(M.CollisionPartner(
            num_col_partner=read_number(folder, C + ".num_col_partner", int),
            orth_or_para_H2=read_word(folder, C + ".orth_or_para_H2"),
            icol=read_list(folder, C + "icol", np.int64),
            jcol=read_list(folder, C + "jcol", np.int64),
            tmp=read_list(folder, C + "tmp"),
            Cd=read_array(folder, C + "Cd"), Ce=read_array(folder, C + "Ce")))
    ld = M.Linedata(num=read_number(folder, L + ".num", int),
                    inverse_mass=read_number(folder, L + ".inverse_mass"),
                    energy=read_list(folder, L + "energy"), weight=read_list(folder, L + "weight"),
                    irad=read_list(folder, L + "irad", np.int64),
                    jrad=read_list(folder, L + "jrad", np.int64),
                    A=read_list(folder, L + "A"), colpar=colpar)
    mwf = read_number(folder, ".max_width_fraction") if exists(folder, ".max_width_fraction") else 0.5
    model = M.Model(position=pos, velocity=vel, nbr_offsets=offs, nbr_list=nbr,
                    boundary2cell=b2c, boundary_temperature=bT, rays=rays, ray_weights=rw,
                    temperature=T, vturb2=vt2, abundance=abn, linedata=ld,
                    quad_roots=read_list(folder, LSPEC + "Quadrature/roots"),
                    quad_weights=read_list(folder, LSPEC + "Quadrature/weights"),
                    pop_prec=read_number(folder, ".pop_prec") if exists(folder, ".pop_prec") else 1e-6,
                    max_width_fraction=mwf, name=name or os.path.basename(os.path.normpath(folder)),
                    meta={"kind": "text", "folder": folder})
    return model.contiguous()


# ------------------------------------------------------------ checkpoints

def write_populations(folder: str, pop, prev=None, Jlin=None, Jeff=None, tag: str = ""):
    """Populations [ncells, nlev] as ``population<tag>`` (and ``J_lin<tag>``,
    ``J_eff<tag>`` when given), plus the previous iterates
    ``population_prev1..3`` that Ng acceleration reads."""
    write_array(folder, LSPEC + "population" + tag, pop)
    if Jlin is not None:
        write_array(folder, LSPEC + "J_lin" + tag, Jlin)
    if Jeff is not None:
        write_array(folder, LSPEC + "J_eff" + tag, Jeff)
    if prev is not None:
        for i, p in enumerate(prev):
            write_array(folder, LSPEC + f"population_prev{i + 1}", p)


def read_populations(folder: str, tag: str = "") -> Dict[str, np.ndarray]:
    out = {"population": read_array(folder, LSPEC + "population" + tag)}
    for i in (1, 2, 3):
        name = LSPEC + f"population_prev{i}"
        if exists(folder, name):
            out[f"prev{i}"] = read_array(folder, name)
    return out
