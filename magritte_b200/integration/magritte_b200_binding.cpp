// magritte_b200_binding.cpp -- the B200 path called from Magritte's own
// Simulation object.
//
// This file is written against Magritte's headers (Simulation/simulation.hpp
// and the Model containers it holds) and the C ABI of include/magritte_b200.h:
// it is what a Magritte build adds to route Simulation::compute_level_populations
// and Simulation::compute_radiation_field (Simulation/sim_lines.tpp:61-164,
// Simulation/sim_radiation.tpp:56-338) to the GPU.  The Simulation keeps
// owning the model; these functions flatten its containers into the
// descriptor the library uploads, run the device path, and write the results
// back into the same containers (populations, J, Jlin, Jeff, error_max), so
// the rest of a Magritte program (writing, imaging, the Python bindings) sees
// what its own CPU path would have left there.
//
// Link with libmagritte_b200.so.  The Python binding is one line beside the
// others in src/bindings/pyBindings.cpp:404-449:
//     .def ("compute_level_populations_b200", &compute_level_populations_b200)
#include "magritte_b200_binding.hpp"

#include <cstring>
#include <string>
#include <vector>

namespace {

// The descriptor of Model::read's containers plus the flat arrays it points
// into (kept alive as long as the descriptor).
struct Flat {
    std::vector<double> pos, vel, rays, T, vt2, ntot, quad_r, quad_w, energy, weight, A, Bs, Ba,
        freq, bdyT;
    std::vector<int64_t> off, nbr, b2c, irad, jrad;
    std::vector<std::vector<int64_t>> icol, jcol;
    std::vector<std::vector<double>> tmp, Cd, Ce, abn;
    std::vector<mgr_colpar_desc> colpar;
    mgr_model_desc d;
};

template <class T, class S>
std::vector<T> copy_as(const S &src) {
    return std::vector<T>(src.begin(), src.end());
}

bool flatten(const Simulation &sim, Flat &f, std::string &why) {
    const LineProducingSpecies &ls = sim.lines.lineProducingSpecies[0];
    const Linedata &ld = ls.linedata;
    const long N = (long)sim.parameters.ncells();
    if (sim.parameters.nlspecs() != 1) { why = "one line-producing species"; return false; }
    if (sim.parameters.n_off_diag < 0 || sim.parameters.n_off_diag > 8) {
        why = "n_off_diag in 0 .. 8";
        return false;
    }
    f.pos.resize(3 * N);
    f.vel.resize(3 * N);
    f.off.assign(N + 1, 0);
    for (long p = 0; p < N; p++) {
        for (int i = 0; i < 3; i++) {
            f.pos[3 * p + i] = sim.geometry.cells.position[p][i];
            f.vel[3 * p + i] = sim.geometry.cells.velocity[p][i];
        }
        for (long n : sim.geometry.cells.neighbors[p]) f.nbr.push_back(n);
        f.off[p + 1] = (int64_t)f.nbr.size();
    }
    const long R = (long)sim.parameters.nrays();
    f.rays.resize(3 * R);
    for (long r = 0; r < R; r++)
        for (int i = 0; i < 3; i++) f.rays[3 * r + i] = sim.geometry.rays.rays[r][i];
    f.b2c = copy_as<int64_t>(sim.geometry.boundary.boundary2cell_nr);
    f.bdyT = copy_as<double>(sim.geometry.boundary.boundary_temperature);
    f.T = copy_as<double>(sim.thermodynamics.temperature.gas);
    f.vt2 = copy_as<double>(sim.thermodynamics.turbulence.vturb2);
    f.ntot.resize(N);
    for (long p = 0; p < N; p++) f.ntot[p] = sim.chemistry.species.abundance[p][ld.num];
    f.energy = copy_as<double>(ld.energy);
    f.weight = copy_as<double>(ld.weight);
    f.irad = copy_as<int64_t>(ld.irad);
    f.jrad = copy_as<int64_t>(ld.jrad);
    f.A = copy_as<double>(ld.A);
    f.Bs = copy_as<double>(ld.Bs);
    f.Ba = copy_as<double>(ld.Ba);
    f.freq = copy_as<double>(ld.frequency);
    f.quad_r = copy_as<double>(ls.quadrature.roots);
    f.quad_w = copy_as<double>(ls.quadrature.weights);
    const size_t nc = ld.colpar.size();
    f.icol.resize(nc); f.jcol.resize(nc); f.tmp.resize(nc); f.Cd.resize(nc); f.Ce.resize(nc);
    f.abn.resize(nc);
    f.colpar.resize(nc);
    for (size_t c = 0; c < nc; c++) {
        const CollisionPartner &cp = ld.colpar[c];
        f.icol[c] = copy_as<int64_t>(cp.icol);
        f.jcol[c] = copy_as<int64_t>(cp.jcol);
        f.tmp[c] = copy_as<double>(cp.tmp);
        for (const auto &row : cp.Cd) f.Cd[c].insert(f.Cd[c].end(), row.begin(), row.end());
        for (const auto &row : cp.Ce) f.Ce[c].insert(f.Ce[c].end(), row.begin(), row.end());
        f.abn[c].resize(N);
        for (long p = 0; p < N; p++) f.abn[c][p] = sim.chemistry.species.abundance[p][cp.num_col_partner];
        mgr_colpar_desc &cd = f.colpar[c];
        std::memset(&cd, 0, sizeof(cd));
        cd.ntmp = (int32_t)cp.tmp.size();
        cd.ncol = (int32_t)cp.icol.size();
        cd.ortho_para = cp.orth_or_para_H2 == "o" ? 1 : cp.orth_or_para_H2 == "p" ? 2 : 0;
        cd.icol = f.icol[c].data();
        cd.jcol = f.jcol[c].data();
        cd.tmp = f.tmp[c].data();
        cd.Cd = f.Cd[c].data();
        cd.Ce = f.Ce[c].data();
        cd.abundance = f.abn[c].data();
    }
    mgr_model_desc &d = f.d;
    std::memset(&d, 0, sizeof(d));
    d.ncells = N;
    d.position = f.pos.data();
    d.velocity = f.vel.data();
    d.nbr_offsets = f.off.data();
    d.nbr_list = f.nbr.data();
    d.nboundary = (int64_t)f.b2c.size();
    d.boundary2cell = f.b2c.data();
    d.boundary_temperature = f.bdyT.data();
    d.nrays = R;
    d.rays = f.rays.data();
    d.ray_weights = sim.geometry.rays.weights.data();
    d.temperature = f.T.data();
    d.vturb2 = f.vt2.data();
    d.nlev = (int32_t)ld.nlev;
    d.nrad = (int32_t)ld.nrad;
    d.energy = f.energy.data();
    d.weight = f.weight.data();
    d.irad = f.irad.data();
    d.jrad = f.jrad.data();
    d.A = f.A.data();
    d.Bs = f.Bs.data();
    d.Ba = f.Ba.data();
    d.frequency = f.freq.data();
    d.inverse_mass = ld.inverse_mass;
    d.population_tot = f.ntot.data();
    d.nquads = (int32_t)f.quad_r.size();
    d.ncolpar = (int32_t)nc;
    d.quad_roots = f.quad_r.data();
    d.quad_weights = f.quad_w.data();
    d.colpar = f.colpar.data();
    d.pop_prec = sim.parameters.pop_prec();
    d.max_width_fraction = sim.parameters.max_width_fraction;
    return true;
}

// Handle with the model and the Simulation's current populations uploaded.
mgr_handle *open(Simulation &sim, int device, Flat &f, std::string &why) {
    if (!flatten(sim, f, why)) return nullptr;
    mgr_handle *h = nullptr;
    if (mgr_create(device, &h) != MGR_OK) { why = "no CUDA device"; return nullptr; }
    mgr_status s = mgr_upload_model(h, &f.d);
    if (s == MGR_OK) s = mgr_set_n_off_diag(h, (int32_t)sim.parameters.n_off_diag);
    if (s == MGR_OK) s = mgr_compute_spectral_discretisation(h);
    if (s == MGR_OK) s = mgr_compute_boundary_intensities(h);
    if (s == MGR_OK) s = mgr_set_populations(h, sim.lines.lineProducingSpecies[0].population.data());
    if (s != MGR_OK) {
        why = mgr_last_error(h);
        mgr_destroy(h);
        return nullptr;
    }
    return h;
}

// Jlin and Jeff [ncells*nrad] into the species' Double2 containers.
void store_line_fields(Simulation &sim, mgr_handle *h) {
    LineProducingSpecies &ls = sim.lines.lineProducingSpecies[0];
    const size_t N = sim.parameters.ncells(), K = ls.linedata.nrad;
    std::vector<double> jl(N * K), je(N * K);
    mgr_get_Jlin(h, jl.data());
    mgr_get_Jeff(h, je.data());
    for (size_t p = 0; p < N; p++)
        for (size_t k = 0; k < K; k++) {
            ls.Jlin[p][k] = jl[p * K + k];
            ls.Jeff[p][k] = je[p * K + k];
        }
}

}  // namespace

long compute_level_populations_b200(Simulation &sim, const bool use_Ng, const long max_niterations,
                                    const int precision, const double tol_max_rel,
                                    const int device) {
    Flat f;
    std::string why;
    mgr_handle *h = open(sim, device, f, why);
    if (!h) {
        sim.logger.write("B200 path not used: " + why);
        return -1;
    }
    mgr_ali_opts o;
    std::memset(&o, 0, sizeof(o));
    o.use_ng = use_Ng ? 1 : 0;
    o.precision = precision;
    o.max_iter = max_niterations;
    o.tol_max_rel = tol_max_rel;   // <= 0: the reference's own stop test
    o.use_graph = 1;
    std::vector<double> hist(max_niterations > 0 ? max_niterations : 1);
    int64_t iters = 0;
    const mgr_status s = mgr_compute_level_populations(h, &o, &iters, hist.data());
    if (s == MGR_OK || s == MGR_ERR_NOT_CONVERGED) {
        mgr_get_populations(h, sim.lines.lineProducingSpecies[0].population.data());
        sim.lines.set_emissivity_and_opacity();
        store_line_fields(sim, h);
        sim.error_max.assign(hist.begin(), hist.begin() + iters);
    } else {
        sim.logger.write(std::string("B200 path failed: ") + mgr_last_error(h));
    }
    mgr_destroy(h);
    return (s == MGR_OK || s == MGR_ERR_NOT_CONVERGED) ? (long)iters : -1;
}

int compute_radiation_field_b200(Simulation &sim, const int precision, const int device) {
    Flat f;
    std::string why;
    mgr_handle *h = open(sim, device, f, why);
    if (!h) {
        sim.logger.write("B200 path not used: " + why);
        return -1;
    }
    mgr_status s = mgr_set_keep_J(h, 1);
    if (s == MGR_OK) s = mgr_compute_radiation_field(h, precision);
    if (s == MGR_OK) s = mgr_compute_Jeff(h);
    if (s == MGR_OK) {
        const size_t N = sim.parameters.ncells(), nf = sim.parameters.nfreqs();
        std::vector<double> J(N * nf);
        mgr_get_J(h, J.data());
        for (size_t i = 0; i < N * nf; i++) sim.radiation.J[i] = J[i];
        store_line_fields(sim, h);
    } else {
        sim.logger.write(std::string("B200 path failed: ") + mgr_last_error(h));
    }
    mgr_destroy(h);
    return s == MGR_OK ? 0 : -1;
}
