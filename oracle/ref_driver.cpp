// ref_driver.cpp -- runs the reference's own C++ (Magritte's CPU path, built
// from its unmodified sources by oracle/ref_build.sh into oracle/_ref) on a
// model folder in Magritte's text layout, and writes what it computes as
// raw little-endian arrays (TEST INFRASTRUCTURE ONLY: a second checker of
// the C oracle, never part of the product).
//
//   magritte_ref <model/> <out/> radiation     J, Jlin, Jeff, ALO after one
//                                              compute_radiation_field (LTE
//                                              populations, or the model's
//                                              population.txt with --pops)
//   magritte_ref <model/> <out/> ali <n>       compute_level_populations(io,
//                                              Ng, n): populations, the
//                                              max and mean relative change
//                                              of every iteration
//   magritte_ref <model/> <out/> trace <o...>  the traced points of every
//                                              ray of the given origins
//   magritte_ref <model/> <out/> sample <file>  timing of the reference's own
//                                              per-origin work of
//                                              compute_radiation_field (the
//                                              body of its loop, sim_radiation.
//                                              tpp:150-264) over each line's
//                                              origins, OpenMP over origins as
//                                              there, one JSON line per sample;
//                                              after the first sample also one
//                                              full Jeff + statistical-
//                                              equilibrium step and one Ng step
//   magritte_ref <model/> <out/> scatter <U> <V>  every ray pair and origin
//                                              through setup_using_scattering
//                                              and solve_using_scattering with
//                                              the scattering terms U, V read
//                                              from raw files ([nrays/2]
//                                              [ncells*nfreqs]): u, v at the
//                                              origins and J (LTE populations)
//   magritte_ref <model/> <out/> image <r> <w> compute_and_write_image along
//                                              ray r on the image grid of
//                                              relative width w (LTE
//                                              populations): written by the
//                                              reference's Image::write
//   magritte_ref_gpu <model/> <out/> gpu <block> <nblocks> <reps>
//                                              (the build with the
//                                              reference's GPU solver only)
//                                              gpu_compute_radiation_field
//                                              with that launch shape, reps
//                                              times, one JSON line of wall
//                                              time each; then J, Jlin, Jeff,
//                                              ALO as for radiation
//
// MGR_REF_N_OFF_DIAG=<M> sets parameters.n_off_diag before anything runs.
//
// The call sequence follows the reference's examples
// (src/examples/example_1.cpp: read, compute_spectral_discretisation,
// compute_boundary_intensities, compute_LTE_level_populations, ...), with
// the boundary temperatures of the model folder passed to
// compute_boundary_intensities (sim_radiation.tpp:17-40).
#include <omp.h>
#include <sys/stat.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "Io/cpp/io_cpp_text.hpp"
#include "Simulation/simulation.hpp"

namespace {

void write_raw(const std::string &path, const std::vector<double> &v) {
    std::ofstream f(path, std::ios::binary);
    f.write(reinterpret_cast<const char *>(v.data()), (std::streamsize)(v.size() * sizeof(double)));
}

void write_raw_long(const std::string &path, const std::vector<long> &v) {
    std::ofstream f(path, std::ios::binary);
    f.write(reinterpret_cast<const char *>(v.data()), (std::streamsize)(v.size() * sizeof(long)));
}

void set_up(Simulation &sim, bool lte) {
    sim.compute_spectral_discretisation();
    sim.compute_boundary_intensities(sim.geometry.boundary.boundary_temperature);
    if (lte) {
        sim.compute_LTE_level_populations();
    } else {
        // populations read from the model folder (Model::read)
        sim.lines.set_emissivity_and_opacity();
    }
}

// Jlin[p][k] and the diagonal ALO element of (p, k) (sum of the elements
// whose position is p itself; with n_off_diag = 0 there is one).
void write_line_fields(Simulation &sim, const std::string &out) {
    const LineProducingSpecies &ls = sim.lines.lineProducingSpecies[0];
    const size_t N = sim.parameters.ncells(), K = ls.linedata.nrad;
    std::vector<double> jl(N * K), je(N * K), lam(N * K, 0.0);
    for (size_t p = 0; p < N; p++)
        for (size_t k = 0; k < K; k++) {
            jl[p * K + k] = ls.Jlin[p][k];
            je[p * K + k] = ls.Jeff[p][k];
            for (size_t i = 0; i < ls.lambda.Ls[p][k].size(); i++)
                if ((size_t)ls.lambda.nr[p][k][i] == p) lam[p * K + k] += ls.lambda.Ls[p][k][i];
        }
    write_raw(out + "/Jlin.bin", jl);
    write_raw(out + "/Jeff.bin", je);
    write_raw(out + "/Lambda.bin", lam);
}

void write_populations(Simulation &sim, const std::string &out) {
    const LineProducingSpecies &ls = sim.lines.lineProducingSpecies[0];
    std::vector<double> pop(ls.population.size());
    for (size_t i = 0; i < pop.size(); i++) pop[i] = ls.population[i];
    write_raw(out + "/population.bin", pop);
}

}  // namespace

int main(int argc, char **argv) {
    if (argc < 4) {
        std::fprintf(stderr,
                     "usage: %s <model/> <out/> radiation [--pops] | ali <n> | trace <o>... | "
                     "image <r> <width>\n", argv[0]);
        return 2;
    }
    const std::string model = argv[1], out = argv[2], cmd = argv[3];
    IoText io(model);
    Simulation sim;
    sim.read(io);
    // parameters.n_off_diag (a plain member, not part of the model folder)
    if (const char *noff = std::getenv("MGR_REF_N_OFF_DIAG")) sim.parameters.n_off_diag = std::atol(noff);
    if (cmd == "radiation") {
        const bool lte = !(argc > 4 && std::string(argv[4]) == "--pops");
        set_up(sim, lte);
        sim.compute_radiation_field();
        sim.compute_Jeff();
        std::vector<double> J(sim.radiation.J.size());
        for (size_t i = 0; i < J.size(); i++) J[i] = sim.radiation.J[i];
        write_raw(out + "/J.bin", J);
        write_line_fields(sim, out);
        write_populations(sim, out);
        return 0;
    }
    if (cmd == "ali" && argc > 4) {
        set_up(sim, true);
        IoText io_out(out + "/");
        const long it = sim.compute_level_populations(io_out, true, std::atol(argv[4]));
        write_populations(sim, out);
        write_raw(out + "/error_max.bin", sim.error_max);
        write_raw(out + "/error_mean.bin", sim.error_mean);
        write_raw_long(out + "/iterations.bin", std::vector<long>{it});
        return 0;
    }
    if (cmd == "trace") {
        sim.compute_spectral_discretisation();
        std::vector<long> head;
        std::vector<long> cells;
        std::vector<double> sh, dz;
        for (int a = 4; a < argc; a++) {
            const long o = std::atol(argv[a]);
            const double dsm = sim.get_dshift_max(o);
            for (size_t r = 0; r < sim.parameters.nrays(); r++) {
                const RayData rd = sim.geometry.trace_ray<CoMoving>(o, r, dsm);
                head.push_back((long)rd.size());
                for (const ProjectedCellData &d : rd) {
                    cells.push_back(d.cellNr);
                    sh.push_back(d.shift);
                    dz.push_back(d.dZ);
                }
            }
        }
        write_raw_long(out + "/trace_len.bin", head);
        write_raw_long(out + "/trace_cell.bin", cells);
        write_raw(out + "/trace_shift.bin", sh);
        write_raw(out + "/trace_dZ.bin", dz);
        return 0;
    }
    if (cmd == "sample" && argc > 4) {
        set_up(sim, true);
        sim.get_max_npoints_on_rays<CoMoving>();
        const int nthr = omp_get_max_threads();
        std::vector<RayPair> pairs(nthr);
        for (auto &rp : pairs) rp.resize(sim.geometry.max_npoints_on_rays, sim.parameters.n_off_diag);
        const size_t nf = sim.parameters.nfreqs_red();
        const auto sec = [](std::chrono::steady_clock::time_point a,
                            std::chrono::steady_clock::time_point b) {
            return std::chrono::duration<double>(b - a).count();
        };
        std::ifstream lists(argv[4]);
        std::string line;
        bool first = true;
        while (std::getline(lists, line)) {
            std::vector<long> origins;
            std::stringstream ss(line);
            long o;
            while (ss >> o) origins.push_back(o);
            if (origins.empty()) continue;
            for (LineProducingSpecies &lspec : sim.lines.lineProducingSpecies) lspec.lambda.clear();
            sim.radiation.initialize_J();
            const auto t0 = std::chrono::steady_clock::now();
            for (size_t r = 0; r < sim.parameters.nrays() / 2; r++) {
                const long R = (long)r;
                const long ar = sim.geometry.rays.antipod[r];
#pragma omp parallel for schedule(static, 1)
                for (long i = 0; i < (long)origins.size(); i++) {
                    RayPair &rp = pairs[omp_get_thread_num()];
                    const long oo = origins[i];
                    const double w = sim.geometry.rays.weight(oo, r);
                    const double dsm = sim.get_dshift_max(oo);
                    RayData rd_r = sim.geometry.trace_ray<CoMoving>(oo, r, dsm);
                    RayData rd_ar = sim.geometry.trace_ray<CoMoving>(oo, ar, dsm);
                    const bool rf = rd_r.size() > rd_ar.size();
                    if (rf) rp.initialize(rd_r.size(), rd_ar.size());
                    else    rp.initialize(rd_ar.size(), rd_r.size());
                    if (rp.ndep > 1) {
                        for (size_t f = 0; f < nf; f++) {
                            if (rf) sim.setup(R, oo, f, rd_r, rd_ar, rp);
                            else    sim.setup(R, oo, f, rd_ar, rd_r, rp);
                            rp.solve();
                            rp.update_Lambda(sim.radiation.frequencies, sim.thermodynamics, oo, f, w,
                                             sim.lines);
                            sim.radiation.J[sim.radiation.index(oo, f)] += 2.0 * w * rp.get_u_at_origin();
                        }
                    } else {
                        const long b = sim.geometry.boundary.cell2boundary_nr[oo];
                        for (size_t f = 0; f < nf; f++)
                            sim.radiation.J[sim.radiation.index(oo, f)] +=
                                2.0 * w * 0.5 * (sim.radiation.I_bdy[R][b][f] + sim.radiation.I_bdy[R][b][f]);
                    }
                }
            }
            const auto t1 = std::chrono::steady_clock::now();
            double stateq_s = -1.0, ng_s = -1.0;
            if (first) {   // the whole model's rate equations and Ng step, once
                sim.compute_Jeff();
                sim.compute_level_populations_from_stateq();
                const auto t2 = std::chrono::steady_clock::now();
                sim.lines.iteration_using_Ng_acceleration(sim.parameters.pop_prec());
                const auto t3 = std::chrono::steady_clock::now();
                stateq_s = sec(t1, t2);
                ng_s = sec(t2, t3);
                first = false;
            }
            std::printf("{\"origins\": %zu, \"threads\": %d, \"formal_solve_s\": %.6f, "
                        "\"stateq_s\": %.6f, \"ng_s\": %.6f}\n",
                        origins.size(), nthr, sec(t0, t1), stateq_s, ng_s);
            std::fflush(stdout);
        }
        return 0;
    }
    if (cmd == "scatter" && argc > 5) {
        set_up(sim, true);
        const size_t N = sim.parameters.ncells(), nf = sim.parameters.nfreqs_red();
        const size_t np = sim.parameters.nrays() / 2;
        std::vector<double> U(np * N * nf), V(np * N * nf);
        {
            std::ifstream fu(argv[4], std::ios::binary), fv(argv[5], std::ios::binary);
            fu.read(reinterpret_cast<char *>(U.data()), (std::streamsize)(U.size() * sizeof(double)));
            fv.read(reinterpret_cast<char *>(V.data()), (std::streamsize)(V.size() * sizeof(double)));
        }
        sim.radiation.U.assign(np, std::vector<double>(N * nf));
        sim.radiation.V.assign(np, std::vector<double>(N * nf));
        for (size_t r = 0; r < np; r++)
            for (size_t i = 0; i < N * nf; i++) {
                sim.radiation.U[r][i] = U[r * N * nf + i];
                sim.radiation.V[r][i] = V[r * N * nf + i];
            }
        sim.get_max_npoints_on_rays<CoMoving>();
        RayPair rp;
        rp.resize(sim.geometry.max_npoints_on_rays, 0);
        std::vector<double> uo(np * N * nf), vo(np * N * nf), J(N * nf, 0.0);
        for (size_t r = 0; r < np; r++) {
            const long ar = sim.geometry.rays.antipod[r];
            for (size_t o = 0; o < N; o++) {
                const double w = sim.geometry.rays.weight(o, r);
                const double dsm = sim.get_dshift_max(o);
                RayData rd_r = sim.geometry.trace_ray<CoMoving>(o, r, dsm);
                RayData rd_ar = sim.geometry.trace_ray<CoMoving>(o, ar, dsm);
                const bool rf = rd_r.size() > rd_ar.size();
                const size_t n_front = rf ? rd_r.size() : rd_ar.size();
                const size_t n_back = rf ? rd_ar.size() : rd_r.size();
                rp.initialize(n_front, n_back);
                for (size_t f = 0; f < nf; f++) {
                    double u, v;
                    if (n_front + n_back + 1 > 1) {
                        if (rf) sim.setup_using_scattering(r, o, f, rd_r, rd_ar, rp);
                        else    sim.setup_using_scattering(r, o, f, rd_ar, rd_r, rp);
                        rp.solve_using_scattering();
                        u = rp.get_u_at_origin();
                        v = rp.get_v_at_origin();
                        if (rf) v = -v;
                    } else {
                        const long b = sim.geometry.boundary.cell2boundary_nr[o];
                        const double I = sim.radiation.I_bdy[r][b][f];
                        u = 0.5 * (I + I);
                        v = 0.5 * (I - I);
                    }
                    J[o * nf + f] += 2.0 * w * u;
                    uo[r * N * nf + o * nf + f] = u;
                    vo[r * N * nf + o * nf + f] = v;
                }
            }
        }
        write_raw(out + "/u.bin", uo);
        write_raw(out + "/v.bin", vo);
        write_raw(out + "/J.bin", J);
        return 0;
    }
    if (cmd == "image" && argc > 5) {
        sim.compute_spectral_discretisation_image(std::atof(argv[5]));
        sim.compute_boundary_intensities(sim.geometry.boundary.boundary_temperature);
        sim.compute_LTE_level_populations();
        mkdir((out + "/Simulation").c_str(), 0755);
        mkdir((out + "/Simulation/Image").c_str(), 0755);
        IoText io_out(out + "/");
        return sim.compute_and_write_image(io_out, std::atol(argv[4]));
    }
#if GPU_ACCELERATION
    if (cmd == "gpu" && argc > 6) {
        // Simulation::gpu_compute_radiation_field (simulation.cu:512-726)
        // as its Python binding calls it, reps times; each call builds its
        // solvers, traces and solves every ray pair and fills J and the ALO
        // again.  The first call also sets max_npoints_on_rays; the CUDA
        // context is created before it.
        set_up(sim, true);
        const size_t block = (size_t)std::atol(argv[4]), nblocks = (size_t)std::atol(argv[5]);
        const int reps = std::atoi(argv[6]);
        if (cudaFree(nullptr) != cudaSuccess) {
            std::fprintf(stderr, "no CUDA device\n");
            return 1;
        }
        for (int k = 0; k < reps; k++) {
            const auto t0 = std::chrono::steady_clock::now();
            const int rc = sim.gpu_compute_radiation_field(1, block, nblocks, 1.0);
            cudaDeviceSynchronize();
            const double s =
                std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            const cudaError_t e = cudaGetLastError();
            std::printf("{\"rep\": %d, \"seconds\": %.6f, \"rc\": %d, \"cuda\": \"%s\", "
                        "\"threads\": %d, \"max_npoints_on_rays\": %ld}\n",
                        k, s, rc, cudaGetErrorString(e), omp_get_max_threads(),
                        (long)sim.geometry.max_npoints_on_rays);
            std::fflush(stdout);
            if (rc != 0 || e != cudaSuccess) return 1;
        }
        sim.compute_Jeff();
        std::vector<double> J(sim.radiation.J.size());
        for (size_t i = 0; i < J.size(); i++) J[i] = sim.radiation.J[i];
        write_raw(out + "/J.bin", J);
        write_line_fields(sim, out);
        return 0;
    }
#endif
    std::fprintf(stderr, "unknown command %s\n", cmd.c_str());
    return 2;
}
