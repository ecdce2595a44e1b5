// ref_b200_driver.cpp -- Magritte's own Simulation, read from a model folder
// by the reference's IoText, routed to the B200 library through
// magritte_b200/integration/magritte_b200_binding.cpp (TEST INFRASTRUCTURE:
// proves the C++ binding compiles against the reference's headers and gives
// the reference's results; built by oracle/ref_build.sh into oracle/_ref).
//
//   magritte_ref_b200 <model/> <out/> ali <n> [mixed]   compute_level_populations_b200
//   magritte_ref_b200 <model/> <out/> radiation         compute_radiation_field_b200
#include <cstdlib>
#include <fstream>
#include <string>
#include <vector>

#include "Io/cpp/io_cpp_text.hpp"
#include "magritte_b200_binding.hpp"

static void write_raw(const std::string &path, const double *v, size_t n) {
    std::ofstream f(path, std::ios::binary);
    f.write(reinterpret_cast<const char *>(v), (std::streamsize)(n * sizeof(double)));
}

int main(int argc, char **argv) {
    if (argc < 4) return 2;
    const std::string model = argv[1], out = argv[2], cmd = argv[3];
    IoText io(model);
    Simulation sim;
    sim.read(io);
    sim.compute_spectral_discretisation();
    sim.compute_boundary_intensities(sim.geometry.boundary.boundary_temperature);
    sim.compute_LTE_level_populations();
    LineProducingSpecies &ls = sim.lines.lineProducingSpecies[0];
    if (cmd == "ali" && argc > 4) {
        const int prec = (argc > 5 && std::string(argv[5]) == "mixed") ? MGR_MIXED : MGR_FP64;
        const long it = compute_level_populations_b200(sim, true, std::atol(argv[4]), prec, 0.0);
        if (it < 0) return 1;
        write_raw(out + "/population.bin", ls.population.data(), ls.population.size());
        write_raw(out + "/error_max.bin", sim.error_max.data(), sim.error_max.size());
        const double itd = (double)it;
        write_raw(out + "/iterations.bin", &itd, 1);
        return 0;
    }
    if (cmd == "radiation") {
        if (compute_radiation_field_b200(sim, MGR_FP64) != 0) return 1;
        write_raw(out + "/J.bin", sim.radiation.J.data(), sim.radiation.J.size());
        const size_t N = sim.parameters.ncells(), K = ls.linedata.nrad;
        std::vector<double> jl(N * K);
        for (size_t p = 0; p < N; p++)
            for (size_t k = 0; k < K; k++) jl[p * K + k] = ls.Jlin[p][k];
        write_raw(out + "/Jlin.bin", jl.data(), jl.size());
        return 0;
    }
    return 2;
}
