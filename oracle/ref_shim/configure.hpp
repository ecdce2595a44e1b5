// configure.hpp for compiling the reference's code as a test oracle: one
// process, OpenMP threads, no MPI, no Grid-SIMD, no Python IO.  The GPU
// path (src/Simulation/Solver/gpu, Simulation::gpu_compute_radiation_field)
// is compiled in only when MGR_REF_GPU is defined, for the build of the
// reference's own GPU solver.  It shadows the reference's checked-in
// src/configure.hpp (which enables MPI and the GPU) through the include path.
#pragma once
#define MAGRITTE_FOLDER "."
#define MAGRITTE_VERSION_MAJOR "0"
#define MAGRITTE_VERSION_MINOR "0"
#define PYTHON_IO false
#define MPI_PARALLEL false
#define OMP_PARALLEL true
#define GRID_SIMD false
#ifdef MGR_REF_GPU
#define GPU_ACCELERATION true
#else
#define GPU_ACCELERATION false
#endif
