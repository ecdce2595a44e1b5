// configure.hpp for compiling the reference's CPU path as a test oracle:
// one process, OpenMP threads, no MPI, no Grid-SIMD, no GPU, no Python IO.
// It shadows the reference's checked-in src/configure.hpp (which enables MPI
// and the GPU) through the include path.
#pragma once
#define MAGRITTE_FOLDER "."
#define MAGRITTE_VERSION_MAJOR "0"
#define MAGRITTE_VERSION_MINOR "0"
#define PYTHON_IO false
#define MPI_PARALLEL false
#define OMP_PARALLEL true
#define GRID_SIMD false
#define GPU_ACCELERATION false
