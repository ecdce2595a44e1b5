#!/usr/bin/env bash
# Builds the reference's CPU path (Magritte's own C++, unmodified, read where
# it lies) into oracle/_ref/magritte_ref, a second checker for the C oracle
# (TEST INFRASTRUCTURE ONLY).  Nothing from the reference is copied into the
# repository: the sources are compiled in place, and the one translation unit
# that needs a fix is generated into oracle/_ref (git-ignored).
#
# What the build supplies, because the reference's own CMake build needs
# Eigen, MPI and CUDA that this image lacks:
#   oracle/ref_shim/configure.hpp  shadows src/configure.hpp (which enables
#                                  MPI and the GPU): OpenMP only
#   oracle/ref_shim/Eigen/*        a project-written subset of Eigen's API
#   oracle/_ref/raypair_fixed.cpp  src/Simulation/Raypair/raypair.cpp with
#                                  `return 0;` appended to RayPair::resize,
#                                  an int function that falls off its end
#                                  (undefined behaviour; g++ 13 emits a trap)
#
#   oracle/ref_build.sh [reference root, default /root/reference]
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${1:-/root/reference}"
SRC="$REF/src"
OUT="$HERE/_ref"
if [ ! -d "$SRC" ]; then
    echo "reference sources not found at $SRC" >&2
    exit 1
fi
mkdir -p "$OUT/obj"
CXX="${MGR_REF_CXX:-g++}"   # the system g++ (with OpenMP), not $CXX
FLAGS=(-std=c++14 -O2 -fopenmp -ffp-contract=off -w -I "$HERE/ref_shim" -I "$SRC" -I "$REF/dependencies")

# the fixed translation unit: the reference's file with one statement added
python3 - "$SRC/Simulation/Raypair/raypair.cpp" "$OUT/raypair_fixed.cpp" <<'EOF'
import sys
src = open(sys.argv[1]).read()
end = src.rstrip().rfind("}")
assert end > 0 and "return" not in src[src.find("resize"):end].split("End of RayPair constructor")[-1]
open(sys.argv[2], "w").write(src[:end] + "    return 0;\n" + src[end:])
EOF

UNITS=(
  Io/cpp/io_cpp_text.cpp Model/model.cpp Model/parameters.cpp
  Model/Geometry/geometry.cpp Model/Geometry/Cells/cells.cpp Model/Geometry/Rays/rays.cpp
  Model/Geometry/Boundary/boundary.cpp Model/Chemistry/chemistry.cpp
  Model/Chemistry/Species/species.cpp Model/Lines/lines.cpp
  Model/Lines/LineProducingSpecies/lineProducingSpecies.cpp
  Model/Lines/LineProducingSpecies/Quadrature/quadrature.cpp
  Model/Lines/LineProducingSpecies/Linedata/linedata.cpp
  Model/Lines/LineProducingSpecies/Linedata/CollisionPartner/collisionPartner.cpp
  Model/Radiation/radiation.cpp Model/Radiation/Frequencies/frequencies.cpp
  Model/Thermodynamics/thermodynamics.cpp Model/Thermodynamics/Temperature/temperature.cpp
  Model/Thermodynamics/Turbulence/turbulence.cpp Functions/heapsort.cpp
  Simulation/simulation.cpp Simulation/Solver/cpu/cpu_solver.cpp Simulation/Image/image.cpp
)
# compile in parallel, a few units at a time
compile() { "$CXX" "${FLAGS[@]}" "$@"; }
objs=()
jobs_running=0
for u in "${UNITS[@]}"; do
    o="$OUT/obj/$(echo "$u" | tr / _).o"
    objs+=("$o")
    compile -c "$SRC/$u" -o "$o" &
    jobs_running=$((jobs_running + 1))
    if [ "$jobs_running" -ge 6 ]; then wait -n; jobs_running=$((jobs_running - 1)); fi
done
compile -I "$SRC/Simulation/Raypair" -c "$OUT/raypair_fixed.cpp" -o "$OUT/obj/raypair_fixed.o" &
compile -c "$HERE/ref_driver.cpp" -o "$OUT/obj/ref_driver.o" &
while [ "$(jobs -rp | wc -l)" -gt 0 ]; do wait -n; done
"$CXX" -fopenmp -o "$OUT/magritte_ref" "${objs[@]}" "$OUT/obj/raypair_fixed.o" "$OUT/obj/ref_driver.o"
echo "$OUT/magritte_ref"

# The reference's GPU solver (Simulation::gpu_compute_radiation_field,
# src/Simulation/simulation.cu, src/Simulation/Solver/gpu/gpu_solver.cu) in a
# second build of the same sources with GPU_ACCELERATION on, as the
# reference's CMake build makes it (src/CMakeLists.txt:50-88): the C++ units
# by the host compiler, the two .cu units by nvcc with the reference's own
# CUDA_NVCC_FLAGS "-O5 -use_fast_math" (CMakeLists.txt:20), for sm_100a.
if command -v nvcc > /dev/null 2>&1; then
    CUDA_HOME="${CUDA_HOME:-$(dirname "$(dirname "$(command -v nvcc)")")}"
    mkdir -p "$OUT/obj_gpu"
    GFLAGS=(-DMGR_REF_GPU -I "$CUDA_HOME/include")
    gobjs=()
    jobs_running=0
    for u in "${UNITS[@]}"; do
        o="$OUT/obj_gpu/$(echo "$u" | tr / _).o"
        gobjs+=("$o")
        compile "${GFLAGS[@]}" -c "$SRC/$u" -o "$o" &
        jobs_running=$((jobs_running + 1))
        if [ "$jobs_running" -ge 6 ]; then wait -n; jobs_running=$((jobs_running - 1)); fi
    done
    compile "${GFLAGS[@]}" -I "$SRC/Simulation/Raypair" -c "$OUT/raypair_fixed.cpp" \
        -o "$OUT/obj_gpu/raypair_fixed.o" &
    compile "${GFLAGS[@]}" -c "$HERE/ref_driver.cpp" -o "$OUT/obj_gpu/ref_driver.o" &
    for u in Simulation/simulation.cu Simulation/Solver/gpu/gpu_solver.cu; do
        o="$OUT/obj_gpu/$(echo "$u" | tr / _).o"
        gobjs+=("$o")
        nvcc -std=c++14 -O5 -use_fast_math -gencode arch=compute_100a,code=sm_100a -w \
            -Xcompiler -fopenmp -DMGR_REF_GPU -I "$HERE/ref_shim" -I "$SRC" -I "$REF/dependencies" \
            -c "$SRC/$u" -o "$o" &
    done
    while [ "$(jobs -rp | wc -l)" -gt 0 ]; do wait -n; done
    "$CXX" -fopenmp -o "$OUT/magritte_ref_gpu" "${gobjs[@]}" "$OUT/obj_gpu/raypair_fixed.o" \
        "$OUT/obj_gpu/ref_driver.o" -L "$CUDA_HOME/lib64" -lcudart -Wl,-rpath,"$CUDA_HOME/lib64"
    echo "$OUT/magritte_ref_gpu"
fi

# Magritte's Simulation routed to the B200 library through the C++ binding
# of magritte_b200/integration (needs libmagritte_b200.so built first)
LIBDIR="$(cd "$HERE/.." && pwd)/magritte_b200"
if [ -f "$LIBDIR/libmagritte_b200.so" ]; then
    INC=(-I "$(cd "$HERE/.." && pwd)/include" -I "$LIBDIR/integration")
    compile "${INC[@]}" -c "$LIBDIR/integration/magritte_b200_binding.cpp" -o "$OUT/obj/binding.o"
    compile "${INC[@]}" -c "$HERE/ref_b200_driver.cpp" -o "$OUT/obj/ref_b200_driver.o"
    "$CXX" -fopenmp -o "$OUT/magritte_ref_b200" "${objs[@]}" "$OUT/obj/raypair_fixed.o" \
        "$OUT/obj/binding.o" "$OUT/obj/ref_b200_driver.o" -L "$LIBDIR" -lmagritte_b200 \
        -Wl,-rpath,'$ORIGIN/../../magritte_b200'
    echo "$OUT/magritte_ref_b200"
fi
