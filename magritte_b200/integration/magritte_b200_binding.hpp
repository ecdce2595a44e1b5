// magritte_b200_binding.hpp -- Magritte's Simulation routed to the B200 path.
//
// Declarations a Magritte build adds next to Simulation (src/Simulation/
// simulation.hpp:49-166).  Both functions take the Simulation as Magritte
// leaves it after read(), compute_spectral_discretisation(),
// compute_boundary_intensities() and a start for the populations
// (compute_LTE_level_populations() or populations read from a model), and
// leave their results in its containers.  parameters.n_off_diag is honoured
// (0 .. 8; 2 and more: the non-local ALO of mgr_set_n_off_diag).
#pragma once

#include "Simulation/simulation.hpp"
#include "magritte_b200.h"

// Simulation::compute_level_populations(io, use_Ng, max_niterations)
// (Simulation/sim_lines.tpp:61-164) on the GPU: the ALI + Ng loop from the
// Simulation's current populations; precision is MGR_FP64 or MGR_MIXED;
// tol_max_rel > 0 stops at that max relative change, <= 0 uses the
// reference's own test (fraction_not_converged <= 0.005).  Writes the
// populations, emissivities/opacities, Jlin, Jeff and error_max back.
// Returns the number of iterations, -1 on failure (logged).
long compute_level_populations_b200(Simulation &sim, bool use_Ng, long max_niterations,
                                    int precision = MGR_FP64, double tol_max_rel = 0.0,
                                    int device = 0);

// Simulation::compute_radiation_field (Simulation/sim_radiation.tpp:56-338)
// followed by compute_Jeff, on the GPU: radiation.J, Jlin and Jeff written
// back.  Returns 0, or -1 on failure (logged).
int compute_radiation_field_b200(Simulation &sim, int precision = MGR_FP64, int device = 0);
