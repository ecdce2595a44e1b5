/*
 * magritte_b200.h -- C ABI of the B200 radiation hot path.
 *
 * One opaque handle owns one model resident on one GPU.  Every entry point
 * returns an mgr_status (0 = success); mgr_last_error() gives the message of
 * the last failure on a handle.  No entry point aborts, asserts or traps:
 * device-side failures (a ray that cannot be traced, a singular rate matrix)
 * are counted on the device and reported as status codes.
 *
 * Each entry point names the Magritte member it replaces (paths inside the
 * UCL/Magritte source tree).  The reference's Simulation is single-threaded
 * at its interface; so is a handle (one host thread and one CUDA stream per
 * handle).
 */
#ifndef MAGRITTE_B200_H
#define MAGRITTE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    MGR_OK = 0,
    MGR_ERR_INVALID_ARG = 1,   /* bad pointer, size or order of calls        */
    MGR_ERR_TRACE = 2,         /* a ray found no neighbour ahead of it       */
    MGR_ERR_LU_SINGULAR = 3,   /* a cell's rate matrix had a zero pivot      */
    MGR_ERR_NOT_CONVERGED = 4, /* ALI stopped at max_iter                    */
    MGR_ERR_CUDA = 5,          /* a CUDA runtime call failed                 */
    MGR_ERR_TIMEOUT = 6,       /* a bounded device wait ran out              */
    MGR_ERR_UNSUPPORTED = 7,   /* input outside what the device path covers  */
    MGR_ERR_STATE = 8,         /* called before the step it depends on       */
    MGR_ERR_NO_MEMORY = 9,     /* a device allocation failed                 */
    MGR_ERR_TOO_LARGE = 10     /* input larger than a fixed capacity         */
} mgr_status;

typedef enum {
    MGR_FP64 = 0,   /* every step in double precision                        */
    MGR_MIXED = 1   /* opacities, source functions and optical depths in
                       float, Feautrier elimination and rate equations in
                       double                                                */
} mgr_precision;

/* One collision partner of the line species
 * (Lines/LineProducingSpecies/Linedata/CollisionPartner/collisionPartner.hpp). */
typedef struct {
    int32_t ntmp;              /* temperatures in the rate table            */
    int32_t ncol;              /* collisional transitions                   */
    int32_t ortho_para;        /* 0 'n', 1 ortho-H2 ('o'), 2 para-H2 ('p')  */
    int32_t reserved;
    const int64_t *icol;       /* [ncol] upper level                        */
    const int64_t *jcol;       /* [ncol] lower level                        */
    const double  *tmp;        /* [ntmp] K, ascending                       */
    const double  *Cd;         /* [ntmp*ncol] downward rates, m^3 s^-1      */
    const double  *Ce;         /* [ntmp*ncol] upward rates, m^3 s^-1        */
    const double  *abundance;  /* [ncells] partner number density, m^-3     */
} mgr_colpar_desc;

/* The model as Magritte's Model holds it (Model/model.hpp:23-44), with one
 * line-producing species.  Host pointers; mgr_upload_model copies them. */
typedef struct {
    int64_t ncells;
    const double  *position;       /* [ncells*3] m                          */
    const double  *velocity;       /* [ncells*3] fraction of c              */
    const int64_t *nbr_offsets;    /* [ncells+1] CSR offsets                */
    const int64_t *nbr_list;       /* neighbour cells, in list order        */
    int64_t nboundary;
    const int64_t *boundary2cell;  /* [nboundary]                           */
    const double  *boundary_temperature; /* [nboundary] K, NULL: T_CMB      */
    int64_t nrays;
    const double  *rays;           /* [nrays*3] unit vectors                */
    const double  *ray_weights;    /* [nrays]                               */
    const double  *temperature;    /* [ncells] K                            */
    const double  *vturb2;         /* [ncells] (v_turb/c)^2                 */
    int32_t nlev;
    int32_t nrad;
    const double  *energy;         /* [nlev] J                              */
    const double  *weight;         /* [nlev] statistical weights            */
    const int64_t *irad;           /* [nrad] upper level of each line       */
    const int64_t *jrad;           /* [nrad] lower level                    */
    const double  *A;              /* [nrad] s^-1                           */
    const double  *Bs;             /* [nrad] stimulated emission            */
    const double  *Ba;             /* [nrad] absorption                     */
    const double  *frequency;      /* [nrad] Hz                             */
    double inverse_mass;           /* 1 / (mass in amu)                     */
    const double  *population_tot; /* [ncells] m^-3                         */
    int32_t nquads;
    int32_t ncolpar;
    const double  *quad_roots;     /* [nquads] ascending, Doppler widths    */
    const double  *quad_weights;   /* [nquads]                              */
    const mgr_colpar_desc *colpar; /* [ncolpar]                             */
    double pop_prec;               /* Parameters::pop_prec                  */
    double max_width_fraction;     /* Parameters::max_width_fraction (0.5)  */
} mgr_model_desc;

/* Options of the ALI loop.  Replaces the arguments of
 * Simulation::compute_level_populations(io, use_Ng, max_niterations).
 * A zeroed struct with use_ng, precision and max_iter set is the
 * reference's loop. */
typedef struct {
    int32_t use_ng;        /* Ng acceleration after every ng_every normal
                              iterations (the reference: every 5th
                              iteration, i.e. after 4)                     */
    int32_t precision;     /* mgr_precision                                */
    int64_t max_iter;      /* 1000 in the reference's default overload     */
    double  tol_max_rel;   /* > 0: stop once max over (cell, level) of
                              2|n - n_prev|/(n + n_prev) < tol (levels with
                              n > 1e-10 n_tot); <= 0: the reference's stop
                              test, fraction_not_converged <= 0.005        */
    int32_t use_graph;     /* replay each iteration as a CUDA graph        */
    int32_t ng_every;      /* normal iterations before each Ng step: 0 for
                              the reference's 4, else >= 3 (the step reads
                              the populations and three previous iterates) */
} mgr_ali_opts;

typedef struct mgr_handle mgr_handle;

/* --- lifetime ----------------------------------------------------------- */

/* New handle on CUDA device `device`.  Replaces constructing Simulation
 * (Simulation/simulation.hpp:49-166). */
mgr_status mgr_create(int device, mgr_handle **out);

/* Frees every device buffer of the handle. */
mgr_status mgr_destroy(mgr_handle *h);

/* Message of the last failed call on h (never NULL). */
const char *mgr_last_error(const mgr_handle *h);

/* Library version string. */
const char *mgr_version(void);

/* Copies the model to the device and derives antipodal rays
 * (Rays::setup_antipodal_rays, Model/Geometry/Rays/rays.cpp:90-102) and the
 * boundary maps.  Replaces Simulation::read (Model/model.cpp). */
mgr_status mgr_upload_model(mgr_handle *h, const mgr_model_desc *model);

/* Caps device memory used for stored ray traces (bytes; 0 = automatic):
 * the traced points and, for models the staged kernels solve, the far-end
 * boundary cache of the mixed solve (8 B per ray pair and bin per origin).
 * Beyond it, traces are recomputed per batch of origins each solve. */
mgr_status mgr_set_trace_budget(mgr_handle *h, int64_t bytes);

/* --- set-up steps (Simulation/simulation.hpp) --------------------------- */

/* Per-cell frequency grids nu = line + width*root.  The device path needs
 * each cell's grid to be already ascending (lines apart by more than their
 * quadrature span), i.e. the reference's heapsort to be the identity;
 * otherwise MGR_ERR_UNSUPPORTED.  Replaces
 * Simulation::compute_spectral_discretisation (Simulation/sim_spectrum.tpp:13-196). */
mgr_status mgr_compute_spectral_discretisation(mgr_handle *h);

/* Boundary intensities: Planck at each boundary cell's temperature
 * (the model's, or T_CMB).  Replaces Simulation::compute_boundary_intensities
 * (Simulation/sim_radiation.tpp:17-48). */
mgr_status mgr_compute_boundary_intensities(mgr_handle *h);

/* Boltzmann populations scaled to n_tot, then emissivities and opacities.
 * Replaces Simulation::compute_LTE_level_populations
 * (Simulation/sim_lines.tpp:10-16). */
mgr_status mgr_compute_LTE_level_populations(mgr_handle *h);

/* --- geometry ----------------------------------------------------------- */

/* Traces every ray of every origin on the device (bit-exact with
 * Geometry::trace_ray<CoMoving>, Model/Geometry/geometry.tpp:21-207) and
 * keeps the traces while they fit the trace budget. */
mgr_status mgr_trace(mgr_handle *h);

/* npoints[r*ncells + o] = n_ar + n_r + 1 for r < nrays/2.  Replaces
 * Simulation::get_npoints_on_rays<CoMoving> (Simulation/simulation.tpp:540-552). */
mgr_status mgr_get_npoints_on_rays(mgr_handle *h, int64_t *npoints);

/* Points of the trace of (origin o, ray r): cell numbers, Doppler shifts and
 * distance increments (ProjectedCellData, Model/Geometry/raydata.hpp:17-35).
 * *n receives the length; at most cap entries are written. */
mgr_status mgr_get_trace(mgr_handle *h, int64_t o, int64_t r, int64_t cap,
                         int64_t *cell, double *shift, double *dZ, int64_t *n);

/* --- radiation field ---------------------------------------------------- */

/* Formal solve over all ray pairs and frequencies: J (when kept), the line
 * integrals Jlin and the diagonal ALO.  Replaces
 * Simulation::compute_radiation_field (Simulation/sim_radiation.tpp:56-338). */
mgr_status mgr_compute_radiation_field(mgr_handle *h, int32_t precision);

/* Keep (1) or skip (0) the full J[ncells*nfreqs] in device memory; Jlin and
 * the ALO are always produced.  Off by default. */
mgr_status mgr_set_keep_J(mgr_handle *h, int32_t keep);

/* --- level populations -------------------------------------------------- */

/* Jeff = Jlin - (h/4 pi) Ls n_i.  Replaces Simulation::compute_Jeff
 * (Simulation/sim_lines.tpp:176-220). */
mgr_status mgr_compute_Jeff(mgr_handle *h);

/* Statistical equilibrium per cell, convergence statistics, emissivities and
 * opacities.  Replaces Simulation::compute_level_populations_from_stateq
 * (Simulation/sim_lines.tpp:24-30 -> lineProducingSpecies.tpp:120-171, 249-495). */
mgr_status mgr_compute_level_populations_from_stateq(mgr_handle *h);

/* One Ng-accelerated step, convergence statistics, emissivities and
 * opacities.  Replaces Lines::iteration_using_Ng_acceleration
 * (Model/Lines/lines.cpp:131-149). */
mgr_status mgr_ng_acceleration(mgr_handle *h);

/* fraction_not_converged, relative_change_mean and the max relative change
 * of the last population update (lineProducingSpecies.tpp:120-171). */
mgr_status mgr_get_convergence(mgr_handle *h, double *fnc, double *rcm, double *max_rel);

/* The full ALI loop.  *iterations receives the count, as the reference's
 * return value; err_max_hist (optional, max_iter entries) the max relative
 * change of every iteration.  Returns MGR_ERR_NOT_CONVERGED when max_iter is
 * reached.  Replaces Simulation::compute_level_populations
 * (Simulation/sim_lines.tpp:42-164). */
mgr_status mgr_compute_level_populations(mgr_handle *h, const mgr_ali_opts *opts,
                                         int64_t *iterations, double *err_max_hist);

/* --- data movement ------------------------------------------------------ */

mgr_status mgr_set_populations(mgr_handle *h, const double *pop);     /* [ncells*nlev] */
mgr_status mgr_get_populations(mgr_handle *h, double *pop);           /* [ncells*nlev] */
mgr_status mgr_get_J(mgr_handle *h, double *J);                       /* [ncells*nfreqs] */
mgr_status mgr_get_Jlin(mgr_handle *h, double *Jlin);                 /* [ncells*nrad] */
mgr_status mgr_get_Jeff(mgr_handle *h, double *Jeff);                 /* [ncells*nrad] */
mgr_status mgr_get_lambda(mgr_handle *h, double *Ls);                 /* [ncells*nrad] */
mgr_status mgr_get_emissivity_opacity(mgr_handle *h, double *eta, double *chi); /* [ncells*nrad] */

/* The three previous iterates that Ng acceleration reads ([ncells*nlev]
 * each; NULL skips one): with the populations they are what
 * LineProducingSpecies::write stores (population, population_prev1..3,
 * Model/Lines/LineProducingSpecies/lineProducingSpecies.cpp:105-135), so a
 * run can be checkpointed and resumed exactly. */
mgr_status mgr_get_population_history(mgr_handle *h, double *prev1, double *prev2, double *prev3);

/* Restores populations and their history (a NULL previous iterate is set
 * to zero, as the reference leaves it when the file is absent,
 * lineProducingSpecies.cpp:60-95), then the emissivities and opacities. */
mgr_status mgr_set_population_history(mgr_handle *h, const double *pop, const double *prev1,
                                      const double *prev2, const double *prev3);
mgr_status mgr_get_frequencies(mgr_handle *h, double *nu);            /* [ncells*nfreqs] */

/* Device time of the last formal solve (ms, CUDA events on the handle's
 * stream) and the ray-point-frequency updates it did. */
mgr_status mgr_get_solve_stats(mgr_handle *h, double *ms, double *updates);

/* Of the last formal solve's device time: the milliseconds spent
 * rebuilding traces, batch by batch of origins, when the traces exceed the
 * trace budget (0 when they are stored).  No reference counterpart. */
mgr_status mgr_get_solve_breakdown(mgr_handle *h, double *trace_ms);

/* Mixed precision: (origin, pair, bin) solves of the last formal solve that
 * were redone in double (inverted lines driving the opacity below half its
 * 1e-26 floor, or a float failure), and the number of origins since
 * mgr_create that were solved again entirely in double because their
 * failures did not fit that list.  No reference counterpart (the reference
 * solves in double). */
mgr_status mgr_get_patch_stats(mgr_handle *h, int64_t *patched, int64_t *fallbacks);

/* Entries of the mixed solve's list of (origin, pair, bin) solves to redo
 * in double (16 bytes each; 0 = automatic: 1 % of all solves, 1M to 64M
 * entries).  Failures beyond it send their origins to a re-solve in
 * double.  No reference counterpart. */
mgr_status mgr_set_patch_capacity(mgr_handle *h, int64_t entries);

/* parameters.n_off_diag (Model/parameters.hpp:87): 0 or 1 keep the
 * diagonal ALO (the reference's n_off_diag = 1 adds no off-diagonal
 * element, raypair_lambda.tpp:129); M = 2 .. 8 keep, for every cell, line
 * and ray pair, the M-1 nearest off-diagonal elements of the origin's row on
 * each side (RayPair::solve's non-local branch, raypair_solver.tpp:336-388,
 * with RayPair::update_Lambda's weights, raypair_lambda.tpp:94-149), use
 * them in compute_Jeff (sim_lines.tpp:176-220), and solve the rate
 * equations of all cells as one system (lineProducingSpecies.tpp:249-495,
 * SparseLU there, block-Jacobi sweeps here).  Where the reference reads
 * other elements (L_lower[m][n_ar-m] is the element (n_ar+1, n_ar-m)) and
 * places the upper-level term of an element at (I(nr), I(nr)) instead of
 * (I(p), I(nr)), this follows the origin's row and the placement whose
 * terms cancel at convergence, so the iteration keeps the local-ALO fixed
 * point.  One whole model only (MGR_ERR_UNSUPPORTED with a batch or an
 * origin range); each formal solve adds one FP64 kernel, and the ALI
 * iteration is not graph-captured. */
mgr_status mgr_set_n_off_diag(mgr_handle *h, int32_t n_off_diag);

/* The non-local ALO elements of the last formal solve (n_off_diag = M >= 2):
 * Loff [ncells][nrad][nrays/2][2][M-1] (side 0: the front trace, the longer
 * one of the pair, side 1 the back trace; distance 1 .. M-1 from the
 * origin) and their cells Loff_nr [ncells][nrays/2][2][M-1] (-1: no point
 * there).  Either pointer may be NULL. */
mgr_status mgr_get_alo_nonlocal(mgr_handle *h, double *Loff, int64_t *Loff_nr);

/* Block-Jacobi sweeps of the last non-local statistical-equilibrium solve. */
mgr_status mgr_get_nonlocal_sweeps(mgr_handle *h, int64_t *sweeps);

/* Synchronises the handle's stream. */
mgr_status mgr_synchronize(mgr_handle *h);

/* Device timing of a region of calls on the handle's stream: start records
 * a CUDA event, stop records another, waits for it and returns the elapsed
 * milliseconds.  Benchmark support; no reference counterpart (the reference
 * times with its host Timer, Tools/timer.hpp:26-143). */
mgr_status mgr_timer_start(mgr_handle *h);
mgr_status mgr_timer_stop(mgr_handle *h, double *ms);

/* Number of this library's kernels launched on the handle since it was
 * created (library kernels such as CUB's prefix sum are not counted). */
mgr_status mgr_get_launch_count(mgr_handle *h, int64_t *count);

/* --- learned warm start ------------------------------------------------- */

/* Per-cell features and hidden width of the warm-start network. */
#define MGR_MLP_FEATURES 10
#define MGR_MLP_HIDDEN 128

/* A 3 x 128 tanh MLP mapping standardised features to a correction of the
 * LTE log level fractions: n = n_tot softmax(log x_LTE + MLP(f)).
 * params holds W0 [128 x nin], b0, W1 [128 x 128], b1, W2, b2,
 * W3 [nout x 128], b3 (row-major, out x in). */
typedef struct {
    int32_t nin;           /* MGR_MLP_FEATURES                            */
    int32_t nout;          /* number of levels                            */
    float *params;         /* [mgr_mlp_param_count]                       */
    const float *feat_mean;   /* [nin] feature standardisation            */
    const float *feat_istd;   /* [nin]                                    */
} mgr_mlp;

typedef struct {
    int32_t epochs;
    int32_t batch;
    float lr;
    float weight_decay;
    uint64_t seed;         /* shuffling                                   */
} mgr_train_opts;

/* Number of floats in params for a network with nout levels. */
mgr_status mgr_mlp_param_count(int32_t nout, int64_t *count);

/* Features [ncells*MGR_MLP_FEATURES] of the uploaded model: log10 of the
 * collision-partner density, n_tot, T, line width, velocity-gradient
 * length, mean/min column density and mean/min velocity-coherent column
 * along the traced rays, mean ray length.  No counterpart in the reference. */
mgr_status mgr_get_features(mgr_handle *h, float *features);

/* LTE log fractions [ncells*nlev] of the uploaded model. */
mgr_status mgr_get_lte_logfrac(mgr_handle *h, float *logfrac);

/* Warm start: features, network and populations on the device, then
 * emissivities and opacities; replaces the LTE start
 * (Simulation::compute_LTE_level_populations, Simulation/sim_lines.tpp:10-16)
 * before mgr_compute_level_populations.  No counterpart in the reference. */
mgr_status mgr_warm_start(mgr_handle *h, const mgr_mlp *net);

/* Trains net->params in place on device `device` with this library's own
 * forward, backward and Adam kernels.  X [n*nin] raw features, lte and
 * target [n*nout] log fractions (target: converged populations).
 * loss_hist (optional) receives the mean loss of each epoch. */
mgr_status mgr_mlp_train(int device, mgr_mlp *net, const float *X, const float *lte,
                         const float *target, int64_t n, const mgr_train_opts *opts,
                         float *loss_hist);

/* Network output (the log-fraction correction) [n*nout] for features X. */
mgr_status mgr_mlp_forward(int device, const mgr_mlp *net, const float *X, int64_t n,
                           float *delta);

/* Summed loss over n samples and its gradient with respect to params
 * (for gradient checks). */
mgr_status mgr_mlp_loss_grad(int device, const mgr_mlp *net, const float *X, const float *lte,
                             const float *target, int64_t n, float *loss, float *grad);

/* --- without allocation ------------------------------------------------- */

/* --- scattering ---------------------------------------------------------- */

/* Scattering terms U and V of every ray pair, cell and bin
 * ([nrays/2][ncells][nfreqs] host arrays; NULL sets zeros), as Radiation
 * holds them (Model/Radiation/radiation.hpp:33-34). */
mgr_status mgr_set_scattering_terms(mgr_handle *h, const double *U, const double *V);
mgr_status mgr_get_scattering_terms(mgr_handle *h, double *U, double *V);

/* The formal solve with scattering terms, FP64: every ray pair and origin
 * set up as Simulation::setup_using_scattering (Simulation/simulation.tpp:51-171:
 * term1 = (U + eta)/chi, term2 = V/chi, U and V interpolated on each cell's
 * grid) and solved as RayPair::solve_using_scattering
 * (Simulation/Raypair/raypair_solver.tpp:10-190) for u and v at the origin;
 * J (when kept), Jlin and the ALO follow as in compute_radiation_field.
 * The longer trace is in front, and v is stored with its sign flipped when
 * that is the ray rather than its antipode (Simulation/sim_radiation.tpp:226-236).
 * Needs the traces stored (within the trace budget).  The reference defines
 * these two functions but its compute_radiation_field does not call them. */
mgr_status mgr_compute_radiation_field_scattering(mgr_handle *h);

/* u and v at the origins of the last scattering solve, [nrays/2][ncells][nfreqs]. */
mgr_status mgr_get_scattering_uv(mgr_handle *h, double *u, double *v);

/* U[r1] = sum over ray pairs r2 of u[r2] and V likewise, for every r1 (the
 * phase function is one), from the last scattering solve: the scattering
 * terms of the next one.  Replaces Radiation::calc_U_and_V
 * (Model/Radiation/radiation.cpp:330-434, one process). */
mgr_status mgr_calc_U_and_V(mgr_handle *h);

/* --- images -------------------------------------------------------------- */

/* An image along ray `ray`: the emergent intensity through every cell, on
 * the image grid nu[f] = line + line*width*root (the same in every cell,
 * sorted ascending; width is relative, e.g. a few times v_max/c).  For each
 * origin both rays are traced in the rest frame, the antipode's trace in
 * front, and the ray pair is solved in FP64 with the current populations;
 * I_m is the intensity leaving through the front (far end of the antipode's
 * trace), I_p the one leaving through the end (far end of the ray's trace).
 * ImX, ImY: each cell's coordinates on the image plane.  Replaces
 * Simulation::compute_spectral_discretisation_image (sim_spectrum.tpp:200-250)
 * + compute_boundary_intensities + compute_and_write_image
 * (Simulation/sim_radiation.tpp:348-478, Image::set_coordinates in
 * Simulation/Image/image.cpp:86-127).  Outputs: nu [nfreqs], I_m and I_p
 * [ncells*nfreqs], ImX and ImY [ncells]; any may be NULL.  The radiation
 * field's own grid and boundary table are left unchanged. */
mgr_status mgr_compute_image(mgr_handle *h, int64_t ray, double width, double *nu, double *I_m,
                             double *I_p, double *ImX, double *ImY);

/* --- partitioned runs (one shard per GPU) -------------------------------- */

/* Restricts the handle to the origins [o_begin, o_end) of its model: the
 * formal solve computes Jlin and the ALO of those origins only, and the
 * statistical equilibrium updates those cells only.  Every shard keeps the
 * whole model and the whole population history; after each rate-equation
 * step the shards exchange the populations of their cells and their
 * convergence partials (an all-gather over the shards), after which every
 * shard holds the same arrays as an unpartitioned run and the Ng step and
 * the emissivity update run on each shard alike.  Bounds must be multiples
 * of 4 (or ncells).  Replaces the reference's split of the ray directions
 * over MPI ranks with its reduction of J and gather of the ALO
 * (Simulation/sim_radiation.tpp:130, Model/Radiation/radiation.cpp:292-325,
 * Model/Lines/LineProducingSpecies/Lambda/lambda.tpp:191-317): partitioning
 * by origin leaves each cell's J, ALO and rate equations on one shard, so no
 * reduction of J is needed.  Not for batches of models. */
mgr_status mgr_set_origin_range(mgr_handle *h, int64_t o_begin, int64_t o_end);

/* Jeff and the statistical equilibrium of the shard's cells (the history
 * of the other cells shifts as well); their convergence partials are left
 * in MGR_BUF_CONVERGENCE_PARTIALS at the positions of their 4-cell blocks.
 * The local half of Simulation::compute_level_populations_from_stateq
 * (sim_lines.tpp:24-30) for a shard. */
mgr_status mgr_stateq_local(mgr_handle *h);

/* After the exchange: emissivities and opacities of every cell from the
 * populations, and the convergence statistics from every block's partials
 * (read them with mgr_get_convergence). */
mgr_status mgr_stateq_finish(mgr_handle *h);

typedef enum {
    MGR_BUF_POPULATION = 0,            /* double [ncells*nlev] */
    MGR_BUF_PREV1 = 1,                 /* double [ncells*nlev] */
    MGR_BUF_PREV2 = 2,                 /* double [ncells*nlev] */
    MGR_BUF_PREV3 = 3,                 /* double [ncells*nlev] */
    MGR_BUF_JLIN = 4,                  /* double [ncells*nrad] */
    MGR_BUF_LAMBDA = 5,                /* double [ncells*nrad] */
    MGR_BUF_CONVERGENCE_PARTIALS = 6   /* double [3*ceil(ncells/4)]: count, sum, max per 4 cells */
} mgr_buffer;

/* Device address and element count of one of the handle's state arrays,
 * for collectives that read and write them in place (an all-gather over
 * NCCL).  The address stays valid until mgr_upload_model or mgr_destroy.
 * No reference counterpart. */
mgr_status mgr_get_device_buffer(mgr_handle *h, int32_t which, void **ptr, int64_t *count);

/* --- batches of independent models ------------------------------------- */

/* Declares the uploaded point cloud to be the union of `nseg` independent
 * models that share species, rays and quadrature and whose neighbour graphs
 * are disjoint: model s owns cells [seg_begin[s], seg_begin[s+1]) with
 * seg_begin[0] = 0 and seg_begin[nseg] = ncells (nseg+1 entries).
 * mgr_compute_level_populations then iterates every model to its own
 * convergence: statistics and Ng coefficients per model, and a model that
 * has converged is frozen (populations kept, its origins skipped by the
 * formal solve).  The reference runs one Simulation per model
 * (Simulation::compute_level_populations, sim_lines.tpp:61-164, per model);
 * no single reference function corresponds.  nseg = 1 returns to the
 * single-model path.  Cleared by mgr_upload_model. */
mgr_status mgr_set_segments(mgr_handle *h, int64_t nseg, const int64_t *seg_begin);

/* After mgr_compute_level_populations on a batch: stats[3*s .. 3*s+2] =
 * fraction not converged, mean and max relative population change of model
 * s at its last iteration; iterations[s] = the iteration at which model s
 * converged (the total when it did not).  Either pointer may be NULL.
 * No reference counterpart. */
mgr_status mgr_get_segment_results(mgr_handle *h, double *stats, int64_t *iterations);

/* --- autotuning of the formal solve -------------------------------------- */

/* Which formal-solve kernel ran and with what block shape.  No reference
 * counterpart. */
typedef struct {
    int32_t kernel;           /* 0 generic, 1 staged (shared-memory) mixed kernel, -1 none yet */
    int32_t min_blocks;       /* resident blocks per SM it is compiled for */
    int32_t warps_per_block;
    int32_t tuned;            /* 1 once every candidate has been timed */
    float ms[8];              /* time of each candidate's solve (0: not timed) */
} mgr_tuning;

/* With mode 1 or 2 the next formal solves of each precision each run one of
 * the compiled candidates (register budgets for 6, 7 and 8 resident blocks
 * per SM), timed with CUDA events; every later solve uses the fastest.  Mode
 * 1 first reuses a result that another handle of this process found for the
 * same device, precision and problem shape; mode 2 always re-times.  The
 * candidates compute identical results.  Tuning restarts when a retrace
 * changes the longest ray pair.  Mode 0 (default) turns tuning off.
 * No reference counterpart. */
mgr_status mgr_set_autotune(mgr_handle *h, int32_t enable);
mgr_status mgr_get_tuning(mgr_handle *h, int32_t precision, mgr_tuning *out);

/* Largest ncells * nlev that mgr_convergence_noalloc accepts. */
#define MGR_NOALLOC_MAX_ELEMENTS 67108864LL

/* Convergence statistics of populations `pop` against `prev`, for callers
 * that cannot allocate device memory: applications that reserve all of the
 * GPU's memory up front in their own pool and do not allow cudaMalloc (which
 * would also synchronise the device).  No counterpart in the reference; it
 * computes what check_for_convergence does, with no handle.
 *   pop, prev  [ncells*nlev] device arrays, cell-major
 *   pop_tot    [ncells] device array (total population per cell)
 *   stats      device array of 3 doubles, receives the fraction of levels
 *              (with n > 1e-10 n_tot) whose 2|n-n'|/(n+n') exceeds
 *              pop_prec, the mean of that change over ncells*nlev, its max
 *   stream     cudaStream_t to run on (NULL: the default stream)
 * Calls no allocator.  Its scratch is a fixed 1.5 MiB array inside the
 * library that every GPU loading the library holds until the process exits;
 * ncells*nlev above MGR_NOALLOC_MAX_ELEMENTS returns MGR_ERR_TOO_LARGE.
 * Every call on a stream that is not capturing looks up the array's device
 * address in the current context (so a cudaDeviceReset between calls is
 * harmless); a call on a capturing stream reuses the address that the last
 * call outside capture found on this device, and returns MGR_ERR_STATE when
 * there was none: make the first call on each device before any stream
 * capture, and again after a cudaDeviceReset.  A CUDA error already pending
 * on the calling thread from earlier work is reported as MGR_ERR_CUDA
 * without launching anything and is left in place for the caller.  All
 * calls share the array: calls that overlap on the GPU (on different
 * streams) race; nothing in it needs clearing between calls.  Asynchronous:
 * results are in `stats` once the stream reaches that point. */
mgr_status mgr_convergence_noalloc(const double *pop, const double *prev, const double *pop_tot,
                                   int64_t ncells, int32_t nlev, double pop_prec, double *stats,
                                   void *stream);

#ifdef __cplusplus
}
#endif
#endif
