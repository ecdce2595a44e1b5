/*
 * magritte_oracle.h -- CPU restatement of Magritte's radiation hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA path
 * is compared against and the CPU baseline that is timed beside it.  Only the
 * tests, the smoke check and the CPU-baseline leg of the benchmark load it;
 * the product library never links or calls it.
 *
 * Every function restates one reference function (cited per function in
 * magritte_oracle.c) in plain C, compiled with -ffp-contract=off so that each
 * multiply and add rounds separately, as the reference's scalar (non
 * Grid-SIMD) build does.
 *
 * Parity pins: the oracle is checked against the reference's own unit tests
 * and analytic tests restated as known-answer tests (Doppler shifts of
 * tests/unit/Model/Geometry/test_geometry.cpp:46-59, T L = I of
 * tests/unit/Simulation/Raypair/test_raypair.cpp:83-163, the constant slab of
 * tests/integration/test_0_1D_all_constant.py:240-244, statistical-equilibrium
 * balance of tests/unit/Model/Lines/test_lineProducingSpecies.cpp:157-160).
 * The reference's Eigen dependency is absent here, so Eigen-level results
 * (vector dot-product order, SparseLU pivoting) are restated, not pinned.
 */
#ifndef MAGRITTE_ORACLE_H
#define MAGRITTE_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int32_t ntmp;
    int32_t ncol;
    int32_t ortho_para;        /* 0: 'n', 1: 'o' (ortho H2), 2: 'p' (para H2) */
    int32_t pad_;
    const int64_t *icol;       /* [ncol] upper level */
    const int64_t *jcol;       /* [ncol] lower level */
    const double  *tmp;        /* [ntmp] K */
    const double  *Cd;         /* [ntmp*ncol] m^3/s */
    const double  *Ce;         /* [ntmp*ncol] m^3/s */
    const double  *abundance;  /* [ncells] partner density, m^-3 */
} orc_colpar;

typedef struct {
    int64_t ncells;
    const double  *position;       /* [ncells*3] m */
    const double  *velocity;       /* [ncells*3] fraction of c */
    const int64_t *nbr_offsets;    /* [ncells+1] */
    const int64_t *nbr_list;
    const uint8_t *boundary;       /* [ncells] 1 on boundary cells */
    const int64_t *cell2boundary;  /* [ncells] boundary number, ncells if none */
    int64_t nboundary;
    const int64_t *boundary2cell;  /* [nboundary] */
    const double  *boundary_temperature; /* [nboundary] K */
    int64_t nrays;
    const double  *rays;           /* [nrays*3] */
    const double  *ray_weights;    /* [nrays] */
    const double  *temperature;    /* [ncells] K */
    const double  *vturb2;         /* [ncells] (v_turb/c)^2 */
    /* one line-producing species */
    int32_t nlev;
    int32_t nrad;
    const double  *energy;         /* [nlev] J */
    const double  *weight;         /* [nlev] */
    const int64_t *irad;           /* [nrad] upper */
    const int64_t *jrad;           /* [nrad] lower */
    const double  *A;              /* [nrad] */
    const double  *Bs;             /* [nrad] */
    const double  *Ba;             /* [nrad] */
    const double  *frequency;      /* [nrad] Hz */
    double inverse_mass;           /* 1/amu */
    const double  *population_tot; /* [ncells] m^-3 */
    int32_t nquads;
    int32_t ncolpar;
    const double  *quad_roots;     /* [nquads] */
    const double  *quad_weights;   /* [nquads] */
    const orc_colpar *colpar;      /* [ncolpar] */
    double pop_prec;
    double max_width_fraction;
} orc_model;

/* Mutable state.  Every array is owned by the caller. */
typedef struct {
    int64_t nfreqs;                /* nrad*nquads */
    double  *nu;                   /* [ncells*nfreqs] sorted per cell */
    int64_t *nr_line;              /* [ncells*nrad*nquads] sorted bin of (k,z) */
    int64_t *corr_k;               /* [nfreqs] global maps (indexed by bin) */
    int64_t *corr_z;               /* [nfreqs] */
    uint8_t *appears;              /* [nfreqs] */
    double  *I_bdy;                /* [nboundary*nfreqs] */
    double  *pop;                  /* [ncells*nlev] */
    double  *prev1, *prev2, *prev3;
    double  *emissivity;           /* [ncells*nrad] */
    double  *opacity;              /* [ncells*nrad] */
    double  *J;                    /* [ncells*nfreqs] */
    double  *Ls;                   /* [ncells*nrad] local ALO element */
    double  *Jlin, *Jeff, *Jdif;   /* [ncells*nrad] */
    double  fnc;                   /* fraction_not_converged */
    double  rcm;                   /* relative_change_mean */
    double  max_rel;               /* max relative change over n > 1e-10 n_tot */
    int64_t trace_errors;
    int64_t lu_errors;
    /* non-local ALO (parameters.n_off_diag = M >= 2; 0 or 1 leaves Loff
     * unused): for origin o, line k, ray pair r, side (0 the front trace, 1
     * the back trace) and distance d = 1..M-1 from the origin, the element
     * Loff[(((o*nrad + k)*npairs + r)*2 + side)*(M-1) + d-1] of the cell
     * Loff_nr[((o*npairs + r)*2 + side)*(M-1) + d-1] (-1: no such point) */
    int64_t n_off_diag;
    double  *Loff;
    int64_t *Loff_nr;
} orc_state;

/* Constants, exposed so tests can reuse the reference's values. */
double orc_const(int which);

/* geometry */
double  orc_dshift_max(const orc_model *m, int64_t o);
double  orc_doppler_shift(const orc_model *m, int64_t origin, int64_t ray,
                          int64_t current, int rest_frame, const int64_t *antipod);
int64_t orc_npoints_on_ray(const orc_model *m, int64_t o, int64_t r, double dshift_max,
                           int64_t *err);
int64_t orc_trace_ray(const orc_model *m, int64_t o, int64_t r, double dshift_max,
                      int64_t cap, int64_t *cell, double *shift, double *dZ, int64_t *err);

/* spectral discretisation + boundary intensities + LTE */
int orc_spectral_discretisation(const orc_model *m, orc_state *s);
int orc_boundary_intensities(const orc_model *m, orc_state *s);
void orc_lte(const orc_model *m, orc_state *s);
void orc_set_emissivity_opacity(const orc_model *m, orc_state *s);

/* formal solve over all ray pairs (or a subset of origins / pairs) */
int orc_compute_radiation_field_scattering(const orc_model *m, orc_state *s,
                                           const int64_t *antipod, const double *U,
                                           const double *V, double *u_out, double *v_out,
                                           int nthreads);
void orc_calc_U_and_V(const orc_model *m, const orc_state *s, const double *u, const double *v,
                      double *U, double *V);
int orc_image_discretisation(const orc_model *m, orc_state *s, double width);
int orc_compute_image(const orc_model *m, orc_state *s, const int64_t *antipod, int64_t r,
                      double *I_m, double *I_p, int nthreads);
int orc_compute_radiation_field(const orc_model *m, orc_state *s, const int64_t *antipod,
                                const int64_t *origins, int64_t norigins,
                                int64_t npairs, int nthreads);

/* one ray pair: reference elimination + back substitution on given arrays */
void orc_solve_raypair(int64_t n_ar, int64_t ndep, const double *term1, const double *dtau,
                       double I_bdy_0, double I_bdy_n, double *u_origin, double *L_origin);

/* one ray pair, n_off_diag > 0: the diagonal element at the origin and the
 * n_off_diag-1 elements of the origin's row on each side (0 where the pair
 * has no such point) */
void orc_raypair_lambda_row(int64_t n_ar, int64_t ndep, const double *term1, const double *dtau,
                            int64_t n_off_diag, double *diag, double *lower, double *upper);

/* level populations */
void orc_compute_jeff(const orc_model *m, orc_state *s);
int  orc_statistical_equilibrium(const orc_model *m, orc_state *s);
void orc_check_convergence(const orc_model *m, orc_state *s);
void orc_ng_acceleration(const orc_model *m, orc_state *s);
int64_t orc_compute_level_populations(const orc_model *m, orc_state *s, const int64_t *antipod,
                                      int use_ng, int64_t max_iter, double tol_max_rel,
                                      int nthreads, double *iter_max_rel);
/* The same with ng_every normal iterations before each Ng step. */
int64_t orc_compute_level_populations_ng(const orc_model *m, orc_state *s,
                                         const int64_t *antipod, int use_ng, int64_t max_iter,
                                         double tol_max_rel, int nthreads, double *iter_max_rel,
                                         int ng_every);

#ifdef __cplusplus
}
#endif
#endif
