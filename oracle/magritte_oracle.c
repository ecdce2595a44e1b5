/*
 * magritte_oracle.c -- CPU restatement of Magritte's radiation hot path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker and the timed CPU baseline; see
 * magritte_oracle.h).  Reference citations are paths inside the UCL/Magritte
 * source tree.  Compile with -ffp-contract=off.
 */
#include "magritte_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* src/Tools/constants.hpp:25-46, same literals and the same folding order */
#define O_CC        2.99792458E+8
#define O_HH        6.62607004E-34
#define O_KB        1.38064852E-23
#define O_AMU       1.66053904E-27
#define O_T_CMB     2.7254800
#define O_C_SQUARED 8.98755179E+16
#define O_FOUR_PI   (4.0 * M_PI)
#define O_INVERSE_SQRT_PI (0.5 * M_2_SQRTPI)
#define O_TWO_KB_OVER_AMU_C_SQUARED (2.0 * O_KB / (O_AMU * O_C_SQUARED))
#define O_TWO_HH_OVER_CC_SQUARED    (2.0 * O_HH / O_C_SQUARED)
#define O_HH_OVER_KB      (O_HH / O_KB)
#define O_HH_OVER_FOUR_PI (O_HH / O_FOUR_PI)

double orc_const(int which)
{
    switch (which) {
    case 0: return O_CC;
    case 1: return O_HH;
    case 2: return O_KB;
    case 3: return O_AMU;
    case 4: return O_T_CMB;
    case 5: return O_C_SQUARED;
    case 6: return O_TWO_KB_OVER_AMU_C_SQUARED;
    case 7: return O_TWO_HH_OVER_CC_SQUARED;
    case 8: return O_HH_OVER_KB;
    case 9: return O_HH_OVER_FOUR_PI;
    case 10: return O_INVERSE_SQRT_PI;
    default: return NAN;
    }
}

/* ------------------------------------------------------------------ helpers */

/* Eigen's Vector3d::dot as restated here: (x x' + y y') + z z'.  Eigen is
 * not available, so this order defines the oracle (see header). */
static inline double dot3(const double *a, const double *b)
{
    return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2];
}

/* Thermodynamics::profile_width(inverse_mass, p), thermodynamics.tpp:62-69 */
static inline double profile_width(const orc_model *m, int64_t p)
{
    return sqrt(O_TWO_KB_OVER_AMU_C_SQUARED * m->inverse_mass * m->temperature[p]
                + m->vturb2[p]);
}

/* Thermodynamics::profile(width, freq_diff), thermodynamics.tpp:16-29, with
 * vExpMinus(x) = 1/exp(x) (Tools/Parallel/wrap_Grid.hpp:160-163). */
static inline double profile(double width, double freq_diff)
{
    const double inverse_width = 1.0 / width;
    const double sqrtExponent  = inverse_width * freq_diff;
    const double exponent      = sqrtExponent * sqrtExponent;
    return inverse_width * O_INVERSE_SQRT_PI * (1.0 / exp(exponent));
}

/* planck(T, nu), Functions/planck.tpp:15-23 */
static inline double planck(double temperature, double freq)
{
    const double h_over_kbT = O_HH_OVER_KB / temperature;
    return O_TWO_HH_OVER_CC_SQUARED * (freq * freq * freq) / expm1(h_over_kbT * freq);
}

/* Simulation::get_dshift_max, Simulation/simulation.tpp:15-37 (one species) */
double orc_dshift_max(const orc_model *m, int64_t o)
{
    double dshift_max = DBL_MAX;
    const double nd = m->max_width_fraction * profile_width(m, o);
    if (dshift_max > nd) dshift_max = nd;
    return dshift_max;
}

/* ----------------------------------------------------------------- tracer */

/* Geometry::get_doppler_shift<frame>, Model/Geometry/geometry.tpp:433-465 */
double orc_doppler_shift(const orc_model *m, int64_t origin, int64_t ray, int64_t current,
                         int rest_frame, const int64_t *antipod)
{
    if (!rest_frame) {
        const double *vc = m->velocity + 3 * current;
        const double *vo = m->velocity + 3 * origin;
        const double dv[3] = {vc[0] - vo[0], vc[1] - vo[1], vc[2] - vo[2]};
        return 1.0 - dot3(dv, m->rays + 3 * ray);
    }
    int64_t ray_correct = ray;
    if (ray >= m->nrays / 2) ray_correct = antipod[ray];
    return 1.0 - dot3(m->velocity + 3 * current, m->rays + 3 * ray_correct);
}

/* Geometry::get_next_general, Model/Geometry/geometry.tpp:328-421 */
static int64_t get_next_general(const orc_model *m, int64_t origin, const double *ray,
                                int64_t current, double *Z, double *dZ)
{
    double  dmin = DBL_MAX;
    int64_t next = -1;
    const double *po = m->position + 3 * origin;
    for (int64_t k = m->nbr_offsets[current]; k < m->nbr_offsets[current + 1]; k++) {
        const int64_t nb = m->nbr_list[k];
        const double *pn = m->position + 3 * nb;
        const double R[3] = {pn[0] - po[0], pn[1] - po[1], pn[2] - po[2]};
        const double Z_new = dot3(R, ray);
        if (Z_new > *Z) {
            const double distance_from_ray2 = dot3(R, R) - Z_new * Z_new;
            if (distance_from_ray2 < dmin) {
                dmin = distance_from_ray2;
                next = nb;
                *dZ  = Z_new - *Z;
            }
        }
    }
    *Z = *Z + *dZ;
    return next;
}

typedef struct {
    int64_t n, cap;
    int64_t *cell;
    double  *shift, *dZ;
    int grow;           /* 1: realloc when full, 0: fixed capacity */
    int overflow;
} trace_buf;

static int tb_push(trace_buf *t, int64_t cell, double shift, double dZ)
{
    if (t->n >= t->cap) {
        if (!t->grow) { t->overflow = 1; t->n++; return -1; }
        int64_t nc = t->cap ? 2 * t->cap : 256;
        t->cell  = (int64_t *)realloc(t->cell,  (size_t)nc * sizeof(int64_t));
        t->shift = (double  *)realloc(t->shift, (size_t)nc * sizeof(double));
        t->dZ    = (double  *)realloc(t->dZ,    (size_t)nc * sizeof(double));
        t->cap   = nc;
    }
    t->cell[t->n] = cell; t->shift[t->n] = shift; t->dZ[t->n] = dZ;
    t->n++;
    return 0;
}

/* Geometry::set_data, Model/Geometry/geometry.tpp:100-207 */
static int set_data(int64_t crt, int64_t nxt, double shift_crt, double shift_nxt,
                    double dZ_loc, double dshift_max, trace_buf *t)
{
    const double dshift     = shift_nxt - shift_crt;
    const double dshift_abs = fabs(dshift);
    if (dshift_abs > dshift_max) {
        const long   n_interpl      = (long)(dshift_abs / dshift_max + 1);
        const long   half_n_interpl = (long)(0.5 * n_interpl);
        const double dZ_interpl     = dZ_loc / n_interpl;
        const double dshift_interpl = dshift / n_interpl;
        if (n_interpl > 10000 || n_interpl < 0) return -1;
        for (long mm = 1; mm < half_n_interpl; mm++)
            tb_push(t, crt, shift_crt + mm * dshift_interpl, dZ_interpl);
        for (long mm = half_n_interpl; mm <= n_interpl; mm++)
            tb_push(t, nxt, shift_crt + mm * dshift_interpl, dZ_interpl);
    } else {
        tb_push(t, nxt, shift_nxt, dZ_loc);
    }
    return 0;
}

/* Geometry::trace_ray<CoMoving> (rest = 0) or <Rest> (rest = 1),
 * Model/Geometry/geometry.tpp:21-95.
 * err: 1 = no neighbour ahead before a boundary cell (the reference prints
 * "No proper neighbor found" and then reads out of bounds), 2 = more than
 * 10000 interpolation points on one step. */
static void trace_frame(const orc_model *m, int64_t origin, int64_t r, double dshift_max,
                        int rest, const int64_t *antipod, trace_buf *t, int64_t *err)
{
    double Z = 0.0, dZ = 0.0;
    const double *ray = m->rays + 3 * r;
    t->n = 0;
    t->overflow = 0;
    *err = 0;
    int64_t nxt = get_next_general(m, origin, ray, origin, &Z, &dZ);
    if (nxt != -1) {
        int64_t crt = origin;
        double shift_crt = orc_doppler_shift(m, origin, r, crt, rest, antipod);
        double shift_nxt = orc_doppler_shift(m, origin, r, nxt, rest, antipod);
        if (set_data(crt, nxt, shift_crt, shift_nxt, dZ, dshift_max, t)) { *err = 2; return; }
        while (!m->boundary[nxt]) {
            shift_crt = shift_nxt;
            crt = nxt;
            nxt = get_next_general(m, origin, ray, nxt, &Z, &dZ);
            if (nxt < 0) { *err = 1; return; }
            shift_nxt = orc_doppler_shift(m, origin, r, nxt, rest, antipod);
            if (set_data(crt, nxt, shift_crt, shift_nxt, dZ, dshift_max, t)) { *err = 2; return; }
        }
    }
}

static void trace(const orc_model *m, int64_t origin, int64_t r, double dshift_max,
                  trace_buf *t, int64_t *err)
{
    trace_frame(m, origin, r, dshift_max, 0, NULL, t, err);
}

int64_t orc_trace_ray(const orc_model *m, int64_t o, int64_t r, double dshift_max,
                      int64_t cap, int64_t *cell, double *shift, double *dZ, int64_t *err)
{
    trace_buf t = {0, cap, cell, shift, dZ, 0, 0};
    trace(m, o, r, dshift_max, &t, err);
    if (t.overflow && *err == 0) *err = 3;
    return t.n;
}

/* Geometry::get_npoints_on_ray<CoMoving>, geometry.tpp:498-543 */
int64_t orc_npoints_on_ray(const orc_model *m, int64_t o, int64_t r, double dshift_max,
                           int64_t *err)
{
    trace_buf t = {0, 0, NULL, NULL, NULL, 1, 0};
    trace(m, o, r, dshift_max, &t, err);
    free(t.cell); free(t.shift); free(t.dZ);
    return t.n;
}

/* ------------------------------------------------- spectral discretisation */

/* Lines::setup line sort (Model/Lines/lines.cpp:43-87): ascending line
 * frequencies with their original transition numbers. */
static void sorted_lines(const orc_model *m, double *line, int64_t *line_index)
{
    for (int64_t k = 0; k < m->nrad; k++) { line[k] = m->frequency[k]; line_index[k] = k; }
    for (int64_t i = 1; i < m->nrad; i++) {          /* insertion sort, stable */
        double v = line[i]; int64_t ix = line_index[i]; int64_t j = i - 1;
        while (j >= 0 && line[j] > v) { line[j + 1] = line[j]; line_index[j + 1] = line_index[j]; j--; }
        line[j + 1] = v; line_index[j + 1] = ix;
    }
}

/* Simulation::compute_spectral_discretisation, Simulation/sim_spectrum.tpp:13-196.
 * The per-cell grid nu = line + width*root is sorted ascending; the global
 * maps corresponding_{k,z} and appears_in_line_integral are indexed by the
 * UNSORTED bin number, exactly as the reference fills them. */
int orc_spectral_discretisation(const orc_model *m, orc_state *s)
{
    const int64_t nf = (int64_t)m->nrad * m->nquads;
    double  *line  = (double *)malloc(sizeof(double) * m->nrad);
    int64_t *lidx  = (int64_t *)malloc(sizeof(int64_t) * m->nrad);
    sorted_lines(m, line, lidx);
    s->nfreqs = nf;
    int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
    for (int64_t p = 0; p < m->ncells; p++) {
        double  *freqs = s->nu + p * nf;
        int64_t *nmbrs = (int64_t *)malloc(sizeof(int64_t) * nf);
        int64_t *inv   = (int64_t *)malloc(sizeof(int64_t) * nf);
        int64_t index1 = 0;
        for (int64_t k = 0; k < m->nrad; k++) {
            const double freqs_line = line[k];
            const double width = freqs_line * profile_width(m, p);
            for (int64_t z = 0; z < m->nquads; z++) {
                freqs[index1] = freqs_line + width * m->quad_roots[z];
                nmbrs[index1] = index1;
                index1++;
            }
        }
        for (int64_t i = 1; i < nf; i++) {              /* ascending, stable */
            double v = freqs[i]; int64_t ix = nmbrs[i]; int64_t j = i - 1;
            while (j >= 0 && freqs[j] > v) { freqs[j + 1] = freqs[j]; nmbrs[j + 1] = nmbrs[j]; j--; }
            freqs[j + 1] = v; nmbrs[j + 1] = ix;
        }
        for (int64_t fl = 0; fl < nf; fl++) {
            inv[nmbrs[fl]] = fl;
            if (nmbrs[fl] != fl) bad = 1;
        }
        for (int64_t i2 = 0; i2 < nf; i2++) s->nr_line[p * nf + i2] = inv[i2];
        free(nmbrs); free(inv);
    }
    for (int64_t i2 = 0; i2 < nf; i2++) {
        s->appears[i2] = 1;
        s->corr_k[i2]  = i2 / m->nquads;
        s->corr_z[i2]  = i2 % m->nquads;
    }
    free(line); free(lidx);
    return bad;   /* 1 when some cell's sort was not the identity */
}

/* Simulation::compute_boundary_intensities, Simulation/sim_radiation.tpp:17-48.
 * Every ray sees the same boundary values, so one [nboundary][nfreqs] table
 * stands for I_bdy[R][b][f]. */
int orc_boundary_intensities(const orc_model *m, orc_state *s)
{
    const int64_t nf = s->nfreqs;
#pragma omp parallel for schedule(static)
    for (int64_t b = 0; b < m->nboundary; b++) {
        const int64_t p = m->boundary2cell[b];
        for (int64_t f = 0; f < nf; f++)
            s->I_bdy[b * nf + f] = planck(m->boundary_temperature[b], s->nu[p * nf + f]);
    }
    return 0;
}

/* LineProducingSpecies::update_using_LTE, lineProducingSpecies.tpp:82-115 */
void orc_lte(const orc_model *m, orc_state *s)
{
    const int64_t nl = m->nlev;
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < m->ncells; p++) {
        double partition_function = 0.0;
        for (int64_t i = 0; i < nl; i++) {
            s->pop[p * nl + i] = m->weight[i] * exp(-m->energy[i] / (O_KB * m->temperature[p]));
            partition_function += s->pop[p * nl + i];
        }
        for (int64_t i = 0; i < nl; i++)
            s->pop[p * nl + i] *= m->population_tot[p] / partition_function;
    }
}

/* Lines::set_emissivity_and_opacity, Model/Lines/lines.tpp:44-60, with
 * get_emissivity / get_opacity, lineProducingSpecies.tpp:41-70. */
void orc_set_emissivity_opacity(const orc_model *m, orc_state *s)
{
    const int64_t nl = m->nlev, nr = m->nrad;
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < m->ncells; p++) {
        for (int64_t k = 0; k < nr; k++) {
            const double ni = s->pop[p * nl + m->irad[k]];
            const double nj = s->pop[p * nl + m->jrad[k]];
            s->emissivity[p * nr + k] = O_HH_OVER_FOUR_PI * m->A[k] * ni;
            s->opacity[p * nr + k]    = O_HH_OVER_FOUR_PI * (nj * m->Ba[k] - ni * m->Bs[k]);
        }
    }
}

/* ----------------------------------------------------------- formal solve */

typedef struct {
    int64_t cap;
    double *term1, *dtau, *chi, *frs, *A, *C, *F, *G, *Su;
    double *inv_A, *inv_C, *inv1pF, *GoG, *inv1pG, *Ld;
    int64_t *nrs, *notch;
} raypair_buf;

static void rp_ensure(raypair_buf *b, int64_t n)
{
    if (n <= b->cap) return;
    int64_t c = n + 64;
#define RP_GROW(x, T) b->x = (T *)realloc(b->x, sizeof(T) * (size_t)c)
    RP_GROW(term1, double); RP_GROW(dtau, double); RP_GROW(chi, double); RP_GROW(frs, double);
    RP_GROW(A, double); RP_GROW(C, double); RP_GROW(F, double); RP_GROW(G, double);
    RP_GROW(Su, double); RP_GROW(inv_A, double); RP_GROW(inv_C, double);
    RP_GROW(inv1pF, double); RP_GROW(GoG, double); RP_GROW(inv1pG, double); RP_GROW(Ld, double);
    RP_GROW(nrs, int64_t); RP_GROW(notch, int64_t);
#undef RP_GROW
    b->cap = c;
}

static void rp_free(raypair_buf *b)
{
    free(b->term1); free(b->dtau); free(b->chi); free(b->frs); free(b->A); free(b->C);
    free(b->F); free(b->G); free(b->Su); free(b->inv_A); free(b->inv_C); free(b->inv1pF);
    free(b->GoG); free(b->inv1pG); free(b->Ld); free(b->nrs); free(b->notch);
}

/* RayPair::solve, Simulation/Raypair/raypair_solver.tpp:200-334 (the
 * n_off_diag == 0 branch): Rybicki-Hummer elimination from `first` to
 * `last`, back substitution down to the origin n_ar, diagonal ALO there. */
static void solve_raypair(raypair_buf *b, int64_t first, int64_t last, int64_t n_ar,
                          double I_bdy_0, double I_bdy_n, double *u, double *L)
{
    double *A = b->A, *C = b->C, *F = b->F, *G = b->G, *Su = b->Su, *dtau = b->dtau;
    double *inv_A = b->inv_A, *inv_C = b->inv_C, *inv1pF = b->inv1pF, *GoG = b->GoG;
    const double *term1 = b->term1;

    const double inverse_dtau0 = 1.0 / dtau[first];
    const double inverse_dtaud = 1.0 / dtau[last - 1];
    C[first] = 2.0 * inverse_dtau0 * inverse_dtau0;
    const double B0_min_C0 = 1.0 + 2.0 * inverse_dtau0;
    const double B0 = B0_min_C0 + C[first];
    const double inverse_B0 = 1.0 / B0;
    Su[first] = term1[first] + 2.0 * I_bdy_0 * inverse_dtau0;
    for (int64_t n = first + 1; n < last; n++) {
        inv_A[n] = 0.5 * (dtau[n - 1] + dtau[n]) * dtau[n - 1];
        A[n] = 1.0 / inv_A[n];
        inv_C[n] = 0.5 * (dtau[n - 1] + dtau[n]) * dtau[n];
        C[n] = 1.0 / inv_C[n];
        Su[n] = term1[n];
    }
    A[last] = 2.0 * inverse_dtaud * inverse_dtaud;
    const double Bd_min_Ad = 1.0 + 2.0 * inverse_dtaud;
    const double Bd = Bd_min_Ad + A[last];
    Su[last] = term1[last] + 2.0 * I_bdy_n * inverse_dtaud;

    Su[first] = Su[first] * inverse_B0;
    F[first] = 0.5 * B0_min_C0 * dtau[first] * dtau[first];
    inv1pF[first] = 1.0 / (1.0 + F[first]);
    for (int64_t n = first + 1; n < last; n++) {
        F[n] = (1.0 + A[n] * F[n - 1] * inv1pF[n - 1]) * inv_C[n];
        inv1pF[n] = 1.0 / (1.0 + F[n]);
        Su[n] = (Su[n] + A[n] * Su[n - 1]) * inv1pF[n] * inv_C[n];
    }
    const double denominator = 1.0 / (Bd_min_Ad + Bd * F[last - 1]);
    Su[last] = (Su[last] + A[last] * Su[last - 1]) * (1.0 + F[last - 1]) * denominator;

    if (n_ar < last) {
        G[last] = 0.5 * Bd_min_Ad * dtau[last - 1] * dtau[last - 1];
        GoG[last] = G[last] / (1.0 + G[last]);
        for (int64_t n = last - 1; n > n_ar; n--) {
            Su[n] = Su[n] + Su[n + 1] * inv1pF[n];
            G[n] = (1.0 + C[n] * GoG[n + 1]) * inv_A[n];
            GoG[n] = G[n] / (1.0 + G[n]);
        }
        Su[n_ar] = Su[n_ar] + Su[n_ar + 1] * inv1pF[n_ar];
        *u = Su[n_ar];
        *L = inv_C[n_ar] / (F[n_ar] + GoG[n_ar + 1]);
    } else {
        *u = Su[last];
        *L = (1.0 + F[last - 1]) / (Bd_min_Ad + Bd * F[last - 1]);
    }
}

/* RayPair::solve with n_off_diag > 0 (raypair_solver.tpp:336-388): the
 * same elimination, back substitution over the whole pair, and the diagonal
 * of the ray pair's Lambda operator at every point (Ld) with the factors
 * 1/(1+F) and 1/(1+G) its off-diagonal elements are built from. */
static void solve_raypair_nonlocal(raypair_buf *b, int64_t first, int64_t last, int64_t n_ar,
                                   double I_bdy_0, double I_bdy_n, double *u, double *L)
{
    double *A = b->A, *C = b->C, *F = b->F, *G = b->G, *Su = b->Su, *dtau = b->dtau;
    double *inv_A = b->inv_A, *inv_C = b->inv_C, *inv1pF = b->inv1pF, *inv1pG = b->inv1pG;
    double *Ld = b->Ld;
    const double *term1 = b->term1;

    const double inverse_dtau0 = 1.0 / dtau[first];
    const double inverse_dtaud = 1.0 / dtau[last - 1];
    C[first] = 2.0 * inverse_dtau0 * inverse_dtau0;
    const double B0_min_C0 = 1.0 + 2.0 * inverse_dtau0;
    const double B0 = B0_min_C0 + C[first];
    const double inverse_B0 = 1.0 / B0;
    Su[first] = term1[first] + 2.0 * I_bdy_0 * inverse_dtau0;
    for (int64_t n = first + 1; n < last; n++) {
        inv_A[n] = 0.5 * (dtau[n - 1] + dtau[n]) * dtau[n - 1];
        A[n] = 1.0 / inv_A[n];
        inv_C[n] = 0.5 * (dtau[n - 1] + dtau[n]) * dtau[n];
        C[n] = 1.0 / inv_C[n];
        Su[n] = term1[n];
    }
    A[last] = 2.0 * inverse_dtaud * inverse_dtaud;
    const double Bd_min_Ad = 1.0 + 2.0 * inverse_dtaud;
    const double Bd = Bd_min_Ad + A[last];
    Su[last] = term1[last] + 2.0 * I_bdy_n * inverse_dtaud;

    Su[first] = Su[first] * inverse_B0;
    F[first] = 0.5 * B0_min_C0 * dtau[first] * dtau[first];
    inv1pF[first] = 1.0 / (1.0 + F[first]);
    for (int64_t n = first + 1; n < last; n++) {
        F[n] = (1.0 + A[n] * F[n - 1] * inv1pF[n - 1]) * inv_C[n];
        inv1pF[n] = 1.0 / (1.0 + F[n]);
        Su[n] = (Su[n] + A[n] * Su[n - 1]) * inv1pF[n] * inv_C[n];
    }
    const double denominator = 1.0 / (Bd_min_Ad + Bd * F[last - 1]);
    Su[last] = (Su[last] + A[last] * Su[last - 1]) * (1.0 + F[last - 1]) * denominator;

    G[last] = 0.5 * Bd_min_Ad * dtau[last - 1] * dtau[last - 1];
    inv1pG[last] = 1.0 / (1.0 + G[last]);
    for (int64_t n = last - 1; n > first; n--) {
        Su[n] = Su[n] + Su[n + 1] * inv1pF[n];
        G[n] = (1.0 + C[n] * G[n + 1] * inv1pG[n + 1]) * inv_A[n];
        inv1pG[n] = 1.0 / (1.0 + G[n]);
    }
    Su[first] = Su[first] + Su[first + 1] * inv1pF[first];

    Ld[last] = (1.0 + F[last - 1]) / (Bd_min_Ad + Bd * F[last - 1]);
    for (int64_t n = last - 1; n >= first + 1; n--)
        Ld[n] = inv_C[n] / (F[n] + G[n + 1] * inv1pG[n + 1]);
    Ld[first] = (1.0 + G[first + 1]) / (B0_min_C0 + B0 * G[first + 1]);
    *u = Su[n_ar];
    *L = Ld[n_ar];
}

/* Element (n_ar, n_ar - d) and (n_ar, n_ar + d) of the ray pair's Lambda
 * operator from the factors of solve_raypair_nonlocal, multiplied in the
 * order of the reference's recursions (raypair_solver.tpp:372-388):
 * L_lower[d-1][n_ar-d] = Ld[n_ar-d] * 1/(1+G[n_ar-d+1]) * ... * 1/(1+G[n_ar]),
 * L_upper[d-1][n_ar]   = Ld[n_ar+d] * 1/(1+F[n_ar+d-1]) * ... * 1/(1+F[n_ar]).
 * These are the origin's row.  RayPair::update_Lambda
 * (raypair_lambda.tpp:129-145) reads L_lower[d][n_ar-d] and
 * L_upper[d][n_ar+d] instead, the elements (n_ar+1, n_ar-d) and
 * (n_ar+d, n_ar+2d+1), and at the ends of the pair (n_ar = last, or
 * n_ar + 2d = last) entries its recursions did not write for this pair. */
static inline double lambda_lower(const raypair_buf *b, int64_t n_ar, int64_t d)
{
    double lam = b->Ld[n_ar - d];
    for (int64_t q = n_ar - d + 1; q <= n_ar; q++) lam *= b->inv1pG[q];
    return lam;
}

static inline double lambda_upper(const raypair_buf *b, int64_t n_ar, int64_t d)
{
    double lam = b->Ld[n_ar + d];
    for (int64_t q = n_ar + d - 1; q >= n_ar; q--) lam *= b->inv1pF[q];
    return lam;
}

void orc_solve_raypair(int64_t n_ar, int64_t ndep, const double *term1, const double *dtau,
                       double I_bdy_0, double I_bdy_n, double *u_origin, double *L_origin)
{
    raypair_buf b;
    memset(&b, 0, sizeof(b));
    rp_ensure(&b, ndep + 1);
    memcpy(b.term1, term1, sizeof(double) * (size_t)ndep);
    memcpy(b.dtau, dtau, sizeof(double) * (size_t)(ndep - 1));
    solve_raypair(&b, 0, ndep - 1, n_ar, I_bdy_0, I_bdy_n, u_origin, L_origin);
    rp_free(&b);
}

void orc_raypair_lambda_row(int64_t n_ar, int64_t ndep, const double *term1, const double *dtau,
                            int64_t n_off_diag, double *diag, double *lower, double *upper)
{
    raypair_buf b;
    memset(&b, 0, sizeof(b));
    rp_ensure(&b, ndep + 1);
    memcpy(b.term1, term1, sizeof(double) * (size_t)ndep);
    memcpy(b.dtau, dtau, sizeof(double) * (size_t)(ndep - 1));
    double u;
    solve_raypair_nonlocal(&b, 0, ndep - 1, n_ar, 0.0, 0.0, &u, diag);
    for (int64_t d = 1; d < n_off_diag; d++) {
        lower[d - 1] = n_ar - d >= 0 ? lambda_lower(&b, n_ar, d) : 0.0;
        upper[d - 1] = n_ar + d <= ndep - 1 ? lambda_upper(&b, n_ar, d) : 0.0;
    }
    rp_free(&b);
}

typedef struct {
    double  *line;
    int64_t *line_index;
} line_table;

/* Simulation::get_eta_and_chi, Simulation/simulation.tpp:385-481, with the
 * notch carried by the caller across frequency bins. */
static inline void get_eta_and_chi(const orc_model *m, const orc_state *s, const line_table *lt,
                                   double freq_scaled, int64_t p, int64_t *lnotch,
                                   double *eta, double *chi)
{
    const int64_t nlines = m->nrad;
    const double pw = profile_width(m, p);
    *eta = 0.0;
    *chi = 1.0E-26;
    const double lower = -11.0, upper = +11.0;
    double freq_diff = freq_scaled - lt->line[*lnotch];
    double width = lt->line[*lnotch] * pw;
    while (freq_diff > upper * width) {
        if (*lnotch >= nlines - 1) break;
        (*lnotch)++;
        freq_diff = freq_scaled - lt->line[*lnotch];
        width = lt->line[*lnotch] * pw;
    }
    int64_t lindex = *lnotch;
    while (freq_diff >= lower * width) {
        const double line_profile = profile(width, freq_diff);
        const int64_t ind = lt->line_index[lindex] + p * nlines;
        *eta += s->emissivity[ind] * freq_scaled * line_profile;
        *chi += s->opacity[ind] * freq_scaled * line_profile;
        if (lindex >= nlines - 1) break;
        lindex++;
        freq_diff = freq_scaled - lt->line[lindex];
        width = lt->line[lindex] * pw;
    }
}

/* search_with_notch, Functions/interpolation.tpp (scalar build) */
static inline void search_with_notch(const double *vec, int64_t n, int64_t *notch, double value)
{
    while (*notch < n) {
        if (value <= vec[*notch]) return;
        (*notch)++;
    }
    *notch = n - 1;
}

/* Radiation::rescale_I_bdy (scalar build), Model/Radiation/radiation.tpp:341-373 */
static inline double rescale_I_bdy(const orc_state *s, double freq_scaled, int64_t p, int64_t b)
{
    const int64_t nf = s->nfreqs;
    int64_t notch = 0;
    search_with_notch(s->nu + p * nf, nf, &notch, freq_scaled);
    if (notch == 0 || notch == nf - 1) return s->I_bdy[b * nf + notch];
    const double nu1 = s->nu[p * nf + notch];
    const double nu2 = s->nu[p * nf + notch - 1];
    const double I1 = s->I_bdy[b * nf + notch];
    const double I2 = s->I_bdy[b * nf + notch - 1];
    return (I2 - I1) / (nu2 - nu1) * (freq_scaled - nu1) + I1;
}

/* Simulation::setup (simulation.tpp:185-353) for bin f of origin o: the
 * front trace's points (far end first), the origin, the back trace's
 * points; term1 = eta/chi, dtau = (chi_n + chi_{n-1}) dZ / 2, the boundary
 * intensities at both far ends (Radiation::rescale_I_bdy).  The origin is
 * evaluated at its own grid frequency nu[o][f], every traced point at
 * shift * nu[o][f].  Notches are carried per point across bins. */
static void setup_pair(const orc_model *m, orc_state *s, const line_table *lt, int64_t o,
                       int64_t f, const trace_buf *front, const trace_buf *back,
                       raypair_buf *rb, int64_t *lnotch_at_origin, int64_t *first_out,
                       int64_t *last_out, double *I0_out, double *In_out)
{
    const int64_t nf = s->nfreqs;
    const int64_t n_ar = front->n, n_r = back->n;
    double eta, chi, I_bdy_0, I_bdy_n;
    int64_t first = 0, last = n_ar;
    double freq_scaled = s->nu[o * nf + f];
    int64_t index = n_ar;
    get_eta_and_chi(m, s, lt, freq_scaled, o, lnotch_at_origin, &eta, &chi);
    rb->term1[index] = eta / chi;
    rb->chi[index] = chi; rb->nrs[index] = o; rb->frs[index] = freq_scaled;
    double chi_prev = chi;
    const double chi_o = chi;
    if (n_ar > 0) {
        index = n_ar - 1;
        for (int64_t j = 0; j < n_ar; j++) {
            freq_scaled = front->shift[j] * s->nu[o * nf + f];
            get_eta_and_chi(m, s, lt, freq_scaled, front->cell[j], &rb->notch[j], &eta, &chi);
            rb->term1[index] = eta / chi;
            rb->dtau[index] = 0.5 * (chi + chi_prev) * front->dZ[j];
            rb->chi[index] = chi; rb->nrs[index] = front->cell[j]; rb->frs[index] = freq_scaled;
            chi_prev = chi;
            index--;
        }
        const int64_t cellNr = front->cell[n_ar - 1];
        I_bdy_0 = rescale_I_bdy(s, freq_scaled, cellNr, m->cell2boundary[cellNr]);
        first = index + 1;
        chi_prev = chi_o;
    } else {
        I_bdy_0 = s->I_bdy[m->cell2boundary[o] * nf + f];
    }
    if (n_r > 0) {
        index = n_ar + 1;
        for (int64_t j = 0; j < n_r; j++) {
            freq_scaled = back->shift[j] * s->nu[o * nf + f];
            get_eta_and_chi(m, s, lt, freq_scaled, back->cell[j], &rb->notch[n_ar + j], &eta, &chi);
            rb->term1[index] = eta / chi;
            rb->dtau[index - 1] = 0.5 * (chi + chi_prev) * back->dZ[j];
            rb->chi[index] = chi; rb->nrs[index] = back->cell[j]; rb->frs[index] = freq_scaled;
            chi_prev = chi;
            index++;
        }
        const int64_t cellNr = back->cell[n_r - 1];
        I_bdy_n = rescale_I_bdy(s, freq_scaled, cellNr, m->cell2boundary[cellNr]);
        last = index - 1;
    } else {
        I_bdy_n = s->I_bdy[m->cell2boundary[o] * nf + f];
    }
    *first_out = first;
    *last_out = last;
    *I0_out = I_bdy_0;
    *In_out = I_bdy_n;
}

/* One origin, one ray pair: Simulation::setup (simulation.tpp:185-353),
 * RayPair::solve, RayPair::update_Lambda (raypair_lambda.tpp:94-149) and the
 * J update (sim_radiation.tpp:150-264) for every frequency bin. */
static void solve_origin_pair(const orc_model *m, orc_state *s, const line_table *lt,
                              int64_t o, int64_t r, int64_t ar, trace_buf *tr, trace_buf *ta,
                              raypair_buf *rb, int64_t *errs)
{
    const int64_t nf = s->nfreqs;
    const double weight_ang = m->ray_weights[r];
    const double dshift_max = orc_dshift_max(m, o);
    int64_t e1 = 0, e2 = 0;
    trace(m, o, r, dshift_max, tr, &e1);
    trace(m, o, ar, dshift_max, ta, &e2);
    if (e1 || e2) { (*errs)++; return; }
    /* the longer trace goes in front (setup's "rayData_ar" argument) */
    const trace_buf *front = (tr->n > ta->n) ? tr : ta;
    const trace_buf *back  = (tr->n > ta->n) ? ta : tr;
    const int64_t n_ar = front->n, n_r = back->n;
    const int64_t ndep = n_ar + n_r + 1;
    if (ndep > 1) {
        rp_ensure(rb, ndep + 1);
        int64_t lnotch_at_origin = 0;                      /* RayPair::initialize */
        for (int64_t i = 0; i < ndep; i++) rb->notch[i] = 0;  /* ProjectedCellData.lnotch */
        if (s->n_off_diag > 1) {
            const int64_t M1 = s->n_off_diag - 1, np = m->nrays / 2;
            for (int64_t d = 1; d <= M1; d++) {
                s->Loff_nr[((o * np + r) * 2 + 0) * M1 + d - 1] = d <= n_ar ? front->cell[d - 1] : -1;
                s->Loff_nr[((o * np + r) * 2 + 1) * M1 + d - 1] = d <= n_r ? back->cell[d - 1] : -1;
            }
        }
        for (int64_t f = 0; f < nf; f++) {
            double I_bdy_0, I_bdy_n;
            int64_t first, last;
            setup_pair(m, s, lt, o, f, front, back, rb, &lnotch_at_origin, &first, &last,
                       &I_bdy_0, &I_bdy_n);
            double u, Ld;
            if (s->n_off_diag > 0)
                solve_raypair_nonlocal(rb, first, last, n_ar, I_bdy_0, I_bdy_n, &u, &Ld);
            else
                solve_raypair(rb, first, last, n_ar, I_bdy_0, I_bdy_n, &u, &Ld);
            if (s->appears[f]) {
                const int64_t k = s->corr_k[f], z = s->corr_z[f];
                const double freq_line = m->frequency[k];
                const double weight = m->quad_weights[z] * 2.0 * weight_ang;
                const double factor = m->A[k] * weight;
                const double prof = profile(freq_line * profile_width(m, rb->nrs[n_ar]),
                                            rb->frs[n_ar] - freq_line);
                const double L = factor * (rb->frs[n_ar] * prof * Ld / rb->chi[n_ar]);
                s->Ls[o * m->nrad + k] += L;
                /* off-diagonal elements (raypair_lambda.tpp:129-145 with the
                 * origin's row, see lambda_lower) */
                const int64_t M1 = s->n_off_diag - 1, np = m->nrays / 2;
                for (int64_t d = 1; d <= M1; d++) {
                    for (int side = 0; side < 2; side++) {
                        const int64_t j = side == 0 ? n_ar - d : n_ar + d;
                        if (j < first || j > last) continue;
                        const double lam = side == 0 ? lambda_lower(rb, n_ar, d)
                                                     : lambda_upper(rb, n_ar, d);
                        const double pj = profile(freq_line * profile_width(m, rb->nrs[j]),
                                                  rb->frs[j] - freq_line);
                        const double Lj = factor * (rb->frs[j] * pj * lam / rb->chi[j]);
                        s->Loff[(((o * m->nrad + k) * np + r) * 2 + side) * M1 + d - 1] += Lj;
                    }
                }
            }
            s->J[o * nf + f] += 2.0 * weight_ang * u;
        }
    } else {
        const int64_t b = m->cell2boundary[o];
        for (int64_t f = 0; f < nf; f++) {
            const double u = 0.5 * (s->I_bdy[b * nf + f] + s->I_bdy[b * nf + f]);
            s->J[o * nf + f] += 2.0 * weight_ang * u;
        }
        if (s->n_off_diag > 1) {
            const int64_t M1 = s->n_off_diag - 1, np = m->nrays / 2;
            for (int64_t i = 0; i < 2 * M1; i++) s->Loff_nr[(o * np + r) * 2 * M1 + i] = -1;
        }
    }
}

/* Simulation::compute_radiation_field, Simulation/sim_radiation.tpp:56-338.
 * origins == NULL means every cell; npairs <= 0 means nrays/2.  J and Ls
 * are cleared for the processed origins only. */
int orc_compute_radiation_field(const orc_model *m, orc_state *s, const int64_t *antipod,
                                const int64_t *origins, int64_t norigins,
                                int64_t npairs, int nthreads)
{
    const int64_t nf = s->nfreqs;
    const int64_t no = origins ? norigins : m->ncells;
    const int64_t np = (npairs > 0 && npairs < m->nrays / 2) ? npairs : m->nrays / 2;
    line_table lt;
    lt.line = (double *)malloc(sizeof(double) * m->nrad);
    lt.line_index = (int64_t *)malloc(sizeof(int64_t) * m->nrad);
    sorted_lines(m, lt.line, lt.line_index);
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    for (int64_t i = 0; i < no; i++) {
        const int64_t o = origins ? origins[i] : i;
        memset(s->J + o * nf, 0, sizeof(double) * (size_t)nf);
        memset(s->Ls + o * m->nrad, 0, sizeof(double) * (size_t)m->nrad);
        if (s->n_off_diag > 1) {
            const int64_t per = m->nrad * (m->nrays / 2) * 2 * (s->n_off_diag - 1);
            memset(s->Loff + o * per, 0, sizeof(double) * (size_t)per);
        }
    }
    int64_t errs = 0;
    for (int64_t r = 0; r < np; r++) {
        const int64_t ar = antipod[r];
#pragma omp parallel reduction(+ : errs)
        {
            trace_buf tr = {0, 0, NULL, NULL, NULL, 1, 0};
            trace_buf ta = {0, 0, NULL, NULL, NULL, 1, 0};
            raypair_buf rb;
            memset(&rb, 0, sizeof(rb));
#pragma omp for schedule(static, 1)
            for (int64_t i = 0; i < no; i++) {
                const int64_t o = origins ? origins[i] : i;
                solve_origin_pair(m, s, &lt, o, r, ar, &tr, &ta, &rb, &errs);
            }
            free(tr.cell); free(tr.shift); free(tr.dZ);
            free(ta.cell); free(ta.shift); free(ta.dZ);
            rp_free(&rb);
        }
    }
    s->trace_errors = errs;
    free(lt.line); free(lt.line_index);
    return errs ? 1 : 0;
}

/* --------------------------------------------------------------- scattering */

/* Radiation::rescale_U_and_V (scalar build, Model/Radiation/radiation.tpp:232-262):
 * U and V of ray pair R on cell p's grid, interpolated linearly at freq. */
static inline void rescale_U_and_V(const orc_state *s, const double *U, const double *V,
                                   int64_t ncells, double freq_scaled, int64_t R, int64_t p,
                                   double *Us, double *Vs)
{
    const int64_t nf = s->nfreqs;
    const double *Ur = U + R * ncells * nf + p * nf;
    const double *Vr = V + R * ncells * nf + p * nf;
    int64_t notch = 0;
    search_with_notch(s->nu + p * nf, nf, &notch, freq_scaled);
    if (notch == 0 || notch == nf - 1) { *Us = Ur[notch]; *Vs = Vr[notch]; return; }
    const double nu1 = s->nu[p * nf + notch], nu2 = s->nu[p * nf + notch - 1];
    *Us = (Ur[notch - 1] - Ur[notch]) / (nu2 - nu1) * (freq_scaled - nu1) + Ur[notch];
    *Vs = (Vr[notch - 1] - Vr[notch]) / (nu2 - nu1) * (freq_scaled - nu1) + Vr[notch];
}

/* Simulation::setup_using_scattering (Simulation/simulation.tpp:51-171) for
 * bin f: as setup, with RayPair::set_term1_and_term2 (raypair.tpp:86-100)
 * term1 = (U + eta)/chi and term2 = V/chi (into term2[]); U and V at the
 * origin are its own bin's, elsewhere interpolated (rescale_U_and_V). */
static void setup_scattering(const orc_model *m, orc_state *s, const line_table *lt, int64_t o,
                             int64_t f, int64_t R, const double *U, const double *V,
                             const trace_buf *front, const trace_buf *back, raypair_buf *rb,
                             double *term2, int64_t *lnotch_at_origin, double *I0_out,
                             double *In_out)
{
    const int64_t nf = s->nfreqs, N = m->ncells;
    const int64_t n_ar = front->n, n_r = back->n;
    double eta, chi, Us, Vs;
    double freq_scaled = s->nu[o * nf + f];
    int64_t index = n_ar;
    Us = U[R * N * nf + o * nf + f];
    Vs = V[R * N * nf + o * nf + f];
    get_eta_and_chi(m, s, lt, freq_scaled, o, lnotch_at_origin, &eta, &chi);
    double inverse_chi = 1.0 / chi;
    rb->term1[index] = (Us + eta) * inverse_chi;
    term2[index] = Vs * inverse_chi;
    rb->chi[index] = chi; rb->nrs[index] = o; rb->frs[index] = freq_scaled;
    double chi_prev = chi;
    const double chi_o = chi;
    if (n_ar > 0) {
        index = n_ar - 1;
        for (int64_t j = 0; j < n_ar; j++) {
            freq_scaled = front->shift[j] * s->nu[o * nf + f];
            rescale_U_and_V(s, U, V, N, freq_scaled, R, front->cell[j], &Us, &Vs);
            get_eta_and_chi(m, s, lt, freq_scaled, front->cell[j], &rb->notch[j], &eta, &chi);
            inverse_chi = 1.0 / chi;
            rb->term1[index] = (Us + eta) * inverse_chi;
            term2[index] = Vs * inverse_chi;
            rb->dtau[index] = 0.5 * (chi + chi_prev) * front->dZ[j];
            rb->chi[index] = chi; rb->nrs[index] = front->cell[j]; rb->frs[index] = freq_scaled;
            chi_prev = chi;
            index--;
        }
        const int64_t cellNr = front->cell[n_ar - 1];
        *I0_out = rescale_I_bdy(s, freq_scaled, cellNr, m->cell2boundary[cellNr]);
        chi_prev = chi_o;
    } else {
        *I0_out = s->I_bdy[m->cell2boundary[o] * nf + f];
    }
    if (n_r > 0) {
        index = n_ar + 1;
        for (int64_t j = 0; j < n_r; j++) {
            freq_scaled = back->shift[j] * s->nu[o * nf + f];
            rescale_U_and_V(s, U, V, N, freq_scaled, R, back->cell[j], &Us, &Vs);
            get_eta_and_chi(m, s, lt, freq_scaled, back->cell[j], &rb->notch[n_ar + j], &eta, &chi);
            inverse_chi = 1.0 / chi;
            rb->term1[index] = (Us + eta) * inverse_chi;
            term2[index] = Vs * inverse_chi;
            rb->dtau[index - 1] = 0.5 * (chi + chi_prev) * back->dZ[j];
            rb->chi[index] = chi; rb->nrs[index] = back->cell[j]; rb->frs[index] = freq_scaled;
            chi_prev = chi;
            index++;
        }
        const int64_t cellNr = back->cell[n_r - 1];
        *In_out = rescale_I_bdy(s, freq_scaled, cellNr, m->cell2boundary[cellNr]);
    } else {
        *In_out = s->I_bdy[m->cell2boundary[o] * nf + f];
    }
}

/* RayPair::solve_using_scattering (Simulation/Raypair/raypair_solver.tpp:10-190,
 * the n_off_diag == 0 branch): the Feautrier system for u and for v (the
 * same matrix, right-hand sides coupled through centred differences of the
 * other term), elimination, back substitution to n_ar, diagonal ALO there. */
static void solve_scattering(raypair_buf *b, const double *term2, double *Sv, int64_t ndep,
                             int64_t n_ar, double I_bdy_0, double I_bdy_n, double *u, double *v,
                             double *L)
{
    double *A = b->A, *C = b->C, *F = b->F, *G = b->G, *Su = b->Su, *dtau = b->dtau;
    double *inv_A = b->inv_A, *inv_C = b->inv_C, *inv1pF = b->inv1pF, *GoG = b->GoG;
    const double *term1 = b->term1;
    const double inverse_dtau0 = 1.0 / dtau[0];
    const double inverse_dtaud = 1.0 / dtau[ndep - 2];
    C[0] = 2.0 * inverse_dtau0 * inverse_dtau0;
    const double B0_min_C0 = 1.0 + 2.0 * inverse_dtau0;
    const double B0 = B0_min_C0 + C[0];
    const double inverse_B0 = 1.0 / B0;
    Su[0] = term1[0] - (term2[1] + term2[0] - 2.0 * I_bdy_0) * inverse_dtau0;
    Sv[0] = term2[0] - (term1[1] + term1[0] - 2.0 * I_bdy_0) * inverse_dtau0;
    for (int64_t n = 1; n < ndep - 1; n++) {
        inv_A[n] = 0.5 * (dtau[n - 1] + dtau[n]) * dtau[n - 1];
        A[n] = 1.0 / inv_A[n];
        inv_C[n] = 0.5 * (dtau[n - 1] + dtau[n]) * dtau[n];
        C[n] = 1.0 / inv_C[n];
        Su[n] = term1[n] - dtau[n] * C[n] * (term2[n + 1] - term2[n - 1]);
        Sv[n] = term2[n] - dtau[n] * C[n] * (term1[n + 1] - term1[n - 1]);
    }
    A[ndep - 1] = 2.0 * inverse_dtaud * inverse_dtaud;
    const double Bd_min_Ad = 1.0 + 2.0 * inverse_dtaud;
    const double Bd = Bd_min_Ad + A[ndep - 1];
    Su[ndep - 1] = term1[ndep - 1] + (term2[ndep - 1] + term2[ndep - 2] + 2.0 * I_bdy_n) * inverse_dtaud;
    Sv[ndep - 1] = term2[ndep - 1] + (term1[ndep - 1] + term1[ndep - 2] - 2.0 * I_bdy_n) * inverse_dtaud;
    Su[0] = Su[0] * inverse_B0;
    Sv[0] = Sv[0] * inverse_B0;
    F[0] = 0.5 * B0_min_C0 * dtau[0] * dtau[0];
    inv1pF[0] = 1.0 / (1.0 + F[0]);
    for (int64_t n = 1; n < ndep - 1; n++) {
        F[n] = (1.0 + A[n] * F[n - 1] * inv1pF[n - 1]) * inv_C[n];
        inv1pF[n] = 1.0 / (1.0 + F[n]);
        Su[n] = (Su[n] + A[n] * Su[n - 1]) * inv1pF[n] * inv_C[n];
        Sv[n] = (Sv[n] + A[n] * Sv[n - 1]) * inv1pF[n] * inv_C[n];
    }
    const double denominator = 1.0 / (Bd_min_Ad + Bd * F[ndep - 2]);
    Su[ndep - 1] = (Su[ndep - 1] + A[ndep - 1] * Su[ndep - 2]) * (1.0 + F[ndep - 2]) * denominator;
    Sv[ndep - 1] = (Sv[ndep - 1] + A[ndep - 1] * Sv[ndep - 2]) * (1.0 + F[ndep - 2]) * denominator;
    if (n_ar < ndep - 1) {
        G[ndep - 1] = 0.5 * Bd_min_Ad * dtau[ndep - 2] * dtau[ndep - 2];
        GoG[ndep - 1] = G[ndep - 1] / (1.0 + G[ndep - 1]);
        for (int64_t n = ndep - 2; n > n_ar; n--) {
            Su[n] = Su[n] + Su[n + 1] * inv1pF[n];
            Sv[n] = Sv[n] + Sv[n + 1] * inv1pF[n];
            G[n] = (1.0 + C[n] * GoG[n + 1]) * inv_A[n];
            GoG[n] = G[n] / (1.0 + G[n]);
        }
        Su[n_ar] = Su[n_ar] + Su[n_ar + 1] * inv1pF[n_ar];
        Sv[n_ar] = Sv[n_ar] + Sv[n_ar + 1] * inv1pF[n_ar];
        *L = inv_C[n_ar] / (F[n_ar] + GoG[n_ar + 1]);
    } else {
        *L = (1.0 + F[ndep - 2]) / (Bd_min_Ad + Bd * F[ndep - 2]);
    }
    *u = Su[n_ar];
    *v = Sv[n_ar];
}

/* The formal solve with scattering terms: for every ray pair R < nrays/2 and
 * origin, setup_using_scattering + solve_using_scattering at every bin, the
 * J and ALO updates of compute_radiation_field (sim_radiation.tpp:150-264),
 * and u, v at the origin per (R, o, f) as Radiation stores them
 * (sim_radiation.tpp:226-236: u as is, v with its sign flipped when the ray
 * r rather than its antipode is in front).  U, V, u_out, v_out:
 * [nrays/2][ncells*nfreqs]. */
int orc_compute_radiation_field_scattering(const orc_model *m, orc_state *s,
                                           const int64_t *antipod, const double *U,
                                           const double *V, double *u_out, double *v_out,
                                           int nthreads)
{
    const int64_t nf = s->nfreqs, N = m->ncells, np = m->nrays / 2;
    line_table lt;
    lt.line = (double *)malloc(sizeof(double) * m->nrad);
    lt.line_index = (int64_t *)malloc(sizeof(int64_t) * m->nrad);
    sorted_lines(m, lt.line, lt.line_index);
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    memset(s->J, 0, sizeof(double) * (size_t)(N * nf));
    memset(s->Ls, 0, sizeof(double) * (size_t)(N * m->nrad));
    int64_t errs = 0;
    for (int64_t r = 0; r < np; r++) {
        const int64_t ar = antipod[r];
        const double weight_ang = m->ray_weights[r];
#pragma omp parallel reduction(+ : errs)
        {
            trace_buf tr = {0, 0, NULL, NULL, NULL, 1, 0};
            trace_buf ta = {0, 0, NULL, NULL, NULL, 1, 0};
            raypair_buf rb;
            memset(&rb, 0, sizeof(rb));
            double *term2 = NULL, *Sv = NULL;
            int64_t cap = 0;
#pragma omp for schedule(static, 1)
            for (int64_t o = 0; o < N; o++) {
                const double dshift_max = orc_dshift_max(m, o);
                int64_t e1 = 0, e2 = 0;
                trace(m, o, r, dshift_max, &tr, &e1);
                trace(m, o, ar, dshift_max, &ta, &e2);
                if (e1 || e2) { errs++; continue; }
                const int r_front = tr.n > ta.n;
                const trace_buf *front = r_front ? &tr : &ta;
                const trace_buf *back = r_front ? &ta : &tr;
                const int64_t n_ar = front->n, ndep = front->n + back->n + 1;
                if (ndep > 1) {
                    rp_ensure(&rb, ndep + 1);
                    if (ndep + 1 > cap) {
                        cap = ndep + 64;
                        term2 = (double *)realloc(term2, sizeof(double) * (size_t)cap);
                        Sv = (double *)realloc(Sv, sizeof(double) * (size_t)cap);
                    }
                    int64_t lnotch_at_origin = 0;
                    for (int64_t i = 0; i < ndep; i++) rb.notch[i] = 0;
                    for (int64_t f = 0; f < nf; f++) {
                        double I0, In, u, v, Ld;
                        setup_scattering(m, s, &lt, o, f, r, U, V, front, back, &rb, term2,
                                         &lnotch_at_origin, &I0, &In);
                        solve_scattering(&rb, term2, Sv, ndep, n_ar, I0, In, &u, &v, &Ld);
                        if (s->appears[f]) {
                            const int64_t k = s->corr_k[f], z = s->corr_z[f];
                            const double freq_line = m->frequency[k];
                            const double weight = m->quad_weights[z] * 2.0 * weight_ang;
                            const double factor = m->A[k] * weight;
                            const double prof = profile(freq_line * profile_width(m, rb.nrs[n_ar]),
                                                        rb.frs[n_ar] - freq_line);
                            s->Ls[o * m->nrad + k] += factor * (rb.frs[n_ar] * prof * Ld / rb.chi[n_ar]);
                        }
                        s->J[o * nf + f] += 2.0 * weight_ang * u;
                        u_out[r * N * nf + o * nf + f] = u;
                        v_out[r * N * nf + o * nf + f] = r_front ? -v : v;
                    }
                } else {
                    const int64_t b = m->cell2boundary[o];
                    for (int64_t f = 0; f < nf; f++) {
                        const double u = 0.5 * (s->I_bdy[b * nf + f] + s->I_bdy[b * nf + f]);
                        const double v = 0.5 * (s->I_bdy[b * nf + f] - s->I_bdy[b * nf + f]);
                        s->J[o * nf + f] += 2.0 * weight_ang * u;
                        u_out[r * N * nf + o * nf + f] = u;
                        v_out[r * N * nf + o * nf + f] = v;
                    }
                }
            }
            free(tr.cell); free(tr.shift); free(tr.dZ);
            free(ta.cell); free(ta.shift); free(ta.dZ);
            rp_free(&rb);
            free(term2); free(Sv);
        }
    }
    s->trace_errors = errs;
    free(lt.line); free(lt.line_index);
    return errs ? 1 : 0;
}

/* Radiation::calc_U_and_V (Model/Radiation/radiation.cpp:330-434, one
 * process): the direction integrals U[r1] = sum over pairs r2 of u[r2] and
 * V[r1] likewise (the phase function is 1), the same for every r1. */
void orc_calc_U_and_V(const orc_model *m, const orc_state *s, const double *u, const double *v,
                      double *U, double *V)
{
    const int64_t n = m->ncells * s->nfreqs, np = m->nrays / 2;
    for (int64_t r1 = 0; r1 < np; r1++) {
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; i++) {
            double su = 0.0, sv = 0.0;
            for (int64_t r2 = 0; r2 < np; r2++) { su += u[r2 * n + i]; sv += v[r2 * n + i]; }
            U[r1 * n + i] = su;
            V[r1 * n + i] = sv;
        }
    }
}

/* ------------------------------------------------------------------ images */

/* Simulation::compute_spectral_discretisation_image, Simulation/sim_spectrum.tpp:200-250:
 * every cell gets the same grid, line + line*width*root over the sorted
 * lines, sorted ascending. */
int orc_image_discretisation(const orc_model *m, orc_state *s, double width)
{
    const int64_t nf = (int64_t)m->nrad * m->nquads;
    double  *line = (double *)malloc(sizeof(double) * m->nrad);
    int64_t *lidx = (int64_t *)malloc(sizeof(int64_t) * m->nrad);
    double  *g    = (double *)malloc(sizeof(double) * nf);
    sorted_lines(m, line, lidx);
    s->nfreqs = nf;
    int64_t index1 = 0;
    for (int64_t k = 0; k < m->nrad; k++)
        for (int64_t z = 0; z < m->nquads; z++) {
            const double freqs_line = line[k];
            g[index1++] = freqs_line + freqs_line * width * m->quad_roots[z];
        }
    for (int64_t i = 1; i < nf; i++) {
        double v = g[i]; int64_t j = i - 1;
        while (j >= 0 && g[j] > v) { g[j + 1] = g[j]; j--; }
        g[j + 1] = v;
    }
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < m->ncells; p++)
        memcpy(s->nu + p * nf, g, sizeof(double) * (size_t)nf);
    free(line); free(lidx); free(g);
    return 0;
}

/* Simulation::compute_and_write_image, Simulation/sim_radiation.tpp:348-478,
 * for the ray r: per origin both rays traced in the rest frame
 * (Geometry::trace_ray<Rest>), the antipode's trace in front, setup as for
 * the radiation field, RayPair::solve_for_image
 * (Simulation/Raypair/raypair_solver.tpp:523-579: elimination from the
 * front, back substitution to the front) and the emergent intensities
 * I_m = 2 u_front - I_bdy_0 and I_p = 2 u_end - I_bdy_n
 * (RayPair::get_Im_at_front / get_Ip_at_end, raypair.tpp:205-229).  A ray
 * pair of one point takes the boundary value of its bin.  I_m, I_p:
 * [ncells*nfreqs]. */
int orc_compute_image(const orc_model *m, orc_state *s, const int64_t *antipod, int64_t r,
                      double *I_m, double *I_p, int nthreads)
{
    const int64_t nf = s->nfreqs;
    const int64_t ar = antipod[r];
    line_table lt;
    lt.line = (double *)malloc(sizeof(double) * m->nrad);
    lt.line_index = (int64_t *)malloc(sizeof(int64_t) * m->nrad);
    sorted_lines(m, lt.line, lt.line_index);
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    int64_t errs = 0;
#pragma omp parallel reduction(+ : errs)
    {
        trace_buf tr = {0, 0, NULL, NULL, NULL, 1, 0};
        trace_buf ta = {0, 0, NULL, NULL, NULL, 1, 0};
        raypair_buf rb;
        memset(&rb, 0, sizeof(rb));
#pragma omp for schedule(static, 1)
        for (int64_t o = 0; o < m->ncells; o++) {
            const double dshift_max = orc_dshift_max(m, o);
            int64_t e1 = 0, e2 = 0;
            trace_frame(m, o, r, dshift_max, 1, antipod, &tr, &e1);
            trace_frame(m, o, ar, dshift_max, 1, antipod, &ta, &e2);
            if (e1 || e2) { errs++; continue; }
            const int64_t ndep = ta.n + tr.n + 1;
            if (ndep > 1) {
                rp_ensure(&rb, ndep + 1);
                int64_t lnotch_at_origin = 0;
                for (int64_t i = 0; i < ndep; i++) rb.notch[i] = 0;
                for (int64_t f = 0; f < nf; f++) {
                    double I0, In, u, Ld;
                    int64_t first, last;
                    setup_pair(m, s, &lt, o, f, &ta, &tr, &rb, &lnotch_at_origin, &first, &last,
                               &I0, &In);
                    /* back substitution all the way to the front (n_ar = first) */
                    solve_raypair(&rb, first, last, first, I0, In, &u, &Ld);
                    I_m[o * nf + f] = 2.0 * rb.Su[0] - I0;
                    I_p[o * nf + f] = 2.0 * rb.Su[ndep - 1] - In;
                }
            } else {
                const int64_t b = m->cell2boundary[o];
                for (int64_t f = 0; f < nf; f++) {
                    I_m[o * nf + f] = s->I_bdy[b * nf + f];
                    I_p[o * nf + f] = s->I_bdy[b * nf + f];
                }
            }
        }
        free(tr.cell); free(tr.shift); free(tr.dZ);
        free(ta.cell); free(ta.shift); free(ta.dZ);
        rp_free(&rb);
    }
    free(lt.line); free(lt.line_index);
    s->trace_errors = errs;
    return errs ? 1 : 0;
}

/* ------------------------------------------------------- level populations */

/* Simulation::compute_Jeff, Simulation/sim_lines.tpp:176-220 (the ALO has
 * one element per (p,k) when n_off_diag = 0, its cell being p). */
void orc_compute_jeff(const orc_model *m, orc_state *s)
{
    const int64_t nr = m->nrad, nq = m->nquads, nf = s->nfreqs, nl = m->nlev;
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < m->ncells; p++) {
        for (int64_t k = 0; k < nr; k++) {
            double jl = 0.0;
            for (int64_t z = 0; z < nq; z++)
                jl += m->quad_weights[z] * s->J[p * nf + s->nr_line[p * nf + k * nq + z]];
            double diff = 0.0;
            diff += s->Ls[p * nr + k] * s->pop[p * nl + m->irad[k]];
            if (s->n_off_diag > 1) {   /* the non-local elements of (p, k) */
                const int64_t M1 = s->n_off_diag - 1, np = m->nrays / 2;
                for (int64_t r = 0; r < np; r++)
                    for (int64_t i = 0; i < 2 * M1; i++) {
                        const int64_t c = s->Loff_nr[(p * np + r) * 2 * M1 + i];
                        if (c < 0) continue;
                        diff += s->Loff[((p * nr + k) * np + r) * 2 * M1 + i] *
                                s->pop[c * nl + m->irad[k]];
                    }
            }
            s->Jlin[p * nr + k] = jl;
            s->Jeff[p * nr + k] = jl - O_HH_OVER_FOUR_PI * diff;
            s->Jdif[p * nr + k] = O_HH_OVER_FOUR_PI * diff;
        }
    }
}

/* CollisionPartner::interpolate_collision_coefficients with search(),
 * collisionPartner.tpp:15-47 and Functions/interpolation.tpp; a partner
 * table is extrapolated linearly above its last temperature. */
static void interpolate_collision(const orc_colpar *c, double T, double *Cd_i, double *Ce_i)
{
    const int64_t ntmp = c->ntmp;
    int64_t t;
    int64_t start = 0, stop = ntmp - 1;
    if (T >= c->tmp[stop]) t = stop;
    else if (T <= c->tmp[start]) t = start;
    else {
        t = -1;
        while (stop > start + 1) {
            const int64_t middle = (stop + start) / 2;
            if (T > c->tmp[middle]) start = middle;
            else if (T < c->tmp[middle]) stop = middle;
            else { t = middle; break; }
        }
        if (t < 0) t = stop;
    }
    if (t == 0) {
        for (int64_t k = 0; k < c->ncol; k++) { Ce_i[k] = c->Ce[k]; Cd_i[k] = c->Cd[k]; }
    } else if (t == ntmp) {
        for (int64_t k = 0; k < c->ncol; k++) { Ce_i[k] = c->Ce[(ntmp - 1) * c->ncol + k]; Cd_i[k] = c->Cd[(ntmp - 1) * c->ncol + k]; }
    } else {
        const double step = (T - c->tmp[t - 1]) / (c->tmp[t] - c->tmp[t - 1]);
        for (int64_t k = 0; k < c->ncol; k++) {
            const double ce0 = c->Ce[(t - 1) * c->ncol + k], ce1 = c->Ce[t * c->ncol + k];
            const double cd0 = c->Cd[(t - 1) * c->ncol + k], cd1 = c->Cd[t * c->ncol + k];
            Ce_i[k] = ce0 + (ce1 - ce0) * step;
            Cd_i[k] = cd0 + (cd1 - cd0) * step;
        }
    }
}

/* dense partial-pivot LU solve of M x = y in place (row-major n x n) */
static int lu_solve(int64_t n, double *M, double *y)
{
    for (int64_t k = 0; k < n; k++) {
        int64_t piv = k;
        double best = fabs(M[k * n + k]);
        for (int64_t i = k + 1; i < n; i++) {
            const double v = fabs(M[i * n + k]);
            if (v > best) { best = v; piv = i; }
        }
        if (!(best > 0.0)) return -1;
        if (piv != k) {
            for (int64_t j = 0; j < n; j++) { double t = M[k * n + j]; M[k * n + j] = M[piv * n + j]; M[piv * n + j] = t; }
            double t = y[k]; y[k] = y[piv]; y[piv] = t;
        }
        const double inv = 1.0 / M[k * n + k];
        for (int64_t i = k + 1; i < n; i++) {
            const double l = M[i * n + k] * inv;
            if (l == 0.0) continue;
            for (int64_t j = k + 1; j < n; j++) M[i * n + j] -= l * M[k * n + j];
            y[i] -= l * y[k];
        }
    }
    for (int64_t i = n - 1; i >= 0; i--) {
        double acc = y[i];
        for (int64_t j = i + 1; j < n; j++) acc -= M[i * n + j] * y[j];
        y[i] = acc / M[i * n + i];
    }
    return 0;
}

/* Collision rates of cell p into the rows of cell block `base` of a dense
 * matrix with leading dimension ld (lineProducingSpecies.tpp:344-378). */
static void add_collisions(const orc_model *m, int64_t p, double *Mrow0, int64_t ld,
                           int64_t base, double *Cd_i, double *Ce_i)
{
    const int64_t last = m->nlev - 1;
    for (int c = 0; c < m->ncolpar; c++) {
        const orc_colpar *cp = &m->colpar[c];
        double abn = cp->abundance[p];
        const double tmp = m->temperature[p];
        if (cp->ortho_para != 0) {
            const double frac_H2_para = 1.0 / (1.0 + 9.0 * exp(-170.5 / tmp));
            if (cp->ortho_para == 1) abn *= (1.0 - frac_H2_para);
            if (cp->ortho_para == 2) abn *= frac_H2_para;
        }
        interpolate_collision(cp, tmp, Cd_i, Ce_i);
        for (int64_t k = 0; k < cp->ncol; k++) {
            const double v_IJ = Cd_i[k] * abn;
            const double v_JI = Ce_i[k] * abn;
            const int64_t I = base + cp->icol[k], J = base + cp->jcol[k];
            if (cp->jcol[k] != last) { Mrow0[J * ld + I] += +v_IJ; Mrow0[J * ld + J] += -v_JI; }
            if (cp->icol[k] != last) { Mrow0[I * ld + J] += +v_JI; Mrow0[I * ld + I] += -v_IJ; }
        }
    }
}

/* update_using_statistical_equilibrium with a non-local ALO (n_off_diag >= 2,
 * lineProducingSpecies.tpp:249-495).  The cell blocks hold the reference's
 * triplets in its order -- radiative rates, then for each line the ALO
 * elements (nr, Ls) of the cell with v = -Ls * opacity(p, k), then
 * collisions, then the conservation row.  An element couples the rows of
 * cell p's lower and upper levels to the upper level of cell nr: v at
 * (J(p), I(nr)) and -v at (I(p), I(nr)), the terms that cancel the
 * element's part of Jeff once the populations stop changing.  (The
 * reference writes the second at (I(nr), I(nr)) (lineProducingSpecies.tpp:
 * 325-338), the same place when nr = p; for nr != p that leaves
 * -Ls*opacity*n_I(nr) uncancelled in cell p's upper-level row and moves the
 * converged populations.)  Elements with nr = p go into p's block; the
 * others couple the blocks.  The global system (SparseLU<COLAMD> there) is
 * solved by block Jacobi: each cell's block by partial-pivot LU with the
 * couplings to the other cells' current populations moved to the right-hand
 * side, from the populations before the solve, until no population changes
 * by more than 1e-14 of itself (of 1e-10 of the cell's total for the levels
 * below that, which the convergence test ignores), or, once below 1e-6, the
 * change has set no new low for five sweeps (the rounding floor of the cell
 * solves); at most 1000 sweeps, a sweep count past that is an error.  Solving cell by cell keeps every block's own scaling,
 * which a dense LU of the whole model (populations over 10 orders of
 * magnitude) loses for the weakly populated levels. */
static int statistical_equilibrium_global(const orc_model *m, orc_state *s)
{
    const int64_t nl = m->nlev, nr = m->nrad, N = m->ncells, n = N * nl;
    const int64_t M1 = s->n_off_diag - 1, np = m->nrays / 2, ne = np * 2 * M1;
    memcpy(s->prev3, s->prev2, sizeof(double) * (size_t)n);
    memcpy(s->prev2, s->prev1, sizeof(double) * (size_t)n);
    memcpy(s->prev1, s->pop, sizeof(double) * (size_t)n);
    double *xa = (double *)malloc(sizeof(double) * (size_t)n);
    double *xb = (double *)malloc(sizeof(double) * (size_t)n);
    memcpy(xa, s->prev1, sizeof(double) * (size_t)n);
    double *B = (double *)malloc(sizeof(double) * (size_t)(nl * nl));
    double *y = (double *)malloc(sizeof(double) * (size_t)nl);
    int64_t maxcol = 1;
    for (int c = 0; c < m->ncolpar; c++) if (m->colpar[c].ncol > maxcol) maxcol = m->colpar[c].ncol;
    double *Cd_i = (double *)malloc(sizeof(double) * (size_t)maxcol);
    double *Ce_i = (double *)malloc(sizeof(double) * (size_t)maxcol);
    const int64_t last = nl - 1;
    int bad = 0, sweep, best_sweep = 0;
    double best = INFINITY;
    for (sweep = 0; sweep < 1000 && !bad; sweep++) {
        double change = 0.0;
        for (int64_t p = 0; p < N && !bad; p++) {
            const double *pop = s->prev1 + p * nl;
            memset(B, 0, sizeof(double) * (size_t)(nl * nl));
            memset(y, 0, sizeof(double) * (size_t)nl);
            for (int64_t k = 0; k < nr; k++) {
                const double Jeff = s->Jeff[p * nr + k];
                const double v_IJ = m->A[k] + m->Bs[k] * Jeff;
                const double v_JI = m->Ba[k] * Jeff;
                const int64_t I = m->irad[k], J = m->jrad[k];
                if (J != last) { B[J * nl + I] += +v_IJ; B[J * nl + J] += -v_JI; }
                if (I != last) { B[I * nl + J] += +v_JI; B[I * nl + I] += -v_IJ; }
            }
            for (int64_t k = 0; k < nr; k++) {
                const double opac = O_HH_OVER_FOUR_PI * (pop[m->jrad[k]] * m->Ba[k] - pop[m->irad[k]] * m->Bs[k]);
                const int64_t I = m->irad[k], J = m->jrad[k];
                for (int64_t e = -1; e < ne; e++) {
                    int64_t c;
                    double Ls;
                    if (e < 0) {
                        c = p;
                        Ls = s->Ls[p * nr + k];
                    } else {
                        c = s->Loff_nr[p * ne + e];
                        if (c < 0) continue;
                        Ls = s->Loff[(p * nr + k) * ne + e];
                    }
                    const double v_IJ = -Ls * opac;
                    if (c == p) {
                        if (J != last) B[J * nl + I] += +v_IJ;
                        if (I != last) B[I * nl + I] += -v_IJ;
                    } else {
                        const double xc = xa[c * nl + I];
                        if (J != last) y[J] -= v_IJ * xc;
                        if (I != last) y[I] += v_IJ * xc;
                    }
                }
            }
            add_collisions(m, p, B, nl, 0, Cd_i, Ce_i);
            for (int64_t i = 0; i < nl; i++) B[last * nl + i] += 1.0;
            y[last] = m->population_tot[p];
            if (lu_solve(nl, B, y)) { bad = 1; break; }
            /* change relative to the population, or to 1e-10 of the cell's
             * total below it (the levels the convergence test ignores) */
            const double floor_p = 1.0E-10 * m->population_tot[p];
            for (int64_t i = 0; i < nl; i++) {
                const double v = y[i];
                const double d = fabs(v - xa[p * nl + i]) / fmax(fabs(v), floor_p);
                if (d > change) change = d;
                xb[p * nl + i] = v;
            }
        }
        double *t = xa; xa = xb; xb = t;
        if (change <= 1.0E-14) { sweep++; break; }
        /* at the rounding floor of the cell solves: no new low in 5 sweeps */
        if (change < best) { best = change; best_sweep = sweep; }
        else if (best < 1.0E-6 && sweep >= best_sweep + 5) { sweep++; break; }
    }
    if (!bad && sweep >= 1000) bad = 2;
    if (!bad) memcpy(s->pop, xa, sizeof(double) * (size_t)n);
    s->lu_errors = bad ? 1 : 0;
    free(xa); free(xb); free(B); free(y); free(Cd_i); free(Ce_i);
    return bad;
}

/* LineProducingSpecies::update_using_statistical_equilibrium,
 * lineProducingSpecies.tpp:249-495.  With n_off_diag = 0 the rate matrix is
 * block diagonal; each cell's block is assembled from the same triplets in
 * the same order (duplicates summed in insertion order, as
 * SparseMatrix::setFromTriplets does) and solved by dense partial-pivot LU
 * in place of SparseLU<COLAMD> (whose pivot order is not pinned here). */
int orc_statistical_equilibrium(const orc_model *m, orc_state *s)
{
    if (s->n_off_diag > 1) return statistical_equilibrium_global(m, s);
    const int64_t nl = m->nlev, nr = m->nrad, N = m->ncells;
    memcpy(s->prev3, s->prev2, sizeof(double) * (size_t)(N * nl));
    memcpy(s->prev2, s->prev1, sizeof(double) * (size_t)(N * nl));
    memcpy(s->prev1, s->pop, sizeof(double) * (size_t)(N * nl));
    int64_t lu_err = 0;
#pragma omp parallel reduction(+ : lu_err)
    {
        double *M = (double *)malloc(sizeof(double) * (size_t)(nl * nl));
        double *y = (double *)malloc(sizeof(double) * (size_t)nl);
        int64_t maxcol = 1;
        for (int c = 0; c < m->ncolpar; c++) if (m->colpar[c].ncol > maxcol) maxcol = m->colpar[c].ncol;
        double *Cd_i = (double *)malloc(sizeof(double) * (size_t)maxcol);
        double *Ce_i = (double *)malloc(sizeof(double) * (size_t)maxcol);
#pragma omp for schedule(static)
        for (int64_t p = 0; p < N; p++) {
            const double *pop = s->prev1 + p * nl;   /* `population` before the solve */
            memset(M, 0, sizeof(double) * (size_t)(nl * nl));
            memset(y, 0, sizeof(double) * (size_t)nl);
            const int64_t last = nl - 1;
            for (int64_t k = 0; k < nr; k++) {
                const double Jeff = s->Jeff[p * nr + k];
                const double v_IJ = m->A[k] + m->Bs[k] * Jeff;
                const double v_JI = m->Ba[k] * Jeff;
                const int64_t I = m->irad[k], J = m->jrad[k];
                if (J != last) { M[J * nl + I] += +v_IJ; M[J * nl + J] += -v_JI; }
                if (I != last) { M[I * nl + J] += +v_JI; M[I * nl + I] += -v_IJ; }
            }
            for (int64_t k = 0; k < nr; k++) {
                const int64_t I = m->irad[k], J = m->jrad[k];
                const double opac = O_HH_OVER_FOUR_PI * (pop[J] * m->Ba[k] - pop[I] * m->Bs[k]);
                const double v_IJ = -s->Ls[p * nr + k] * opac;
                if (J != last) M[J * nl + I] += +v_IJ;
                if (I != last) M[I * nl + I] += -v_IJ;
            }
            for (int c = 0; c < m->ncolpar; c++) {
                const orc_colpar *cp = &m->colpar[c];
                double abn = cp->abundance[p];
                const double tmp = m->temperature[p];
                if (cp->ortho_para != 0) {
                    const double frac_H2_para = 1.0 / (1.0 + 9.0 * exp(-170.5 / tmp));
                    if (cp->ortho_para == 1) abn *= (1.0 - frac_H2_para);
                    if (cp->ortho_para == 2) abn *= frac_H2_para;
                }
                interpolate_collision(cp, tmp, Cd_i, Ce_i);
                for (int64_t k = 0; k < cp->ncol; k++) {
                    const double v_IJ = Cd_i[k] * abn;
                    const double v_JI = Ce_i[k] * abn;
                    const int64_t I = cp->icol[k], J = cp->jcol[k];
                    if (J != last) { M[J * nl + I] += +v_IJ; M[J * nl + J] += -v_JI; }
                    if (I != last) { M[I * nl + J] += +v_JI; M[I * nl + I] += -v_IJ; }
                }
            }
            for (int64_t i = 0; i < nl; i++) M[last * nl + i] += 1.0;
            y[last] = m->population_tot[p];
            if (lu_solve(nl, M, y)) { lu_err++; continue; }
            for (int64_t i = 0; i < nl; i++) s->pop[p * nl + i] = y[i];
        }
        free(M); free(y); free(Cd_i); free(Ce_i);
    }
    s->lu_errors = lu_err;
    return lu_err ? 1 : 0;
}

/* LineProducingSpecies::check_for_convergence, lineProducingSpecies.tpp:120-171,
 * plus the maximum relative change over the same levels. */
void orc_check_convergence(const orc_model *m, orc_state *s)
{
    const int64_t nl = m->nlev, N = m->ncells;
    const double weight = 1.0 / (double)(N * nl);
    double fnc = 0.0, rcm = 0.0, mx = 0.0;
    for (int64_t p = 0; p < N; p++) {
        const double min_pop = 1.0E-10 * m->population_tot[p];
        for (int64_t i = 0; i < nl; i++) {
            const double a = s->pop[p * nl + i], b = s->prev1[p * nl + i];
            if (a > min_pop) {
                double relative_change = 2.0;
                relative_change *= fabs(a - b);
                relative_change /= (a + b);
                if (relative_change > m->pop_prec) fnc += weight;
                rcm += weight * relative_change;
                if (relative_change > mx) mx = relative_change;
            }
        }
    }
    s->fnc = fnc;
    s->rcm = rcm;
    s->max_rel = mx;
}

/* LineProducingSpecies::update_using_Ng_acceleration, lineProducingSpecies.tpp:181-238 */
void orc_ng_acceleration(const orc_model *m, orc_state *s)
{
    const int64_t n = m->ncells * (int64_t)m->nlev;
    double A1 = 0.0, A2 = 0.0, B2 = 0.0, C1 = 0.0, C2 = 0.0;
    for (int64_t i = 0; i < n; i++) {
        const double Q1 = s->pop[i] - 2.0 * s->prev1[i] + s->prev2[i];
        const double Q2 = s->pop[i] - s->prev1[i] - s->prev2[i] + s->prev3[i];
        const double Q3 = s->pop[i] - s->prev1[i];
        A1 += Q1 * Q1; A2 += Q1 * Q2; B2 += Q2 * Q2; C1 += Q1 * Q3; C2 += Q2 * Q3;
    }
    const double B1 = A2;
    const double denominator = A1 * B2 - A2 * B1;
    if (denominator != 0.0) {
        const double a = (C1 * B2 - C2 * B1) / denominator;
        const double b = (C2 * A1 - C1 * A2) / denominator;
        for (int64_t i = 0; i < n; i++) {
            const double tmp = s->pop[i];
            const double np = (1.0 - a - b) * s->pop[i] + a * s->prev1[i] + b * s->prev2[i];
            s->prev3[i] = s->prev2[i];
            s->prev2[i] = s->prev1[i];
            s->prev1[i] = tmp;
            s->pop[i] = np;
        }
    }
}

/* Simulation::compute_level_populations(io, use_Ng, max_niterations),
 * Simulation/sim_lines.tpp:61-164.  tol_max_rel > 0 replaces the stop test
 * "fraction_not_converged <= 0.005" by "max relative change < tol_max_rel".
 * ng_every: normal iterations before each Ng step (the reference: 4). */
int64_t orc_compute_level_populations_ng(const orc_model *m, orc_state *s,
                                         const int64_t *antipod, int use_ng, int64_t max_iter,
                                         double tol_max_rel, int nthreads, double *iter_max_rel,
                                         int ng_every)
{
    int64_t iteration = 0, iteration_normal = 0;
    int some_not_converged = 1;
    while (some_not_converged && iteration < max_iter) {
        iteration++;
        some_not_converged = 0;
        if (use_ng && iteration_normal == ng_every) {
            orc_ng_acceleration(m, s);
            orc_check_convergence(m, s);
            orc_set_emissivity_opacity(m, s);
            iteration_normal = 0;
        } else {
            orc_compute_radiation_field(m, s, antipod, NULL, 0, 0, nthreads);
            orc_compute_jeff(m, s);
            orc_statistical_equilibrium(m, s);
            orc_check_convergence(m, s);
            orc_set_emissivity_opacity(m, s);
            iteration_normal++;
        }
        if (iter_max_rel) iter_max_rel[iteration - 1] = s->max_rel;
        if (tol_max_rel > 0.0) { if (s->max_rel >= tol_max_rel) some_not_converged = 1; }
        else if (s->fnc > 0.005) some_not_converged = 1;
    }
    return iteration;
}

int64_t orc_compute_level_populations(const orc_model *m, orc_state *s, const int64_t *antipod,
                                      int use_ng, int64_t max_iter, double tol_max_rel,
                                      int nthreads, double *iter_max_rel)
{
    return orc_compute_level_populations_ng(m, s, antipod, use_ng, max_iter, tol_max_rel,
                                            nthreads, iter_max_rel, 4);
}
