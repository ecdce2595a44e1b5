// mgr_internal.cuh -- shared definitions of the B200 radiation hot path.
//
// Device layout (all arrays resident in HBM for the handle's lifetime):
//   geometry   pos[3N], vel[3N] (double, AoS), nbr_off[N+1], nbr[.] (int32),
//              boundary[N] (uint8), cell2bdy[N] (int32, -1 if none),
//              rays[3R], dshift_max[N], pw[N] (profile width over c)
//   lines      line[K] (ascending Hz), inv_line[K], A[K], window lo/hi[K]
//   state      pop/prev1..3 [N*nlev], eps/kap [N*K] (double),
//              Ehat/Khat [N*K] (float, scaled), Jlin/Lam/Jeff [N*K]
//   traces     per (direction, origin): offset (int64), length (int32);
//              points as cell (int32), shift (double), dZ (double), and a
//              16-byte record {cell, shift-1, dZ/(2X), 1/pw} in float for
//              the mixed-precision solve (X: the float opacity scale)
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/magritte_b200.h"

namespace mgr {

// Physical constants with the reference's literals and folding order
// (src/Tools/constants.hpp:25-46).
constexpr double kCC = 2.99792458E+8;
constexpr double kHH = 6.62607004E-34;
constexpr double kKB = 1.38064852E-23;
constexpr double kAMU = 1.66053904E-27;
constexpr double kT_CMB = 2.7254800;
constexpr double kC_SQUARED = 8.98755179E+16;
constexpr double kPI = 3.14159265358979323846;
constexpr double kFOUR_PI = 4.0 * kPI;
constexpr double kINVERSE_SQRT_PI = 0.5 * 1.12837916709551257390;  // 0.5*M_2_SQRTPI
constexpr double kTWO_KB_OVER_AMU_C_SQUARED = 2.0 * kKB / (kAMU * kC_SQUARED);
constexpr double kTWO_HH_OVER_CC_SQUARED = 2.0 * kHH / kC_SQUARED;
constexpr double kHH_OVER_KB = kHH / kKB;
constexpr double kHH_OVER_FOUR_PI = kHH / kFOUR_PI;

constexpr int kWarp = 32;
constexpr int kMaxLevels = 32;     // rate-equation solver: one lane per level
constexpr int kMaxColpar = 4;

// ------------------------------------------------------------------------
// Separately rounded double arithmetic (no FMA contraction): the tracer must
// reproduce the oracle's bits, which rounds every operation on its own.
__device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double radd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double rsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double rdiv(double a, double b) { return __ddiv_rn(a, b); }
// (x x' + y y') + z z' -- the dot-product order the oracle restates for
// Eigen's Vector3d::dot.
__device__ __forceinline__ double rdot3(double ax, double ay, double az,
                                        double bx, double by, double bz) {
    return radd(radd(rmul(ax, bx), rmul(ay, by)), rmul(az, bz));
}

// Planck function (Functions/planck.tpp:15-23).
__device__ __forceinline__ double planck(double T, double nu) {
    const double h_over_kbT = kHH_OVER_KB / T;
    return kTWO_HH_OVER_CC_SQUARED * (nu * nu * nu) / expm1(h_over_kbT * nu);
}

// ------------------------------------------------------------------------
struct ColparDev {
    int ntmp, ncol, ortho_para;
    int32_t *icol, *jcol;   // [ncol]
    double *tmp;            // [ntmp]
    double *Cd, *Ce;        // [ntmp*ncol]
    double *abn;            // [N]
};

// Non-owning view of the device model handed to kernels by value.
struct ModelView {
    int64_t N;
    int nrays, npairs, nlev, nrad, nquads, nfreqs, ncolpar;
    const double *pos, *vel, *rays, *ray_w;
    const int32_t *nbr_off, *nbr;
    const uint8_t *boundary;
    const int32_t *cell2bdy;
    const int32_t *antipod;
    const double *bdy_T;
    const double *ibdy;    // [nboundary][nfreqs] boundary intensities
    const double *T, *dshift_max, *pw, *inv_pw;
    const double *line, *inv_line, *A, *Bs, *Ba, *energy, *weight;
    const int32_t *irad, *jrad, *win_lo, *win_hi;
    const double *roots, *qw;
    const double *pop_tot;
    ColparDev colpar[kMaxColpar];
    double pop_prec;
    double root_inv_step;  // (nquads - 1) / (roots[last] - roots[0]), 0 for one root
    double mixed_scale;    // X: power of two scaling the float opacities
    int overlap;           // some line window holds more than its own line
    // batches of independent models (nullptr / 0 for a single model)
    int64_t nseg;
    const int64_t *seg_begin;   // [nseg+1] first cell of each model
    const int32_t *cell_seg;    // [N] model of each cell
    const int32_t *seg_active;  // [nseg] 1 while the model iterates
};

// One traced point in the mixed-precision format (one 16-byte load).
struct __align__(16) MixedPoint {
    int32_t cell;
    float delta;   // Doppler shift - 1
    float dzs;     // dZ / (2 X): dtau = (chi_a + chi_b) * dzs for chi scaled by X
    float ipw;     // 1 / profile width of the cell
};

// Trace store for one batch of origins [o_begin, o_begin + o_count).
struct TraceView {
    int64_t o_begin, o_count;
    int ndir;
    const int64_t *off;    // [ndir*o_count]
    const int32_t *len;    // [ndir*o_count]
    const int32_t *cell;
    const double *shift, *dZ;
    const MixedPoint *mp;  // same points, mixed format
};

// Error counters written by kernels (bounded, never trap).
struct DevFlags {
    unsigned long long trace_err;   // rays without a neighbour ahead
    unsigned long long interp_err;  // > 10000 interpolation points
    unsigned long long lu_err;      // zero pivots
    unsigned long long cap_err;     // trace longer than its slot
    unsigned long long stuck_err;   // step limit reached
    unsigned long long patch_overflow;  // mixed entries beyond the patch list
    unsigned long long redo_count;      // origins listed for an FP64 re-solve (overflow)
};

// Emissivity and opacity at (cell p, frequency freq) over lines [lo, hi]:
// Simulation::get_eta_and_chi (simulation.tpp:385-481) over the lines in the
// bin's window, with Thermodynamics::profile (thermodynamics.tpp:16-29);
// 1/exp(x^2) is written exp(-x^2) and 1/width (1/line)(1/pw).
__device__ __forceinline__ void eta_chi_double(const ModelView &m, const double *__restrict__ eps,
                                               const double *__restrict__ kap, int p, double freq,
                                               int lo, int hi, double &eta, double &chi) {
    eta = 0.0;
    chi = 1.0E-26;
    const double pwp = __ldg(m.pw + p);
    const double ipw = __ldg(m.inv_pw + p);
    const int K = m.nrad;
    for (int l = lo; l <= hi; l++) {
        const double line_l = __ldg(m.line + l);
        const double width = line_l * pwp;
        const double diff = freq - line_l;
        const bool in = diff <= 11.0 * width && diff >= -11.0 * width;
        const double inv_w = __ldg(m.inv_line + l) * ipw;
        const double x = inv_w * diff;
        const double fp = in ? freq * (inv_w * kINVERSE_SQRT_PI * exp(-(x * x))) : 0.0;
        eta += __ldg(eps + (unsigned)p * K + l) * fp;
        chi += __ldg(kap + (unsigned)p * K + l) * fp;
    }
}

// What the boundary condition needs, passed by value to the out-of-line
// helper below.
struct BdyCtx {
    const int32_t *cell2bdy;
    const double *ibdy;            // [nboundary][nfreqs] I_bdy on each boundary cell's grid
    const double *pw, *line, *roots;
    const double *inv_pw, *inv_line;
    double root_inv_step;
    int nq, nf;
};

__device__ __forceinline__ BdyCtx bdy_ctx(const ModelView &m) {
    BdyCtx c;
    c.cell2bdy = m.cell2bdy;
    c.ibdy = m.ibdy;
    c.pw = m.pw;
    c.line = m.line;
    c.roots = m.roots;
    c.inv_pw = m.inv_pw;
    c.inv_line = m.inv_line;
    c.root_inv_step = m.root_inv_step;
    c.nq = m.nquads;
    c.nf = m.nfreqs;
    return c;
}

// Radiation::rescale_I_bdy (scalar build, Model/Radiation/radiation.tpp:341-373)
// on the table of Simulation::compute_boundary_intensities.  The reference
// takes the first bin of cell p's grid with freq <= nu_p(f) by a linear
// search; the grid ascends (lines do not interleave, which the spectral
// discretisation checks), so the same bin is found in two steps: the line
// whose last bin is >= freq (first the hint k_hint, the line of the bin the
// frequency was shifted from, checked against its neighbour; otherwise by
// bisection), then the bin within that line, from a guess on the root grid
// walked up or down to the first bin >= freq (two checks when the guess is
// right, which on an evenly spaced root grid it is but for rounding).
static __device__ __forceinline__ double boundary_intensity(BdyCtx c, double freq, int p,
                                                            DevFlags *flags, int k_hint = -1) {
    const int b = __ldg(c.cell2bdy + p);
    if (b < 0) {
        atomicAdd(&flags->trace_err, 1ull);
        return 0.0;
    }
    const double pwp = __ldg(c.pw + p);
    const int nq = c.nq, nf = c.nf, K = nf / nq;
    auto nu_kz = [&](int k, int z) {
        const double line = __ldg(c.line + k);
        return radd(line, rmul(rmul(line, pwp), __ldg(c.roots + z)));
    };
    int lo = 0, hi = K;
    if (k_hint >= 0 && k_hint < K && freq <= nu_kz(k_hint, nq - 1) &&
        (k_hint == 0 || freq > nu_kz(k_hint - 1, nq - 1))) {
        lo = k_hint;   // the first line whose last bin is >= freq
    } else {
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (freq <= nu_kz(mid, nq - 1)) hi = mid;
            else lo = mid + 1;
        }
    }
    const double *I = c.ibdy + (int64_t)b * nf;
    if (lo == K) return __ldg(I + nf - 1);   // above the grid
    const int k = lo;
    // guess from freq = line (1 + pw root), then the first z with freq <= nu(k, z)
    // (freq <= nu(k, nq-1) holds, so the upward walk ends at or before it)
    const double root = (freq * __ldg(c.inv_line + k) - 1.0) * __ldg(c.inv_pw + p);
    const double zg = ceil((root - __ldg(c.roots)) * c.root_inv_step);
    int zl = (int)fmin(fmax(zg, 0.0), (double)(nq - 1));
    while (zl < nq - 1 && freq > nu_kz(k, zl)) zl++;
    while (zl > 0 && freq <= nu_kz(k, zl - 1)) zl--;
    const int notch = k * nq + zl;
    if (notch == 0 || notch == nf - 1) return __ldg(I + notch);
    const double nu1 = nu_kz(k, zl);
    const double nu2 = zl > 0 ? nu_kz(k, zl - 1) : nu_kz(k - 1, nq - 1);
    const double I1 = __ldg(I + notch), I2 = __ldg(I + notch - 1);
    return (I2 - I1) / (nu2 - nu1) * (freq - nu1) + I1;
}

// ------------------------------------------------------------------------
// Host-side launchers (each file owns its kernels).
// The neighbour each hop of a walk chose, recorded by the counting pass
// so that the filling pass replays the walk without searching: cell[k *
// nrays_total + idx] for hops k < cap of ray idx, and n[idx] = the ray's hop
// count, or -1 when it has more than cap hops (the fill then searches).
struct HopLog {
    int32_t *cell;
    int32_t *n;
    int cap;
};
cudaError_t launch_trace_count(const ModelView &m, int64_t o_begin, int64_t o_count,
                               int32_t *len, DevFlags *flags, cudaStream_t s,
                               const HopLog *hops = nullptr);
// hops: the log of the counting pass over the same rays (o_begin = 0,
// o_count = N), or null to search every walk again.
cudaError_t launch_trace_fill(const ModelView &m, const TraceView &t, int32_t *cell,
                              double *shift, double *dZ, MixedPoint *mp, DevFlags *flags,
                              cudaStream_t s, const HopLog *hops = nullptr);
// Rest-frame traces of the two rays of an image for every origin: slot
// d * N + o walks ray_front (d = 0) or ray_back (d = 1), its shift projected
// on ray shift_front or shift_back.
cudaError_t launch_image_trace_count(const ModelView &m, int ray_front, int ray_back,
                                     int shift_front, int shift_back, int32_t *len,
                                     DevFlags *flags, cudaStream_t s);
cudaError_t launch_image_trace_fill(const ModelView &m, int ray_front, int ray_back,
                                    int shift_front, int shift_back, const int32_t *len,
                                    const int64_t *off, int32_t *cell, double *shift, double *dZ,
                                    DevFlags *flags, cudaStream_t s);

// Images (image.cu): the emergent intensities at both far ends of the ray
// pair through every origin, on an image frequency grid common to all cells.
struct ImageArgs {
    const double *grid;        // [nf] image frequencies, ascending
    const int32_t *lo, *hi;    // [nf] lines whose window can reach the bin
    const double *table;       // [nboundary][nf] boundary intensities on the grid
    const int32_t *len;        // [2N] trace lengths: front (antipode) then back
    const int64_t *off;        // [2N]
    const int32_t *cell;
    const double *shift, *dZ;
    const double *eps, *kap;   // [N*nrad]
    double *I_m, *I_p;         // [N*nf]
    int nf;
};
// The formal solve with scattering terms (scatter.cu): U, V [npairs][N*nf]
// in, u, v at the origins [npairs][N*nf] out, with J (optional), Jlin and
// the ALO.
struct ScatterArgs {
    const double *eps, *kap;
    const double *U, *V;
    double *u, *v;
    double *J, *Jlin, *Lam;
};
cudaError_t launch_scatter(const ModelView &m, const TraceView &t, const ScatterArgs &a,
                           DevFlags *flags, cudaStream_t s);
cudaError_t launch_calc_uv(const ModelView &m, const double *u, const double *v, double *U,
                           double *V, cudaStream_t s);

cudaError_t launch_image_table(const ModelView &m, int64_t nboundary, const int64_t *b2c,
                               const double *grid, int nf, double *table, cudaStream_t s);
cudaError_t launch_image(const ModelView &m, const ImageArgs &a, DevFlags *flags, cudaStream_t s);

// acc[0] = points of all traces, acc[1] = sum over (pair, origin) of ndep
// where ndep > 1 for origins in [u_begin, u_end), acc[2] = the longest ray
// pair (points); pts_origin[N] and
// upd_origin[N] (updates of one formal solve per origin) when not null.
cudaError_t launch_trace_stats(const ModelView &m, const int32_t *len, unsigned long long *acc,
                               int32_t *pts_origin, float *upd_origin, int64_t u_begin,
                               int64_t u_end, cudaStream_t s);

struct SolveArgs {
    const double *eps, *kap;        // [N*K] emissivity, opacity (FP64 path)
    const float2 *ehat_khat;        // [N*K] scaled (mixed path)
    double mixed_scale;             // power of two applied to Ehat/Khat
    double *Jlin, *Lam;             // [N*K]
    double *J;                      // [N*nfreqs] or null
    int warps_per_block;
    int4 *patch;                    // mixed: (origin, pair, bin) to redo in double
    unsigned long long *patch_count;
    int64_t patch_cap;
    int64_t s_begin, s_end;         // origins of the trace store to solve: [s_begin, s_end)
    const int32_t *olist;           // when set: solve origins olist[s_begin .. s_end) instead
    int32_t *redo_flag;             // [N] mixed: 1 once an origin is listed for an FP64 re-solve
    int32_t *redo_list;             // [N] mixed: origins whose failures overflowed the patch list
    const float *bcache;            // staged mixed solve: far-end boundary intensities of the
                                    // trace store, [o_count][npairs][2][nfreqs] (launch_bdy_cache)
};
// Formal solve of the origins of one trace store.  variant selects the
// register budget (one of kSolveVariants compiled resident-block counts;
// < 0: the default); *kind receives 1 when the staged mixed kernel ran.
constexpr int kSolveVariants = 3;
cudaError_t launch_formal_solve(const ModelView &m, const TraceView &t, const SolveArgs &a,
                                int precision, int variant, DevFlags *flags, cudaStream_t s,
                                int *kind);
int solve_variant_blocks(int variant);
// True when a solve of this model runs the staged kernels (no overlapping
// lines, 31+ bins per line): the mixed one reads SolveArgs::bcache.
bool solve_is_staged(const ModelView &m);
// Fills cache[(oi * npairs + r) * 2 + h][f] for the origins [s_begin,
// s_end) of trace store t: the boundary intensity at the far end of half h
// (0: the longer one) of pair r, at bin f's frequency Doppler-shifted there.
cudaError_t launch_bdy_cache(const ModelView &m, const TraceView &t, int64_t s_begin,
                             int64_t s_end, float *cache, DevFlags *flags, cudaStream_t s);

struct LevelArgs {
    double *pop, *prev1, *prev2, *prev3;   // [N*nlev]
    double *eps, *kap;                     // [N*K]
    float2 *ehat_khat;                     // [N*K]
    double mixed_scale;
    double *Jlin, *Lam, *Jeff;             // [N*K]
    double *partials;                      // reduction scratch
    double *stats;                         // [8] device results
    int npartials;
    int64_t c_begin, c_end;                // cells whose Jeff and rate equations are solved
};
cudaError_t launch_lte(const ModelView &m, const LevelArgs &a, cudaStream_t s);
cudaError_t launch_boundary_table(const ModelView &m, int64_t nboundary, const int64_t *b2c,
                                  double *table, cudaStream_t s);
cudaError_t launch_emissivity_opacity(const ModelView &m, const LevelArgs &a, cudaStream_t s);
cudaError_t launch_jeff(const ModelView &m, const LevelArgs &a, cudaStream_t s);
// Statistical equilibrium of cells [c_begin, c_end) (their convergence
// partials at the global positions of their 4-cell blocks); the history of
// the other cells is shifted as well.  With the whole cell range the
// convergence statistics are reduced too; otherwise launch_convergence_final
// reduces them once every shard's partials are in place.
cudaError_t launch_stateq(const ModelView &m, const LevelArgs &a, DevFlags *flags, cudaStream_t s);
cudaError_t launch_convergence_final(const ModelView &m, const LevelArgs &a, cudaStream_t s);

// Non-local ALO (n_off_diag = M1 + 1 >= 2).  Element (o, k, r, side, d) of
// cell o, line k, ray pair r, side 0 (front trace) or 1 (back trace) at
// distance d = 1..M1 from the origin: Loff[(((o*K + k)*npairs + r)*2 +
// side)*M1 + d-1], belonging to cell Loff_nr[((o*npairs + r)*2 + side)*M1 +
// d-1] (-1: the pair has no point there).
struct NonlocalArgs {
    const double *Loff;
    const int32_t *Loff_nr;
    int M1;
    const double *x_in;   // [N*nlev] populations the couplings between cells use
    double *x_out;        // [N*nlev] solution of the sweep
    double *change;       // [nonlocal_sweep_blocks + 1]: per block, then the max
};
struct OffdiagArgs {
    const double *eps, *kap;   // [N*K]
    double *Loff;
    int32_t *Loff_nr;
    int M1;
    int64_t s_begin, s_end;    // origins of the trace store
};
constexpr int kMaxOffDiag = 8;   // n_off_diag accepted: 0 .. kMaxOffDiag
cudaError_t launch_offdiag(const ModelView &m, const TraceView &t, const OffdiagArgs &a,
                           DevFlags *flags, cudaStream_t s);
cudaError_t launch_jeff_nonlocal(const ModelView &m, const LevelArgs &a, const NonlocalArgs &nl,
                                 cudaStream_t s);
// prev3 <- prev2 <- prev1 <- pop for every cell
cudaError_t launch_history_shift(const ModelView &m, const LevelArgs &a, cudaStream_t s);
int nonlocal_sweep_blocks(const ModelView &m);
// One block-Jacobi sweep x_in -> x_out and the max change into
// change[nonlocal_sweep_blocks].
cudaError_t launch_stateq_nonlocal_sweep(const ModelView &m, const LevelArgs &a,
                                         const NonlocalArgs &nl, DevFlags *flags, cudaStream_t s);
constexpr int kCellsPerPartial = 4;   // cells per convergence partial of launch_stateq
cudaError_t launch_convergence(const ModelView &m, const LevelArgs &a, cudaStream_t s);
cudaError_t launch_ng(const ModelView &m, const LevelArgs &a, cudaStream_t s);
int level_partials_needed(const ModelView &m);
// Per-model convergence statistics (3 per model: fraction not converged,
// mean and max relative change) and per-model Ng steps, for batches.
cudaError_t launch_seg_convergence(const ModelView &m, const LevelArgs &a, double *seg_stats,
                                   cudaStream_t s);
cudaError_t launch_seg_ng(const ModelView &m, const LevelArgs &a, cudaStream_t s);

// Warm-start network on the device (pointers into one parameter buffer).
struct MlpDevice {
    int nin, nout;
    float *W[4], *b[4];
    float *mean, *istd;
};
struct MlpGrad {
    float *W[4], *b[4];
};
size_t mlp_smem_bytes(bool train);
cudaError_t mlp_prepare();
cudaError_t launch_mlp_forward(const MlpDevice &d, const float *X, int64_t n, float *out,
                               cudaStream_t s);
cudaError_t launch_mlp_train_batch(const MlpDevice &d, const MlpGrad &g, const float *X,
                                   const float *lte, const float *tgt, const int *idx, int64_t b0,
                                   int64_t bn, float scale, float *loss, cudaStream_t s);
cudaError_t launch_adam(float *p, const float *g, float *m, float *v, int64_t n, float lr,
                        float b1, float b2, int step, float eps, float wd, cudaStream_t s);
cudaError_t launch_features(const ModelView &m, const TraceView &t, float *F, cudaStream_t s);
cudaError_t launch_lte_logfrac(const ModelView &m, int64_t o0, int64_t cnt, float *L, cudaStream_t s);
cudaError_t launch_warm_populations(const ModelView &m, int64_t o0, int64_t cnt, const float *L,
                                    const float *D, double *pop, cudaStream_t s);
// parameter layout: W0,b0,W1,b1,W2,b2,W3,b3
int64_t mlp_param_count(int nin, int nout);
void mlp_bind(float *base, int nin, int nout, float **W, float **b);

}  // namespace mgr
