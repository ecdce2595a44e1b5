// solve.cu -- Feautrier formal solve over all ray pairs and frequency bins.
//
// Work decomposition: one warp per origin cell.  The warp loops over
// 32-bin chunks of the frequency grid (lane = bin) and, inside a chunk, over
// the ray pairs in the reference's order (r = 0 .. nrays/2-1), so that J at
// a bin is summed over pairs in the same order as
// Simulation::compute_radiation_field (Simulation/sim_radiation.tpp:130-220)
// without atomics.  Every lane of the warp walks the same traced points, so
// point records are broadcast loads.
//
// Per (pair, origin, bin) the lane evaluates emissivity and opacity along
// the ray (Simulation::setup / get_eta_and_chi, simulation.tpp:185-481) and
// solves the second-order Feautrier system in Rybicki-Hummer form
// (RayPair::solve, raypair_solver.tpp:200-334).  Instead of eliminating the
// whole ray and substituting back, the front half is eliminated from its far
// end toward the origin and the back half from its far end toward the
// origin; the two meet in the origin's row:
//     u_o  = (S_o + A_o Su_{o-1} + C_o Sb_{o+1}) / (1 + A_o F'_{o-1} + C_o G'_{o+1})
//     L_oo =                                   1 / (1 + A_o F'_{o-1} + C_o G'_{o+1})
// with F' = F/(1+F), G' = G/(1+G) the reference's F and G.  This is the
// same linear system and the same diagonal ALO element (the reference's
// L_diag[n_ar] = inv_C/(F + G/(1+G))), with O(1) state per lane.  The
// elimination runs on half optical depths in projective form (F'/2 = a/b,
// S/2 = c/b), so a step toward the origin needs no division:
//     H = dh_far + dh_near, P = H dh_far, Q = H dh_near, Pb = P b,
//     a <- Q (Pb + a),  c <- Q (t Pb + c),  b <- Pb + 2a
// with a power-of-two rescaling of (a, b, c); the two halves are
// independent chains that a lane advances together for instruction-level
// parallelism, and one division per (pair, bin) joins them at the origin.
//
// Kernels: the staged kernels (lines whose windows do not overlap, 31 or
// more bins per line, FP64 or mixed) stage each ray pair's points window by
// window in shared memory; the generic kernel reads them from the trace
// store and handles overlapping lines.
//
// Precision policies:
//   FP64  every quantity in double, as the reference.
//   MIXED opacity, emissivity, source function and optical-depth increment
//         in float, in dimensionless form (frequency offsets in Doppler
//         widths relative to the line, opacities scaled by a power of two
//         X); the elimination, u, the ALO and all accumulations in double.
//
// Outputs per origin: the line integrals Jlin[o][k] = sum_z w_z J[o][k,z]
// (Simulation::compute_Jeff, sim_lines.tpp:185-198) and the diagonal ALO
// Lam[o][k] (RayPair::update_Lambda, raypair_lambda.tpp:94-149), both
// reduced over the bins of a line with warp shuffles; optionally J itself.
#include <type_traits>

#include "mgr_internal.cuh"

namespace mgr {

namespace {

constexpr int kWarpsPerBlock = 4;
// Resident blocks per SM each solve kernel is compiled for (its register
// budget): the autotuner's candidates.  Defaults when not tuning: 7 for the
// generic and the staged FP64 kernels, 8 for the staged mixed one (measured
// best on the 64^3 wind).
constexpr int kVariantBlocks[kSolveVariants] = {6, 7, 8};
constexpr int kDefaultGeneric = 1, kDefaultStaged = 2, kDefaultStaged64 = 1;

// 1/x for normal x of either sign: hardware estimate refined by two Newton-Raphson
// steps y <- y (2 - x y) (accurate to about one ulp).
__device__ __forceinline__ double rcp_pos(double x) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    double e = fma(-x, y, 1.0);
    y = fma(y, e, y);
    e = fma(-x, y, 1.0);
    return fma(y, e, y);
}

// Per-lane constants of one bin at one origin.
struct BinCtx {
    double nu_o;      // bin frequency at the origin (sim_spectrum.tpp:37-41)
    int k;            // line of the bin
    int lo, hi;       // lines whose +-11-width window can reach this bin
    int f;            // the bin
    float q;          // pw_o * root_z: offset of the bin from its line, in units of nu
};

// ---------------------------------------------------------------- policies

template <bool kOverlap>
struct Fp64Policy {
    using Real = double;
    static constexpr bool kFallback = false;
    struct Pt {
        int cell;
        double shift, dz;
    };
    const int32_t *cell;
    const double *shift, *dZ;
    const double *eps, *kap;

    __device__ __forceinline__ Pt load(int64_t i) const {
        Pt p;
        p.cell = __ldg(cell + i);
        p.shift = __ldg(shift + i);
        p.dz = __ldg(dZ + i);
        return p;
    }
    __device__ __forceinline__ double freq(const Pt &p, const BinCtx &b) const {
        return p.shift * b.nu_o;
    }
    // Without overlapping profiles the window holds the bin's own line only.
    __device__ __forceinline__ void eval(const ModelView &m, int p, double freq, const BinCtx &b,
                                         double &chi, double &t) const {
        double eta;
        eta_chi_double(m, eps, kap, p, freq, kOverlap ? b.lo : b.k, kOverlap ? b.hi : b.k, eta, chi);
        t = eta * rcp_pos(chi);
    }
    __device__ __forceinline__ void eval_pt(const ModelView &m, const Pt &p, const BinCtx &b,
                                            double &chi, double &t) const {
        eval(m, p.cell, freq(p, b), b, chi, t);
    }
    __device__ __forceinline__ static double dtau(double chi_a, double chi_b, double dz) {
        return 0.5 * (chi_a + chi_b) * dz;
    }
    __device__ __forceinline__ static double dz_of(const Pt &p) { return p.dz; }
    // origin: opacity, source function and the opacity in physical units
    __device__ __forceinline__ void origin(const ModelView &m, int o, const BinCtx &b,
                                           double &chi, double &t, double &chi_phys) const {
        eval(m, o, b.nu_o, b, chi, t);
        chi_phys = chi;
    }
};

template <bool kOverlap>
struct MixedPolicy {
    using Real = float;
    static constexpr bool kFallback = true;   // redo non-finite pairs in double
    using Pt = MixedPoint;
    const MixedPoint *mp;
    const float2 *ek;         // [N*K] (eps, kap) * INVSQRTPI / pw * X
    float floor_hat;          // 1e-26 * X
    double inv_scale;         // 1 / X
    const double *eps, *kap;  // for lines other than the bin's own

    __device__ __forceinline__ Pt load(int64_t i) const {
        const float4 v = __ldg(reinterpret_cast<const float4 *>(mp) + i);
        Pt p;
        p.cell = __float_as_int(v.x);
        p.delta = v.y;
        p.dzs = v.z;
        p.ipw = v.w;
        return p;
    }
    __device__ __forceinline__ double freq(const Pt &p, const BinCtx &b) const {
        return (1.0 + (double)p.delta) * b.nu_o;
    }
    // Scaled opacity and source function.  For the bin's own line,
    // x = ((1+delta)(1+q) - 1) / pw_p and nu/line = (1+delta)(1+q), so
    // chi X = 1e-26 X + Khat (nu/line) exp(-x^2), zero outside +-11 widths;
    // other lines in the window (overlapping profiles) come from the double
    // tables.
    __device__ __forceinline__ void eval_pt(const ModelView &m, const Pt &p, const BinCtx &b,
                                            float &chi, float &t) const {
        const float off = fmaf(p.delta, b.q, p.delta + b.q);   // (1+d)(1+q) - 1
        const float x = off * p.ipw;
        const float r = 1.0f + off;
        const int K = m.nrad;
        const float2 e = __ldg(ek + (unsigned)p.cell * K + b.k);
        const float g = fabsf(x) <= 11.0f ? r * __expf(-x * x) : 0.0f;
        float eta = e.x * g;
        chi = fmaf(e.y, g, floor_hat);
        if (kOverlap && b.lo != b.hi) {
            const double fr = freq(p, b);
            const double pwp = __ldg(m.pw + p.cell);
            const double ipw = __ldg(m.inv_pw + p.cell);
            double ea = 0.0, ca = 0.0;
            for (int l = b.lo; l <= b.hi; l++) {
                if (l == b.k) continue;
                const double line_l = __ldg(m.line + l);
                const double width = line_l * pwp;
                const double diff = fr - line_l;
                if (diff <= 11.0 * width && diff >= -11.0 * width) {
                    const double inv_w = __ldg(m.inv_line + l) * ipw;
                    const double xx = inv_w * diff;
                    const double fp = fr * (inv_w * kINVERSE_SQRT_PI * exp(-(xx * xx)));
                    ea += __ldg(eps + (unsigned)p.cell * K + l) * fp;
                    ca += __ldg(kap + (unsigned)p.cell * K + l) * fp;
                }
            }
            eta += (float)(ea * m.mixed_scale);
            chi += (float)(ca * m.mixed_scale);
        }
        // Negative line opacity (population inversion, which the
        // reference's iteration allows) that takes chi below half the floor
        // cancels badly in float: such a point poisons its pair with a NaN
        // source function, and the pair is solved again in double by the
        // patch pass.  Above half the floor the float sum loses at most a
        // factor two of relative precision.
        if (chi < 0.5f * floor_hat) eta = __int_as_float(0x7fc00000);
        t = __fdividef(eta, chi);
    }
    __device__ __forceinline__ static double dtau(float chi_a, float chi_b, float dzs) {
        return (double)((chi_a + chi_b) * dzs);
    }
    __device__ __forceinline__ static float dz_of(const Pt &p) { return p.dzs; }
    // origin: evaluated in double once per chunk (it enters every pair and
    // the ALO), then scaled to the float units of the chains
    __device__ __forceinline__ void origin(const ModelView &m, int o, const BinCtx &b,
                                           float &chi, float &t, double &chi_phys) const {
        double e64, c64;
        eta_chi_double(m, eps, kap, o, b.nu_o, kOverlap ? b.lo : b.k, kOverlap ? b.hi : b.k, e64, c64);
        chi = (float)(c64 * m.mixed_scale);
        t = (float)(e64 / c64);
        chi_phys = c64;
    }
};

// ------------------------------------------------------------------ chains

// 2^-e for the binary exponent e of b > 0 (a normal double), built from the
// exponent field: multiplying by it brings b into [1, 2) exactly.
__device__ __forceinline__ double pow2_recip_scale(double b) {
    const int hi = __double2hiint(b);
    return __hiloint2double(0x7fe00000 - (hi & 0x7ff00000), 0);
}

// Elimination of one half of the ray pair from its far end toward the
// origin, on half optical depths dh = dtau/2 in projective form: the scaled
// Rybicki-Hummer quantities are F~ = a/b and S~ = c/b (F~ = F'/2, S~ = S/2
// for the reference's F' = F/(1+F) and S), and one step toward the origin is
//     H = dh_far + dh_near, P = H dh_far, Q = H dh_near, Pb = P b,
//     a <- Q (Pb + a),  c <- Q (t Pb + c),  b <- Pb + 2a
// which is F~ <- w/(P + 2w), S~ <- (t P + S~) Q/(P + 2w) with
// w = Q (P + F~), multiplied through by b: no division per point.  For
// non-negative opacities every term is non-negative.  a, b, c are brought
// back to b in [1, 2) by a power of two after each step.
template <class Pol>
struct Chain {
    using Real = typename Pol::Real;
    Real chi_a, t_a;      // current point
    Real dz_a;            // its increment toward the origin (policy units)
    double dh_prev, a, b, c;

    // boundary row of the far end: F~ = dh(dh+1)/(2dh(dh+1)+1),
    // S~ = dh(t dh + I)/(2dh(dh+1)+1)
    __device__ __forceinline__ void first(Real chi_b, Real t_b, Real dz_b, double I) {
        const double dh = 0.5 * Pol::dtau(chi_a, chi_b, dz_a);
        a = dh * (dh + 1.0);
        b = fma(2.0, a, 1.0);
        c = dh * fma((double)t_a, dh, I);
        dh_prev = dh;
        chi_a = chi_b;
        t_a = t_b;
        dz_a = dz_b;
    }
    __device__ __forceinline__ void step(Real chi_b, Real t_b, Real dz_b) {
        const double dh = 0.5 * Pol::dtau(chi_a, chi_b, dz_a);
        const double H = dh_prev + dh;
        const double P = H * dh_prev, Q = H * dh;
        const double Pb = P * b;
        a = Q * (Pb + a);
        c = Q * fma((double)t_a, Pb, c);
        b = fma(2.0, a, Pb);
        const double sc = pow2_recip_scale(b);
        a *= sc;
        b *= sc;
        c *= sc;
        dh_prev = dh;
        chi_a = chi_b;
        t_a = t_b;
        dz_a = dz_b;
    }
};

// u and L at the origin for one ray pair.  The front half has nfr >= 1
// points (far end first at index nfr-1), the back half nbk >= 0; both are
// eliminated toward the origin in lock step while both have points left.
template <class Pol>
__device__ __forceinline__ void sweep(const ModelView &m, const Pol &pol, const BinCtx &b,
                                      int64_t ofr, int nfr, int64_t obk, int nbk,
                                      typename Pol::Real chi_o, typename Pol::Real t_o,
                                      int origin, DevFlags *flags, double &u, double &L) {
    using Real = typename Pol::Real;
    Chain<Pol> fr, bk;
    const BdyCtx bc = bdy_ctx(m);
    Real chi, t;
    // front: far end, boundary value, first (boundary-row) step
    double I0;
    {
        const auto p = pol.load(ofr + nfr - 1);
        pol.eval_pt(m, p, b, chi, t);
        fr.chi_a = chi; fr.t_a = t; fr.dz_a = Pol::dz_of(p);
        I0 = boundary_intensity(bc, pol.freq(p, b), p.cell, flags, b.k);
    }
    if (nfr >= 2) {
        const auto p = pol.load(ofr + nfr - 2);
        pol.eval_pt(m, p, b, chi, t);
        fr.first(chi, t, Pol::dz_of(p), I0);
    } else {
        fr.first(chi_o, t_o, Real(0), I0);
    }
    double In = 0.0;
    if (nbk > 0) {
        const auto p = pol.load(obk + nbk - 1);
        pol.eval_pt(m, p, b, chi, t);
        bk.chi_a = chi; bk.t_a = t; bk.dz_a = Pol::dz_of(p);
        In = boundary_intensity(bc, pol.freq(p, b), p.cell, flags, b.k);
        if (nbk >= 2) {
            const auto q = pol.load(obk + nbk - 2);
            pol.eval_pt(m, q, b, chi, t);
            bk.first(chi, t, Pol::dz_of(q), In);
        } else {
            bk.first(chi_o, t_o, Real(0), In);
        }
    } else {
        const int bo = __ldg(m.cell2bdy + origin);
        if (bo >= 0) In = __ldg(m.ibdy + (int64_t)bo * m.nfreqs + b.f);
        else atomicAdd(&flags->trace_err, 1ull);
    }
    // both halves have interior points
    int s = 2;
    for (; s < nbk; s++) {
        const auto p = pol.load(ofr + nfr - 1 - s);
        const auto q = pol.load(obk + nbk - 1 - s);
        Real chi_p, t_p, chi_q, t_q;
        pol.eval_pt(m, p, b, chi_p, t_p);
        pol.eval_pt(m, q, b, chi_q, t_q);
        fr.step(chi_p, t_p, Pol::dz_of(p));
        bk.step(chi_q, t_q, Pol::dz_of(q));
    }
    if (nbk >= 2) bk.step(chi_o, t_o, Real(0));
    // the rest of the front half
    for (; s < nfr; s++) {
        const auto p = pol.load(ofr + nfr - 1 - s);
        pol.eval_pt(m, p, b, chi, t);
        fr.step(chi, t, Pol::dz_of(p));
    }
    if (nfr >= 2) fr.step(chi_o, t_o, Real(0));

    const double to = (double)t_o;
    if (nbk == 0) {
        // the origin is the last row: u = (dh (t dh + In) + S~)/(dh (dh + 1) + F~)
        const double dh = fr.dh_prev;
        const double D = rcp_pos(fma(dh * (dh + 1.0), fr.b, fr.a));
        u = fma(dh * fma(to, dh, In), fr.b, fr.c) * D;
        L = dh * dh * fr.b * D;
        return;
    }
    // origin row: u = (t PQ + S~f Q + S~b P)/(F~f Q + F~b P + PQ), times bf bb
    const double H = fr.dh_prev + bk.dh_prev;
    const double P = H * fr.dh_prev, Q = H * bk.dh_prev;
    const double PQB = P * Q * (fr.b * bk.b);
    const double D = rcp_pos(fma(fr.a * bk.b, Q, fma(bk.a * fr.b, P, PQB)));
    u = fma(to, PQB, fma(fr.c * bk.b, Q, bk.c * fr.b * P)) * D;
    L = PQB * D;
}

// Patch pass of the mixed solve: (origin, pair, bin) entries whose float
// sweep produced a non-finite u or L (near-zero or negative opacities from
// transient population inversion, where float runs out of range) are
// solved again in double, one thread per entry, and added to the outputs.
__device__ __noinline__ void patch_entry(const ModelView &m, const TraceView &t, const SolveArgs &a,
                                         DevFlags *flags, int4 e) {
    const int o = e.x, r = e.y, f = e.z;
    const int64_t oi = o - t.o_begin;
    const int nq = m.nquads, nf = m.nfreqs, K = m.nrad;
    BinCtx b;
    b.f = f;
    b.k = f / nq;
    const int z = f - b.k * nq;
    b.lo = m.win_lo[b.k];
    b.hi = m.win_hi[b.k];
    const double line_k = m.line[b.k];
    const double pw_o = m.pw[o];
    b.nu_o = radd(line_k, rmul(rmul(line_k, pw_o), m.roots[z]));
    b.q = (float)(pw_o * m.roots[z]);
    const int ar = m.antipod[r];
    const int64_t ir = (int64_t)r * t.o_count + oi, iar = (int64_t)ar * t.o_count + oi;
    const int nr_ = t.len[ir], nar_ = t.len[iar];
    const bool rfront = nr_ > nar_;
    Fp64Policy<true> pol;
    pol.cell = t.cell;
    pol.shift = t.shift;
    pol.dZ = t.dZ;
    pol.eps = a.eps;
    pol.kap = a.kap;
    double chi_o, t_o, chi_phys;
    pol.origin(m, o, b, chi_o, t_o, chi_phys);
    double u, L;
    sweep<Fp64Policy<true>>(m, pol, b, rfront ? t.off[ir] : t.off[iar], rfront ? nr_ : nar_,
                            rfront ? t.off[iar] : t.off[ir], rfront ? nar_ : nr_, chi_o, t_o, o,
                            flags, u, L);
    const double wr = m.ray_w[r];
    const double width_o = line_k * pw_o;
    const double iw = 1.0 / width_o;
    const double xo = iw * (b.nu_o - line_k);
    const double prof_o = iw * kINVERSE_SQRT_PI * exp(-(xo * xo));
    const double lam_pre = m.A[b.k] * (m.qw[z] * 2.0) * (b.nu_o * prof_o / chi_phys);
    atomicAdd(a.Jlin + (int64_t)o * K + b.k, m.qw[z] * (2.0 * wr * u));
    atomicAdd(a.Lam + (int64_t)o * K + b.k, lam_pre * wr * L);
    if (a.J) atomicAdd(a.J + (int64_t)o * nf + f, 2.0 * wr * u);
}

// More float failures than the patch list holds: the origin is listed
// (once) to be solved again entirely in double after the patch pass.
__device__ __forceinline__ void list_for_redo(const SolveArgs &a, DevFlags *flags, int o) {
    atomicAdd(&flags->patch_overflow, 1ull);
    if (atomicExch(a.redo_flag + o, 1) == 0) {
        const unsigned long long i = atomicAdd(&flags->redo_count, 1ull);
        a.redo_list[i] = o;
    }
}

__global__ void patch_kernel(ModelView m, TraceView t, SolveArgs a, DevFlags *flags) {
    const int64_t n = min((unsigned long long)*a.patch_count, (unsigned long long)a.patch_cap);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        patch_entry(m, t, a, flags, a.patch[i]);
}

template <class Pol, int kMinBlocks>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, kMinBlocks)
    formal_solve_kernel(ModelView m, TraceView t, SolveArgs a, Pol pol, DevFlags *flags) {
    using Real = typename Pol::Real;
    extern __shared__ double smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t idx = a.s_begin + (int64_t)blockIdx.x * kWarpsPerBlock + warp;
    if (idx >= a.s_end) return;
    const int64_t oi = a.olist ? (int64_t)a.olist[idx] - t.o_begin : idx;
    const int o = (int)(t.o_begin + oi);
    if (m.seg_active && !m.seg_active[m.cell_seg[o]]) return;   // converged model of a batch
    const int K = m.nrad, nq = m.nquads, nf = m.nfreqs;
    double *sJ = smem + (size_t)warp * 2 * K;
    double *sL = sJ + K;
    for (int k = lane; k < K; k += 32) { sJ[k] = 0.0; sL[k] = 0.0; }
    __syncwarp();

    const double pw_o = m.pw[o];
    const int nchunks = (nf + 31) >> 5;
    for (int c = 0; c < nchunks; c++) {
        const int f = c * 32 + lane;
        const bool active = f < nf;
        const int fc = active ? f : nf - 1;
        BinCtx b;
        b.f = fc;
        b.k = fc / nq;
        const int z = fc - b.k * nq;
        b.lo = m.win_lo[b.k];
        b.hi = m.win_hi[b.k];
        const double line_k = m.line[b.k];
        const double root = m.roots[z];
        b.nu_o = radd(line_k, rmul(rmul(line_k, pw_o), root));
        b.q = (float)(pw_o * root);

        // origin: same opacity and source for every pair
        Real chi_o, t_o;
        double chi_o_d;
        pol.origin(m, o, b, chi_o, t_o, chi_o_d);
        // ALO factor without the pair weight (raypair_lambda.tpp:26-29, :115-121)
        const double width_o = line_k * pw_o;
        const double iw = 1.0 / width_o;
        const double xo = iw * (b.nu_o - line_k);
        const double prof_o = iw * kINVERSE_SQRT_PI * exp(-(xo * xo));
        const double lam_pre = m.A[b.k] * (m.qw[z] * 2.0) * (b.nu_o * prof_o / chi_o_d);

        double Jf = 0.0, Lf = 0.0;
        for (int r = 0; r < m.npairs; r++) {
            const int ar = m.antipod[r];
            const double wr = m.ray_w[r];
            const int64_t ir = (int64_t)r * t.o_count + oi;
            const int64_t iar = (int64_t)ar * t.o_count + oi;
            const int nr_ = t.len[ir], nar_ = t.len[iar];
            // the longer trace is the front half (sim_radiation.tpp:164-171)
            const bool rfront = nr_ > nar_;
            const int64_t ofr = rfront ? t.off[ir] : t.off[iar];
            const int64_t obk = rfront ? t.off[iar] : t.off[ir];
            const int nfr = rfront ? nr_ : nar_;
            const int nbk = rfront ? nar_ : nr_;
            if (nfr == 0) {
                // only the origin on the ray pair: J += 2 w I_bdy (sim_radiation.tpp:243-264)
                const int bo = m.cell2bdy[o];
                double I = 0.0;
                if (bo >= 0) I = m.ibdy[(int64_t)bo * nf + fc];
                else if (lane == 0) atomicAdd(&flags->trace_err, 1ull);
                Jf += 2.0 * wr * (0.5 * (I + I));
                continue;
            }
            double u, L;
            sweep<Pol>(m, pol, b, ofr, nfr, obk, nbk, chi_o, t_o, o, flags, u, L);
            if (Pol::kFallback && !(isfinite(u) && isfinite(L))) {
                // leave this pair to the double-precision patch pass
                const unsigned long long slot = atomicAdd(a.patch_count, 1ull);
                if (slot < (unsigned long long)a.patch_cap) a.patch[slot] = make_int4(o, r, fc, 0);
                else list_for_redo(a, flags, o);
                continue;
            }
            Jf += 2.0 * wr * u;
            Lf += lam_pre * wr * L;
        }
        if (a.J && active) a.J[(int64_t)o * nf + f] = Jf;

        // line integrals over the bins of this chunk
        const double jw = active ? m.qw[z] * Jf : 0.0;
        const double lw = active ? Lf : 0.0;
        const int kfirst = (c * 32) / nq;
        const int klast = min(K - 1, (c * 32 + 31) / nq);
        for (int kk = kfirst; kk <= klast; kk++) {
            double vj = (active && b.k == kk) ? jw : 0.0;
            double vl = (active && b.k == kk) ? lw : 0.0;
#pragma unroll
            for (int s = 16; s > 0; s >>= 1) {
                vj += __shfl_xor_sync(0xffffffffu, vj, s);
                vl += __shfl_xor_sync(0xffffffffu, vl, s);
            }
            if (lane == 0) { sJ[kk] += vj; sL[kk] += vl; }
        }
        __syncwarp();
    }
    for (int k = lane; k < K; k += 32) {
        a.Jlin[(int64_t)o * K + k] = sJ[k];
        a.Lam[(int64_t)o * K + k] = sL[k];
    }
}

// ------------------------------------------------------------------ staged mixed solve
//
// The mixed solve with the points of each (ray pair, chunk) staged in
// shared memory.  The warp first gathers every point's record and the
// scaled opacities of the chunk's (at most two) lines with parallel loads,
// then each lane runs its serial elimination on shared memory only.  Used
// when the lines' windows do not overlap, every 32-bin chunk spans at most
// two lines (31 or more bins per line) and ray pairs fit the buffer.
//
// The elimination runs on half optical depths dh = dtau/2 with F~ = F'/2,
// S~ = S/2, which removes constant factors from the step:
//     H = dh_far + dh_near, P = H dh_far, Q = H dh_near,
//     w = Q (P + F~), D = 1/(P + 2w), F~ <- w D, S~ <- (t P + S~) Q D
// (the same recursion as the generic sweep with p = 2P, q = 2Q).  The
// boundary row becomes D = 1/(2dh(dh+1)+1), F~ = dh(dh+1)D, S~ = dh(t dh+I)D
// and the origin row u = (t PQ + S~f Q + S~b P)/(F~f Q + F~b P + PQ),
// L = PQ/(...) with P, Q built from the two segments at the origin.

// One traced point of the staged pair: the float record and the opacity
// pairs (eps, kap) * INVSQRTPI / pw * X of the chunk's two lines.
struct __align__(16) StagedPt {
    float delta;   // Doppler shift - 1
    float dzh;     // dZ / (4 X): dh = (chi_a + chi_b) * dzh for chi scaled by X
    float ipws;    // sqrt(log2 e) / profile width
    int cell;
    float2 e[2];
};

__device__ __forceinline__ float ex2_approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float rcp_approx(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Scaled opacity and source function of a staged point for a lane whose
// bin sits q = pw_o * root widths from its line: with off = nu/line - 1,
// chi X = 1e-26 X + Khat (1 + off) 2^-(off ipws)^2, the profile vanishing
// (flushed to zero) beyond ~9.3 widths, inside the reference's 11-width cut.
// kCheck (windows holding a strongly inverted line): a chi below half the
// floor at this bin poisons the pair with a NaN source function.
template <bool kCheck>
__device__ __forceinline__ void staged_eval(const StagedPt *p, int eo, float q, float floor_hat,
                                            float &chi, float &t) {
    const float4 r = *reinterpret_cast<const float4 *>(p);
    const float2 e = reinterpret_cast<const float2 *>(p)[eo];
    const float off = fmaf(r.x, q, r.x + q);
    const float x = off * r.z;
    const float g = ex2_approx(-x * x);
    const float rg = fmaf(off, g, g);
    chi = fmaf(e.y, rg, floor_hat);
    t = e.x * rg * rcp_approx(chi);
    if (kCheck && chi < 0.5f * floor_hat) t = __int_as_float(0x7fc00000);
}


// Scaled Rybicki-Hummer state in projective form: F~ = a/b, S~ = c/b.  A
// step then needs no division:
//     X = dh' b,  Pb = H X,  a <- dh (Pb + a),  b <- X + 2a,  c <- dh (t Pb + c)
// with dh' the previous half optical depth and H = dh' + dh (from
// F~ <- w/(P + 2w), w = Q (P + F~), and S~ <- (t P + S~) Q/(P + 2w), where
// P = H dh' and Q = H dh, multiplied through by b/H).  Every term is
// non-negative for non-negative opacities, so nothing cancels; per step b
// shrinks by at most dh' and grows by at most about 4 dh^3, and a, b, c are
// rescaled by a power of two every few steps, which keeps them in range for
// any optical depth.
// R is the type of the staged point values (float in mixed precision,
// double in FP64); the elimination itself is always double.
template <class R>
struct ProjChainT {
    R chi_a, t_a, dzh_a;   // current point
    double dh_prev, a, b, c;

    __device__ __forceinline__ void start(R chi, R t, R dzh) {
        chi_a = chi; t_a = t; dzh_a = dzh;
    }
    // boundary row of the far end: F~ = dh(dh+1)/(2dh(dh+1)+1),
    // S~ = dh(t dh + I)/(2dh(dh+1)+1)
    __device__ __forceinline__ void first(R chi_b, R t_b, R dzh_b, double I) {
        const double dh = (double)((chi_a + chi_b) * dzh_a);
        a = dh * (dh + 1.0);
        b = fma(2.0, a, 1.0);
        c = dh * fma((double)t_a, dh, I);
        dh_prev = dh;
        chi_a = chi_b; t_a = t_b; dzh_a = dzh_b;
    }
    __device__ __forceinline__ void step(R chi_b, R t_b, R dzh_b) {
        const double dh = (double)((chi_a + chi_b) * dzh_a);
        const double H = dh_prev + dh;
        const double X = dh_prev * b;
        const double Pb = H * X;
        a = dh * (Pb + a);
        c = dh * fma((double)t_a, Pb, c);
        b = fma(2.0, a, X);
        dh_prev = dh;
        chi_a = chi_b; t_a = t_b; dzh_a = dzh_b;
    }
    __device__ __forceinline__ void renorm() {
        const double sc = pow2_recip_scale(b);
        a *= sc; b *= sc; c *= sc;
    }
};
using ProjChain = ProjChainT<float>;

// Steps of the sweep held in shared memory at a time (per half).
#ifndef MGR_STAGE_STEPS
#define MGR_STAGE_STEPS 64
#endif
constexpr int kStageSteps = MGR_STAGE_STEPS;

// The sweep steps [s0, s1) of one staged window (front step s at F[s], back
// step s at B[s]).
// I0 and In are the boundary intensities at the two far ends.
template <bool kCheck>
__device__ __forceinline__ void staged_window(const StagedPt *F, const StagedPt *B, int s0, int s1,
                                              int nbk, int eo, float q, float floor_hat,
                                              ProjChain &fr, ProjChain &bk, double I0, double In) {
    float chi, t_, chi2, t2;
    int s = s0;
    if (s == 0) {
        staged_eval<kCheck>(F, eo, q, floor_hat, chi, t_);
        fr.start(chi, t_, F->dzh);
        if (nbk > 0) {
            staged_eval<kCheck>(B, eo, q, floor_hat, chi, t_);
            bk.start(chi, t_, B->dzh);
        }
        s = 1;
    }
    if (s == 1 && s < s1) {
        staged_eval<kCheck>(F + 1, eo, q, floor_hat, chi, t_);
        fr.first(chi, t_, F[1].dzh, I0);
        if (nbk > 1) {
            staged_eval<kCheck>(B + 1, eo, q, floor_hat, chi, t_);
            bk.first(chi, t_, B[1].dzh, In);
        }
        s = 2;
    }
    // both halves: four steps between renormalisations (per step b shrinks
    // by at most dh >= ~5e-20, on floor-opacity sub-points, and grows by at
    // most ~4 dh^3, so four steps stay inside the double range for half
    // optical depths up to ~1e19)
    const int e1 = min(s1, nbk);
    for (; s + 3 < e1; s += 4) {
#pragma unroll
        for (int j = 0; j < 4; j++) {
            staged_eval<kCheck>(F + s + j, eo, q, floor_hat, chi, t_);
            staged_eval<kCheck>(B + s + j, eo, q, floor_hat, chi2, t2);
            fr.step(chi, t_, F[s + j].dzh);
            bk.step(chi2, t2, B[s + j].dzh);
        }
        fr.renorm();
        bk.renorm();
    }
    for (; s + 1 < e1; s += 2) {
        staged_eval<kCheck>(F + s, eo, q, floor_hat, chi, t_);
        staged_eval<kCheck>(B + s, eo, q, floor_hat, chi2, t2);
        fr.step(chi, t_, F[s].dzh);
        bk.step(chi2, t2, B[s].dzh);
        staged_eval<kCheck>(F + s + 1, eo, q, floor_hat, chi, t_);
        staged_eval<kCheck>(B + s + 1, eo, q, floor_hat, chi2, t2);
        fr.step(chi, t_, F[s + 1].dzh);
        bk.step(chi2, t2, B[s + 1].dzh);
        fr.renorm();
        bk.renorm();
    }
    if (s < e1) {
        staged_eval<kCheck>(F + s, eo, q, floor_hat, chi, t_);
        staged_eval<kCheck>(B + s, eo, q, floor_hat, chi2, t2);
        fr.step(chi, t_, F[s].dzh);
        bk.step(chi2, t2, B[s].dzh);
        fr.renorm();
        bk.renorm();
        s++;
    }
    // the rest of the front half
    for (; s + 3 < s1; s += 4) {
#pragma unroll
        for (int j = 0; j < 4; j++) {
            staged_eval<kCheck>(F + s + j, eo, q, floor_hat, chi, t_);
            fr.step(chi, t_, F[s + j].dzh);
        }
        fr.renorm();
    }
    for (; s + 1 < s1; s += 2) {
        staged_eval<kCheck>(F + s, eo, q, floor_hat, chi, t_);
        fr.step(chi, t_, F[s].dzh);
        staged_eval<kCheck>(F + s + 1, eo, q, floor_hat, chi, t_);
        fr.step(chi, t_, F[s + 1].dzh);
        fr.renorm();
    }
    if (s < s1) {
        staged_eval<kCheck>(F + s, eo, q, floor_hat, chi, t_);
        fr.step(chi, t_, F[s].dzh);
        fr.renorm();
    }
}

// u and L at the origin for one (pair, bin): the warp stages the two halves
// window by window (kStageSteps steps of each), step s of the front being
// its point nfr-1-s (the far end first) and likewise for the back; each
// lane eliminates both halves toward the origin, in lock step while both
// have points.  A window with a line whose inverted opacity can take chi
// below half the floor runs the checking variant of the sweep.  bc_pair
// holds the far ends' boundary intensities of this pair (front, then back;
// nfreqs each), loaded before the first window is staged so that their
// latency overlaps the staging.
__device__ __forceinline__ void staged_pair(StagedPt *buf, const TraceView &t, const float2 *ek,
                                            int K, int k0, int k1, int64_t ofr, int nfr,
                                            int64_t obk, int nbk, int eo, float q, float floor_hat,
                                            const float *bc_pair, const BinCtx &b, float chi_o,
                                            float t_o, const ModelView &m, int origin, int lane,
                                            DevFlags *flags, double &u, double &L) {
    constexpr float kSqrtLog2e = 1.2011224087864498f;
    // an inverted line whose opacity can take chi below half the floor
    // (the profile factor (1 + off) exp(-x^2) stays below 1.001)
    const float neg_cut = -0.499f * floor_hat;
    ProjChain fr, bk;
    double I0 = (double)__ldcs(bc_pair + b.f);
    double In = nbk > 0 ? (double)__ldcs(bc_pair + m.nfreqs + b.f) : 0.0;
    for (int s0 = 0; s0 < nfr; s0 += kStageSteps) {
        const int s1 = min(s0 + kStageSteps, nfr);
        const int nF = s1 - s0;
        const int nB = max(0, min(s1, nbk) - s0);
        bool inverted = false;
        for (int j = lane; j < nF + nB; j += 32) {
            const bool front = j < nF;
            const int st = s0 + (front ? j : j - nF);
            const int64_t gi = front ? ofr + (nfr - 1 - st) : obk + (nbk - 1 - st);
            const float4 v = __ldg(reinterpret_cast<const float4 *>(t.mp) + gi);
            const unsigned cell = (unsigned)__float_as_int(v.x);
            const float2 e0 = __ldg(ek + cell * K + k0);
            const float2 e1 = __ldg(ek + cell * K + k1);
            inverted |= (e0.y < neg_cut) | (e1.y < neg_cut);
            float4 *dst = reinterpret_cast<float4 *>(buf + (front ? j : kStageSteps + (j - nF)));
            dst[0] = make_float4(v.y, 0.5f * v.z, v.w * kSqrtLog2e, v.x);
            dst[1] = make_float4(e0.x, e0.y, e1.x, e1.y);
        }
        const bool check = __any_sync(0xffffffffu, inverted);
        __syncwarp();
        const StagedPt *F = buf - s0;                 // front step s at F[s]
        const StagedPt *B = buf + kStageSteps - s0;   // back step s at B[s]
        if (check)
            staged_window<true>(F, B, s0, s1, nbk, eo, q, floor_hat, fr, bk, I0, In);
        else
            staged_window<false>(F, B, s0, s1, nbk, eo, q, floor_hat, fr, bk, I0, In);
        __syncwarp();
    }
    // the origin row
    if (nfr == 1) fr.first(chi_o, t_o, 0.0f, I0);
    else fr.step(chi_o, t_o, 0.0f);
    const double to = (double)t_o;
    if (nbk == 0) {
        const int bo = __ldg(m.cell2bdy + origin);
        if (bo >= 0) In = __ldg(m.ibdy + (int64_t)bo * m.nfreqs + b.f);
        else atomicAdd(&flags->trace_err, 1ull);
        // u = (dh (t dh + In) + S~)/(dh (dh + 1) + F~), times b
        const double dh = fr.dh_prev;
        const double D = rcp_pos(fma(dh * (dh + 1.0), fr.b, fr.a));
        u = fma(dh * fma(to, dh, In), fr.b, fr.c) * D;
        L = dh * dh * fr.b * D;
        return;
    }
    if (nbk == 1) bk.first(chi_o, t_o, 0.0f, In);
    else bk.step(chi_o, t_o, 0.0f);
    // u = (t PQ + S~f Q + S~b P)/(F~f Q + F~b P + PQ), times bf bb
    const double H = fr.dh_prev + bk.dh_prev;
    const double P = H * fr.dh_prev, Q = H * bk.dh_prev;
    const double PQB = P * Q * (fr.b * bk.b);
    const double D = rcp_pos(fma(fr.a * bk.b, Q, fma(bk.a * fr.b, P, PQB)));
    u = fma(to, PQB, fma(fr.c * bk.b, Q, bk.c * fr.b * P)) * D;
    L = PQB * D;
}

// ------------------------------------------------------------------ staged FP64 solve
//
// The FP64 solve with the same staging: per window the warp gathers each
// point's shift, dZ/4, profile width and its inverse, and the (eps, kap) of
// the chunk's two lines; each lane then evaluates emissivity and opacity
// exactly as Simulation::get_eta_and_chi does (simulation.tpp:385-481, its
// own line only: the lines' windows do not overlap) and eliminates in the
// same projective form.

struct __align__(8) StagedPt64 {
    double shift, dzq, pw, inv_pw;   // dzq = dZ / 4: dh = (chi_a + chi_b) dzq
    double e[4];                     // eps, kap of the chunk's first and second line
    int64_t cell;
};

constexpr int kStageSteps64 = 32;

struct Lane64 {
    double nu_o, line, inv_line;
    int eo;   // 0 or 2: this lane's line in StagedPt64::e
    int k;    // this lane's line
};

__device__ __forceinline__ void staged_eval64(const StagedPt64 *p, const Lane64 &l, double &chi,
                                              double &t) {
    const double freq = p->shift * l.nu_o;
    const double width = l.line * p->pw;
    const double diff = freq - l.line;
    const bool in = diff <= 11.0 * width && diff >= -11.0 * width;
    const double inv_w = l.inv_line * p->inv_pw;
    const double x = inv_w * diff;
    const double fp = in ? freq * (inv_w * kINVERSE_SQRT_PI * exp(-(x * x))) : 0.0;
    const double eta = p->e[l.eo] * fp;
    chi = 1.0E-26 + p->e[l.eo + 1] * fp;
    t = eta * rcp_pos(chi);
}

__device__ __forceinline__ void staged_window64(const StagedPt64 *F, const StagedPt64 *B, int s0,
                                                int s1, int nbk, const Lane64 &ln,
                                                const BdyCtx &bc, DevFlags *flags,
                                                ProjChainT<double> &fr, ProjChainT<double> &bk,
                                                double &I0, double &In) {
    double chi, t_, chi2, t2;
    int s = s0;
    if (s == 0) {
        staged_eval64(F, ln, chi, t_);
        fr.start(chi, t_, F->dzq);
        I0 = boundary_intensity(bc, F->shift * ln.nu_o, (int)F->cell, flags, ln.k);
        if (nbk > 0) {
            staged_eval64(B, ln, chi, t_);
            bk.start(chi, t_, B->dzq);
            In = boundary_intensity(bc, B->shift * ln.nu_o, (int)B->cell, flags, ln.k);
        }
        s = 1;
    }
    if (s == 1 && s < s1) {
        staged_eval64(F + 1, ln, chi, t_);
        fr.first(chi, t_, F[1].dzq, I0);
        if (nbk > 1) {
            staged_eval64(B + 1, ln, chi, t_);
            bk.first(chi, t_, B[1].dzq, In);
        }
        s = 2;
    }
    // renormalised every second step: a four-step unrolled body with the
    // double exp inlined eight times spills and runs 1.6x slower
    const int e1 = min(s1, nbk);
    for (; s + 1 < e1; s += 2) {
        staged_eval64(F + s, ln, chi, t_);
        staged_eval64(B + s, ln, chi2, t2);
        fr.step(chi, t_, F[s].dzq);
        bk.step(chi2, t2, B[s].dzq);
        staged_eval64(F + s + 1, ln, chi, t_);
        staged_eval64(B + s + 1, ln, chi2, t2);
        fr.step(chi, t_, F[s + 1].dzq);
        bk.step(chi2, t2, B[s + 1].dzq);
        fr.renorm();
        bk.renorm();
    }
    if (s < e1) {
        staged_eval64(F + s, ln, chi, t_);
        staged_eval64(B + s, ln, chi2, t2);
        fr.step(chi, t_, F[s].dzq);
        bk.step(chi2, t2, B[s].dzq);
        fr.renorm();
        bk.renorm();
        s++;
    }
    for (; s + 1 < s1; s += 2) {
        staged_eval64(F + s, ln, chi, t_);
        fr.step(chi, t_, F[s].dzq);
        staged_eval64(F + s + 1, ln, chi, t_);
        fr.step(chi, t_, F[s + 1].dzq);
        fr.renorm();
    }
    if (s < s1) {
        staged_eval64(F + s, ln, chi, t_);
        fr.step(chi, t_, F[s].dzq);
        fr.renorm();
    }
}

__device__ __forceinline__ void staged_pair64(StagedPt64 *buf, const TraceView &t, const double *eps,
                                              const double *kap, int K, int k0, int k1, int64_t ofr,
                                              int nfr, int64_t obk, int nbk, const Lane64 &ln,
                                              const BdyCtx &bc, const BinCtx &b, double chi_o,
                                              double t_o, const ModelView &m, int origin, int lane,
                                              DevFlags *flags, double &u, double &L) {
    ProjChainT<double> fr, bk;
    double I0 = 0.0, In = 0.0;
    for (int s0 = 0; s0 < nfr; s0 += kStageSteps64) {
        const int s1 = min(s0 + kStageSteps64, nfr);
        const int nF = s1 - s0;
        const int nB = max(0, min(s1, nbk) - s0);
        for (int j = lane; j < nF + nB; j += 32) {
            const bool front = j < nF;
            const int st = s0 + (front ? j : j - nF);
            const int64_t gi = front ? ofr + (nfr - 1 - st) : obk + (nbk - 1 - st);
            const int cell = __ldg(t.cell + gi);
            StagedPt64 *d = buf + (front ? j : kStageSteps64 + (j - nF));
            d->shift = __ldg(t.shift + gi);
            d->dzq = 0.25 * __ldg(t.dZ + gi);
            d->pw = __ldg(m.pw + cell);
            d->inv_pw = __ldg(m.inv_pw + cell);
            d->e[0] = __ldg(eps + (unsigned)cell * K + k0);
            d->e[1] = __ldg(kap + (unsigned)cell * K + k0);
            d->e[2] = __ldg(eps + (unsigned)cell * K + k1);
            d->e[3] = __ldg(kap + (unsigned)cell * K + k1);
            d->cell = cell;
        }
        __syncwarp();
        staged_window64(buf - s0, buf + kStageSteps64 - s0, s0, s1, nbk, ln, bc, flags, fr, bk, I0,
                        In);
        __syncwarp();
    }
    if (nfr == 1) fr.first(chi_o, t_o, 0.0, I0);
    else fr.step(chi_o, t_o, 0.0);
    if (nbk == 0) {
        const int bo = __ldg(m.cell2bdy + origin);
        if (bo >= 0) In = __ldg(m.ibdy + (int64_t)bo * m.nfreqs + b.f);
        else atomicAdd(&flags->trace_err, 1ull);
        const double dh = fr.dh_prev;
        const double D = rcp_pos(fma(dh * (dh + 1.0), fr.b, fr.a));
        u = fma(dh * fma(t_o, dh, In), fr.b, fr.c) * D;
        L = dh * dh * fr.b * D;
        return;
    }
    if (nbk == 1) bk.first(chi_o, t_o, 0.0, In);
    else bk.step(chi_o, t_o, 0.0);
    const double H = fr.dh_prev + bk.dh_prev;
    const double P = H * fr.dh_prev, Q = H * bk.dh_prev;
    const double PQB = P * Q * (fr.b * bk.b);
    const double D = rcp_pos(fma(fr.a * bk.b, Q, fma(bk.a * fr.b, P, PQB)));
    u = fma(t_o, PQB, fma(fr.c * bk.b, Q, bk.c * fr.b * P)) * D;
    L = PQB * D;
}

template <int kMinBlocks, bool kFp64>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, kMinBlocks)
    formal_solve_staged_kernel(ModelView m, TraceView t, SolveArgs a, DevFlags *flags) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t idx = a.s_begin + (int64_t)blockIdx.x * kWarpsPerBlock + warp;
    if (idx >= a.s_end) return;
    const int64_t oi = a.olist ? (int64_t)a.olist[idx] - t.o_begin : idx;
    const int o = (int)(t.o_begin + oi);
    if (m.seg_active && !m.seg_active[m.cell_seg[o]]) return;   // converged model of a batch
    const int K = m.nrad, nq = m.nquads, nf = m.nfreqs;
    using Pt = typename std::conditional<kFp64, StagedPt64, StagedPt>::type;
    constexpr int cap = 2 * (kFp64 ? kStageSteps64 : kStageSteps);
    Pt *pts = reinterpret_cast<Pt *>(smem_raw) + (size_t)warp * cap;
    double *sJ = reinterpret_cast<double *>(reinterpret_cast<Pt *>(smem_raw) +
                                            (size_t)kWarpsPerBlock * cap) + (size_t)warp * 2 * K;
    double *sL = sJ + K;
    for (int k = lane; k < K; k += 32) { sJ[k] = 0.0; sL[k] = 0.0; }
    __syncwarp();
    const float2 *ek = a.ehat_khat;
    const BdyCtx bc = bdy_ctx(m);
    const float floor_hat = (float)(1.0E-26 * a.mixed_scale);
    const double pw_o = m.pw[o];
    const int nchunks = (nf + 31) >> 5;
    for (int c = 0; c < nchunks; c++) {
        const int f = c * 32 + lane;
        const bool active = f < nf;
        const int fc = active ? f : nf - 1;
        BinCtx b;
        b.f = fc;
        b.k = fc / nq;
        const int z = fc - b.k * nq;
        b.lo = b.hi = b.k;
        const double line_k = m.line[b.k];
        const double root = m.roots[z];
        b.nu_o = radd(line_k, rmul(rmul(line_k, pw_o), root));
        b.q = (float)(pw_o * root);
        const int k0 = (c * 32) / nq;
        const int k1 = min(K - 1, k0 + 1);
        const int eo = b.k != k0 ? 3 : 2;   // float2 index of this lane's line in a StagedPt

        // origin in double; in mixed precision an inverted line taking chi
        // below half the floor there poisons the bin
        double e64, c64;
        eta_chi_double(m, a.eps, a.kap, o, b.nu_o, b.k, b.k, e64, c64);
        const float chi_o = (float)(c64 * m.mixed_scale);
        const float t_o = c64 < 0.5E-26 ? __int_as_float(0x7fc00000) : (float)(e64 / c64);
        const double t_o64 = e64 * rcp_pos(c64);
        Lane64 ln;
        ln.nu_o = b.nu_o;
        ln.line = line_k;
        ln.inv_line = m.inv_line[b.k];
        ln.eo = b.k != k0 ? 2 : 0;
        ln.k = b.k;
        const double width_o = line_k * pw_o;
        const double iw = 1.0 / width_o;
        const double xo = iw * (b.nu_o - line_k);
        const double prof_o = iw * kINVERSE_SQRT_PI * exp(-(xo * xo));
        const double lam_pre = m.A[b.k] * (m.qw[z] * 2.0) * (b.nu_o * prof_o / c64);

        double Jf = 0.0, Lf = 0.0;
        for (int r = 0; r < m.npairs; r++) {
            const int ar = m.antipod[r];
            const double wr = m.ray_w[r];
            const int64_t ir = (int64_t)r * t.o_count + oi;
            const int64_t iar = (int64_t)ar * t.o_count + oi;
            const int nr_ = t.len[ir], nar_ = t.len[iar];
            const bool rfront = nr_ > nar_;
            const int64_t ofr = rfront ? t.off[ir] : t.off[iar];
            const int64_t obk = rfront ? t.off[iar] : t.off[ir];
            const int nfr = rfront ? nr_ : nar_;
            const int nbk = rfront ? nar_ : nr_;
            if (nfr == 0) {
                const int bo = m.cell2bdy[o];
                double I = 0.0;
                if (bo >= 0) I = m.ibdy[(int64_t)bo * nf + fc];
                else if (lane == 0) atomicAdd(&flags->trace_err, 1ull);
                Jf += 2.0 * wr * (0.5 * (I + I));
                continue;
            }
            double u, L;
            if constexpr (kFp64) {
                staged_pair64(pts, t, a.eps, a.kap, K, k0, k1, ofr, nfr, obk, nbk, ln, bc, b, c64,
                              t_o64, m, o, lane, flags, u, L);
            } else {
                staged_pair(pts, t, ek, K, k0, k1, ofr, nfr, obk, nbk, eo, b.q, floor_hat,
                            a.bcache + ((oi * m.npairs + r) * 2) * (int64_t)nf, b, chi_o, t_o, m,
                            o, lane, flags, u, L);
            }
            if (!kFp64 && !(isfinite(u) && isfinite(L))) {
                const unsigned long long slot = atomicAdd(a.patch_count, 1ull);
                if (slot < (unsigned long long)a.patch_cap) a.patch[slot] = make_int4(o, r, fc, 0);
                else list_for_redo(a, flags, o);
                continue;
            }
            Jf += 2.0 * wr * u;
            Lf += lam_pre * wr * L;
        }
        if (a.J && active) a.J[(int64_t)o * nf + f] = Jf;
        const double jw = active ? m.qw[z] * Jf : 0.0;
        const double lw = active ? Lf : 0.0;
        const int klast = min(K - 1, (c * 32 + 31) / nq);
        for (int kk = k0; kk <= klast; kk++) {
            double vj = (active && b.k == kk) ? jw : 0.0;
            double vl = (active && b.k == kk) ? lw : 0.0;
#pragma unroll
            for (int sh = 16; sh > 0; sh >>= 1) {
                vj += __shfl_xor_sync(0xffffffffu, vj, sh);
                vl += __shfl_xor_sync(0xffffffffu, vl, sh);
            }
            if (lane == 0) { sJ[kk] += vj; sL[kk] += vl; }
        }
        __syncwarp();
    }
    for (int k = lane; k < K; k += 32) {
        a.Jlin[(int64_t)o * K + k] = sJ[k];
        a.Lam[(int64_t)o * K + k] = sL[k];
    }
}

// The far end of one half for the boundary cache: its boundary row and
// its profile width, resolved once per (origin, pair).
struct FarEnd {
    const double *I;   // I_bdy on the far cell's grid, or null (not a boundary cell)
    double pwp, ipwp;
    double shift;      // 1 + Doppler shift - 1 of the far end
};

__device__ __forceinline__ FarEnd far_end(const BdyCtx &c, float4 rec, DevFlags *flags) {
    FarEnd e;
    const int p = __float_as_int(rec.x);
    const int b = __ldg(c.cell2bdy + p);
    e.I = nullptr;
    if (b >= 0) e.I = c.ibdy + (int64_t)b * c.nf;
    else atomicAdd(&flags->trace_err, 1ull);
    e.pwp = __ldg(c.pw + p);
    e.ipwp = __ldg(c.inv_pw + p);
    e.shift = 1.0 + (double)rec.y;
    return e;
}

// boundary_intensity's bin search on the far cell's grid, with the
// interpolation weight formed in double and applied with one float
// division (the cache holds floats).  The line is searched from the lane's
// own line k: a Doppler shift of many profile widths moves the frequency
// out of line k's window, but on a grid of separated lines only to the gap
// below line k (line k or k - 1 then holds the first bin at or above it)
// or the gap above (line k + 1); a bisection covers the rest.  The bin is
// then found from the root-grid guess and walked.
__device__ __forceinline__ float far_end_intensity(const BdyCtx &c, const FarEnd &e, double freq,
                                                   int k) {
    const int nq = c.nq, nf = c.nf, K = nf / nq;
    if (!e.I) return 0.0f;
    auto nu_kz = [&](int kk, int z) {
        const double line = __ldg(c.line + kk);
        return radd(line, rmul(rmul(line, e.pwp), __ldg(c.roots + z)));
    };
    // the first line whose last bin is >= freq, within [lo, hi)
    auto bisect = [&](int lo, int hi) {
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (freq <= nu_kz(mid, nq - 1)) hi = mid;
            else lo = mid + 1;
        }
        return lo;
    };
    int lo;
    if (freq <= nu_kz(k, nq - 1)) {
        if (k == 0 || freq > nu_kz(k - 1, nq - 1)) lo = k;
        else if (k == 1 || freq > nu_kz(k - 2, nq - 1)) lo = k - 1;
        else lo = bisect(0, k - 1);
    } else {
        if (k + 1 < K && freq <= nu_kz(k + 1, nq - 1)) lo = k + 1;
        else lo = bisect(k + 1, K);
        if (lo == K) return (float)__ldg(e.I + nf - 1);   // above the grid
    }
    const double root = (freq * __ldg(c.inv_line + lo) - 1.0) * e.ipwp;
    const double zg = ceil((root - __ldg(c.roots)) * c.root_inv_step);
    int zl = (int)fmin(fmax(zg, 0.0), (double)(nq - 1));
    double nu1 = nu_kz(lo, zl);
    while (zl < nq - 1 && freq > nu1) nu1 = nu_kz(lo, ++zl);
    double nu2 = zl > 0 ? nu_kz(lo, zl - 1) : (lo > 0 ? nu_kz(lo - 1, nq - 1) : 0.0);
    while (zl > 0 && freq <= nu2) {
        nu1 = nu2;
        zl--;
        nu2 = zl > 0 ? nu_kz(lo, zl - 1) : (lo > 0 ? nu_kz(lo - 1, nq - 1) : 0.0);
    }
    const int notch = lo * nq + zl;
    const double I1 = __ldg(e.I + notch);
    if (notch == 0 || notch == nf - 1) return (float)I1;
    const double I2 = __ldg(e.I + notch - 1);
    const float w = __fdividef((float)(freq - nu1), (float)(nu2 - nu1));
    return (float)fma((double)w, I2 - I1, I1);
}

// One warp per (origin, pair) of a trace store, lanes over bins: the far
// ends' boundary intensities that the staged mixed solve reads
// (Radiation::rescale_I_bdy at the Doppler-shifted frequency, from the same
// far-end records and origin frequencies as the solve).  They depend only
// on the traces, the frequency grid and the boundary table, so one fill
// serves every solve over a store.
__global__ void __launch_bounds__(256)
    bdy_cache_kernel(ModelView m, TraceView t, int64_t s_begin, int64_t s_end, float *cache,
                     DevFlags *flags) {
    const int lane = threadIdx.x & 31;
    const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
    const int np = m.npairs;
    const int64_t ntask = (s_end - s_begin) * np;
    const BdyCtx bc = bdy_ctx(m);
    const int nq = m.nquads, nf = m.nfreqs;
    // this lane's first bin: line k0, root z0; each further chunk moves
    // 32 bins on (32 - nq wraps to the next line at most twice for nq >= 11)
    const int k0 = lane / nq, z0 = lane - k0 * nq;
    for (int64_t task = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
         task < ntask; task += nwarps) {
        const int64_t oi = s_begin + task / np;
        const int r = (int)(task - (oi - s_begin) * np);
        const int o = (int)(t.o_begin + oi);
        const int ar = m.antipod[r];
        const int64_t ir = (int64_t)r * t.o_count + oi;
        const int64_t iar = (int64_t)ar * t.o_count + oi;
        const int nr_ = t.len[ir], nar_ = t.len[iar];
        const bool rfront = nr_ > nar_;
        const int nfr = rfront ? nr_ : nar_;
        const int nbk = rfront ? nar_ : nr_;
        if (nfr == 0) continue;   // the solve takes this origin's own boundary value
        const int64_t ofr = rfront ? t.off[ir] : t.off[iar];
        const int64_t obk = rfront ? t.off[iar] : t.off[ir];
        // far-end records: x = cell (bits), y = Doppler shift - 1
        const FarEnd ef = far_end(bc, __ldg(reinterpret_cast<const float4 *>(t.mp) + ofr + nfr - 1),
                                  flags);
        FarEnd eb{nullptr, 0.0, 0.0, 1.0};
        if (nbk > 0)
            eb = far_end(bc, __ldg(reinterpret_cast<const float4 *>(t.mp) + obk + nbk - 1), flags);
        const double pw_o = m.pw[o];
        float *row = cache + (oi * np + r) * 2 * (int64_t)nf;
        int k = k0, z = z0;
        for (int f = lane; f < nf; f += 32) {
            const double line_k = __ldg(m.line + k);
            const double nu_o = radd(line_k, rmul(rmul(line_k, pw_o), __ldg(m.roots + z)));
            __stcs(row + f, far_end_intensity(bc, ef, ef.shift * nu_o, k));
            if (nbk > 0) __stcs(row + nf + f, far_end_intensity(bc, eb, eb.shift * nu_o, k));
            z += 32;
            while (z >= nq) { z -= nq; k++; }
        }
    }
}

}  // namespace

bool solve_is_staged(const ModelView &m) { return !m.overlap && m.nquads >= 31; }

cudaError_t launch_bdy_cache(const ModelView &m, const TraceView &t, int64_t s_begin,
                             int64_t s_end, float *cache, DevFlags *flags, cudaStream_t s) {
    if (s_end <= s_begin) return cudaSuccess;
    if (!cache) return cudaErrorInvalidValue;
    const int64_t warps = (s_end - s_begin) * m.npairs;
    const unsigned blocks = (unsigned)std::min<int64_t>((warps + 7) / 8, 148 * 32);
    bdy_cache_kernel<<<blocks, 256, 0, s>>>(m, t, s_begin, s_end, cache, flags);
    return cudaGetLastError();
}

cudaError_t launch_formal_solve(const ModelView &m, const TraceView &t, const SolveArgs &a,
                                int precision, int variant, DevFlags *flags, cudaStream_t s,
                                int *kind) {
    if (a.s_end <= a.s_begin) return cudaSuccess;
    const int64_t blocks = (a.s_end - a.s_begin + kWarpsPerBlock - 1) / kWarpsPerBlock;
    const size_t shmem = (size_t)kWarpsPerBlock * 2 * m.nrad * sizeof(double);
    // the staged kernels need each 32-bin chunk within two lines and lines
    // whose windows do not overlap
    const bool staged = solve_is_staged(m);
    if (staged && precision == MGR_MIXED && !a.bcache) return cudaErrorInvalidValue;
    if (kind) *kind = staged ? 1 : 0;
    if (variant < 0 || variant >= kSolveVariants)
        variant = !staged ? kDefaultGeneric : precision == MGR_FP64 ? kDefaultStaged64 : kDefaultStaged;
    auto run = [&](auto pol) {
        using P = decltype(pol);
        auto go = [&](auto kern) {
            kern<<<(unsigned)blocks, kWarpsPerBlock * 32, shmem, s>>>(m, t, a, pol, flags);
        };
        switch (variant) {
            case 0: go(formal_solve_kernel<P, kVariantBlocks[0]>); break;
            case 1: go(formal_solve_kernel<P, kVariantBlocks[1]>); break;
            default: go(formal_solve_kernel<P, kVariantBlocks[2]>); break;
        }
    };
    auto mixed = [&](auto pol) {
        pol.mp = t.mp;
        pol.ek = a.ehat_khat;
        pol.floor_hat = (float)(1.0E-26 * a.mixed_scale);
        pol.inv_scale = 1.0 / a.mixed_scale;
        pol.eps = a.eps;
        pol.kap = a.kap;
        run(pol);
    };
    auto fp64 = [&](auto pol) {
        pol.cell = t.cell;
        pol.shift = t.shift;
        pol.dZ = t.dZ;
        pol.eps = a.eps;
        pol.kap = a.kap;
        run(pol);
    };
    if (staged) {
        const bool f64 = precision == MGR_FP64;
        const size_t sm = (f64 ? (size_t)kWarpsPerBlock * 2 * kStageSteps64 * sizeof(StagedPt64)
                               : (size_t)kWarpsPerBlock * 2 * kStageSteps * sizeof(StagedPt)) +
                          (size_t)kWarpsPerBlock * 2 * m.nrad * sizeof(double);
        auto go = [&](auto kern) -> cudaError_t {
            cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)sm);
            if (e != cudaSuccess) return e;
            kern<<<(unsigned)blocks, kWarpsPerBlock * 32, sm, s>>>(m, t, a, flags);
            return cudaSuccess;
        };
        cudaError_t e;
        if (f64) {
            switch (variant) {
                case 0: e = go(formal_solve_staged_kernel<kVariantBlocks[0], true>); break;
                case 1: e = go(formal_solve_staged_kernel<kVariantBlocks[1], true>); break;
                default: e = go(formal_solve_staged_kernel<kVariantBlocks[2], true>); break;
            }
        } else {
            switch (variant) {
                case 0: e = go(formal_solve_staged_kernel<kVariantBlocks[0], false>); break;
                case 1: e = go(formal_solve_staged_kernel<kVariantBlocks[1], false>); break;
                default: e = go(formal_solve_staged_kernel<kVariantBlocks[2], false>); break;
            }
        }
        if (e != cudaSuccess) return e;
    } else if (precision == MGR_MIXED) {
        if (m.overlap) mixed(MixedPolicy<true>{});
        else mixed(MixedPolicy<false>{});
    }
    if (precision == MGR_MIXED) {
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        // entries beyond patch_cap are counted in DevFlags; the host then
        // solves again in double
        const unsigned pblocks = (unsigned)std::min<int64_t>((a.patch_cap + 127) / 128, 148 * 16);
        patch_kernel<<<pblocks, 128, 0, s>>>(m, t, a, flags);
    } else if (!staged) {
        if (m.overlap) fp64(Fp64Policy<true>{});
        else fp64(Fp64Policy<false>{});
    }
    return cudaGetLastError();
}

int solve_variant_blocks(int variant) {
    return variant >= 0 && variant < kSolveVariants ? kVariantBlocks[variant] : 0;
}

}  // namespace mgr
