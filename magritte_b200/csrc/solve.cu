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
// with F' = F/(1+F), G' = G/(1+G) the reference's F and G.  This is the same
// linear system and the same diagonal ALO element (the reference's
// L_diag[n_ar] = inv_C/(F + G/(1+G))), with O(1) state per lane and a single
// division per point for the recursion.
//
// Outputs per origin: the line integrals Jlin[o][k] = sum_z w_z J[o][k,z]
// (Simulation::compute_Jeff, sim_lines.tpp:185-198) and the diagonal ALO
// Lam[o][k] (RayPair::update_Lambda, raypair_lambda.tpp:94-149), both
// reduced over the bins of a line with warp shuffles; optionally J itself.
#include "mgr_internal.cuh"

namespace mgr {

namespace {

constexpr int kWarpsPerBlock = 4;

// Per-lane frequency context of one bin at one origin.
struct BinCtx {
    double nu_o;      // bin frequency at the origin (sim_spectrum.tpp:37-41)
    int k;            // line of the bin
    int lo, hi;       // lines whose profile window can reach this bin
};

// ---------------------------------------------------------------- FP64 path
// Thermodynamics::profile with 1/exp(x^2) written as exp(-x^2) and
// 1/width as (1/line)(1/pw); same function to a few ulp.
__device__ __forceinline__ void eta_chi_fp64(const ModelView &m, const double *__restrict__ eps,
                                             const double *__restrict__ kap, int64_t p,
                                             double freq, const BinCtx &b, double &eta,
                                             double &chi) {
    eta = 0.0;
    chi = 1.0E-26;
    const double pwp = __ldg(m.pw + p);
    const double ipw = __ldg(m.inv_pw + p);
    const int K = m.nrad;
    for (int l = b.lo; l <= b.hi; l++) {
        const double line_l = __ldg(m.line + l);
        const double width = line_l * pwp;
        const double diff = freq - line_l;
        if (diff <= 11.0 * width && diff >= -11.0 * width) {
            const double inv_w = __ldg(m.inv_line + l) * ipw;
            const double x = inv_w * diff;
            const double prof = inv_w * kINVERSE_SQRT_PI * exp(-(x * x));
            const double fp = freq * prof;
            eta += __ldg(eps + p * K + l) * fp;
            chi += __ldg(kap + p * K + l) * fp;
        }
    }
}

// Radiation::rescale_I_bdy (scalar build, Model/Radiation/radiation.tpp:341-373)
// with I_bdy = planck(T_b, nu_p) evaluated on the fly.  The grid of cell p is
// ascending, so the reference's linear notch search equals a lower bound.
__device__ __forceinline__ double boundary_intensity(const ModelView &m, double freq, int64_t p,
                                                     DevFlags *flags) {
    const int b = __ldg(m.cell2bdy + p);
    if (b < 0) {
        atomicAdd(&flags->trace_err, 1ull);
        return 0.0;
    }
    const double T = __ldg(m.bdy_T + b);
    const double pwp = __ldg(m.pw + p);
    const int nq = m.nquads, nf = m.nfreqs;
    auto nu_at = [&](int f) {
        const int k = f / nq;
        const double line = __ldg(m.line + k);
        return radd(line, rmul(rmul(line, pwp), __ldg(m.roots + (f - k * nq))));
    };
    int lo = 0, hi = nf;   // first f with freq <= nu(f), or nf
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (freq <= nu_at(mid)) hi = mid;
        else lo = mid + 1;
    }
    int notch = lo < nf ? lo : nf - 1;
    if (notch == 0 || notch == nf - 1) return planck(T, nu_at(notch));
    const double nu1 = nu_at(notch), nu2 = nu_at(notch - 1);
    const double I1 = planck(T, nu1), I2 = planck(T, nu2);
    return (I2 - I1) / (nu2 - nu1) * (freq - nu1) + I1;
}

struct Trace {
    const int32_t *cell;
    const double *shift, *dZ;
    int n;
};

// Forward elimination over the front half (far end first) and backward
// elimination over the back half, meeting at the origin.
__device__ __forceinline__ void sweep_fp64(const ModelView &m, const double *__restrict__ eps,
                                           const double *__restrict__ kap, const BinCtx &b,
                                           const Trace &fr, const Trace &bk, double t_o,
                                           double chi_o, int64_t origin, DevFlags *flags,
                                           double &u, double &L) {
    // ---- front: positions 0 .. n_ar-1 are elements n_ar-1 .. 0
    int j = fr.n - 1;
    int32_t p = __ldg(fr.cell + j);
    double freq = __ldg(fr.shift + j) * b.nu_o;
    double eta, chi;
    eta_chi_fp64(m, eps, kap, p, freq, b, eta, chi);
    double chi_a = chi, t_a = eta / chi, dz_a = __ldg(fr.dZ + j);
    const double I0 = boundary_intensity(m, freq, p, flags);
    double Fp = 0.0, Su = 0.0, dtau_prev = 0.0;
    for (int n = 1; n <= fr.n; n++) {
        double chi_b, t_b, dz_b = 0.0;
        if (n < fr.n) {
            j = fr.n - 1 - n;
            p = __ldg(fr.cell + j);
            freq = __ldg(fr.shift + j) * b.nu_o;
            eta_chi_fp64(m, eps, kap, p, freq, b, eta, chi);
            chi_b = chi;
            t_b = eta / chi;
            dz_b = __ldg(fr.dZ + j);
        } else {
            chi_b = chi_o;
            t_b = t_o;
        }
        const double dtau = 0.5 * (chi_a + chi_b) * dz_a;
        if (n == 1) {
            // row 0: B0 = 1 + 2/dtau + 2/dtau^2, S0 = t + 2 I0/dtau
            const double D = 1.0 / (dtau * dtau + 2.0 * dtau + 2.0);
            Fp = (dtau * dtau + 2.0 * dtau) * D;
            Su = (t_a * dtau * dtau + 2.0 * I0 * dtau) * D;
        } else {
            const double h = 0.5 * (dtau_prev + dtau);
            const double invA = h * dtau_prev, invC = h * dtau;
            const double D = 1.0 / (invA * (1.0 + invC) + invC * Fp);
            const double Su_new = (t_a * invA + Su) * D * invC;
            Fp = invC * (invA + Fp) * D;
            Su = Su_new;
        }
        dtau_prev = dtau;
        chi_a = chi_b;
        t_a = t_b;
        dz_a = dz_b;
    }
    const double dtau_front = dtau_prev;   // dtau[o-1]

    if (bk.n == 0) {
        // the origin is the last row: S_d = t + 2 I_n / dtau with the
        // origin's own boundary value at this bin (simulation.tpp:343-348)
        const int bo = __ldg(m.cell2bdy + origin);
        double In = 0.0;
        if (bo >= 0) In = planck(__ldg(m.bdy_T + bo), b.nu_o);
        else atomicAdd(&flags->trace_err, 1ull);
        const double d = dtau_front;
        const double den = 1.0 / (d * d + 2.0 * d + 2.0 * Fp);
        u = (t_o * d * d + 2.0 * In * d + 2.0 * Su) * den;
        L = d * d * den;
        return;
    }

    // ---- back: positions last .. o+1 are elements n_r-1 .. 0
    j = bk.n - 1;
    p = __ldg(bk.cell + j);
    freq = __ldg(bk.shift + j) * b.nu_o;
    eta_chi_fp64(m, eps, kap, p, freq, b, eta, chi);
    chi_a = chi;
    t_a = eta / chi;
    dz_a = __ldg(bk.dZ + j);
    const double In = boundary_intensity(m, freq, p, flags);
    double Gp = 0.0, Sb = 0.0;
    dtau_prev = 0.0;
    for (int n = 1; n <= bk.n; n++) {
        double chi_b, t_b, dz_b = 0.0;
        if (n < bk.n) {
            j = bk.n - 1 - n;
            p = __ldg(bk.cell + j);
            freq = __ldg(bk.shift + j) * b.nu_o;
            eta_chi_fp64(m, eps, kap, p, freq, b, eta, chi);
            chi_b = chi;
            t_b = eta / chi;
            dz_b = __ldg(bk.dZ + j);
        } else {
            chi_b = chi_o;
            t_b = t_o;
        }
        const double dtau = 0.5 * (chi_a + chi_b) * dz_a;
        if (n == 1) {
            const double D = 1.0 / (dtau * dtau + 2.0 * dtau + 2.0);
            Gp = (dtau * dtau + 2.0 * dtau) * D;
            Sb = (t_a * dtau * dtau + 2.0 * In * dtau) * D;
        } else {
            // backward row: A uses the step toward the origin (dtau),
            // C the step toward the far end (dtau_prev)
            const double h = 0.5 * (dtau_prev + dtau);
            const double invA = h * dtau, invC = h * dtau_prev;
            const double D = 1.0 / (invC * (1.0 + invA) + invA * Gp);
            const double Sb_new = (t_a * invC + Sb) * D * invA;
            Gp = invA * (invC + Gp) * D;
            Sb = Sb_new;
        }
        dtau_prev = dtau;
        chi_a = chi_b;
        t_a = t_b;
        dz_a = dz_b;
    }
    const double dtau_back = dtau_prev;   // dtau[o]

    // ---- origin row
    const double h = 0.5 * (dtau_front + dtau_back);
    const double invA = h * dtau_front, invC = h * dtau_back;
    const double invAC = invA * invC;
    const double den = 1.0 / (invAC + Fp * invC + Gp * invA);
    u = (t_o * invAC + Su * invC + Sb * invA) * den;
    L = invAC * den;
}

__global__ void __launch_bounds__(kWarpsPerBlock * 32)
    formal_solve_fp64_kernel(ModelView m, TraceView t, SolveArgs a, DevFlags *flags) {
    extern __shared__ double smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t oi = (int64_t)blockIdx.x * kWarpsPerBlock + warp;
    if (oi >= t.o_count) return;
    const int64_t o = t.o_begin + oi;
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
        b.k = fc / nq;
        const int z = fc - b.k * nq;
        b.lo = m.win_lo[b.k];
        b.hi = m.win_hi[b.k];
        const double line_k = m.line[b.k];
        b.nu_o = radd(line_k, rmul(rmul(line_k, pw_o), m.roots[z]));

        // origin: same opacity and source for every pair
        double eta_o, chi_o;
        eta_chi_fp64(m, a.eps, a.kap, o, b.nu_o, b, eta_o, chi_o);
        const double t_o = eta_o / chi_o;
        // ALO factor without the pair weight (raypair_lambda.tpp:26-29, :115-121)
        const double width_o = line_k * pw_o;
        const double d_o = b.nu_o - line_k;
        const double iw = 1.0 / width_o;
        const double xo = iw * d_o;
        const double prof_o = iw * kINVERSE_SQRT_PI * exp(-(xo * xo));
        const double lam_pre = m.A[b.k] * (m.qw[z] * 2.0) * (b.nu_o * prof_o / chi_o);

        double Jf = 0.0, Lf = 0.0;
        for (int r = 0; r < m.npairs; r++) {
            const int ar = m.antipod[r];
            const double wr = m.ray_w[r];
            const int64_t ir = (int64_t)r * t.o_count + oi;
            const int64_t iar = (int64_t)ar * t.o_count + oi;
            const int nr_ = t.len[ir], nar_ = t.len[iar];
            // the longer trace is the front half (sim_radiation.tpp:164-171)
            const bool rfront = nr_ > nar_;
            Trace fr, bk;
            const int64_t ofr = rfront ? t.off[ir] : t.off[iar];
            const int64_t obk = rfront ? t.off[iar] : t.off[ir];
            fr.n = rfront ? nr_ : nar_;
            bk.n = rfront ? nar_ : nr_;
            fr.cell = t.cell + ofr; fr.shift = t.shift + ofr; fr.dZ = t.dZ + ofr;
            bk.cell = t.cell + obk; bk.shift = t.shift + obk; bk.dZ = t.dZ + obk;
            if (fr.n == 0) {
                // only the origin on the ray pair: J += 2 w I_bdy (sim_radiation.tpp:243-264)
                const int bo = m.cell2bdy[o];
                double I = 0.0;
                if (bo >= 0) I = planck(m.bdy_T[bo], b.nu_o);
                else if (lane == 0) atomicAdd(&flags->trace_err, 1ull);
                Jf += 2.0 * wr * (0.5 * (I + I));
                continue;
            }
            double u, L;
            sweep_fp64(m, a.eps, a.kap, b, fr, bk, t_o, chi_o, o, flags, u, L);
            Jf += 2.0 * wr * u;
            Lf += lam_pre * wr * L;
        }
        if (a.J && active) a.J[o * nf + f] = Jf;

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
        a.Jlin[o * K + k] = sJ[k];
        a.Lam[o * K + k] = sL[k];
    }
}

}  // namespace

cudaError_t launch_formal_solve(const ModelView &m, const TraceView &t, const SolveArgs &a,
                                int precision, DevFlags *flags, cudaStream_t s) {
    if (t.o_count == 0) return cudaSuccess;
    const int64_t blocks = (t.o_count + kWarpsPerBlock - 1) / kWarpsPerBlock;
    const size_t shmem = (size_t)kWarpsPerBlock * 2 * m.nrad * sizeof(double);
    (void)precision;
    formal_solve_fp64_kernel<<<(unsigned)blocks, kWarpsPerBlock * 32, shmem, s>>>(m, t, a, flags);
    return cudaGetLastError();
}

}  // namespace mgr
