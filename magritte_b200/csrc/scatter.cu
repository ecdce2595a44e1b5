// scatter.cu -- the formal solve with scattering terms.
//
// Simulation::setup_using_scattering (Simulation/simulation.tpp:51-171) puts
// term1 = (U + eta)/chi and term2 = V/chi on every point of a ray pair, U and
// V being the direction-integrated scattering terms of the pair (the
// origin's own bin, elsewhere interpolated on the cell's grid,
// Radiation::rescale_U_and_V, radiation.tpp:232-262).
// RayPair::solve_using_scattering (raypair_solver.tpp:10-190) then solves the
// Feautrier system twice with one matrix: for u with sources
//     Su[n] = term1[n] - (term2[n+1] - term2[n-1]) * 2/(dtau[n-1] + dtau[n])
// and for v with term1 and term2 exchanged, the boundary rows carrying
//     Su[0] = term1[0] - (term2[1] + term2[0] - 2 I_0)/dtau[0],
//     Sv[0] = term2[0] - (term1[1] + term1[0] - 2 I_0)/dtau[0]
// and their mirror images at the far end.
//
// The device solves it like the formal solve: one warp per origin, lanes
// over 32-bin chunks, each half of the pair eliminated from its far end
// toward the origin in projective form (F~ = a/b, S~ = c/b on half optical
// depths).  The matrix is the same for u and v, so each half carries one
// pair (a, b) and two right-hand sides (c_u, c_v); a boundary row is the
// non-scattering one with an effective boundary intensity (I_0 minus half
// the sum of the other term at the two end points), and an interior
// point's source is formed when the chain leaves it, when its neighbours on
// both sides are known.  FP64 throughout.
#include "mgr_internal.cuh"

namespace mgr {

namespace {

constexpr int kScatWarps = 4;

__device__ __forceinline__ double inv2pow(double b) {
    const int hi = __double2hiint(b);
    return __hiloint2double(0x7fe00000 - (hi & 0x7ff00000), 0);
}

// Position of freq on cell p's grid nu = line + line pw root (ascending):
// the first bin with nu >= freq, by bisection over lines and then bins
// (search_with_notch of the scalar build finds the same bin linearly).
__device__ int cell_notch(const ModelView &m, int p, double freq) {
    const int nq = m.nquads, K = m.nrad;
    const double pwp = __ldg(m.pw + p);
    auto nu_kz = [&](int k, int z) {
        const double line = __ldg(m.line + k);
        return radd(line, rmul(rmul(line, pwp), __ldg(m.roots + z)));
    };
    int lo = 0, hi = K;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (freq <= nu_kz(mid, nq - 1)) hi = mid;
        else lo = mid + 1;
    }
    if (lo == K) return m.nfreqs - 1;
    const int k = lo;
    int zl = 0, zh = nq - 1;
    while (zl < zh) {
        const int mid = (zl + zh) >> 1;
        if (freq <= nu_kz(k, mid)) zh = mid;
        else zl = mid + 1;
    }
    return k * nq + zl;
}

__device__ __forceinline__ double cell_nu(const ModelView &m, int p, int f) {
    const int k = f / m.nquads, z = f - k * m.nquads;
    const double line = __ldg(m.line + k);
    return radd(line, rmul(rmul(line, __ldg(m.pw + p)), __ldg(m.roots + z)));
}

struct PointTerms {
    double chi, t1, t2;
};

struct ScatChain {
    double chi_a, t1_a, t2_a, dz_a;   // point being left next and its segment toward the origin
    double t1_p, t2_p;                // the point before it (farther from the origin)
    double dh_prev, a, b, cu, cv;
};

// Terms of one point: emissivity and opacity over the bin's line window,
// U and V interpolated on the point's cell grid (or the origin's own bin).
struct ScatCtx {
    const ModelView *m;
    const double *eps, *kap, *U, *V;   // U, V: this pair's [N*nf]
    int lo, hi, f;
    int64_t N;
};

__device__ PointTerms terms_at(const ScatCtx &c, int cell, double freq, bool origin) {
    const ModelView &m = *c.m;
    const int nf = m.nfreqs;
    double eta, chi;
    eta_chi_double(m, c.eps, c.kap, cell, freq, c.lo, c.hi, eta, chi);
    double Us, Vs;
    const double *Ur = c.U + (int64_t)cell * nf, *Vr = c.V + (int64_t)cell * nf;
    if (origin) {
        Us = Ur[c.f];
        Vs = Vr[c.f];
    } else {
        const int n = cell_notch(m, cell, freq);
        if (n == 0 || n == nf - 1) {
            Us = Ur[n];
            Vs = Vr[n];
        } else {
            const double nu1 = cell_nu(m, cell, n), nu2 = cell_nu(m, cell, n - 1);
            Us = (Ur[n - 1] - Ur[n]) / (nu2 - nu1) * (freq - nu1) + Ur[n];
            Vs = (Vr[n - 1] - Vr[n]) / (nu2 - nu1) * (freq - nu1) + Vr[n];
        }
    }
    PointTerms t;
    const double ic = 1.0 / chi;
    t.chi = chi;
    t.t1 = (Us + eta) * ic;
    t.t2 = Vs * ic;
    return t;
}

// The far end's boundary row (intensity I at the end point) and the step
// onto the next point q; `toward_origin_is_up`: the chain walks toward
// increasing index of the reference's pair (the front half).
__device__ __forceinline__ void chain_first(ScatChain &s, const PointTerms &q, double dz_q,
                                            double I, bool up) {
    const double dh = 0.25 * (s.chi_a + q.chi) * s.dz_a;
    // effective intensities: I - (term_other[end] + term_other[next])/2 for
    // the front's first row; the back's (index end) row adds instead and
    // flips v's sign of I
    const double Iu = up ? I - 0.5 * (s.t2_a + q.t2) : I + 0.5 * (s.t2_a + q.t2);
    const double Iv = up ? I - 0.5 * (s.t1_a + q.t1) : 0.5 * (s.t1_a + q.t1) - I;
    s.a = dh * (dh + 1.0);
    s.b = fma(2.0, s.a, 1.0);
    s.cu = dh * fma(s.t1_a, dh, Iu);
    s.cv = dh * fma(s.t2_a, dh, Iv);
    s.dh_prev = dh;
    s.t1_p = s.t1_a; s.t2_p = s.t2_a;
    s.chi_a = q.chi; s.t1_a = q.t1; s.t2_a = q.t2; s.dz_a = dz_q;
}

// Leaves point a (its sources formed from its neighbours p and q) for q.
__device__ __forceinline__ void chain_step(ScatChain &s, const PointTerms &q, double dz_q, bool up) {
    const double dh = 0.25 * (s.chi_a + q.chi) * s.dz_a;
    const double H = s.dh_prev + dh;
    const double iH = 1.0 / H;   // 2 / (dtau[n-1] + dtau[n])
    // term_other[n+1] - term_other[n-1]: q is n+1 walking up, n-1 walking down
    const double d2 = up ? q.t2 - s.t2_p : s.t2_p - q.t2;
    const double d1 = up ? q.t1 - s.t1_p : s.t1_p - q.t1;
    const double su = s.t1_a - d2 * iH;
    const double sv = s.t2_a - d1 * iH;
    const double P = H * s.dh_prev, Q = H * dh;
    const double Pb = P * s.b;
    s.a = Q * (Pb + s.a);
    s.cu = Q * fma(su, Pb, s.cu);
    s.cv = Q * fma(sv, Pb, s.cv);
    s.b = fma(2.0, s.a, Pb);
    const double sc = inv2pow(s.b);
    s.a *= sc; s.b *= sc; s.cu *= sc; s.cv *= sc;
    s.dh_prev = dh;
    s.t1_p = s.t1_a; s.t2_p = s.t2_a;
    s.chi_a = q.chi; s.t1_a = q.t1; s.t2_a = q.t2; s.dz_a = dz_q;
}

__global__ void __launch_bounds__(kScatWarps * 32) scatter_kernel(ModelView m, TraceView t,
                                                                 ScatterArgs a, DevFlags *flags) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t oi = (int64_t)blockIdx.x * kScatWarps + warp;
    if (oi >= t.o_count) return;
    const int o = (int)(t.o_begin + oi);
    const int K = m.nrad, nq = m.nquads, nf = m.nfreqs;
    const int64_t N = m.N;
    const double pw_o = m.pw[o];
    const int bo = m.cell2bdy[o];
    for (int kk = lane; kk < K; kk += 32) {
        a.Jlin[(int64_t)o * K + kk] = 0.0;
        a.Lam[(int64_t)o * K + kk] = 0.0;
    }
    __syncwarp();
    for (int f0 = 0; f0 < nf; f0 += 32) {
        const int f = f0 + lane;
        const bool active = f < nf;
        const int fc = active ? f : nf - 1;
        const int k = fc / nq, z = fc - k * nq;
        const double line_k = m.line[k];
        const double nu_o = radd(line_k, rmul(rmul(line_k, pw_o), m.roots[z]));
        double Jf = 0.0, Lf = 0.0;
        // ALO factor without the pair weight (raypair_lambda.tpp:26-29, :115-121)
        double e64, c64;
        eta_chi_double(m, a.eps, a.kap, o, nu_o, m.win_lo[k], m.win_hi[k], e64, c64);
        const double width_o = line_k * pw_o;
        const double iw = 1.0 / width_o;
        const double xo = iw * (nu_o - line_k);
        const double prof_o = iw * kINVERSE_SQRT_PI * exp(-(xo * xo));
        const double lam_pre = m.A[k] * (m.qw[z] * 2.0) * (nu_o * prof_o / c64);
        for (int r = 0; r < m.npairs; r++) {
            const int ar = m.antipod[r];
            const double wr = m.ray_w[r];
            const int64_t ir = (int64_t)r * t.o_count + oi, iar = (int64_t)ar * t.o_count + oi;
            const int nr_ = t.len[ir], nar_ = t.len[iar];
            const bool rfront = nr_ > nar_;
            const int64_t ofr = rfront ? t.off[ir] : t.off[iar];
            const int64_t obk = rfront ? t.off[iar] : t.off[ir];
            const int nfr = rfront ? nr_ : nar_, nbk = rfront ? nar_ : nr_;
            double u, v, L = 0.0;
            const int64_t uv = ((int64_t)r * N + o) * nf + fc;
            if (nfr == 0) {
                double I = 0.0;
                if (bo >= 0) I = m.ibdy[(int64_t)bo * nf + fc];
                else if (lane == 0) atomicAdd(&flags->trace_err, 1ull);
                u = 0.5 * (I + I);
                v = 0.5 * (I - I);
            } else {
                ScatCtx c;
                c.m = &m; c.eps = a.eps; c.kap = a.kap;
                c.U = a.U + (int64_t)r * N * nf;
                c.V = a.V + (int64_t)r * N * nf;
                c.lo = m.win_lo[k]; c.hi = m.win_hi[k]; c.f = fc; c.N = N;
                const PointTerms to = terms_at(c, o, nu_o, true);
                const BdyCtx bl = bdy_ctx(m);
                // front half: far end first (reference index 0 upward)
                ScatChain F;
                {
                    const int64_t g = ofr + nfr - 1;
                    const int cell = t.cell[g];
                    const double fr = t.shift[g] * nu_o;
                    const PointTerms p0 = terms_at(c, cell, fr, false);
                    F.chi_a = p0.chi; F.t1_a = p0.t1; F.t2_a = p0.t2; F.dz_a = t.dZ[g];
                    const double I0 = boundary_intensity(bl, fr, cell, flags);
                    PointTerms q;
                    double dzq = 0.0;
                    if (nfr >= 2) {
                        const int64_t g1 = ofr + nfr - 2;
                        q = terms_at(c, t.cell[g1], t.shift[g1] * nu_o, false);
                        dzq = t.dZ[g1];
                    } else {
                        q = to;
                    }
                    chain_first(F, q, dzq, I0, true);
                    for (int s = 2; s < nfr; s++) {
                        const int64_t gs = ofr + nfr - 1 - s;
                        const PointTerms qs = terms_at(c, t.cell[gs], t.shift[gs] * nu_o, false);
                        chain_step(F, qs, t.dZ[gs], true);
                    }
                    if (nfr >= 2) chain_step(F, to, 0.0, true);
                }
                if (nbk == 0) {
                    // the origin is the last row, with the origin's boundary value
                    double In = 0.0;
                    if (bo >= 0) In = m.ibdy[(int64_t)bo * nf + fc];
                    else atomicAdd(&flags->trace_err, 1ull);
                    const double Iu = In + 0.5 * (to.t2 + F.t2_p);
                    const double Iv = 0.5 * (to.t1 + F.t1_p) - In;
                    const double dh = F.dh_prev;
                    const double D = 1.0 / fma(dh * (dh + 1.0), F.b, F.a);
                    u = fma(dh * fma(to.t1, dh, Iu), F.b, F.cu) * D;
                    v = fma(dh * fma(to.t2, dh, Iv), F.b, F.cv) * D;
                    L = dh * dh * F.b * D;
                } else {
                    // back half: its far end first (reference index ndep-1 downward)
                    ScatChain B;
                    const int64_t g = obk + nbk - 1;
                    const int cell = t.cell[g];
                    const double fr = t.shift[g] * nu_o;
                    const PointTerms p0 = terms_at(c, cell, fr, false);
                    B.chi_a = p0.chi; B.t1_a = p0.t1; B.t2_a = p0.t2; B.dz_a = t.dZ[g];
                    const double In = boundary_intensity(bl, fr, cell, flags);
                    PointTerms q;
                    double dzq = 0.0;
                    if (nbk >= 2) {
                        const int64_t g1 = obk + nbk - 2;
                        q = terms_at(c, t.cell[g1], t.shift[g1] * nu_o, false);
                        dzq = t.dZ[g1];
                    } else {
                        q = to;
                    }
                    chain_first(B, q, dzq, In, false);
                    for (int s = 2; s < nbk; s++) {
                        const int64_t gs = obk + nbk - 1 - s;
                        const PointTerms qs = terms_at(c, t.cell[gs], t.shift[gs] * nu_o, false);
                        chain_step(B, qs, t.dZ[gs], false);
                    }
                    if (nbk >= 2) chain_step(B, to, 0.0, false);
                    // the origin's row: Su[n_ar] with term_other[n_ar + 1] on the
                    // back side (B's last point) and [n_ar - 1] on the front side
                    const double H = F.dh_prev + B.dh_prev;
                    const double iH = 1.0 / H;
                    const double su = to.t1 - (B.t2_p - F.t2_p) * iH;
                    const double sv = to.t2 - (B.t1_p - F.t1_p) * iH;
                    const double P = H * F.dh_prev, Q = H * B.dh_prev;
                    const double PQB = P * Q * (F.b * B.b);
                    const double D = 1.0 / fma(F.a * B.b, Q, fma(B.a * F.b, P, PQB));
                    u = fma(su, PQB, fma(F.cu * B.b, Q, B.cu * F.b * P)) * D;
                    v = fma(sv, PQB, fma(F.cv * B.b, Q, B.cv * F.b * P)) * D;
                    L = PQB * D;
                }
                if (rfront) v = -v;
            }
            if (active) {
                a.u[uv] = u;
                a.v[uv] = v;
            }
            Jf += 2.0 * wr * u;
            if (nfr > 0) Lf += lam_pre * wr * L;
        }
        if (a.J && active) a.J[(int64_t)o * nf + f] = Jf;
        // line integrals over the bins of this chunk (one writer per origin)
        const double jw = active ? m.qw[z] * Jf : 0.0;
        const double lw = active ? Lf : 0.0;
        const int kfirst = f0 / nq, klast = min(K - 1, (f0 + 31) / nq);
        for (int kk = kfirst; kk <= klast; kk++) {
            double vj = (active && k == kk) ? jw : 0.0;
            double vl = (active && k == kk) ? lw : 0.0;
#pragma unroll
            for (int sh = 16; sh > 0; sh >>= 1) {
                vj += __shfl_xor_sync(0xffffffffu, vj, sh);
                vl += __shfl_xor_sync(0xffffffffu, vl, sh);
            }
            if (lane == 0) {
                a.Jlin[(int64_t)o * K + kk] += vj;
                a.Lam[(int64_t)o * K + kk] += vl;
            }
        }
        __syncwarp();
    }
}

// Radiation::calc_U_and_V (Model/Radiation/radiation.cpp:330-434, one
// process): U[r1] = sum over pairs r2 of u[r2] for every r1 (the phase
// function is 1), V from v alike.
__global__ void calc_uv_kernel(const double *u, const double *v, double *U, double *V, int64_t n,
                               int npairs) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double su = 0.0, sv = 0.0;
    for (int r = 0; r < npairs; r++) {
        su += u[(int64_t)r * n + i];
        sv += v[(int64_t)r * n + i];
    }
    for (int r = 0; r < npairs; r++) {
        U[(int64_t)r * n + i] = su;
        V[(int64_t)r * n + i] = sv;
    }
}

}  // namespace

cudaError_t launch_scatter(const ModelView &m, const TraceView &t, const ScatterArgs &a,
                           DevFlags *flags, cudaStream_t s) {
    if (t.o_count == 0) return cudaSuccess;
    const int64_t blocks = (t.o_count + kScatWarps - 1) / kScatWarps;
    scatter_kernel<<<(unsigned)blocks, kScatWarps * 32, 0, s>>>(m, t, a, flags);
    return cudaGetLastError();
}

cudaError_t launch_calc_uv(const ModelView &m, const double *u, const double *v, double *U,
                           double *V, cudaStream_t s) {
    const int64_t n = m.N * m.nfreqs;
    calc_uv_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(u, v, U, V, n, m.npairs);
    return cudaGetLastError();
}

}  // namespace mgr
