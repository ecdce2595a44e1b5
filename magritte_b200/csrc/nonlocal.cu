// nonlocal.cu -- the off-diagonal elements of the approximated Lambda
// operator (parameters.n_off_diag = M >= 2).
//
// RayPair::solve with n_off_diag > 0 (Simulation/Raypair/raypair_solver.tpp:
// 336-388) eliminates the whole ray pair, substitutes back over all of it
// and forms the diagonal of the pair's Lambda operator at every point,
// Ld[n], with the factors 1/(1+F[n]) and 1/(1+G[n]) its off-diagonal
// elements are products of.  Here, for every (origin, pair, bin), one lane
// runs the forward recursion F from the front far end to M-1 points past
// the origin and the backward recursion G from the back far end to M-1
// points before it, in the reference's own (divide) form, keeping the
// values of the 2M points around the origin; the elements of the origin's
// row at distance d = 1..M-1,
//     Lambda(o, o-d) = Ld[o-d] / ((1+G[o-d+1]) ... (1+G[o])),
//     Lambda(o, o+d) = Ld[o+d] / ((1+F[o+d-1]) ... (1+F[o])),
// are weighted like the diagonal element (raypair_lambda.tpp:19-30, with the
// profile and opacity of the point they belong to) and summed over the
// bins of each line by warp shuffles.  RayPair::update_Lambda
// (raypair_lambda.tpp:129-145) reads L_lower[d][n_ar-d] and L_upper[d][n_ar+d]
// instead -- the elements (n_ar+1, n_ar-d) and (n_ar+d, n_ar+2d+1), not the
// origin's row, and at the ends of a pair entries its recursions did not
// write for that pair -- so this is where the two differ.
//
// Work decomposition as in the generic formal solve: one warp per origin,
// lanes over 32-bin chunks, all lanes walking the same traced points.  FP64.
#include "mgr_internal.cuh"

namespace mgr {

namespace {

constexpr int kOffWarps = 4;
constexpr int kWin = 2 * (kMaxOffDiag - 1) + 2;   // points kept around the origin

// The points of one ray pair in the reference's order: index 0 is the far
// end of the front trace (the longer one), nfr the origin, last = nfr + nbk
// the far end of the back trace.
struct PairPts {
    const TraceView *t;
    int64_t ofr, obk;
    int nfr, nbk, o;
    __device__ __forceinline__ void point(int i, int &cell, double &shift) const {
        if (i < nfr) {
            const int64_t g = ofr + (nfr - 1 - i);
            cell = __ldg(t->cell + g);
            shift = __ldg(t->shift + g);
        } else if (i == nfr) {
            cell = o;
            shift = 1.0;
        } else {
            const int64_t g = obk + (i - nfr - 1);
            cell = __ldg(t->cell + g);
            shift = __ldg(t->shift + g);
        }
    }
    // length of the segment between points i-1 and i
    __device__ __forceinline__ double dz_to(int i) const {
        return i <= nfr ? __ldg(t->dZ + ofr + (nfr - i)) : __ldg(t->dZ + obk + (i - nfr - 1));
    }
};

__global__ void __launch_bounds__(kOffWarps * 32) offdiag_kernel(ModelView m, TraceView t,
                                                                 OffdiagArgs a) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t oi = a.s_begin + (int64_t)blockIdx.x * kOffWarps + warp;
    if (oi >= a.s_end) return;
    const int o = (int)(t.o_begin + oi);
    const int K = m.nrad, nq = m.nquads, nf = m.nfreqs, M1 = a.M1, np = m.npairs;
    const int64_t ne = (int64_t)np * 2 * M1;
    double *Lo = a.Loff + (int64_t)o * K * ne;
    for (int64_t i = lane; i < (int64_t)K * ne; i += 32) Lo[i] = 0.0;
    for (int r = 0; r < np; r++) {
        const int ar = m.antipod[r];
        const int nr_ = t.len[(int64_t)r * t.o_count + oi], nar_ = t.len[(int64_t)ar * t.o_count + oi];
        const bool rfront = nr_ > nar_;
        const int64_t g_fr = rfront ? t.off[(int64_t)r * t.o_count + oi]
                                    : t.off[(int64_t)ar * t.o_count + oi];
        const int64_t g_bk = rfront ? t.off[(int64_t)ar * t.o_count + oi]
                                    : t.off[(int64_t)r * t.o_count + oi];
        const int nfr = rfront ? nr_ : nar_, nbk = rfront ? nar_ : nr_;
        for (int e = lane; e < 2 * M1; e += 32) {
            const int side = e / M1, d = e - side * M1 + 1;
            const int n = side == 0 ? nfr : nbk;
            const int64_t g = side == 0 ? g_fr : g_bk;
            a.Loff_nr[((int64_t)o * np + r) * 2 * M1 + e] = d <= n ? __ldg(t.cell + g + d - 1) : -1;
        }
    }
    __syncwarp();

    const double pw_o = m.pw[o];
    const int nchunks = (nf + 31) >> 5;
    double Ld_lo[kMaxOffDiag - 1], Ld_up[kMaxOffDiag - 1];
    for (int c = 0; c < nchunks; c++) {
        const int f = c * 32 + lane;
        const bool active = f < nf;
        const int fc = active ? f : nf - 1;
        const int k = fc / nq, z = fc - k * nq;
        const int lo = m.overlap ? m.win_lo[k] : k, hi = m.overlap ? m.win_hi[k] : k;
        const double line_k = m.line[k];
        const double nu_o = radd(line_k, rmul(rmul(line_k, pw_o), m.roots[z]));
        for (int r = 0; r < np; r++) {
            const int ar = m.antipod[r];
            const int64_t ir = (int64_t)r * t.o_count + oi, iar = (int64_t)ar * t.o_count + oi;
            const int nr_ = t.len[ir], nar_ = t.len[iar];
            const bool rfront = nr_ > nar_;
            PairPts P;
            P.t = &t;
            P.o = o;
            P.ofr = rfront ? t.off[ir] : t.off[iar];
            P.obk = rfront ? t.off[iar] : t.off[ir];
            P.nfr = rfront ? nr_ : nar_;
            P.nbk = rfront ? nar_ : nr_;
            if (P.nfr == 0) continue;   // the origin alone: no off-diagonal element
            const int nfr = P.nfr, last = P.nfr + P.nbk;
            const int base = nfr - M1;   // window: points base .. base + kWin - 1
            double wF[kWin], wi1F[kWin], wiC[kWin], wchi[kWin], wG[kWin], wi1G[kWin];
            int wcell[kWin];
            double wfr[kWin];
            auto in_win = [&](int i) { return i >= base && i < base + kWin; };
            auto eval = [&](int i, double &chi, int &cell, double &fr) {
                double shift, eta;
                P.point(i, cell, shift);
                fr = i == nfr ? nu_o : shift * nu_o;
                eta_chi_double(m, a.eps, a.kap, cell, fr, lo, hi, eta, chi);
            };
            // forward: F from the front far end to min(nfr + M1, last - 1)
            double chi_a, fr_a, chi_b, fr_b;
            int cell_a, cell_b;
            eval(0, chi_a, cell_a, fr_a);
            eval(1, chi_b, cell_b, fr_b);
            double dtau_prev = 0.5 * (chi_a + chi_b) * P.dz_to(1);
            const double inverse_dtau0 = 1.0 / dtau_prev;
            const double C0 = 2.0 * inverse_dtau0 * inverse_dtau0;
            const double B0_min_C0 = 1.0 + 2.0 * inverse_dtau0;
            const double B0 = B0_min_C0 + C0;
            double F = 0.5 * B0_min_C0 * dtau_prev * dtau_prev;
            double i1F = 1.0 / (1.0 + F);
            if (in_win(0)) {
                wF[0 - base] = F; wi1F[0 - base] = i1F; wchi[0 - base] = chi_a;
                wcell[0 - base] = cell_a; wfr[0 - base] = fr_a;
            }
            if (in_win(1)) { wchi[1 - base] = chi_b; wcell[1 - base] = cell_b; wfr[1 - base] = fr_b; }
            const int f_end = min(nfr + M1, last - 1);
            for (int n = 1; n <= f_end; n++) {
                double chi_c, fr_c;
                int cell_c;
                eval(n + 1, chi_c, cell_c, fr_c);
                const double dtau_n = 0.5 * (chi_b + chi_c) * P.dz_to(n + 1);
                const double inv_A = 0.5 * (dtau_prev + dtau_n) * dtau_prev;
                const double A = 1.0 / inv_A;
                const double inv_C = 0.5 * (dtau_prev + dtau_n) * dtau_n;
                F = (1.0 + A * F * i1F) * inv_C;
                i1F = 1.0 / (1.0 + F);
                if (in_win(n)) { wF[n - base] = F; wi1F[n - base] = i1F; wiC[n - base] = inv_C; }
                if (in_win(n + 1)) { wchi[n + 1 - base] = chi_c; wcell[n + 1 - base] = cell_c; wfr[n + 1 - base] = fr_c; }
                chi_b = chi_c;
                dtau_prev = dtau_n;
            }
            // backward: G from the back far end to max(nfr - M1 + 1, 1)
            eval(last, chi_a, cell_a, fr_a);
            eval(last - 1, chi_b, cell_b, fr_b);
            double dtau_next = 0.5 * (chi_b + chi_a) * P.dz_to(last);
            const double inverse_dtaud = 1.0 / dtau_next;
            const double Ad = 2.0 * inverse_dtaud * inverse_dtaud;
            const double Bd_min_Ad = 1.0 + 2.0 * inverse_dtaud;
            const double Bd = Bd_min_Ad + Ad;
            double G = 0.5 * Bd_min_Ad * dtau_next * dtau_next;
            double i1G = 1.0 / (1.0 + G);
            if (in_win(last)) {
                wG[last - base] = G; wi1G[last - base] = i1G; wchi[last - base] = chi_a;
                wcell[last - base] = cell_a; wfr[last - base] = fr_a;
            }
            const int g_end = max(nfr - M1 + 1, 1);
            for (int n = last - 1; n >= g_end; n--) {
                double chi_c, fr_c;
                int cell_c;
                eval(n - 1, chi_c, cell_c, fr_c);
                const double dtau_p = 0.5 * (chi_c + chi_b) * P.dz_to(n);
                const double inv_A = 0.5 * (dtau_p + dtau_next) * dtau_p;
                const double C = 1.0 / (0.5 * (dtau_p + dtau_next) * dtau_next);
                G = (1.0 + C * G * i1G) * inv_A;
                i1G = 1.0 / (1.0 + G);
                if (in_win(n)) { wG[n - base] = G; wi1G[n - base] = i1G; }
                if (in_win(n - 1)) { wchi[n - 1 - base] = chi_c; wcell[n - 1 - base] = cell_c; wfr[n - 1 - base] = fr_c; }
                chi_b = chi_c;
                dtau_next = dtau_p;
            }
            // the origin's row at distance d, weighted as the diagonal element
            const double wr = m.ray_w[r];
            const double pre = m.A[k] * (m.qw[z] * 2.0) * wr;
            auto weight_at = [&](int j, double lam) {
                const double width = line_k * __ldg(m.pw + wcell[j - base]);
                const double iw = 1.0 / width;
                const double x = iw * (wfr[j - base] - line_k);
                const double prof = iw * kINVERSE_SQRT_PI * exp(-(x * x));
                return pre * (wfr[j - base] * prof * lam / wchi[j - base]);
            };
            for (int d = 1; d <= M1; d++) {
                double vlo = 0.0, vup = 0.0;
                const int jl = nfr - d;
                if (active && jl >= 0) {
                    const double Ld = jl == 0
                        ? (1.0 + wG[1 - base]) / (B0_min_C0 + B0 * wG[1 - base])
                        : wiC[jl - base] / (wF[jl - base] + wG[jl + 1 - base] * wi1G[jl + 1 - base]);
                    double lam = Ld;
                    for (int q = jl + 1; q <= nfr; q++) lam *= wi1G[q - base];
                    vlo = weight_at(jl, lam);
                }
                const int ju = nfr + d;
                if (active && ju <= last) {
                    const double Ld = ju == last
                        ? (1.0 + wF[last - 1 - base]) / (Bd_min_Ad + Bd * wF[last - 1 - base])
                        : wiC[ju - base] / (wF[ju - base] + wG[ju + 1 - base] * wi1G[ju + 1 - base]);
                    double lam = Ld;
                    for (int q = ju - 1; q >= nfr; q--) lam *= wi1F[q - base];
                    vup = weight_at(ju, lam);
                }
                Ld_lo[d - 1] = vlo;
                Ld_up[d - 1] = vup;
            }
            // sums over the bins of each line of this chunk
            const int kfirst = (c * 32) / nq, klast = min(K - 1, (c * 32 + 31) / nq);
            for (int kk = kfirst; kk <= klast; kk++) {
                for (int d = 1; d <= M1; d++) {
                    double vl = (active && k == kk) ? Ld_lo[d - 1] : 0.0;
                    double vu = (active && k == kk) ? Ld_up[d - 1] : 0.0;
#pragma unroll
                    for (int s = 16; s > 0; s >>= 1) {
                        vl += __shfl_xor_sync(0xffffffffu, vl, s);
                        vu += __shfl_xor_sync(0xffffffffu, vu, s);
                    }
                    if (lane == 0) {
                        double *dst = Lo + ((int64_t)kk * np + r) * 2 * M1;
                        dst[d - 1] += vl;
                        dst[M1 + d - 1] += vu;
                    }
                }
            }
            __syncwarp();
        }
    }
}

}  // namespace

cudaError_t launch_offdiag(const ModelView &m, const TraceView &t, const OffdiagArgs &a,
                           DevFlags *flags, cudaStream_t s) {
    const int64_t n = a.s_end - a.s_begin;
    if (n <= 0) return cudaSuccess;
    (void)flags;   // the traces it walks were checked when they were built
    offdiag_kernel<<<(unsigned)((n + kOffWarps - 1) / kOffWarps), kOffWarps * 32, 0, s>>>(m, t, a);
    return cudaGetLastError();
}

}  // namespace mgr
