// image.cu -- images of the model: the emergent intensity along one ray
// direction through every cell (Simulation::compute_and_write_image,
// Simulation/sim_radiation.tpp:348-478).
//
// For origin o the ray pair is the rest-frame trace of the antipode (in
// front, far end first), the origin, and the trace of the ray itself.  The
// reference eliminates the whole pair and substitutes back to its front
// (RayPair::solve_for_image, Simulation/Raypair/raypair_solver.tpp:523-579),
// then reads I_m = 2 u_front - I_bdy_0 and I_p = 2 u_end - I_bdy_n
// (RayPair::get_Im_at_front / get_Ip_at_end, raypair.tpp:205-229).  Here a
// lane runs two one-sided eliminations in projective form (the scaled
// Rybicki-Hummer quantities F~ = a/b, S~ = c/b of the formal solve), one
// from each far end to the other; each ends in the other end's boundary
// row, which gives u there directly.  Same linear system, no back
// substitution and O(1) state per lane; the two chains are independent and
// advance together.
//
// Work decomposition as in the formal solve: one warp per origin, lanes
// over 32-bin chunks of the image grid, every lane walking the same traced
// points (broadcast loads).  FP64 throughout.
#include "mgr_internal.cuh"

namespace mgr {

namespace {

constexpr int kImageWarps = 4;

// Radiation::rescale_I_bdy (Model/Radiation/radiation.tpp:341-373) on the
// image grid, which is the same for every cell: the first bin whose
// frequency is >= freq (found by bisection on the ascending grid, where the
// reference searches linearly), then linear interpolation from the bin
// below it.
__device__ double image_boundary(const ImageArgs &a, const ModelView &m, double freq, int cell,
                                 DevFlags *flags) {
    const int b = __ldg(m.cell2bdy + cell);
    if (b < 0) {
        atomicAdd(&flags->trace_err, 1ull);
        return 0.0;
    }
    const int nf = a.nf;
    int lo = 0, hi = nf;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (freq <= __ldg(a.grid + mid)) hi = mid;
        else lo = mid + 1;
    }
    const double *I = a.table + (int64_t)b * nf;
    const int notch = lo < nf ? lo : nf - 1;
    if (notch == 0 || notch == nf - 1) return __ldg(I + notch);
    const double nu1 = __ldg(a.grid + notch), nu2 = __ldg(a.grid + notch - 1);
    const double I1 = __ldg(I + notch), I2 = __ldg(I + notch - 1);
    return (I2 - I1) / (nu2 - nu1) * (freq - nu1) + I1;
}

// 2^-e for the binary exponent e of b > 0: brings b into [1, 2) exactly.
__device__ __forceinline__ double pow2_inv(double b) {
    const int hi = __double2hiint(b);
    return __hiloint2double(0x7fe00000 - (hi & 0x7ff00000), 0);
}

// One-sided elimination in projective form on half optical depths
// dh = dtau/2: F~ = a/b, S~ = c/b.
struct ImageChain {
    double t_a, dh_prev, a, b, c;
    // boundary row of the starting end (source t0, boundary intensity I),
    // then the first step, across a segment of half optical depth dh
    __device__ __forceinline__ void first(double t0, double dh, double I) {
        a = dh * (dh + 1.0);
        b = fma(2.0, a, 1.0);
        c = dh * fma(t0, dh, I);
        dh_prev = dh;
    }
    // onto the next point across a segment of half optical depth dh; t_a is
    // the source of the point being left
    __device__ __forceinline__ void step(double dh) {
        const double H = dh_prev + dh;
        const double P = H * dh_prev, Q = H * dh;
        const double Pb = P * b;
        a = Q * (Pb + a);
        c = Q * fma(t_a, Pb, c);
        b = fma(2.0, a, Pb);
        const double sc = pow2_inv(b);
        a *= sc;
        b *= sc;
        c *= sc;
        dh_prev = dh;
    }
    // u at the last point: its boundary row with source t_end and I_end
    __device__ __forceinline__ double finish(double t_end, double I_end) const {
        const double dh = dh_prev;
        const double D = 1.0 / fma(dh * (dh + 1.0), b, a);
        return fma(dh * fma(t_end, dh, I_end), b, c) * D;
    }
};

__global__ void __launch_bounds__(kImageWarps * 32) image_kernel(ModelView m, ImageArgs a,
                                                                 DevFlags *flags) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t o = (int64_t)blockIdx.x * kImageWarps + warp;
    if (o >= m.N) return;
    const int64_t N = m.N;
    const int nf = a.nf;
    const int n_ar = a.len[o], n_r = a.len[N + o];
    const int64_t off_ar = a.off[o], off_r = a.off[N + o];
    const int ndep = n_ar + n_r + 1;
    const int bo = m.cell2bdy[o];
    for (int f0 = 0; f0 < nf; f0 += 32) {
        const int f = f0 + lane;
        if (f >= nf) break;
        if (ndep <= 1) {
            // a ray pair of the origin alone: its boundary value
            const double I = bo >= 0 ? a.table[(int64_t)bo * nf + f] : 0.0;
            if (bo < 0) atomicAdd(&flags->trace_err, 1ull);
            a.I_m[o * nf + f] = I;
            a.I_p[o * nf + f] = I;
            continue;
        }
        const double nu = a.grid[f];
        const int lo = a.lo[f], hi = a.hi[f];
        // point i of the pair (front far end first): cell and frequency;
        // the origin is evaluated at its grid frequency, as Simulation::setup
        // does (simulation.tpp:214-222), every traced point at shift * nu
        auto point = [&](int i, int &cell, double &freq) {
            if (i < n_ar) {
                const int64_t g = off_ar + (n_ar - 1 - i);
                cell = a.cell[g];
                freq = a.shift[g] * nu;
            } else if (i == n_ar) {
                cell = (int)o;
                freq = nu;
            } else {
                const int64_t g = off_r + (i - n_ar - 1);
                cell = a.cell[g];
                freq = a.shift[g] * nu;
            }
        };
        // length of the segment between points i and i + 1
        auto seg = [&](int i) {
            return i < n_ar ? a.dZ[off_ar + (n_ar - 1 - i)] : a.dZ[off_r + (i - n_ar)];
        };
        auto eval = [&](int i, double &chi, double &t, double &freq, int &cell) {
            point(i, cell, freq);
            double eta;
            eta_chi_double(m, a.eps, a.kap, cell, freq, lo, hi, eta, chi);
            t = eta / chi;
        };
        // both far ends: sources and boundary intensities
        double chi0, t0, fr0, chiN, tN, frN;
        int c0, cN;
        eval(0, chi0, t0, fr0, c0);
        eval(ndep - 1, chiN, tN, frN, cN);
        const double I0 = n_ar > 0 ? image_boundary(a, m, fr0, c0, flags)
                                   : (bo >= 0 ? a.table[(int64_t)bo * nf + f] : 0.0);
        const double In = n_r > 0 ? image_boundary(a, m, frN, cN, flags)
                                  : (bo >= 0 ? a.table[(int64_t)bo * nf + f] : 0.0);
        // forward chain (front -> end) and backward chain (end -> front)
        ImageChain F, B;
        double chiF = chi0, chiB = chiN;
        F.t_a = t0;
        B.t_a = tN;
        for (int s = 1; s < ndep; s++) {
            double chi1, t1, fr1, chi2, t2, fr2;
            int c1, c2;
            eval(s, chi1, t1, fr1, c1);               // forward chain's next point
            eval(ndep - 1 - s, chi2, t2, fr2, c2);    // backward chain's next point
            const double dhF = 0.25 * (chiF + chi1) * seg(s - 1);
            const double dhB = 0.25 * (chiB + chi2) * seg(ndep - 1 - s);
            if (s == 1) {
                F.first(t0, dhF, I0);
                B.first(tN, dhB, In);
            } else {
                F.step(dhF);
                B.step(dhB);
            }
            F.t_a = t1;
            B.t_a = t2;
            chiF = chi1;
            chiB = chi2;
        }
        const double u_end = F.finish(F.t_a, In);
        const double u_front = B.finish(B.t_a, I0);
        a.I_p[o * nf + f] = 2.0 * u_end - In;
        a.I_m[o * nf + f] = 2.0 * u_front - I0;
    }
}

// Simulation::compute_boundary_intensities (sim_radiation.tpp:17-48) on the
// image grid: Planck at each boundary cell's temperature.
__global__ void image_table_kernel(ModelView m, int64_t nb, const double *grid, int nf,
                                   double *table) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nb * nf) return;
    const int64_t b = idx / nf;
    table[idx] = planck(m.bdy_T[b], grid[idx - b * nf]);
}

}  // namespace

cudaError_t launch_image_table(const ModelView &m, int64_t nboundary, const int64_t *b2c,
                               const double *grid, int nf, double *table, cudaStream_t s) {
    (void)b2c;
    const int64_t n = nboundary * nf;
    image_table_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(m, nboundary, grid, nf, table);
    return cudaGetLastError();
}

cudaError_t launch_image(const ModelView &m, const ImageArgs &a, DevFlags *flags, cudaStream_t s) {
    const int64_t blocks = (m.N + kImageWarps - 1) / kImageWarps;
    image_kernel<<<(unsigned)blocks, kImageWarps * 32, 0, s>>>(m, a, flags);
    return cudaGetLastError();
}

}  // namespace mgr
