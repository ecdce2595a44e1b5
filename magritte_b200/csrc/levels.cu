// levels.cu -- level populations on the device: LTE start, line
// emissivities/opacities, Jeff, per-cell statistical equilibrium, the
// convergence statistics and Ng acceleration.
//
// With a local (diagonal) ALO the global rate matrix of
// LineProducingSpecies::update_using_statistical_equilibrium
// (Model/Lines/LineProducingSpecies/lineProducingSpecies.tpp:249-495) is
// block diagonal, one nlev x nlev block per cell; each block is assembled
// from the reference's triplets and solved by a warp (lane = row, partial
// pivoting, rows staged in shared memory).  Reductions are two-level with a
// fixed block count so results do not depend on scheduling.
#include "mgr_internal.cuh"

namespace mgr {

namespace {

constexpr int kStateqWarps = 4;
constexpr int kRowPitch = kMaxLevels + 1;
constexpr int kReduceBlocks = 1184;   // 8 x 148 SMs

__device__ __forceinline__ void write_emissivity_opacity(const ModelView &m, const LevelArgs &a,
                                                         int64_t p, int k, const double *pop) {
    const int K = m.nrad;
    const double ni = pop[m.irad[k]], nj = pop[m.jrad[k]];
    const double eps = kHH_OVER_FOUR_PI * m.A[k] * ni;
    const double kap = kHH_OVER_FOUR_PI * (nj * m.Ba[k] - ni * m.Bs[k]);
    a.eps[p * K + k] = eps;
    a.kap[p * K + k] = kap;
    const double g = kINVERSE_SQRT_PI * m.inv_pw[p] * a.mixed_scale;
    a.ehat_khat[p * K + k] = make_float2((float)(eps * g), (float)(kap * g));
}

// LineProducingSpecies::update_using_LTE (lineProducingSpecies.tpp:82-115)
__global__ void lte_kernel(ModelView m, LevelArgs a) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= m.N) return;
    const int nl = m.nlev;
    double *pop = a.pop + p * nl;
    double Z = 0.0;
    for (int i = 0; i < nl; i++) {
        pop[i] = m.weight[i] * exp(-m.energy[i] / (kKB * m.T[p]));
        Z += pop[i];
    }
    for (int i = 0; i < nl; i++) pop[i] *= m.pop_tot[p] / Z;
}

// Lines::set_emissivity_and_opacity (Model/Lines/lines.tpp:44-60)
__global__ void emissivity_opacity_kernel(ModelView m, LevelArgs a) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= m.N * m.nrad) return;
    const int64_t p = idx / m.nrad;
    const int k = (int)(idx - p * m.nrad);
    write_emissivity_opacity(m, a, p, k, a.pop + p * m.nlev);
}

// Simulation::compute_Jeff (Simulation/sim_lines.tpp:176-220), local ALO,
// for cells [c_begin, c_end)
__global__ void jeff_kernel(ModelView m, LevelArgs a) {
    const int64_t idx = a.c_begin * m.nrad + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= a.c_end * m.nrad) return;
    const int64_t p = idx / m.nrad;
    const int k = (int)(idx - p * m.nrad);
    const double diff = a.Lam[idx] * a.pop[p * m.nlev + m.irad[k]];
    a.Jeff[idx] = a.Jlin[idx] - kHH_OVER_FOUR_PI * diff;
}

// CollisionPartner::interpolate_collision_coefficients' table position:
// search() of Functions/interpolation.tpp, then t == 0 -> first column,
// otherwise linear between t-1 and t (extrapolating above the table).
__device__ __forceinline__ void colpar_position(const ColparDev &c, double T, int &t, double &step) {
    int start = 0, stop = c.ntmp - 1;
    if (T >= c.tmp[stop]) t = stop;
    else if (T <= c.tmp[start]) t = start;
    else {
        t = -1;
        while (stop > start + 1) {
            const int middle = (stop + start) / 2;
            if (T > c.tmp[middle]) start = middle;
            else if (T < c.tmp[middle]) stop = middle;
            else { t = middle; break; }
        }
        if (t < 0) t = stop;
    }
    step = (t == 0) ? 0.0 : (T - c.tmp[t - 1]) / (c.tmp[t] - c.tmp[t - 1]);
}

__device__ __forceinline__ void block_reduce3(double &cnt, double &sum, double &mx, double *red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) {
        cnt += __shfl_xor_sync(0xffffffffu, cnt, s);
        sum += __shfl_xor_sync(0xffffffffu, sum, s);
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, s));
    }
    if (lane == 0) { red[3 * warp] = cnt; red[3 * warp + 1] = sum; red[3 * warp + 2] = mx; }
    __syncthreads();
    if (threadIdx.x == 0) {
        const int nw = blockDim.x >> 5;
        cnt = 0.0; sum = 0.0; mx = 0.0;
        for (int w = 0; w < nw; w++) {
            cnt += red[3 * w]; sum += red[3 * w + 1]; mx = fmax(mx, red[3 * w + 2]);
        }
    }
}

// Rows of cell p's block of RT (transpose convention,
// lineProducingSpecies.tpp:282-389) owned by lane i: radiative rates, the
// local ALO element (nr = p) with the opacity of the populations `old`,
// collisions, and the conservation row replacing the last level's.
__device__ __forceinline__ void assemble_rows(const ModelView &m, const LevelArgs &a, int64_t p,
                                              int i, double *row, double *y, const double *old) {
    const int nl = m.nlev, K = m.nrad, last = nl - 1;
    // radiative transitions
    for (int k = 0; k < K; k++) {
        const int I = m.irad[k], J = m.jrad[k];
        if (i != I && i != J) continue;
        const double Jeff = a.Jeff[p * K + k];
        const double v_IJ = m.A[k] + m.Bs[k] * Jeff;
        const double v_JI = m.Ba[k] * Jeff;
        if (J != last && i == J) { row[I] += v_IJ; row[J] += -v_JI; }
        if (I != last && i == I) { row[J] += v_JI; row[I] += -v_IJ; }
    }
    // approximated Lambda operator (nr = p)
    for (int k = 0; k < K; k++) {
        const int I = m.irad[k], J = m.jrad[k];
        if (i != I && i != J) continue;
        const double opac = kHH_OVER_FOUR_PI * (old[J] * m.Ba[k] - old[I] * m.Bs[k]);
        const double v_IJ = -a.Lam[p * K + k] * opac;
        if (J != last && i == J) row[I] += v_IJ;
        if (I != last && i == I) row[I] += -v_IJ;
    }
    // collisions
    for (int c = 0; c < m.ncolpar; c++) {
        const ColparDev &cp = m.colpar[c];
        double abn = cp.abn[p];
        const double tmp = m.T[p];
        if (cp.ortho_para != 0) {
            const double frac_H2_para = 1.0 / (1.0 + 9.0 * exp(-170.5 / tmp));
            if (cp.ortho_para == 1) abn *= (1.0 - frac_H2_para);
            if (cp.ortho_para == 2) abn *= frac_H2_para;
        }
        int t;
        double step;
        colpar_position(cp, tmp, t, step);
        for (int k = 0; k < cp.ncol; k++) {
            const int I = cp.icol[k], J = cp.jcol[k];
            if (i != I && i != J) continue;
            double Cd, Ce;
            if (t == 0) {
                Cd = cp.Cd[k];
                Ce = cp.Ce[k];
            } else {
                const double cd0 = cp.Cd[(t - 1) * cp.ncol + k], cd1 = cp.Cd[t * cp.ncol + k];
                const double ce0 = cp.Ce[(t - 1) * cp.ncol + k], ce1 = cp.Ce[t * cp.ncol + k];
                Cd = cd0 + (cd1 - cd0) * step;
                Ce = ce0 + (ce1 - ce0) * step;
            }
            const double v_IJ = Cd * abn, v_JI = Ce * abn;
            if (J != last && i == J) { row[I] += v_IJ; row[J] += -v_JI; }
            if (I != last && i == I) { row[J] += v_JI; row[I] += -v_IJ; }
        }
    }
    if (i == last) {
        for (int j = 0; j < nl; j++) row[j] += 1.0;
        y[last] = m.pop_tot[p];
    }
}

// Partial-pivot LU of the nl x nl rows M (pitch kRowPitch) with right-hand
// side y, one lane per row; returns true on a zero pivot.  The pivot search
// is a butterfly over the lanes, its result taken from lane 0.
__device__ __forceinline__ bool warp_lu(double *M, double *y, int nl, int i) {
    bool singular = false;
    for (int kc = 0; kc < nl; kc++) {
        double v = (i >= kc && i < nl) ? fabs(M[i * kRowPitch + kc]) : -1.0;
        int idx = i;
#pragma unroll
        for (int s = 16; s > 0; s >>= 1) {
            const double ov = __shfl_xor_sync(0xffffffffu, v, s);
            const int oi = __shfl_xor_sync(0xffffffffu, idx, s);
            if (ov > v || (ov == v && oi < idx)) { v = ov; idx = oi; }
        }
        // lane 0's result for everyone: NaNs can make the butterfly
        // disagree between lanes, and the loop must stay warp-uniform
        v = __shfl_sync(0xffffffffu, v, 0);
        idx = __shfl_sync(0xffffffffu, idx, 0);
        if (!(v > 0.0) || idx >= nl) { singular = true; break; }
        if (idx != kc) {
            if (i < nl) {
                const double t0 = M[kc * kRowPitch + i];
                M[kc * kRowPitch + i] = M[idx * kRowPitch + i];
                M[idx * kRowPitch + i] = t0;
            }
            if (i == 0) { const double t1 = y[kc]; y[kc] = y[idx]; y[idx] = t1; }
        }
        __syncwarp();
        if (i > kc && i < nl) {
            const double l = M[i * kRowPitch + kc] * (1.0 / M[kc * kRowPitch + kc]);
            if (l != 0.0) {
                for (int j = kc + 1; j < nl; j++) M[i * kRowPitch + j] -= l * M[kc * kRowPitch + j];
                y[i] -= l * y[kc];
            }
        }
        __syncwarp();
    }
    return singular;
}

// Back substitution after warp_lu: y becomes the solution.
__device__ __forceinline__ void warp_back_substitute(const double *M, double *y, int nl, int i) {
    for (int jc = nl - 1; jc >= 0; jc--) {
        if (i == jc) y[jc] = y[jc] / M[jc * kRowPitch + jc];
        __syncwarp();
        if (i < jc) y[i] -= M[i * kRowPitch + jc] * y[jc];
        __syncwarp();
    }
}

// One warp per cell: assemble the cell's block of RT (transpose convention,
// lineProducingSpecies.tpp:282-389), solve it, update populations and their
// history, then convergence partials and the cell's emissivities/opacities.
__global__ void __launch_bounds__(kStateqWarps * 32) stateq_kernel(ModelView m, LevelArgs a,
                                                                   DevFlags *flags) {
    __shared__ double Msh[kStateqWarps][kMaxLevels * kRowPitch];
    __shared__ double ysh[kStateqWarps][kMaxLevels];
    __shared__ double popsh[kStateqWarps][kMaxLevels];
    __shared__ double red[kStateqWarps * 3];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t p = a.c_begin + (int64_t)blockIdx.x * kStateqWarps + warp;
    // cells of a converged model of a batch keep their populations
    const bool valid = p < a.c_end && !(m.seg_active && !m.seg_active[m.cell_seg[p]]);
    const int nl = m.nlev, K = m.nrad;
    double *M = Msh[warp];
    double *y = ysh[warp];
    double *old = popsh[warp];
    double cnt = 0.0, rsum = 0.0, rmax = 0.0;
    if (valid) {
        const int i = lane;
        if (i < nl) {
            const int64_t q = p * nl + i;
            const double o = a.pop[q];
            a.prev3[q] = a.prev2[q];
            a.prev2[q] = a.prev1[q];
            a.prev1[q] = o;
            old[i] = o;
            for (int j = 0; j < nl; j++) M[i * kRowPitch + j] = 0.0;
            y[i] = 0.0;
        }
        __syncwarp();
        if (i < nl) assemble_rows(m, a, p, i, M + i * kRowPitch, y, old);
        __syncwarp();
        const bool singular = warp_lu(M, y, nl, i);
        if (singular) {
            if (lane == 0) atomicAdd(&flags->lu_err, 1ull);
        } else {
            warp_back_substitute(M, y, nl, i);
            if (i < nl) {
                const double nw = y[i];
                a.pop[p * nl + i] = nw;
                old[i] = nw;   // new populations for the opacity update below
            }
        }
        __syncwarp();
        // convergence statistics (lineProducingSpecies.tpp:120-171)
        if (i < nl) {
            const double nw = a.pop[p * nl + i], pv = a.prev1[p * nl + i];
            if (nw > 1.0E-10 * m.pop_tot[p]) {
                double rc = 2.0;
                rc *= fabs(nw - pv);
                rc /= (nw + pv);
                if (rc > m.pop_prec) cnt = 1.0;
                rsum = rc;
                rmax = rc;
            }
        }
        for (int k = lane; k < K; k += 32) write_emissivity_opacity(m, a, p, k, old);
    }
    block_reduce3(cnt, rsum, rmax, red);
    if (threadIdx.x == 0) {
        // at the global position of this block of cells
        const int64_t g = a.c_begin / kStateqWarps + blockIdx.x;
        a.partials[3 * g + 0] = cnt;
        a.partials[3 * g + 1] = rsum;
        a.partials[3 * g + 2] = rmax;
    }
}

// ------------------------------------------------------------ non-local ALO
//
// With n_off_diag = M >= 2 every (cell p, line k) also holds the M-1 nearest
// off-diagonal ALO elements on each side of every ray pair (NonlocalArgs),
// each belonging to the cell nr the ray passes there.

// compute_Jeff (sim_lines.tpp:176-220) over every element of (p, k): the
// diagonal one, then the non-local ones in (pair, side, distance) order.
__global__ void jeff_nonlocal_kernel(ModelView m, LevelArgs a, NonlocalArgs nl) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= m.N * m.nrad) return;
    const int64_t p = idx / m.nrad;
    const int k = (int)(idx - p * m.nrad);
    const int I = m.irad[k], nlev = m.nlev;
    const int64_t ne = (int64_t)m.npairs * 2 * nl.M1;
    double diff = a.Lam[idx] * a.pop[p * nlev + I];
    for (int64_t e = 0; e < ne; e++) {
        const int c = nl.Loff_nr[p * ne + e];
        if (c < 0) continue;
        diff += nl.Loff[idx * ne + e] * a.pop[(int64_t)c * nlev + I];
    }
    a.Jeff[idx] = a.Jlin[idx] - kHH_OVER_FOUR_PI * diff;
}

// One block-Jacobi sweep of the rate equations of all cells
// (lineProducingSpecies.tpp:249-495 with n_off_diag > 0): cell p's block as
// stateq_kernel assembles it from the populations before the solve (prev1,
// the history already shifted), plus every non-local element (nr, Ls) of
// the cell with v = -Ls * opacity(p, k): v at (J(p), I(nr)) and -v at
// (I(p), I(nr)) -- in the block when nr = p, otherwise moved to the
// right-hand side with nr's populations from x_in.  The solution goes to
// x_out; change[block] receives the largest change of the block's cells
// relative to the population (or to 1e-10 of the cell's total below that).
__global__ void __launch_bounds__(kStateqWarps * 32) stateq_nonlocal_kernel(ModelView m,
                                                                            LevelArgs a,
                                                                            NonlocalArgs nl,
                                                                            DevFlags *flags) {
    __shared__ double Msh[kStateqWarps][kMaxLevels * kRowPitch];
    __shared__ double ysh[kStateqWarps][kMaxLevels];
    __shared__ double popsh[kStateqWarps][kMaxLevels];
    __shared__ double red[kStateqWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t p = (int64_t)blockIdx.x * kStateqWarps + warp;
    const int nlev = m.nlev, K = m.nrad, last = nlev - 1;
    const int64_t ne = (int64_t)m.npairs * 2 * nl.M1;
    double *M = Msh[warp];
    double *y = ysh[warp];
    double *old = popsh[warp];
    double change = 0.0;
    if (p < m.N) {
        const int i = lane;
        if (i < nlev) {
            old[i] = a.prev1[p * nlev + i];
            for (int j = 0; j < nlev; j++) M[i * kRowPitch + j] = 0.0;
            y[i] = 0.0;
        }
        __syncwarp();
        if (i < nlev) {
            double *row = M + i * kRowPitch;
            assemble_rows(m, a, p, i, row, y, old);
            for (int k = 0; k < K; k++) {
                const int I = m.irad[k], J = m.jrad[k];
                if (i != I && i != J) continue;
                const double opac = kHH_OVER_FOUR_PI * (old[J] * m.Ba[k] - old[I] * m.Bs[k]);
                for (int64_t e = 0; e < ne; e++) {
                    const int c = nl.Loff_nr[p * ne + e];
                    if (c < 0) continue;
                    const double v = -nl.Loff[(p * K + k) * ne + e] * opac;
                    if (c == p) {
                        if (J != last && i == J) row[I] += v;
                        if (I != last && i == I) row[I] += -v;
                    } else {
                        const double xc = nl.x_in[(int64_t)c * nlev + I];
                        if (J != last && i == J) y[J] -= v * xc;
                        if (I != last && i == I) y[I] += v * xc;
                    }
                }
            }
        }
        __syncwarp();
        const bool singular = warp_lu(M, y, nlev, i);
        if (singular) {
            // the cell keeps its populations; the solve reports the zero pivot
            if (lane == 0) atomicAdd(&flags->lu_err, 1ull);
            if (i < nlev) nl.x_out[p * nlev + i] = nl.x_in[p * nlev + i];
        } else {
            warp_back_substitute(M, y, nlev, i);
            if (i < nlev) {
                const double v = y[i];
                const double prev = nl.x_in[p * nlev + i];
                change = fabs(v - prev) / fmax(fabs(v), 1.0E-10 * m.pop_tot[p]);
                nl.x_out[p * nlev + i] = v;
            }
        }
    }
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) change = fmax(change, __shfl_xor_sync(0xffffffffu, change, s));
    if (lane == 0) red[warp] = change;
    __syncthreads();
    if (threadIdx.x == 0) {
        double mx = 0.0;
        for (int w = 0; w < kStateqWarps; w++) mx = fmax(mx, red[w]);
        nl.change[blockIdx.x] = mx;
    }
}

// Largest of the per-block changes into change[nblocks] (one block).
__global__ void max_reduce_kernel(double *change, int nblocks) {
    __shared__ double red[32];
    double mx = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) mx = fmax(mx, change[b]);
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, s));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) mx = fmax(mx, red[w]);
        change[nblocks] = mx;
    }
}

// Population history of the cells outside [c_begin, c_end), shifted as the
// statistical-equilibrium kernel shifts it for its own cells; their new
// populations come from the shard that owns them.
__global__ void history_shift_kernel(ModelView m, LevelArgs a) {
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= m.N * m.nlev) return;
    const int64_t p = q / m.nlev;
    if (p >= a.c_begin && p < a.c_end) return;
    a.prev3[q] = a.prev2[q];
    a.prev2[q] = a.prev1[q];
    a.prev1[q] = a.pop[q];
}

// Per-cell convergence partials (after an Ng step).
__global__ void convergence_partials_kernel(ModelView m, LevelArgs a) {
    __shared__ double red[32 * 3];
    double cnt = 0.0, rsum = 0.0, rmax = 0.0;
    const int64_t n = m.N * m.nlev;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
         q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = q / m.nlev;
        const double nw = a.pop[q], pv = a.prev1[q];
        if (nw > 1.0E-10 * m.pop_tot[p]) {
            double rc = 2.0;
            rc *= fabs(nw - pv);
            rc /= (nw + pv);
            if (rc > m.pop_prec) cnt += 1.0;
            rsum += rc;
            rmax = fmax(rmax, rc);
        }
    }
    block_reduce3(cnt, rsum, rmax, red);
    if (threadIdx.x == 0) {
        a.partials[3 * blockIdx.x + 0] = cnt;
        a.partials[3 * blockIdx.x + 1] = rsum;
        a.partials[3 * blockIdx.x + 2] = rmax;
    }
}

static_assert(kStateqWarps == kCellsPerPartial, "one convergence partial per stateq block");

// Final reduction of (count, sum, max) partials: stats[0] = fraction not
// converged, stats[1] = mean relative change, stats[2] = max relative change.
__global__ void convergence_final_kernel(ModelView m, LevelArgs a, int nparts) {
    __shared__ double red[32 * 3];
    double cnt = 0.0, rsum = 0.0, rmax = 0.0;
    for (int b = threadIdx.x; b < nparts; b += blockDim.x) {
        cnt += a.partials[3 * b];
        rsum += a.partials[3 * b + 1];
        rmax = fmax(rmax, a.partials[3 * b + 2]);
    }
    block_reduce3(cnt, rsum, rmax, red);
    if (threadIdx.x == 0) {
        const double weight = 1.0 / (double)(m.N * m.nlev);
        a.stats[0] = cnt * weight;
        a.stats[1] = rsum * weight;
        a.stats[2] = rmax;
    }
}

// Ng acceleration (lineProducingSpecies.tpp:181-238): five dot products ...
__global__ void ng_dots_kernel(ModelView m, LevelArgs a) {
    __shared__ double red[32][5];
    double s[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    const int64_t n = m.N * m.nlev;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
         q += (int64_t)gridDim.x * blockDim.x) {
        const double P = a.pop[q], p1 = a.prev1[q], p2 = a.prev2[q], p3 = a.prev3[q];
        const double Q1 = P - 2.0 * p1 + p2;
        const double Q2 = P - p1 - p2 + p3;
        const double Q3 = P - p1;
        s[0] += Q1 * Q1; s[1] += Q1 * Q2; s[2] += Q2 * Q2; s[3] += Q1 * Q3; s[4] += Q2 * Q3;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < 5; j++)
        for (int o = 16; o > 0; o >>= 1) s[j] += __shfl_xor_sync(0xffffffffu, s[j], o);
    if (lane == 0) for (int j = 0; j < 5; j++) red[warp][j] = s[j];
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int j = 0; j < 5; j++) {
            double t = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w][j];
            a.partials[5 * blockIdx.x + j] = t;
        }
    }
}

// ... their sum and the extrapolation coefficients: stats[4] = a,
// stats[5] = b, stats[6] = 1 when the denominator is non-zero.
__global__ void ng_coeff_kernel(LevelArgs a, int nparts) {
    if (threadIdx.x != 0) return;
    double s[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (int b = 0; b < nparts; b++)
        for (int j = 0; j < 5; j++) s[j] += a.partials[5 * b + j];
    const double A1 = s[0], A2 = s[1], B2 = s[2], C1 = s[3], C2 = s[4];
    const double B1 = A2;
    const double denominator = A1 * B2 - A2 * B1;
    if (denominator != 0.0) {
        a.stats[4] = (C1 * B2 - C2 * B1) / denominator;
        a.stats[5] = (C2 * A1 - C1 * A2) / denominator;
        a.stats[6] = 1.0;
    } else {
        a.stats[4] = 0.0;
        a.stats[5] = 0.0;
        a.stats[6] = 0.0;
    }
}

__global__ void ng_update_kernel(ModelView m, LevelArgs a) {
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= m.N * m.nlev) return;
    if (a.stats[6] == 0.0) return;
    const double ca = a.stats[4], cb = a.stats[5];
    const double P = a.pop[q], p1 = a.prev1[q], p2 = a.prev2[q];
    a.pop[q] = (1.0 - ca - cb) * P + ca * p1 + cb * p2;
    a.prev3[q] = p2;
    a.prev2[q] = p1;
    a.prev1[q] = P;
}

// Simulation::compute_boundary_intensities (Simulation/sim_radiation.tpp:17-48):
// I_bdy[b][f] = planck(T_b, nu_p[f]) on the grid of the boundary cell p.
__global__ void boundary_table_kernel(ModelView m, int64_t nb, const int64_t *b2c, double *table) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nb * m.nfreqs) return;
    const int64_t b = idx / m.nfreqs;
    const int f = (int)(idx - b * m.nfreqs);
    const int64_t p = b2c[b];
    const int k = f / m.nquads;
    const double line = m.line[k];
    const double nu = radd(line, rmul(rmul(line, m.pw[p]), m.roots[f - k * m.nquads]));
    table[idx] = planck(m.bdy_T[b], nu);
}

}  // namespace

int level_partials_needed(const ModelView &m) {
    const int64_t sb = (m.N + kStateqWarps - 1) / kStateqWarps;
    const int64_t need = sb > kReduceBlocks ? sb : kReduceBlocks;
    return (int)need;
}

static inline unsigned blocks_for(int64_t n, int threads) {
    return (unsigned)((n + threads - 1) / threads);
}

cudaError_t launch_boundary_table(const ModelView &m, int64_t nboundary, const int64_t *b2c,
                                  double *table, cudaStream_t s) {
    boundary_table_kernel<<<blocks_for(nboundary * m.nfreqs, 256), 256, 0, s>>>(m, nboundary, b2c,
                                                                                 table);
    return cudaGetLastError();
}

cudaError_t launch_lte(const ModelView &m, const LevelArgs &a, cudaStream_t s) {
    lte_kernel<<<blocks_for(m.N, 256), 256, 0, s>>>(m, a);
    return cudaGetLastError();
}

cudaError_t launch_emissivity_opacity(const ModelView &m, const LevelArgs &a, cudaStream_t s) {
    emissivity_opacity_kernel<<<blocks_for(m.N * m.nrad, 256), 256, 0, s>>>(m, a);
    return cudaGetLastError();
}

cudaError_t launch_jeff(const ModelView &m, const LevelArgs &a, cudaStream_t s) {
    if (a.c_end <= a.c_begin) return cudaSuccess;
    jeff_kernel<<<blocks_for((a.c_end - a.c_begin) * m.nrad, 256), 256, 0, s>>>(m, a);
    return cudaGetLastError();
}

cudaError_t launch_stateq(const ModelView &m, const LevelArgs &a, DevFlags *flags, cudaStream_t s) {
    const bool whole = a.c_begin == 0 && a.c_end == m.N;
    if (a.c_end > a.c_begin) {
        stateq_kernel<<<blocks_for(a.c_end - a.c_begin, kStateqWarps), kStateqWarps * 32, 0, s>>>(
            m, a, flags);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    if (!whole) {
        history_shift_kernel<<<blocks_for(m.N * m.nlev, 256), 256, 0, s>>>(m, a);
        return cudaGetLastError();
    }
    return launch_convergence_final(m, a, s);
}

cudaError_t launch_jeff_nonlocal(const ModelView &m, const LevelArgs &a, const NonlocalArgs &nl,
                                 cudaStream_t s) {
    jeff_nonlocal_kernel<<<blocks_for(m.N * m.nrad, 256), 256, 0, s>>>(m, a, nl);
    return cudaGetLastError();
}

int nonlocal_sweep_blocks(const ModelView &m) { return (int)blocks_for(m.N, kStateqWarps); }

cudaError_t launch_history_shift(const ModelView &m, const LevelArgs &a, cudaStream_t s) {
    LevelArgs b = a;
    b.c_begin = b.c_end = 0;   // every cell
    history_shift_kernel<<<blocks_for(m.N * m.nlev, 256), 256, 0, s>>>(m, b);
    return cudaGetLastError();
}

cudaError_t launch_stateq_nonlocal_sweep(const ModelView &m, const LevelArgs &a,
                                         const NonlocalArgs &nl, DevFlags *flags, cudaStream_t s) {
    const unsigned nb = blocks_for(m.N, kStateqWarps);
    stateq_nonlocal_kernel<<<nb, kStateqWarps * 32, 0, s>>>(m, a, nl, flags);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    max_reduce_kernel<<<1, 1024, 0, s>>>(nl.change, (int)nb);
    return cudaGetLastError();
}

cudaError_t launch_convergence_final(const ModelView &m, const LevelArgs &a, cudaStream_t s) {
    convergence_final_kernel<<<1, 1024, 0, s>>>(m, a, (int)blocks_for(m.N, kStateqWarps));
    return cudaGetLastError();
}

cudaError_t launch_convergence(const ModelView &m, const LevelArgs &a, cudaStream_t s) {
    convergence_partials_kernel<<<kReduceBlocks, 256, 0, s>>>(m, a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    convergence_final_kernel<<<1, 1024, 0, s>>>(m, a, kReduceBlocks);
    return cudaGetLastError();
}

cudaError_t launch_ng(const ModelView &m, const LevelArgs &a, cudaStream_t s) {
    ng_dots_kernel<<<kReduceBlocks, 256, 0, s>>>(m, a);
    ng_coeff_kernel<<<1, 32, 0, s>>>(a, kReduceBlocks);
    ng_update_kernel<<<blocks_for(m.N * m.nlev, 256), 256, 0, s>>>(m, a);
    return cudaGetLastError();
}

}  // namespace mgr
