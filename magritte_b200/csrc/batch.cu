// batch.cu -- per-model reductions for a batch of independent models held
// as one point cloud.
//
// The reference iterates one model per Simulation
// (Simulation::compute_level_populations, sim_lines.tpp:61-164): its
// convergence test (LineProducingSpecies::check_for_convergence,
// lineProducingSpecies.tpp:120-171) and Ng step
// (update_using_Ng_acceleration, lineProducingSpecies.tpp:181-238) reduce
// over that model's cells only.  A batch keeps that meaning with one block
// per model: each block reduces its model's cell range in a fixed order (so
// results do not depend on scheduling) and models that have converged are
// skipped.
#include "mgr_internal.cuh"

namespace mgr {

namespace {

constexpr int kSegThreads = 512;

template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double (*red)[NV]) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < NV; j++)
        for (int s = 16; s > 0; s >>= 1) v[j] += __shfl_xor_sync(0xffffffffu, v[j], s);
    if (lane == 0)
        for (int j = 0; j < NV; j++) red[warp][j] = v[j];
    __syncthreads();
    for (int j = 0; j < NV; j++) {
        double t = 0.0;
        for (int w = 0; w < kSegThreads / 32; w++) t += red[w][j];
        v[j] = t;   // every thread holds the block total
    }
    __syncthreads();
}

// seg_stats[3 s + (0, 1, 2)] = fraction of the model's (cell, level) pairs
// not converged, mean relative change, max relative change.
__global__ void __launch_bounds__(kSegThreads) seg_convergence_kernel(ModelView m, LevelArgs a,
                                                                      double *seg_stats) {
    __shared__ double red[kSegThreads / 32][2];
    __shared__ double redm[kSegThreads / 32];
    const int64_t sg = blockIdx.x;
    if (!m.seg_active[sg]) return;
    const int64_t c0 = m.seg_begin[sg], c1 = m.seg_begin[sg + 1];
    const int nl = m.nlev;
    double v[2] = {0.0, 0.0};
    double mx = 0.0;
    for (int64_t q = c0 * nl + threadIdx.x; q < c1 * nl; q += kSegThreads) {
        const int64_t p = q / nl;
        const double nw = a.pop[q], pv = a.prev1[q];
        if (nw > 1.0E-10 * m.pop_tot[p]) {
            double rc = 2.0;
            rc *= fabs(nw - pv);
            rc /= (nw + pv);
            if (rc > m.pop_prec) v[0] += 1.0;
            v[1] += rc;
            mx = fmax(mx, rc);
        }
    }
    for (int s = 16; s > 0; s >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, s));
    if ((threadIdx.x & 31) == 0) redm[threadIdx.x >> 5] = mx;
    block_sum<2>(v, red);
    if (threadIdx.x == 0) {
        double m2 = 0.0;
        for (int w = 0; w < kSegThreads / 32; w++) m2 = fmax(m2, redm[w]);
        const double weight = 1.0 / (double)((c1 - c0) * nl);
        seg_stats[3 * sg + 0] = v[0] * weight;
        seg_stats[3 * sg + 1] = v[1] * weight;
        seg_stats[3 * sg + 2] = m2;
    }
}

// One Ng step per active model: the five dot products over the model's
// populations, the extrapolation coefficients, and the update with the
// history shift (the single-model kernels in levels.cu, per model).
__global__ void __launch_bounds__(kSegThreads) seg_ng_kernel(ModelView m, LevelArgs a) {
    __shared__ double red[kSegThreads / 32][5];
    const int64_t sg = blockIdx.x;
    if (!m.seg_active[sg]) return;
    const int64_t q0 = m.seg_begin[sg] * m.nlev, q1 = m.seg_begin[sg + 1] * m.nlev;
    double s[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (int64_t q = q0 + threadIdx.x; q < q1; q += kSegThreads) {
        const double P = a.pop[q], p1 = a.prev1[q], p2 = a.prev2[q], p3 = a.prev3[q];
        const double Q1 = P - 2.0 * p1 + p2;
        const double Q2 = P - p1 - p2 + p3;
        const double Q3 = P - p1;
        s[0] += Q1 * Q1; s[1] += Q1 * Q2; s[2] += Q2 * Q2; s[3] += Q1 * Q3; s[4] += Q2 * Q3;
    }
    block_sum<5>(s, red);
    const double A1 = s[0], A2 = s[1], B2 = s[2], C1 = s[3], C2 = s[4];
    const double B1 = A2;
    const double denominator = A1 * B2 - A2 * B1;
    if (denominator == 0.0) return;
    const double ca = (C1 * B2 - C2 * B1) / denominator;
    const double cb = (C2 * A1 - C1 * A2) / denominator;
    for (int64_t q = q0 + threadIdx.x; q < q1; q += kSegThreads) {
        const double P = a.pop[q], p1 = a.prev1[q], p2 = a.prev2[q];
        a.pop[q] = (1.0 - ca - cb) * P + ca * p1 + cb * p2;
        a.prev3[q] = p2;
        a.prev2[q] = p1;
        a.prev1[q] = P;
    }
}

}  // namespace

cudaError_t launch_seg_convergence(const ModelView &m, const LevelArgs &a, double *seg_stats,
                                   cudaStream_t s) {
    if (m.nseg <= 0) return cudaSuccess;
    seg_convergence_kernel<<<(unsigned)m.nseg, kSegThreads, 0, s>>>(m, a, seg_stats);
    return cudaGetLastError();
}

cudaError_t launch_seg_ng(const ModelView &m, const LevelArgs &a, cudaStream_t s) {
    if (m.nseg <= 0) return cudaSuccess;
    seg_ng_kernel<<<(unsigned)m.nseg, kSegThreads, 0, s>>>(m, a);
    return cudaGetLastError();
}

}  // namespace mgr
