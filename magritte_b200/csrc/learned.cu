// learned.cu -- learned warm start for the level populations.
//
// A small MLP maps per-cell features (densities, temperature, line width,
// velocity-gradient length, column densities along the traced rays) to a
// correction of the LTE level populations:
//     log x = log_softmax(log x_LTE + MLP(features)),   n = n_tot x
// so a zero network reproduces the LTE start of
// LineProducingSpecies::update_using_LTE (lineProducingSpecies.tpp:82-115),
// which stays the fallback.  The ALI iteration then runs to the same
// tolerance from this start, so it also checks the network's error.
//
// Everything here is hand-written SIMT FP32: the network is tiny
// (10 -> 128 -> 128 -> 128 -> nlev, 35k parameters) and runs once per solve;
// one thread block handles 32 samples with all activations in shared memory.
// Training: forward, weighted log-fraction loss, backward, per-block weight
// gradient sums added to global accumulators, Adam.
#include <algorithm>
#include <vector>

#include "mgr_internal.cuh"

namespace mgr {

namespace {

constexpr int kS = 32;          // samples per block
constexpr int kT = 256;         // threads per block
constexpr int kH = MGR_MLP_HIDDEN;
constexpr int kL = 4;           // dense layers (3 hidden + output)

struct NetView {
    int nin, nout;
    const float *W[kL];   // [out][in]
    const float *b[kL];
    const float *mean, *istd;   // feature standardisation
};

struct GradView {
    float *W[kL];
    float *b[kL];
};

__device__ __forceinline__ int layer_in(const NetView &n, int l) { return l == 0 ? n.nin : kH; }
__device__ __forceinline__ int layer_out(const NetView &n, int l) { return l == kL - 1 ? n.nout : kH; }

constexpr int kWPitch = kH + 1;   // row pitch of the staged transposed weights

// act[l] holds the input of layer l ([kS][kH] floats, columns past the
// layer's width zero up to a multiple of 4); act[kL] the output.  Each
// layer's weights are staged transposed in shared memory (ws[k][j], pitch
// kH+1: conflict-free both when staged and when read); thread t computes
// output j = t % kH for samples (t / kH) * kS/2 ... + kS/2-1, four inputs
// at a time from one float4 of the activations.
__device__ void forward_block(const NetView &n, float (*act)[kS * kH], float *ws, int ns) {
    constexpr int kSG = kS / (kT / kH);   // samples per thread
    const int j = threadIdx.x % kH, sg = threadIdx.x / kH;
    for (int l = 0; l < kL; l++) {
        const int in = layer_in(n, l), out = layer_out(n, l);
        const int in4 = (in + 3) & ~3;
        const float *W = n.W[l];
        for (int idx = threadIdx.x; idx < out * in; idx += kT) {
            const int jj = idx / in, k = idx - jj * in;
            ws[k * kWPitch + jj] = __ldg(W + idx);
        }
        for (int idx = threadIdx.x; idx < (in4 - in) * kH; idx += kT)
            ws[(in + idx / kH) * kWPitch + idx % kH] = 0.0f;
        __syncthreads();
        const float *A = act[l] + sg * kSG * kH;
        float acc[kSG];
        const float bj = j < out ? __ldg(n.b[l] + j) : 0.0f;
#pragma unroll
        for (int s = 0; s < kSG; s++) acc[s] = bj;
        for (int k = 0; k < in4; k += 4) {
            const float w0 = ws[k * kWPitch + j], w1 = ws[(k + 1) * kWPitch + j];
            const float w2 = ws[(k + 2) * kWPitch + j], w3 = ws[(k + 3) * kWPitch + j];
#pragma unroll
            for (int s = 0; s < kSG; s++) {
                const float4 a4 = *reinterpret_cast<const float4 *>(A + s * kH + k);
                acc[s] = fmaf(w0, a4.x, fmaf(w1, a4.y, fmaf(w2, a4.z, fmaf(w3, a4.w, acc[s]))));
            }
        }
        float *Y = act[l + 1] + sg * kSG * kH;
        if (j < out) {
#pragma unroll
            for (int s = 0; s < kSG; s++)
                if (sg * kSG + s < ns) Y[s * kH + j] = (l < kL - 1) ? tanhf(acc[s]) : acc[s];
        }
        __syncthreads();
    }
}

// Loads and standardises the features of samples [s0, s0+ns).
__device__ void load_inputs(const NetView &n, const float *X, const int *idx, int64_t s0, int ns,
                            float *A0) {
    const int nin4 = (n.nin + 3) & ~3;
    for (int t = threadIdx.x; t < kS * nin4; t += kT) {
        const int s = t / nin4, f = t - s * nin4;
        float v = 0.0f;
        if (s < ns && f < n.nin) {
            const int64_t row = idx ? idx[s0 + s] : s0 + s;
            v = (X[row * n.nin + f] - n.mean[f]) * n.istd[f];
        }
        A0[s * kH + f] = v;
    }
    __syncthreads();
}

__global__ void __launch_bounds__(kT) mlp_forward_kernel(NetView n, const float *X, int64_t ns_total,
                                                         float *out) {
    extern __shared__ float sm[];
    float(*act)[kS * kH] = reinterpret_cast<float(*)[kS * kH]>(sm);
    const int64_t s0 = (int64_t)blockIdx.x * kS;
    const int ns = (int)(ns_total - s0 < (int64_t)kS ? ns_total - s0 : (int64_t)kS);
    load_inputs(n, X, nullptr, s0, ns, act[0]);
    forward_block(n, act, sm + (kL + 1) * kS * kH, ns);
    for (int t = threadIdx.x; t < ns * n.nout; t += kT) {
        const int s = t / n.nout, j = t - s * n.nout;
        out[(s0 + s) * n.nout + j] = act[kL][s * kH + j];
    }
}

// Loss of one sample: z = lte + delta, p = z - logsumexp(z), r = p - target,
// L = sum_i w_i r_i^2 with w_i = 1 for target fractions above 1e-8, 0.1 for
// 1e-12 .. 1e-8 and 0 below.  dL/ddelta_j = 2 (w_j r_j - softmax_j sum_i w_i r_i).
__device__ __forceinline__ float sample_loss_grad(const float *delta, const float *lte,
                                                  const float *tgt, int nout, float *g) {
    float zmax = -3.0e38f;
    for (int i = 0; i < nout; i++) zmax = fmaxf(zmax, lte[i] + delta[i]);
    float se = 0.0f;
    for (int i = 0; i < nout; i++) se += __expf(lte[i] + delta[i] - zmax);
    const float c = zmax + __logf(se);
    float L = 0.0f, swr = 0.0f;
    for (int i = 0; i < nout; i++) {
        const float r = lte[i] + delta[i] - c - tgt[i];
        // log(1e-8), log(1e-12): levels that the convergence test sees
        // (n > 1e-10 n_tot) carry the loss; far-depleted ones none
        const float w = tgt[i] > -18.420681f ? 1.0f : (tgt[i] > -27.631021f ? 0.1f : 0.0f);
        L += w * r * r;
        swr += w * r;
        g[i] = w * r;
    }
    for (int i = 0; i < nout; i++) {
        const float sm = __expf(lte[i] + delta[i] - c);
        g[i] = 2.0f * (g[i] - sm * swr);
    }
    return L;
}

__global__ void __launch_bounds__(kT) mlp_train_kernel(NetView n, GradView gr, const float *X,
                                                       const float *lte, const float *tgt,
                                                       const int *idx, int64_t b0, int64_t bn,
                                                       float scale, float *loss) {
    extern __shared__ float sm[];
    float(*act)[kS * kH] = reinterpret_cast<float(*)[kS * kH]>(sm);
    float *dA = sm + (kL + 1) * kS * kH;     // gradient w.r.t. a layer's output
    float *dB = dA + kS * kH;                // ... and w.r.t. its input
    float *ws = dB + kS * kH;                // staged weights of the forward pass
    __shared__ float red[kT / 32];
    const int64_t s0 = b0 + (int64_t)blockIdx.x * kS;
    const int ns = (int)(b0 + bn - s0 < (int64_t)kS ? b0 + bn - s0 : (int64_t)kS);
    if (ns <= 0) return;
    load_inputs(n, X, idx, s0, ns, act[0]);
    forward_block(n, act, ws, ns);
    // output gradient
    float lsum = 0.0f;
    if (threadIdx.x < ns) {
        const int s = threadIdx.x;
        const int64_t row = idx[s0 + s];
        float d[kMaxLevels], l[kMaxLevels], t[kMaxLevels], g[kMaxLevels];
        for (int i = 0; i < n.nout; i++) {
            d[i] = act[kL][s * kH + i];
            l[i] = lte[row * n.nout + i];
            t[i] = tgt[row * n.nout + i];
        }
        lsum = sample_loss_grad(d, l, t, n.nout, g);
        for (int i = 0; i < n.nout; i++) dA[s * kH + i] = g[i] * scale;
    }
    for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = lsum;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.0f;
        for (int w = 0; w < kT / 32; w++) t += red[w];
        atomicAdd(loss, t);
    }
    // backward through the layers
    for (int l = kL - 1; l >= 0; l--) {
        const int in = layer_in(n, l), out = layer_out(n, l);
        const float *A = act[l];
        // dZ = dA * act'(Z) for hidden layers (tanh' = 1 - a^2)
        if (l < kL - 1) {
            const float *Y = act[l + 1];
            for (int t = threadIdx.x; t < ns * out; t += kT) {
                const int s = t / out, j = t - s * out;
                const float a = Y[s * kH + j];
                dA[s * kH + j] *= (1.0f - a * a);
            }
            __syncthreads();
        }
        // weight and bias gradients, summed over the block's samples
        for (int t = threadIdx.x; t < out * in; t += kT) {
            const int j = t / in, k = t - j * in;
            float acc = 0.0f;
            for (int s = 0; s < ns; s++) acc = fmaf(dA[s * kH + j], A[s * kH + k], acc);
            atomicAdd(gr.W[l] + t, acc);
        }
        for (int j = threadIdx.x; j < out; j += kT) {
            float acc = 0.0f;
            for (int s = 0; s < ns; s++) acc += dA[s * kH + j];
            atomicAdd(gr.b[l] + j, acc);
        }
        if (l > 0) {
            for (int t = threadIdx.x; t < ns * in; t += kT) {
                const int s = t / in, k = t - s * in;
                float acc = 0.0f;
                for (int j = 0; j < out; j++) acc = fmaf(dA[s * kH + j], __ldg(n.W[l] + (size_t)j * in + k), acc);
                dB[s * kH + k] = acc;
            }
            __syncthreads();
            for (int t = threadIdx.x; t < ns * kH; t += kT) dA[t] = dB[t];
            __syncthreads();
        }
    }
}

__global__ void adam_kernel(float *p, const float *g, float *m, float *v, int64_t n, float lr,
                            float b1, float b2, float c1, float c2, float eps, float wd) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i] + wd * p[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
}

}  // namespace

// ---------------------------------------------------------------- features

namespace {

// Per-cell features from the model and the stored traces:
//  0 log10 collision-partner density     5 log10 mean column n_tot dZ over rays
//  1 log10 n_tot                         6 log10 min column over rays
//  2 log10 T                             7 log10 mean coherent column (points
//  3 log10 profile width over c            within one Doppler width of the origin)
//  4 log10 velocity-gradient length      8 log10 min coherent column
//    pw / <|dv . dr| / |dr|^2>           9 log10 mean ray length
__global__ void features_kernel(ModelView m, TraceView t, float *F) {
    const int64_t oi = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (oi >= t.o_count) return;
    const int64_t o = t.o_begin + oi;
    double ncol = 0.0;
    for (int c = 0; c < m.ncolpar; c++) ncol += m.colpar[c].abn[o];
    const double pw = m.pw[o];
    // velocity gradient over the neighbours
    double g = 0.0;
    const int b = m.nbr_off[o], e = m.nbr_off[o + 1];
    for (int k = b; k < e; k++) {
        const int nb = m.nbr[k];
        double dr[3], dv[3];
        for (int i = 0; i < 3; i++) {
            dr[i] = m.pos[3 * nb + i] - m.pos[3 * o + i];
            dv[i] = m.vel[3 * nb + i] - m.vel[3 * o + i];
        }
        const double r2 = dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2];
        if (r2 > 0.0) g += fabs(dv[0] * dr[0] + dv[1] * dr[1] + dv[2] * dr[2]) / r2;
    }
    if (e > b) g /= (e - b);
    double cmean = 0.0, cmin = 1e300, hmean = 0.0, hmin = 1e300, lmean = 0.0;
    for (int d = 0; d < t.ndir; d++) {
        const int64_t ix = (int64_t)d * t.o_count + oi;
        const int64_t off = t.off[ix];
        const int n = t.len[ix];
        double col = 0.0, coh = 0.0, len = 0.0;
        for (int j = 0; j < n; j++) {
            const int c = t.cell[off + j];
            const double dz = t.dZ[off + j];
            const double nd = m.pop_tot[c] * dz;
            col += nd;
            len += dz;
            if (fabs(t.shift[off + j] - 1.0) < pw) coh += nd;
        }
        cmean += col; cmin = fmin(cmin, col);
        hmean += coh; hmin = fmin(hmin, coh);
        lmean += len;
    }
    const double nd = (double)t.ndir;
    const double tiny = 1e-30;
    float *f = F + oi * MGR_MLP_FEATURES;
    f[0] = (float)log10(ncol + tiny);
    f[1] = (float)log10(m.pop_tot[o] + tiny);
    f[2] = (float)log10(m.T[o]);
    f[3] = (float)log10(pw);
    f[4] = (float)log10(pw / (g + 1e-300) + tiny);
    f[5] = (float)log10(cmean / nd + tiny);
    f[6] = (float)log10(cmin + tiny);
    f[7] = (float)log10(hmean / nd + tiny);
    f[8] = (float)log10(hmin + tiny);
    f[9] = (float)log10(lmean / nd + tiny);
}

// LTE log-fractions (lineProducingSpecies.tpp:82-115, in logarithms).
__global__ void lte_logfrac_kernel(ModelView m, int64_t o0, int64_t cnt, float *L) {
    const int64_t oi = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (oi >= cnt) return;
    const int64_t p = o0 + oi;
    const int nl = m.nlev;
    double e[kMaxLevels];
    double emax = -1e300;
    for (int i = 0; i < nl; i++) {
        e[i] = log(m.weight[i]) - m.energy[i] / (kKB * m.T[p]);
        emax = fmax(emax, e[i]);
    }
    double s = 0.0;
    for (int i = 0; i < nl; i++) s += exp(e[i] - emax);
    const double c = emax + log(s);
    for (int i = 0; i < nl; i++) L[oi * nl + i] = (float)(e[i] - c);
}

// n = n_tot softmax(lte + delta), written as populations.
__global__ void warm_populations_kernel(ModelView m, int64_t o0, int64_t cnt, const float *L,
                                        const float *D, double *pop) {
    const int64_t oi = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (oi >= cnt) return;
    const int64_t p = o0 + oi;
    const int nl = m.nlev;
    double z[kMaxLevels];
    double zmax = -1e300;
    for (int i = 0; i < nl; i++) {
        z[i] = (double)L[oi * nl + i] + (double)D[oi * nl + i];
        zmax = fmax(zmax, z[i]);
    }
    double s = 0.0;
    for (int i = 0; i < nl; i++) s += exp(z[i] - zmax);
    for (int i = 0; i < nl; i++) pop[p * nl + i] = m.pop_tot[p] * exp(z[i] - zmax) / s;
}

}  // namespace

// ---------------------------------------------------------------- launchers

static NetView net_view(const MlpDevice &d) {
    NetView n;
    n.nin = d.nin;
    n.nout = d.nout;
    for (int l = 0; l < kL; l++) { n.W[l] = d.W[l]; n.b[l] = d.b[l]; }
    n.mean = d.mean;
    n.istd = d.istd;
    return n;
}

size_t mlp_smem_bytes(bool train) {
    return ((size_t)((kL + 1) + (train ? 2 : 0)) * kS * kH + (size_t)kH * kWPitch) * sizeof(float);
}

cudaError_t mlp_prepare() {
    cudaError_t e = cudaFuncSetAttribute(mlp_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)mlp_smem_bytes(false));
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(mlp_train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)mlp_smem_bytes(true));
}

cudaError_t launch_mlp_forward(const MlpDevice &d, const float *X, int64_t n, float *out,
                               cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    const unsigned blocks = (unsigned)((n + kS - 1) / kS);
    mlp_forward_kernel<<<blocks, kT, mlp_smem_bytes(false), s>>>(net_view(d), X, n, out);
    return cudaGetLastError();
}

cudaError_t launch_mlp_train_batch(const MlpDevice &d, const MlpGrad &g, const float *X,
                                   const float *lte, const float *tgt, const int *idx, int64_t b0,
                                   int64_t bn, float scale, float *loss, cudaStream_t s) {
    if (bn <= 0) return cudaSuccess;
    GradView gv;
    for (int l = 0; l < kL; l++) { gv.W[l] = g.W[l]; gv.b[l] = g.b[l]; }
    const unsigned blocks = (unsigned)((bn + kS - 1) / kS);
    mlp_train_kernel<<<blocks, kT, mlp_smem_bytes(true), s>>>(net_view(d), gv, X, lte, tgt, idx,
                                                              b0, bn, scale, loss);
    return cudaGetLastError();
}

cudaError_t launch_adam(float *p, const float *g, float *m, float *v, int64_t n, float lr,
                        float b1, float b2, int step, float eps, float wd, cudaStream_t s) {
    const float c1 = 1.0f / (1.0f - powf(b1, (float)step));
    const float c2 = 1.0f / (1.0f - powf(b2, (float)step));
    adam_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(p, g, m, v, n, lr, b1, b2, c1, c2, eps, wd);
    return cudaGetLastError();
}

cudaError_t launch_features(const ModelView &m, const TraceView &t, float *F, cudaStream_t s) {
    if (t.o_count == 0) return cudaSuccess;
    features_kernel<<<(unsigned)((t.o_count + 127) / 128), 128, 0, s>>>(m, t, F);
    return cudaGetLastError();
}

cudaError_t launch_lte_logfrac(const ModelView &m, int64_t o0, int64_t cnt, float *L, cudaStream_t s) {
    if (cnt == 0) return cudaSuccess;
    lte_logfrac_kernel<<<(unsigned)((cnt + 127) / 128), 128, 0, s>>>(m, o0, cnt, L);
    return cudaGetLastError();
}

cudaError_t launch_warm_populations(const ModelView &m, int64_t o0, int64_t cnt, const float *L,
                                    const float *D, double *pop, cudaStream_t s) {
    if (cnt == 0) return cudaSuccess;
    warm_populations_kernel<<<(unsigned)((cnt + 127) / 128), 128, 0, s>>>(m, o0, cnt, L, D, pop);
    return cudaGetLastError();
}

}  // namespace mgr

// ================================================================ C ABI

namespace mgr {

int64_t mlp_param_count(int nin, int nout) {
    return (int64_t)kH * nin + kH + 2 * ((int64_t)kH * kH + kH) + (int64_t)nout * kH + nout;
}

void mlp_bind(float *base, int nin, int nout, float **W, float **b) {
    float *p = base;
    const int ins[kL] = {nin, kH, kH, kH}, outs[kL] = {kH, kH, kH, nout};
    for (int l = 0; l < kL; l++) {
        W[l] = p;
        p += (int64_t)ins[l] * outs[l];
        b[l] = p;
        p += outs[l];
    }
}

}  // namespace mgr

namespace {

using namespace mgr;

// Device buffers of one standalone call, freed on every exit path.
struct Scratch {
    std::vector<void *> ptrs;
    cudaStream_t stream = nullptr;
    ~Scratch() {
        if (stream) cudaStreamSynchronize(stream);
        for (void *p : ptrs) cudaFree(p);
        if (stream) cudaStreamDestroy(stream);
    }
    template <class T>
    T *alloc(int64_t n, cudaError_t &e) {
        void *p = nullptr;
        if (e == cudaSuccess) e = cudaMalloc(&p, (size_t)std::max<int64_t>(n, 1) * sizeof(T));
        if (e == cudaSuccess) ptrs.push_back(p);
        return (T *)p;
    }
    template <class T>
    T *upload(const T *src, int64_t n, cudaError_t &e) {
        T *d = alloc<T>(n, e);
        if (e == cudaSuccess && n > 0) e = cudaMemcpy(d, src, (size_t)n * sizeof(T), cudaMemcpyHostToDevice);
        return d;
    }
};

mgr_status cuda_status(cudaError_t e) {
    if (e == cudaSuccess) return MGR_OK;
    return e == cudaErrorMemoryAllocation ? MGR_ERR_NO_MEMORY : MGR_ERR_CUDA;
}

bool net_ok(const mgr_mlp *net) {
    return net && net->params && net->feat_mean && net->feat_istd &&
           net->nin == MGR_MLP_FEATURES && net->nout >= 1 && net->nout <= kMaxLevels;
}

// Uploads the network; d.W/d.b point into the returned parameter buffer.
float *upload_net(Scratch &sc, const mgr_mlp *net, MlpDevice &d, cudaError_t &e) {
    const int64_t np = mlp_param_count(net->nin, net->nout);
    float *P = sc.upload(net->params, np, e);
    d.nin = net->nin;
    d.nout = net->nout;
    d.mean = sc.upload(net->feat_mean, net->nin, e);
    d.istd = sc.upload(net->feat_istd, net->nin, e);
    if (e == cudaSuccess) mlp_bind(P, d.nin, d.nout, d.W, d.b);
    return P;
}

}  // namespace

extern "C" mgr_status mgr_mlp_param_count(int32_t nout, int64_t *count) {
    if (!count || nout < 1 || nout > kMaxLevels) return MGR_ERR_INVALID_ARG;
    *count = mlp_param_count(MGR_MLP_FEATURES, nout);
    return MGR_OK;
}

extern "C" mgr_status mgr_mlp_forward(int device, const mgr_mlp *net, const float *X, int64_t n,
                                      float *delta) {
    if (!net_ok(net) || !X || !delta || n <= 0) return MGR_ERR_INVALID_ARG;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return MGR_ERR_CUDA;
    Scratch sc;
    e = cudaStreamCreateWithFlags(&sc.stream, cudaStreamNonBlocking);
    MlpDevice d;
    upload_net(sc, net, d, e);
    float *dX = sc.upload(X, n * net->nin, e);
    float *dY = sc.alloc<float>(n * net->nout, e);
    if (e == cudaSuccess) e = mlp_prepare();
    if (e == cudaSuccess) e = launch_mlp_forward(d, dX, n, dY, sc.stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(delta, dY, (size_t)n * net->nout * sizeof(float),
                                              cudaMemcpyDeviceToHost, sc.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(sc.stream);
    return cuda_status(e);
}

extern "C" mgr_status mgr_mlp_loss_grad(int device, const mgr_mlp *net, const float *X,
                                        const float *lte, const float *target, int64_t n,
                                        float *loss, float *grad) {
    if (!net_ok(net) || !X || !lte || !target || !loss || !grad || n <= 0) return MGR_ERR_INVALID_ARG;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return MGR_ERR_CUDA;
    Scratch sc;
    e = cudaStreamCreateWithFlags(&sc.stream, cudaStreamNonBlocking);
    MlpDevice d;
    upload_net(sc, net, d, e);
    const int64_t np = mlp_param_count(net->nin, net->nout);
    float *dX = sc.upload(X, n * net->nin, e);
    float *dL = sc.upload(lte, n * net->nout, e);
    float *dT = sc.upload(target, n * net->nout, e);
    std::vector<int> idx(n);
    for (int64_t i = 0; i < n; i++) idx[i] = (int)i;
    int *dI = sc.upload(idx.data(), n, e);
    float *G = sc.alloc<float>(np, e);
    float *dloss = sc.alloc<float>(1, e);
    MlpGrad g;
    if (e == cudaSuccess) mlp_bind(G, net->nin, net->nout, g.W, g.b);
    if (e == cudaSuccess) e = cudaMemsetAsync(G, 0, np * sizeof(float), sc.stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(dloss, 0, sizeof(float), sc.stream);
    if (e == cudaSuccess) e = mlp_prepare();
    if (e == cudaSuccess) e = launch_mlp_train_batch(d, g, dX, dL, dT, dI, 0, n, 1.0f, dloss, sc.stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(grad, G, np * sizeof(float), cudaMemcpyDeviceToHost, sc.stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(loss, dloss, sizeof(float), cudaMemcpyDeviceToHost, sc.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(sc.stream);
    return cuda_status(e);
}

extern "C" mgr_status mgr_mlp_train(int device, mgr_mlp *net, const float *X, const float *lte,
                                    const float *target, int64_t n, const mgr_train_opts *opts,
                                    float *loss_hist) {
    if (!net_ok(net) || !X || !lte || !target || !opts || n <= 0 || opts->epochs < 1 ||
        opts->batch < 1 || !(opts->lr > 0.0f))
        return MGR_ERR_INVALID_ARG;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return MGR_ERR_CUDA;
    Scratch sc;
    e = cudaStreamCreateWithFlags(&sc.stream, cudaStreamNonBlocking);
    MlpDevice d;
    float *P = upload_net(sc, net, d, e);
    const int64_t np = mlp_param_count(net->nin, net->nout);
    float *dX = sc.upload(X, n * net->nin, e);
    float *dL = sc.upload(lte, n * net->nout, e);
    float *dT = sc.upload(target, n * net->nout, e);
    int *dI = sc.alloc<int>(n, e);
    float *G = sc.alloc<float>(np, e);
    float *Mo = sc.alloc<float>(np, e);
    float *Vo = sc.alloc<float>(np, e);
    float *dloss = sc.alloc<float>(1, e);
    MlpGrad g;
    if (e == cudaSuccess) mlp_bind(G, net->nin, net->nout, g.W, g.b);
    if (e == cudaSuccess) e = cudaMemsetAsync(Mo, 0, np * sizeof(float), sc.stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(Vo, 0, np * sizeof(float), sc.stream);
    if (e == cudaSuccess) e = mlp_prepare();
    std::vector<int> idx(n);
    for (int64_t i = 0; i < n; i++) idx[i] = (int)i;
    uint64_t state = opts->seed * 6364136223846793005ull + 1442695040888963407ull;
    auto rnd = [&]() {   // 64-bit LCG, high bits
        state = state * 6364136223846793005ull + 1442695040888963407ull;
        return state >> 33;
    };
    int step = 0;
    float host_loss = 0.0f;
    for (int ep = 0; ep < opts->epochs && e == cudaSuccess; ep++) {
        for (int64_t i = n - 1; i > 0; i--) std::swap(idx[i], idx[rnd() % (uint64_t)(i + 1)]);
        e = cudaMemcpyAsync(dI, idx.data(), n * sizeof(int), cudaMemcpyHostToDevice, sc.stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(dloss, 0, sizeof(float), sc.stream);
        for (int64_t b0 = 0; b0 < n && e == cudaSuccess; b0 += opts->batch) {
            const int64_t bn = std::min<int64_t>(opts->batch, n - b0);
            e = cudaMemsetAsync(G, 0, np * sizeof(float), sc.stream);
            if (e == cudaSuccess)
                e = launch_mlp_train_batch(d, g, dX, dL, dT, dI, b0, bn, 1.0f / (float)bn, dloss, sc.stream);
            if (e == cudaSuccess)
                e = launch_adam(P, G, Mo, Vo, np, opts->lr, 0.9f, 0.999f, ++step, 1e-8f,
                                opts->weight_decay, sc.stream);
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(&host_loss, dloss, sizeof(float), cudaMemcpyDeviceToHost, sc.stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(sc.stream);
        if (e == cudaSuccess && loss_hist) loss_hist[ep] = host_loss / (float)n;
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(net->params, P, np * sizeof(float), cudaMemcpyDeviceToHost, sc.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(sc.stream);
    return cuda_status(e);
}
