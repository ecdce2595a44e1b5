// noalloc.cu -- convergence statistics for callers that cannot allocate.
//
// Some host applications own all of the GPU's memory: they reserve it once
// through their own pool and do not allow further cudaMalloc calls (which
// would also synchronise the whole device).  They hand this library pointers
// into memory they already own.  mgr_convergence_noalloc computes the same
// statistics as the handle-based path (fraction of (cell, level) pairs whose
// relative change exceeds pop_prec, the mean and the maximum relative change,
// as LineProducingSpecies::check_for_convergence defines them) from caller
// buffers only.  Its reduction scratch is the file-scope device array below:
// every GPU that loads this library holds it until the process exits.
#include <mutex>

#include "mgr_internal.cuh"

namespace {

constexpr int kThreads = 256;
constexpr int kPerThread = 4;
constexpr int kPerBlock = kThreads * kPerThread;                  // 1024 elements
constexpr int kMaxBlocks = (int)(MGR_NOALLOC_MAX_ELEMENTS / kPerBlock);
constexpr int kMaxDevices = 64;

// Partial (count, sum, max) of each block of the first pass.  Every slot
// the second pass reads is written by the first pass of the same call, so
// nothing here has to start at zero.  Calls that overlap on the GPU share
// this array and race.
static __device__ __align__(256) double g_noalloc_partials[3 * kMaxBlocks];

std::mutex g_setup_mutex;
double *g_partials_dev[kMaxDevices];   // device address of the array, per device

__global__ void noalloc_partials_kernel(const double *__restrict__ pop,
                                        const double *__restrict__ prev,
                                        const double *__restrict__ pop_tot, int64_t n, int nlev,
                                        double pop_prec, double *partials) {
    __shared__ double red[3 * (kThreads / 32)];
    double cnt = 0.0, sum = 0.0, mx = 0.0;
    const int64_t base = (int64_t)blockIdx.x * kPerBlock + threadIdx.x;
    for (int j = 0; j < kPerThread; j++) {
        const int64_t q = base + (int64_t)j * kThreads;
        if (q < n) {
            const double a = pop[q], b = prev[q];
            if (a > 1.0E-10 * pop_tot[q / nlev]) {
                double rc = 2.0;
                rc *= fabs(a - b);
                rc /= (a + b);
                if (rc > pop_prec) cnt += 1.0;
                sum += rc;
                mx = fmax(mx, rc);
            }
        }
    }
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) {
        cnt += __shfl_xor_sync(0xffffffffu, cnt, s);
        sum += __shfl_xor_sync(0xffffffffu, sum, s);
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, s));
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) { red[3 * warp] = cnt; red[3 * warp + 1] = sum; red[3 * warp + 2] = mx; }
    __syncthreads();
    if (threadIdx.x == 0) {
        cnt = 0.0; sum = 0.0; mx = 0.0;
        for (int w = 0; w < kThreads / 32; w++) {
            cnt += red[3 * w]; sum += red[3 * w + 1]; mx = fmax(mx, red[3 * w + 2]);
        }
        partials[3 * blockIdx.x + 0] = cnt;
        partials[3 * blockIdx.x + 1] = sum;
        partials[3 * blockIdx.x + 2] = mx;
    }
}

__global__ void noalloc_final_kernel(const double *partials, int nblocks, double inv_n,
                                     double *stats) {
    __shared__ double red[3 * 32];
    double cnt = 0.0, sum = 0.0, mx = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
        cnt += partials[3 * b];
        sum += partials[3 * b + 1];
        mx = fmax(mx, partials[3 * b + 2]);
    }
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) {
        cnt += __shfl_xor_sync(0xffffffffu, cnt, s);
        sum += __shfl_xor_sync(0xffffffffu, sum, s);
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, s));
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) { red[3 * warp] = cnt; red[3 * warp + 1] = sum; red[3 * warp + 2] = mx; }
    __syncthreads();
    if (threadIdx.x == 0) {
        cnt = 0.0; sum = 0.0; mx = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
            cnt += red[3 * w]; sum += red[3 * w + 1]; mx = fmax(mx, red[3 * w + 2]);
        }
        stats[0] = cnt * inv_n;
        stats[1] = sum * inv_n;
        stats[2] = mx;
    }
}

// Device address of the scratch array on the current device.  The array's
// host-side name is only a stand-in and must never be given to a kernel;
// cudaGetSymbolAddress gives the address in the current context.  A call on
// a stream that is not capturing looks the address up again (a host-side
// table lookup, no allocation), so a cudaDeviceReset or a new primary
// context between calls cannot leave a stale address behind.  A call on a
// capturing stream uses the address that the last call outside capture
// found on this device; with none yet it returns cudaErrorStreamCaptureUnsupported
// without touching the runtime's module state inside the capture.
cudaError_t partials_on_current_device(cudaStream_t s, double **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    e = cudaStreamIsCapturing(s, &cap);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (cap == cudaStreamCaptureStatusNone) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_partials);
        if (e != cudaSuccess) return e;
        g_partials_dev[dev] = static_cast<double *>(p);
    } else if (!g_partials_dev[dev]) {
        return cudaErrorStreamCaptureUnsupported;
    }
    *out = g_partials_dev[dev];
    return cudaSuccess;
}

}  // namespace

extern "C" mgr_status mgr_convergence_noalloc(const double *pop, const double *prev,
                                              const double *pop_tot, int64_t ncells,
                                              int32_t nlev, double pop_prec, double *stats,
                                              void *stream) {
    if (!pop || !prev || !pop_tot || !stats || ncells <= 0 || nlev <= 0) return MGR_ERR_INVALID_ARG;
    if (ncells > MGR_NOALLOC_MAX_ELEMENTS / nlev) return MGR_ERR_TOO_LARGE;
    const int64_t n = ncells * (int64_t)nlev;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // an error left pending on this host thread by earlier work is the
    // caller's: report it without launching and leave it in place
    if (cudaPeekAtLastError() != cudaSuccess) return MGR_ERR_CUDA;
    double *partials = nullptr;
    const cudaError_t e = partials_on_current_device(s, &partials);
    if (e == cudaErrorStreamCaptureUnsupported) return MGR_ERR_STATE;
    if (e != cudaSuccess) return MGR_ERR_CUDA;
    const int nblocks = (int)((n + kPerBlock - 1) / kPerBlock);
    noalloc_partials_kernel<<<nblocks, kThreads, 0, s>>>(pop, prev, pop_tot, n, nlev, pop_prec,
                                                         partials);
    if (cudaGetLastError() != cudaSuccess) return MGR_ERR_CUDA;
    noalloc_final_kernel<<<1, 1024, 0, s>>>(partials, nblocks, 1.0 / (double)n, stats);
    if (cudaGetLastError() != cudaSuccess) return MGR_ERR_CUDA;
    return MGR_OK;
}
