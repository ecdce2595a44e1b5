// capi.cu -- the handle, device memory and the extern "C" entry points.
//
// A handle owns one model on one GPU.  Host code here validates inputs,
// derives the small per-model tables (antipodal rays, profile widths, line
// windows) with separately rounded double arithmetic, moves data, and runs
// the kernels of trace.cu, solve.cu and levels.cu on the handle's stream.
// C++ exceptions are used internally and never cross the C boundary.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <map>
#include <mutex>
#include <limits>
#include <memory>
#include <stdexcept>

#include "mgr_internal.cuh"

using namespace mgr;

namespace {

struct Failure {
    mgr_status code;
    std::string msg;
};

[[noreturn]] void fail(mgr_status c, const std::string &m) { throw Failure{c, m}; }

void ck(cudaError_t e, const char *what) {
    if (e != cudaSuccess) {
        if (e == cudaErrorMemoryAllocation) fail(MGR_ERR_NO_MEMORY, std::string(what) + ": " + cudaGetErrorString(e));
        fail(MGR_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    }
}

__global__ void widen_kernel(const int32_t *in, int64_t *out, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = in[i];
}

}  // namespace

struct mgr_handle {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, tev0 = nullptr, tev1 = nullptr;
    std::string err;
    int64_t launches = 0;

    // sizes
    int64_t N = 0;
    int nrays = 0, npairs = 0, nlev = 0, nrad = 0, nquads = 0, nfreqs = 0, ncolpar = 0;

    std::vector<void *> model_allocs;
    ModelView mv{};

    // state
    double *pop = nullptr, *prev1 = nullptr, *prev2 = nullptr, *prev3 = nullptr;
    double *eps = nullptr, *kap = nullptr, *Jlin = nullptr, *Lam = nullptr, *Jeff = nullptr;
    double *J = nullptr, *partials = nullptr, *stats = nullptr;
    float2 *ek = nullptr;
    DevFlags *flags = nullptr;
    double *h_stats = nullptr;
    DevFlags *h_flags = nullptr;
    double mixed_scale = 1.0;

    // traces
    int32_t *len_all = nullptr;        // [nrays*N]
    int64_t *off_all = nullptr;        // [nrays*N] when stored
    int32_t *tcell = nullptr;
    double *tshift = nullptr, *tdz = nullptr;
    MixedPoint *tmp_ = nullptr;        // mixed-format records
    int64_t tcap = 0;                  // point capacity of tcell/tshift/tdz
    // far-end boundary intensities of the trace store for the staged mixed
    // solve, [origins][npairs][2][nfreqs]; valid while bc_stamp == bc_serial
    // (bc_serial counts changes of the traces, grid and boundary table)
    float *bcache = nullptr;
    int64_t bcache_cap = 0;            // origins
    uint64_t bc_serial = 1, bc_stamp = 0;
    // hop log of the counting pass (HopLog): the fill of a stored trace
    // replays it instead of searching; [kHopCap][nrays*N] cells and
    // [nrays*N] counts
    int32_t *hop_cell = nullptr, *hop_n = nullptr;
    int64_t hop_rays = 0;
    int32_t *blen = nullptr;           // batch lengths [nrays*bcap]
    int64_t *boff = nullptr;           // batch offsets
    int64_t bcap = 0;                  // origins per batch capacity
    void *scan_tmp = nullptr;
    size_t scan_tmp_bytes = 0;
    bool traced = false, stored = false;
    int64_t total_points = 0;
    int64_t batch_origins = 0;
    int64_t trace_budget = 0;
    double updates_per_solve = 0.0;
    int max_pair_points = 0;
    std::vector<int32_t> h_len;        // [nrays*N] host copy for npoints, made on demand
    bool h_len_valid = false;
    std::vector<float> upd_origin;     // [N] updates of one formal solve per origin (batches)
    unsigned long long *tstats_d = nullptr, *h_tstats = nullptr;   // trace statistics [3]
    int32_t *pts_origin_d = nullptr;   // [N] points of each origin's traces
    float *upd_origin_d = nullptr;     // [N] updates per origin (batches)

    double pw_max = 0.0, vmax = 0.0;  // largest profile width (over c) and speed (over c)
    bool model_loaded = false, line_set = false, bdy_set = false, pops_valid = false;
    bool keep_J = false;
    double last_solve_ms = 0.0, last_updates = 0.0;
    double last_trace_ms = 0.0;        // of the last solve: rebuilding traces per batch of origins
    std::vector<cudaEvent_t> batch_ev; // [2 per batch] around each batch's trace rebuild

    std::vector<int64_t> antipod;
    int64_t nboundary = 0;
    int64_t *b2c_dev = nullptr;        // boundary -> cell (int64)
    double *ibdy = nullptr;            // [nboundary][nfreqs]
    int4 *patch = nullptr;             // mixed solve: entries redone in double
    unsigned long long *patch_count = nullptr;
    unsigned long long *h_patch = nullptr;   // pinned copy of patch_count
    int64_t patch_cap = 0;
    int64_t patch_cap_set = 0;         // capacity fixed by the caller (0: automatic)
    int64_t last_patched = 0;
    int64_t fp64_fallbacks = 0;        // origins re-solved in double (patch list full), cumulative
    int32_t *redo_flag = nullptr, *redo_list = nullptr;   // [N] each

    // scattering: terms U, V and the origins' u, v per (pair, cell, bin)
    double *scat_U = nullptr, *scat_V = nullptr, *scat_u = nullptr, *scat_v = nullptr;

    // non-local ALO (parameters.n_off_diag >= 2): the off-diagonal elements
    // and their cells, the block-Jacobi iterates and the sweep's max change
    int noff = 0;
    double *Loff = nullptr;
    int32_t *Loff_nr = nullptr;
    double *nl_x[2] = {nullptr, nullptr};
    double *nl_change = nullptr;
    double *h_nl_change = nullptr;     // pinned
    int64_t nl_sweeps = 0;             // block-Jacobi sweeps of the last solve
    double nl_best_change = 0.0;       // their smallest max relative change

    // warm start: features, LTE log fractions, network output and the
    // network's parameters, kept between calls (allocated once per model)
    float *ws_F = nullptr, *ws_L = nullptr, *ws_D = nullptr, *ws_P = nullptr;
    float *ws_mean = nullptr, *ws_istd = nullptr;
    int64_t ws_np = 0;

    // origins (= cells) this handle solves: a shard of a partitioned run
    int64_t o_begin = 0, o_end = 0;
    bool whole() const { return o_begin == 0 && o_end == N; }

    // batch of independent models (nseg > 0)
    int64_t nseg = 0;
    int64_t *seg_begin_d = nullptr;
    int32_t *cell_seg_d = nullptr, *seg_active_d = nullptr;
    double *seg_stats_d = nullptr;
    double *h_seg_stats = nullptr;     // pinned [3*nseg]
    int32_t *h_seg_active = nullptr;   // pinned [nseg]
    std::vector<int64_t> seg_iters;

    // online autotuner of the formal solve: per precision, the first solves
    // each run one compiled variant; later solves use the fastest
    int autotune = 0;   // 0 off, 1 tune (reuse this process's results), 2 always re-time
    struct Tune {
        int next = 0, best = -1, kind = -1;
        float ms[kSolveVariants] = {};
    } tune[2];

    // CUDA graphs of the ALI iteration (rebuilt when gen or the key changes)
    int64_t gen = 0;
    struct Graph {
        cudaGraphExec_t exec = nullptr;
        int64_t gen = -1;
        int key = 0;
        int kernels = 0;   // kernels per replay
    } g_solve, g_level, g_ng;
};

namespace {

template <class T>
T *dalloc(mgr_handle *h, int64_t count, std::vector<void *> *track) {
    if (count <= 0) count = 1;
    void *p = nullptr;
    ck(cudaMalloc(&p, (size_t)count * sizeof(T)), "cudaMalloc");
    if (track) track->push_back(p);
    return (T *)p;
}

template <class T>
T *upload(mgr_handle *h, const T *src, int64_t count, std::vector<void *> *track) {
    T *d = dalloc<T>(h, count, track);
    if (count > 0) ck(cudaMemcpy(d, src, (size_t)count * sizeof(T), cudaMemcpyHostToDevice), "upload");
    return d;
}

void free_ptr(void *&p) {
    if (p) cudaFree(p);
    p = nullptr;
}

void free_traces(mgr_handle *h) {
    free_ptr((void *&)h->off_all);
    free_ptr((void *&)h->tcell);
    free_ptr((void *&)h->tshift);
    free_ptr((void *&)h->tdz);
    free_ptr((void *&)h->tmp_);
    free_ptr((void *&)h->blen);
    free_ptr((void *&)h->boff);
    free_ptr((void *&)h->bcache);
    free_ptr((void *&)h->hop_cell);
    free_ptr((void *&)h->hop_n);
    h->hop_rays = 0;
    free_ptr(h->scan_tmp);
    h->scan_tmp_bytes = 0;
    h->tcap = 0;
    h->bcap = 0;
    h->bcache_cap = 0;
    h->bc_serial++;
    h->traced = false;
    h->stored = false;
    h->gen++;
}

void free_graph(mgr_handle::Graph &g) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    g.exec = nullptr;
    g.gen = -1;
}

void free_segments(mgr_handle *h) {
    free_ptr((void *&)h->seg_begin_d);
    free_ptr((void *&)h->cell_seg_d);
    free_ptr((void *&)h->seg_active_d);
    free_ptr((void *&)h->seg_stats_d);
    if (h->h_seg_stats) cudaFreeHost(h->h_seg_stats);
    if (h->h_seg_active) cudaFreeHost(h->h_seg_active);
    h->h_seg_stats = nullptr;
    h->h_seg_active = nullptr;
    h->nseg = 0;
    h->seg_iters.clear();
    h->mv.nseg = 0;
    h->mv.seg_begin = nullptr;
    h->mv.cell_seg = nullptr;
    h->mv.seg_active = nullptr;
    h->gen++;
}

void free_model(mgr_handle *h) {
    free_graph(h->g_solve);
    free_graph(h->g_level);
    free_graph(h->g_ng);
    free_segments(h);
    free_traces(h);
    free_ptr((void *&)h->len_all);
    free_ptr((void *&)h->tstats_d);
    free_ptr((void *&)h->pts_origin_d);
    free_ptr((void *&)h->upd_origin_d);
    h->h_len.clear();
    h->h_len_valid = false;
    for (void *p : h->model_allocs) cudaFree(p);
    h->model_allocs.clear();
    void **ws[] = {(void **)&h->ws_F, (void **)&h->ws_L, (void **)&h->ws_D, (void **)&h->ws_P,
                   (void **)&h->ws_mean, (void **)&h->ws_istd, (void **)&h->scat_U,
                   (void **)&h->scat_V, (void **)&h->scat_u, (void **)&h->scat_v,
                   (void **)&h->Loff, (void **)&h->Loff_nr, (void **)&h->nl_x[0],
                   (void **)&h->nl_x[1], (void **)&h->nl_change};
    for (void **p : ws) free_ptr(*p);
    h->noff = 0;
    h->ws_np = 0;
    void **state[] = {(void **)&h->pop, (void **)&h->prev1, (void **)&h->prev2, (void **)&h->prev3,
                      (void **)&h->eps, (void **)&h->kap, (void **)&h->Jlin, (void **)&h->Lam,
                      (void **)&h->Jeff, (void **)&h->J, (void **)&h->partials, (void **)&h->stats,
                      (void **)&h->ek, (void **)&h->flags, (void **)&h->ibdy,
                      (void **)&h->patch, (void **)&h->patch_count, (void **)&h->redo_flag,
                      (void **)&h->redo_list};
    for (void **p : state) free_ptr(*p);
    h->model_loaded = h->line_set = h->bdy_set = h->pops_valid = false;
}

void set_device(mgr_handle *h) { ck(cudaSetDevice(h->device), "cudaSetDevice"); }

void reset_flags(mgr_handle *h) {
    ck(cudaMemsetAsync(h->flags, 0, sizeof(DevFlags), h->stream), "reset flags");
}

// Raises the status that the device error counters (already copied to the
// pinned host copy) imply.
void check_flags_copied(mgr_handle *h, const char *what) {
    const DevFlags &f = *h->h_flags;
    if (f.trace_err || f.stuck_err)
        fail(MGR_ERR_TRACE, std::string(what) + ": " + std::to_string(f.trace_err + f.stuck_err) +
                                " ray(s) found no neighbour ahead before reaching a boundary cell");
    if (f.interp_err)
        fail(MGR_ERR_TRACE, std::string(what) + ": more than 10000 interpolation points needed on " +
                                std::to_string(f.interp_err) + " ray step(s)");
    if (f.cap_err) fail(MGR_ERR_CUDA, std::string(what) + ": trace slot overflow (internal)");
    if (f.lu_err)
        fail(MGR_ERR_LU_SINGULAR, std::string(what) + ": zero pivot in the rate equations of " +
                                      std::to_string(f.lu_err) + " cell(s)");
}

// Reads the device error counters; raises the status they imply.
void check_flags(mgr_handle *h, const char *what) {
    ck(cudaMemcpyAsync(h->h_flags, h->flags, sizeof(DevFlags), cudaMemcpyDeviceToHost, h->stream),
       "read flags");
    ck(cudaStreamSynchronize(h->stream), what);
    check_flags_copied(h, what);
}

LevelArgs level_args(mgr_handle *h) {
    LevelArgs a{};
    a.pop = h->pop; a.prev1 = h->prev1; a.prev2 = h->prev2; a.prev3 = h->prev3;
    a.eps = h->eps; a.kap = h->kap; a.ehat_khat = h->ek; a.mixed_scale = h->mixed_scale;
    a.Jlin = h->Jlin; a.Lam = h->Lam; a.Jeff = h->Jeff;
    a.partials = h->partials; a.stats = h->stats;
    a.npartials = level_partials_needed(h->mv);
    a.c_begin = h->o_begin;
    a.c_end = h->o_end;
    return a;
}

void need(bool ok, mgr_status c, const char *msg) {
    if (!ok) fail(c, msg);
}

// Profile width over c, Thermodynamics::profile_width (thermodynamics.tpp:62-69).
// Separately rounded (this file is compiled with -ffp-contract=off).
double profile_width_host(double inverse_mass, double T, double vturb2) {
    volatile double a = kTWO_KB_OVER_AMU_C_SQUARED * inverse_mass;
    volatile double b = a * T;
    volatile double c = b + vturb2;
    return std::sqrt((double)c);
}

// ------------------------------------------------------------------ upload
void do_upload(mgr_handle *h, const mgr_model_desc *d) {
    need(d != nullptr, MGR_ERR_INVALID_ARG, "model descriptor is NULL");
    need(d->ncells > 0 && d->ncells < (int64_t)INT32_MAX, MGR_ERR_INVALID_ARG, "ncells out of range");
    need(d->position && d->velocity && d->nbr_offsets && d->nbr_list && d->boundary2cell &&
             d->rays && d->ray_weights && d->temperature && d->vturb2 && d->energy && d->weight &&
             d->irad && d->jrad && d->A && d->Bs && d->Ba && d->frequency && d->population_tot &&
             d->quad_roots && d->quad_weights,
         MGR_ERR_INVALID_ARG, "a required model array is NULL");
    need(d->nlev >= 2 && d->nlev <= kMaxLevels, MGR_ERR_UNSUPPORTED, "nlev must be in [2, 32]");
    need(d->nrad >= 1, MGR_ERR_INVALID_ARG, "nrad must be >= 1");
    need(d->nquads >= 1, MGR_ERR_INVALID_ARG, "nquads must be >= 1");
    need(d->nrays >= 2 && d->nrays % 2 == 0, MGR_ERR_INVALID_ARG, "nrays must be even and >= 2");
    need(d->ncolpar >= 0 && d->ncolpar <= kMaxColpar, MGR_ERR_UNSUPPORTED, "at most 4 collision partners");
    need(d->ncolpar == 0 || d->colpar, MGR_ERR_INVALID_ARG, "colpar is NULL");
    need(d->nboundary >= 1, MGR_ERR_INVALID_ARG, "nboundary must be >= 1");
    need((int64_t)d->nrad * d->nquads < (int64_t)INT32_MAX, MGR_ERR_INVALID_ARG, "too many bins");

    free_model(h);
    set_device(h);
    const int64_t N = d->ncells;
    h->N = N;
    h->o_begin = 0;
    h->o_end = N;
    h->nrays = (int)d->nrays;
    h->npairs = (int)(d->nrays / 2);
    h->nlev = d->nlev;
    h->nrad = d->nrad;
    h->nquads = d->nquads;
    h->nfreqs = d->nrad * d->nquads;
    h->ncolpar = d->ncolpar;
    auto *T = &h->model_allocs;

    // neighbours (int32 on the device)
    const int64_t nnb = d->nbr_offsets[N];
    need(d->nbr_offsets[0] == 0 && nnb >= 0 && nnb < (int64_t)INT32_MAX, MGR_ERR_INVALID_ARG,
         "neighbour offsets out of range");
    std::vector<int32_t> off32(N + 1), nb32(std::max<int64_t>(nnb, 1));
    for (int64_t p = 0; p <= N; p++) {
        if (p < N) need(d->nbr_offsets[p + 1] >= d->nbr_offsets[p], MGR_ERR_INVALID_ARG, "neighbour offsets not ascending");
        off32[p] = (int32_t)d->nbr_offsets[p];
    }
    for (int64_t k = 0; k < nnb; k++) {
        need(d->nbr_list[k] >= 0 && d->nbr_list[k] < N, MGR_ERR_INVALID_ARG, "neighbour index out of range");
        nb32[k] = (int32_t)d->nbr_list[k];
    }

    // boundary
    std::vector<uint8_t> bmask(N, 0);
    std::vector<int32_t> c2b(N, -1);
    for (int64_t b = 0; b < d->nboundary; b++) {
        const int64_t c = d->boundary2cell[b];
        need(c >= 0 && c < N, MGR_ERR_INVALID_ARG, "boundary cell out of range");
        bmask[c] = 1;
        c2b[c] = (int32_t)b;
    }
    std::vector<double> bT(d->nboundary, kT_CMB);
    if (d->boundary_temperature)
        for (int64_t b = 0; b < d->nboundary; b++) bT[b] = d->boundary_temperature[b];

    // rays and antipodes (Rays::setup_antipodal_rays, rays.cpp:90-102)
    h->antipod.assign(d->nrays, -1);
    for (int64_t r1 = 0; r1 < d->nrays; r1++)
        for (int64_t r2 = 0; r2 < d->nrays; r2++) {
            const double *a = d->rays + 3 * r1, *b = d->rays + 3 * r2;
            const double sx = a[0] + b[0], sy = a[1] + b[1], sz = a[2] + b[2];
            if ((sx * sx + sy * sy) + sz * sz < 1.0E-9) h->antipod[r1] = r2;
        }
    std::vector<int32_t> ap32(d->nrays);
    for (int64_t r = 0; r < d->nrays; r++) {
        if (r < d->nrays / 2) need(h->antipod[r] >= 0, MGR_ERR_INVALID_ARG, "a ray of the first half has no antipode");
        ap32[r] = (int32_t)h->antipod[r];
    }

    // thermodynamics
    std::vector<double> pw(N), ipw(N), dsm(N);
    double pw_max = 0.0, pw_min = std::numeric_limits<double>::max(), vmax = 0.0;
    for (int64_t p = 0; p < N; p++) {
        pw[p] = profile_width_host(d->inverse_mass, d->temperature[p], d->vturb2[p]);
        need(pw[p] > 0.0 && std::isfinite(pw[p]), MGR_ERR_INVALID_ARG, "non-positive profile width");
        ipw[p] = 1.0 / pw[p];
        dsm[p] = d->max_width_fraction * pw[p];
        pw_max = std::max(pw_max, pw[p]);
        pw_min = std::min(pw_min, pw[p]);
        const double *v = d->velocity + 3 * p;
        vmax = std::max(vmax, std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]));
    }

    h->pw_max = pw_max;
    h->vmax = vmax;

    // lines: the device path keeps the transitions' order, which must be
    // ascending in frequency (Lines::setup's heapsort then is the identity)
    std::vector<double> line(d->nrad), iline(d->nrad);
    for (int k = 0; k < d->nrad; k++) {
        line[k] = d->frequency[k];
        need(line[k] > 0.0, MGR_ERR_INVALID_ARG, "non-positive line frequency");
        if (k) need(line[k] > line[k - 1], MGR_ERR_UNSUPPORTED, "line frequencies must be ascending");
        iline[k] = 1.0 / line[k];
        need(d->irad[k] >= 0 && d->irad[k] < d->nlev && d->jrad[k] >= 0 && d->jrad[k] < d->nlev,
             MGR_ERR_INVALID_ARG, "irad/jrad out of range");
    }
    for (int z = 1; z < d->nquads; z++)
        need(d->quad_roots[z] > d->quad_roots[z - 1], MGR_ERR_UNSUPPORTED, "quadrature roots must be ascending");

    // conservative window of lines a bin can see (+-11 widths around any
    // Doppler-shifted frequency of the bin)
    std::vector<int32_t> wlo(d->nrad), whi(d->nrad);
    {
        const double sdev = 2.0 * vmax * (1.0 + 1e-9) + 1e-15;
        const double rlo = std::min(d->quad_roots[0], 0.0), rhi = std::max(d->quad_roots[d->nquads - 1], 0.0);
        for (int k = 0; k < d->nrad; k++) {
            const double nlo = line[k] * (1.0 + pw_max * rlo) * (1.0 - sdev) * (1.0 - 1e-12);
            const double nhi = line[k] * (1.0 + pw_max * rhi) * (1.0 + sdev) * (1.0 + 1e-12);
            int lo = k, hi = k;
            for (int l = 0; l < d->nrad; l++) {
                const double wl = line[l] * (1.0 - 11.0 * pw_max) * (1.0 - 1e-12);
                const double wh = line[l] * (1.0 + 11.0 * pw_max) * (1.0 + 1e-12);
                if (nhi >= wl && nlo <= wh) { lo = std::min(lo, l); hi = std::max(hi, l); }
            }
            wlo[k] = lo;
            whi[k] = hi;
        }
    }

    // scale of the float opacities: a power of two that brings the largest
    // possible line-centre opacity (over c) near one
    {
        double bamax = 0.0, ptmax = 0.0;
        for (int k = 0; k < d->nrad; k++) bamax = std::max(bamax, std::fabs(d->Ba[k]));
        for (int64_t p = 0; p < N; p++) ptmax = std::max(ptmax, d->population_tot[p]);
        const double kest = kHH_OVER_FOUR_PI * ptmax * bamax * kINVERSE_SQRT_PI / pw_min;
        int e = 0;
        if (kest > 0.0 && std::isfinite(kest)) e = -(int)std::lround(std::log2(kest));
        e = std::max(-100, std::min(120, e));
        h->mixed_scale = std::ldexp(1.0, e);
    }

    // upload
    ModelView &m = h->mv;
    m = ModelView{};
    m.N = N;
    m.nrays = h->nrays;
    m.npairs = h->npairs;
    m.nlev = h->nlev;
    m.nrad = h->nrad;
    m.nquads = h->nquads;
    m.nfreqs = h->nfreqs;
    m.ncolpar = h->ncolpar;
    m.pop_prec = d->pop_prec;
    m.mixed_scale = h->mixed_scale;
    m.overlap = 0;
    for (int k = 0; k < d->nrad; k++) m.overlap |= (wlo[k] != whi[k]);
    m.pos = upload(h, d->position, 3 * N, T);
    m.vel = upload(h, d->velocity, 3 * N, T);
    m.rays = upload(h, d->rays, 3 * (int64_t)d->nrays, T);
    m.ray_w = upload(h, d->ray_weights, d->nrays, T);
    m.nbr_off = upload(h, off32.data(), N + 1, T);
    m.nbr = upload(h, nb32.data(), (int64_t)nb32.size(), T);
    m.boundary = upload(h, bmask.data(), N, T);
    m.cell2bdy = upload(h, c2b.data(), N, T);
    m.antipod = upload(h, ap32.data(), d->nrays, T);
    m.bdy_T = upload(h, bT.data(), d->nboundary, T);
    h->nboundary = d->nboundary;
    h->b2c_dev = upload(h, d->boundary2cell, d->nboundary, T);
    m.T = upload(h, d->temperature, N, T);
    m.dshift_max = upload(h, dsm.data(), N, T);
    m.pw = upload(h, pw.data(), N, T);
    m.inv_pw = upload(h, ipw.data(), N, T);
    m.line = upload(h, line.data(), d->nrad, T);
    m.inv_line = upload(h, iline.data(), d->nrad, T);
    m.A = upload(h, d->A, d->nrad, T);
    m.Bs = upload(h, d->Bs, d->nrad, T);
    m.Ba = upload(h, d->Ba, d->nrad, T);
    m.energy = upload(h, d->energy, d->nlev, T);
    m.weight = upload(h, d->weight, d->nlev, T);
    std::vector<int32_t> ir(d->nrad), jr(d->nrad);
    for (int k = 0; k < d->nrad; k++) { ir[k] = (int32_t)d->irad[k]; jr[k] = (int32_t)d->jrad[k]; }
    m.irad = upload(h, ir.data(), d->nrad, T);
    m.jrad = upload(h, jr.data(), d->nrad, T);
    m.win_lo = upload(h, wlo.data(), d->nrad, T);
    m.win_hi = upload(h, whi.data(), d->nrad, T);
    m.roots = upload(h, d->quad_roots, d->nquads, T);
    {
        const double span = d->quad_roots[d->nquads - 1] - d->quad_roots[0];
        m.root_inv_step = (d->nquads > 1 && span > 0.0) ? (double)(d->nquads - 1) / span : 0.0;
    }
    m.qw = upload(h, d->quad_weights, d->nquads, T);
    m.pop_tot = upload(h, d->population_tot, N, T);
    for (int c = 0; c < d->ncolpar; c++) {
        const mgr_colpar_desc &s = d->colpar[c];
        need(s.ntmp >= 1 && s.ncol >= 0 && s.icol && s.jcol && s.tmp && s.Cd && s.Ce && s.abundance,
             MGR_ERR_INVALID_ARG, "bad collision partner");
        need(s.ortho_para >= 0 && s.ortho_para <= 2, MGR_ERR_INVALID_ARG, "bad ortho_para");
        std::vector<int32_t> ic(std::max(1, s.ncol)), jc(std::max(1, s.ncol));
        for (int k = 0; k < s.ncol; k++) {
            need(s.icol[k] >= 0 && s.icol[k] < d->nlev && s.jcol[k] >= 0 && s.jcol[k] < d->nlev,
                 MGR_ERR_INVALID_ARG, "icol/jcol out of range");
            ic[k] = (int32_t)s.icol[k];
            jc[k] = (int32_t)s.jcol[k];
        }
        ColparDev &cd = m.colpar[c];
        cd.ntmp = s.ntmp;
        cd.ncol = s.ncol;
        cd.ortho_para = s.ortho_para;
        cd.icol = upload(h, ic.data(), (int64_t)ic.size(), T);
        cd.jcol = upload(h, jc.data(), (int64_t)jc.size(), T);
        cd.tmp = upload(h, s.tmp, s.ntmp, T);
        cd.Cd = upload(h, s.Cd, (int64_t)s.ntmp * s.ncol, T);
        cd.Ce = upload(h, s.Ce, (int64_t)s.ntmp * s.ncol, T);
        cd.abn = upload(h, s.abundance, N, T);
    }

    // state
    const int64_t NL = N * h->nlev, NK = N * h->nrad;
    h->pop = dalloc<double>(h, NL, nullptr);
    h->prev1 = dalloc<double>(h, NL, nullptr);
    h->prev2 = dalloc<double>(h, NL, nullptr);
    h->prev3 = dalloc<double>(h, NL, nullptr);
    h->eps = dalloc<double>(h, NK, nullptr);
    h->kap = dalloc<double>(h, NK, nullptr);
    h->ek = dalloc<float2>(h, NK, nullptr);
    h->Jlin = dalloc<double>(h, NK, nullptr);
    h->Lam = dalloc<double>(h, NK, nullptr);
    h->Jeff = dalloc<double>(h, NK, nullptr);
    h->partials = dalloc<double>(h, 5 * (int64_t)level_partials_needed(m), nullptr);
    h->stats = dalloc<double>(h, 8, nullptr);
    h->flags = dalloc<DevFlags>(h, 1, nullptr);
    ck(cudaMemset(h->pop, 0, NL * sizeof(double)), "memset");
    ck(cudaMemset(h->prev1, 0, NL * sizeof(double)), "memset");
    ck(cudaMemset(h->prev2, 0, NL * sizeof(double)), "memset");
    ck(cudaMemset(h->prev3, 0, NL * sizeof(double)), "memset");
    ck(cudaMemset(h->Jlin, 0, NK * sizeof(double)), "memset");
    ck(cudaMemset(h->Lam, 0, NK * sizeof(double)), "memset");
    ck(cudaMemset(h->Jeff, 0, NK * sizeof(double)), "memset");
    ck(cudaMemset(h->stats, 0, 8 * sizeof(double)), "memset");
    ck(cudaMemset(h->flags, 0, sizeof(DevFlags)), "memset");
    h->model_loaded = true;
}

// ------------------------------------------------------------------ traces
void ensure_scan_tmp(mgr_handle *h, int64_t n) {
    size_t bytes = 0;
    ck(cub::DeviceScan::ExclusiveSum(nullptr, bytes, (int64_t *)nullptr, (int64_t *)nullptr, n, h->stream),
       "scan size");
    if (bytes > h->scan_tmp_bytes) {
        free_ptr(h->scan_tmp);
        ck(cudaMalloc(&h->scan_tmp, bytes), "cudaMalloc scan");
        h->scan_tmp_bytes = bytes;
    }
}

// Offsets of lens[0..n) (int32) into off (int64); returns the total.
int64_t scan_lengths(mgr_handle *h, const int32_t *lens, int64_t *off, int64_t n) {
    widen_kernel<<<(unsigned)((n + 255) / 256), 256, 0, h->stream>>>(lens, off, n);
    ck(cudaGetLastError(), "widen");
    h->launches += 1;
    ensure_scan_tmp(h, n);
    size_t bytes = h->scan_tmp_bytes;
    ck(cub::DeviceScan::ExclusiveSum(h->scan_tmp, bytes, off, off, n, h->stream), "scan");
    int64_t last_off = 0;
    int32_t last_len = 0;
    ck(cudaMemcpyAsync(&last_off, off + n - 1, sizeof(int64_t), cudaMemcpyDeviceToHost, h->stream), "d2h");
    ck(cudaMemcpyAsync(&last_len, lens + n - 1, sizeof(int32_t), cudaMemcpyDeviceToHost, h->stream), "d2h");
    ck(cudaStreamSynchronize(h->stream), "scan sync");
    return last_off + last_len;
}

void ensure_points(mgr_handle *h, int64_t npts) {
    if (npts <= h->tcap) return;
    free_ptr((void *&)h->tcell);
    free_ptr((void *&)h->tshift);
    free_ptr((void *&)h->tdz);
    free_ptr((void *&)h->tmp_);
    const int64_t cap = std::max<int64_t>(npts, 1);
    h->tcell = dalloc<int32_t>(h, cap, nullptr);
    h->tshift = dalloc<double>(h, cap, nullptr);
    h->tdz = dalloc<double>(h, cap, nullptr);
    h->tmp_ = dalloc<MixedPoint>(h, cap, nullptr);
    h->tcap = cap;
}

constexpr int64_t kBytesPerPoint = sizeof(int32_t) + 2 * sizeof(double) + sizeof(MixedPoint);
// Hops of a walk the counting pass logs (longer walks are searched again).
constexpr int64_t kHopCap = 128;

// Bytes per origin of the boundary cache (staged shapes only).
int64_t bcache_bytes_per_origin(mgr_handle *h) {
    return solve_is_staged(h->mv) ? (int64_t)h->npairs * 2 * h->nfreqs * (int64_t)sizeof(float) : 0;
}

// 60% of the free device memory plus what the handle's trace buffers hold.
int64_t default_budget(mgr_handle *h) {
    size_t fr = 0, tot = 0;
    ck(cudaMemGetInfo(&fr, &tot), "cudaMemGetInfo");
    return (int64_t)(0.6 * (double)fr) + h->tcap * kBytesPerPoint +
           h->bcache_cap * h->npairs * 2 * h->nfreqs * (int64_t)sizeof(float);
}

// Room for the boundary cache of `origins` origins (a new buffer changes the
// captured graphs' arguments).
void ensure_bcache(mgr_handle *h, int64_t origins) {
    if (origins <= h->bcache_cap) return;
    free_ptr((void *&)h->bcache);
    h->bcache = dalloc<float>(h, origins * h->npairs * 2 * (int64_t)h->nfreqs, nullptr);
    h->bcache_cap = origins;
    h->bc_stamp = 0;
    h->gen++;
}

// Host copy of the trace lengths (for get_npoints_on_rays and get_trace).
void host_lens(mgr_handle *h) {
    if (h->h_len_valid) return;
    const int64_t n = (int64_t)h->nrays * h->N;
    h->h_len.resize(n);
    ck(cudaMemcpy(h->h_len.data(), h->len_all, n * sizeof(int32_t), cudaMemcpyDeviceToHost), "d2h lens");
    h->h_len_valid = true;
}

void do_trace(mgr_handle *h) {
    need(h->model_loaded, MGR_ERR_STATE, "no model uploaded");
    set_device(h);
    // keep the point buffers of an earlier trace for reuse (freeing and
    // allocating several GB costs more than the trace itself); captured
    // graphs stay valid unless a buffer or the storage mode changes
    const void *old_bufs[] = {h->tcell, h->tshift, h->tdz, h->tmp_, h->off_all};
    const bool old_stored = h->stored;
    h->traced = false;
    h->bc_serial++;
    h->stored = false;
    h->h_len_valid = false;
    const int old_max_pair = h->max_pair_points;
    const int64_t N = h->N, R = h->nrays, n = R * N;
    if (!h->len_all) h->len_all = dalloc<int32_t>(h, n, nullptr);
    if (!h->tstats_d) {
        h->tstats_d = dalloc<unsigned long long>(h, 3, nullptr);
        h->pts_origin_d = dalloc<int32_t>(h, N, nullptr);
        if (!h->h_tstats) ck(cudaMallocHost(&h->h_tstats, 3 * sizeof(unsigned long long)), "pinned");
    }
    if (h->nseg > 0 && !h->upd_origin_d) h->upd_origin_d = dalloc<float>(h, N, nullptr);
    // log the walks' hops when the log takes at most a tenth of the free
    // memory (and the caller set no trace budget): the fill then replays them
    bool logged = false;
    if (h->trace_budget == 0) {
        const int64_t bytes = n * (kHopCap + 1) * (int64_t)sizeof(int32_t);
        size_t fr = 0, tot = 0;
        ck(cudaMemGetInfo(&fr, &tot), "cudaMemGetInfo");
        const int64_t held = h->hop_rays * (kHopCap + 1) * (int64_t)sizeof(int32_t);
        if (bytes <= ((int64_t)fr + held) / 10) {
            if (h->hop_rays != n) {
                free_ptr((void *&)h->hop_cell);
                free_ptr((void *&)h->hop_n);
                h->hop_cell = dalloc<int32_t>(h, n * kHopCap, nullptr);
                h->hop_n = dalloc<int32_t>(h, n, nullptr);
                h->hop_rays = n;
            }
            logged = true;
        }
    }
    if (!logged && h->hop_rays) {   // a log kept from an earlier trace is not used again
        free_ptr((void *&)h->hop_cell);
        free_ptr((void *&)h->hop_n);
        h->hop_rays = 0;
    }
    const HopLog hop_log{h->hop_cell, h->hop_n, (int)kHopCap};
    reset_flags(h);
    ck(launch_trace_count(h->mv, 0, N, h->len_all, h->flags, h->stream, logged ? &hop_log : nullptr),
       "trace count");
    // ray-point-frequency updates of one formal solve, the longest pair and
    // the points per origin, reduced on the device
    ck(launch_trace_stats(h->mv, h->len_all, h->tstats_d, h->pts_origin_d,
                          h->nseg > 0 ? h->upd_origin_d : nullptr, h->o_begin, h->o_end, h->stream),
       "trace stats");
    h->launches += 2;
    ck(cudaMemcpyAsync(h->h_tstats, h->tstats_d, 3 * sizeof(unsigned long long),
                       cudaMemcpyDeviceToHost, h->stream), "trace stats");
    check_flags(h, "trace");
    const int64_t total = (int64_t)h->h_tstats[0];
    h->updates_per_solve = (double)h->h_tstats[1] * h->nfreqs;
    h->max_pair_points = (int)h->h_tstats[2];
    if (h->nseg > 0) {
        h->upd_origin.resize(N);
        ck(cudaMemcpy(h->upd_origin.data(), h->upd_origin_d, N * sizeof(float),
                      cudaMemcpyDeviceToHost), "d2h updates");
    } else {
        h->upd_origin.clear();
    }
    if (h->max_pair_points != old_max_pair) {   // tuned shapes depend on the ray lengths
        h->tune[0] = mgr_handle::Tune{};
        h->tune[1] = mgr_handle::Tune{};
    }
    h->total_points = total;
    const int64_t budget = h->trace_budget > 0 ? h->trace_budget : default_budget(h);
    const int64_t per_origin_cache = bcache_bytes_per_origin(h);
    if (total * kBytesPerPoint + N * per_origin_cache <= budget) {
        if (!h->off_all) h->off_all = dalloc<int64_t>(h, n, nullptr);
        const int64_t tot = scan_lengths(h, h->len_all, h->off_all, n);
        ensure_points(h, tot);
        TraceView t{0, N, (int)R, h->off_all, h->len_all, h->tcell, h->tshift, h->tdz, h->tmp_};
        reset_flags(h);
        ck(launch_trace_fill(h->mv, t, h->tcell, h->tshift, h->tdz, h->tmp_, h->flags, h->stream,
                             logged ? &hop_log : nullptr),
           "trace fill");
        h->launches += 1;
        check_flags(h, "trace fill");
        h->stored = true;
        h->batch_origins = N;
    } else {
        // origins per batch so that the largest batch fits the budget
        std::vector<int32_t> per_origin(N);
        ck(cudaMemcpy(per_origin.data(), h->pts_origin_d, N * sizeof(int32_t),
                      cudaMemcpyDeviceToHost), "d2h points");
        int64_t best = N;
        for (;;) {
            int64_t worst = 0;
            for (int64_t o0 = 0; o0 < N; o0 += best) {
                const int64_t o1 = std::min(N, o0 + best);
                int64_t s = 0;
                for (int64_t o = o0; o < o1; o++) s += per_origin[o];
                worst = std::max(worst, s * kBytesPerPoint + (o1 - o0) * per_origin_cache);
            }
            if (worst <= budget || best == 1) break;
            best = std::max<int64_t>(1, best / 2);
        }
        h->batch_origins = best;
        h->stored = false;
    }
    const void *new_bufs[] = {h->tcell, h->tshift, h->tdz, h->tmp_, h->off_all};
    if (old_stored != h->stored || !std::equal(old_bufs, old_bufs + 5, new_bufs)) h->gen++;
    h->traced = true;
}

// Fills the trace store for origins [o0, o0+cnt) and returns its view.
TraceView build_batch(mgr_handle *h, int64_t o0, int64_t cnt) {
    const int64_t R = h->nrays;
    if (cnt > h->bcap) {
        free_ptr((void *&)h->blen);
        free_ptr((void *&)h->boff);
        h->blen = dalloc<int32_t>(h, R * cnt, nullptr);
        h->boff = dalloc<int64_t>(h, R * cnt, nullptr);
        h->bcap = cnt;
    }
    ck(cudaMemcpy2DAsync(h->blen, cnt * sizeof(int32_t), h->len_all + o0, h->N * sizeof(int32_t),
                         cnt * sizeof(int32_t), R, cudaMemcpyDeviceToDevice, h->stream),
       "batch lens");
    const int64_t tot = scan_lengths(h, h->blen, h->boff, R * cnt);
    ensure_points(h, tot);
    TraceView t{o0, cnt, (int)R, h->boff, h->blen, h->tcell, h->tshift, h->tdz, h->tmp_};
    ck(launch_trace_fill(h->mv, t, h->tcell, h->tshift, h->tdz, h->tmp_, h->flags, h->stream),
       "trace fill");
    h->launches += 1;
    return t;
}

void boundary_table(mgr_handle *h) {
    if (!h->ibdy) {
        h->ibdy = dalloc<double>(h, h->nboundary * (int64_t)h->nfreqs, nullptr);
        h->mv.ibdy = h->ibdy;
    }
    ck(launch_boundary_table(h->mv, h->nboundary, h->b2c_dev, h->ibdy, h->stream), "boundary table");
    h->launches += 1;
    ck(cudaStreamSynchronize(h->stream), "boundary sync");
    h->bdy_set = true;
    h->bc_serial++;
}

void do_solve(mgr_handle *h, int precision, bool use_graph);

SolveArgs solve_args(mgr_handle *h) {
    SolveArgs a{};
    a.eps = h->eps;
    a.kap = h->kap;
    a.ehat_khat = h->ek;
    a.mixed_scale = h->mixed_scale;
    a.Jlin = h->Jlin;
    a.Lam = h->Lam;
    a.J = h->keep_J ? h->J : nullptr;
    a.patch = h->patch;
    a.patch_count = h->patch_count;
    a.patch_cap = h->patch_cap;
    a.s_begin = h->o_begin;   // origins of the stored trace (index = origin)
    a.s_end = h->o_end;
    a.olist = nullptr;
    a.redo_flag = h->redo_flag;
    a.redo_list = h->redo_list;
    a.bcache = h->bcache;
    return a;
}

// A mixed solve of a staged shape reads the boundary cache; enqueue_bcache
// fills it for origins [s_begin, s_end) of trace store t (stream work only).
bool bcache_needed(mgr_handle *h, int precision) {
    return precision == MGR_MIXED && solve_is_staged(h->mv);
}
void enqueue_bcache(mgr_handle *h, const TraceView &t, int64_t s_begin, int64_t s_end) {
    ck(launch_bdy_cache(h->mv, t, s_begin, s_end, h->bcache, h->flags, h->stream),
       "boundary cache");
    h->launches += 1;
}

void solve_prepare(mgr_handle *h, int precision) {
    need(h->line_set, MGR_ERR_STATE, "compute_spectral_discretisation first");
    need(h->pops_valid, MGR_ERR_STATE, "no level populations yet (LTE or set_populations)");
    need(precision == MGR_FP64 || precision == MGR_MIXED, MGR_ERR_INVALID_ARG, "bad precision");
    set_device(h);
    if (!h->traced) do_trace(h);
    if (!h->bdy_set) boundary_table(h);
    if (h->keep_J && !h->J) h->J = dalloc<double>(h, h->N * (int64_t)h->nfreqs, nullptr);
    if (precision == MGR_MIXED && !h->patch) {
        // room for 1 in 100 (origin, pair, bin) solves, 1M..64M entries,
        // unless the caller fixed the capacity
        const double all = (double)h->N * h->npairs * h->nfreqs;
        h->patch_cap = h->patch_cap_set > 0 ? h->patch_cap_set
                     : (int64_t)std::min(std::max(all / 100.0, (double)(1 << 20)), (double)(1 << 26));
        h->patch = dalloc<int4>(h, h->patch_cap, nullptr);
        h->patch_count = dalloc<unsigned long long>(h, 1, nullptr);
        h->redo_flag = dalloc<int32_t>(h, h->N, nullptr);
        h->redo_list = dalloc<int32_t>(h, h->N, nullptr);
        ck(cudaMemset(h->redo_flag, 0, h->N * sizeof(int32_t)), "memset");
        h->gen++;
    }
}

// Tuning results shared by the handles of this process, keyed by device,
// precision and the shape that decides the kernel's behaviour.
std::mutex g_tune_mu;
std::map<std::string, int> g_tune_cache;

std::string tune_key(mgr_handle *h, int precision) {
    return std::to_string(h->device) + "/" + std::to_string(precision) + "/" +
           std::to_string(h->nfreqs) + "/" + std::to_string(h->nquads) + "/" +
           std::to_string(h->nrad) + "/" + std::to_string(h->mv.overlap) + "/" +
           std::to_string(h->max_pair_points / 32) + "/" + std::to_string(h->stored ? 1 : 0);
}

// The compiled variant for the next solve: a candidate still to be timed
// while autotuning, else the fastest timed one, else the default (-1).
int solve_variant(mgr_handle *h, int precision, bool *timing) {
    mgr_handle::Tune &tu = h->tune[precision == MGR_MIXED];
    *timing = false;
    if (tu.best >= 0) return tu.best;
    if (h->autotune == 1) {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune_cache.find(tune_key(h, precision));
        if (it != g_tune_cache.end()) {
            tu.best = it->second;
            return tu.best;
        }
    }
    if (h->autotune && tu.next < kSolveVariants) {
        *timing = true;
        return tu.next;
    }
    return -1;
}

void tune_record(mgr_handle *h, int precision, int variant, float ms) {
    mgr_handle::Tune &tu = h->tune[precision == MGR_MIXED];
    tu.ms[variant] = ms;
    tu.next = variant + 1;
    if (tu.next == kSolveVariants) {
        int best = 0;
        for (int v = 1; v < kSolveVariants; v++)
            if (tu.ms[v] < tu.ms[best]) best = v;
        tu.best = best;
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune_cache[tune_key(h, precision)] = best;
    }
}

// Enqueues one formal solve over the stored trace (asynchronous, capturable).
int enqueue_stored_solve(mgr_handle *h, int precision, int variant) {
    const SolveArgs a = solve_args(h);
    reset_flags(h);
    if (precision == MGR_MIXED)
        ck(cudaMemsetAsync(h->patch_count, 0, sizeof(unsigned long long), h->stream), "patch reset");
    TraceView t{0, h->N, h->nrays, h->off_all, h->len_all, h->tcell, h->tshift, h->tdz, h->tmp_};
    int kind = 0;
    ck(launch_formal_solve(h->mv, t, a, precision, variant, h->flags, h->stream, &kind),
       "formal solve");
    h->tune[precision == MGR_MIXED].kind = kind;
    ck(cudaMemcpyAsync(h->h_flags, h->flags, sizeof(DevFlags), cudaMemcpyDeviceToHost, h->stream),
       "flags");
    if (precision == MGR_MIXED)
        ck(cudaMemcpyAsync(h->h_patch, h->patch_count, sizeof(unsigned long long),
                           cudaMemcpyDeviceToHost, h->stream), "patch count");
    return precision == MGR_MIXED ? 2 : 1;
}

// Runs `body` (stream work only; returns the kernels it launches) through a
// CUDA graph captured on first use and replayed while neither the handle's
// generation nor `key` changed.  Returns the kernels per replay.
int graph_run(mgr_handle *h, mgr_handle::Graph &g, int key, const std::function<int()> &body) {
    if (!g.exec || g.gen != h->gen || g.key != key) {
        free_graph(g);
        ck(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeRelaxed), "begin capture");
        cudaGraph_t graph = nullptr;
        try {
            g.kernels = body();
        } catch (...) {
            cudaStreamEndCapture(h->stream, &graph);
            if (graph) cudaGraphDestroy(graph);
            throw;
        }
        ck(cudaStreamEndCapture(h->stream, &graph), "end capture");
        const cudaError_t e = cudaGraphInstantiate(&g.exec, graph, 0);
        cudaGraphDestroy(graph);
        ck(e, "graph instantiate");
        g.gen = h->gen;
        g.key = key;
    }
    ck(cudaGraphLaunch(g.exec, h->stream), "graph launch");
    return g.kernels;
}

// Origins [done, count) of the redo list, whose float failures overflowed
// the patch list, solved again entirely in double over the trace store t
// (their Jlin, ALO and J are overwritten, after the patch pass added to
// them).  Stream work only.
void enqueue_redo(mgr_handle *h, const TraceView &t, int64_t done, int64_t count) {
    if (count <= done) return;
    SolveArgs a = solve_args(h);
    a.olist = h->redo_list;
    a.s_begin = done;
    a.s_end = count;
    int kind = 0;
    ck(launch_formal_solve(h->mv, t, a, MGR_FP64, -1, h->flags, h->stream, &kind), "fp64 redo");
    h->launches += 1;
    h->fp64_fallbacks += count - done;
}

// The non-local ALO elements of origins [s_begin, s_end) of a trace store
// (FP64, whatever the precision of the solve).
void enqueue_offdiag(mgr_handle *h, const TraceView &t, int64_t s_begin, int64_t s_end) {
    OffdiagArgs oa{h->eps, h->kap, h->Loff, h->Loff_nr, h->noff - 1, s_begin, s_end};
    ck(launch_offdiag(h->mv, t, oa, h->flags, h->stream), "off-diagonal ALO");
    h->launches += 1;
}

void finish_solve(mgr_handle *h, int precision, int variant, bool timing, int64_t patched) {
    if (precision == MGR_MIXED && h->stored && h->h_flags->redo_count > 0) {
        // more float failures than the patch list holds: the listed origins
        // again in double, then clear their marks for the next solve
        TraceView t{0, h->N, h->nrays, h->off_all, h->len_all, h->tcell, h->tshift, h->tdz, h->tmp_};
        enqueue_redo(h, t, 0, (int64_t)h->h_flags->redo_count);
        ck(cudaMemsetAsync(h->redo_flag, 0, h->N * sizeof(int32_t), h->stream), "redo reset");
        ck(cudaEventRecord(h->ev1, h->stream), "event");
        ck(cudaStreamSynchronize(h->stream), "fp64 redo");
    }
    check_flags(h, "formal solve");
    float ms = 0.f;
    ck(cudaEventElapsedTime(&ms, h->ev0, h->ev1), "elapsed");
    if (timing) tune_record(h, precision, variant, ms);
    h->last_solve_ms = ms;
    h->last_updates = h->updates_per_solve;
    if (h->nseg > 0 && (int64_t)h->upd_origin.size() == h->N) {
        // a batch: only the origins of models still iterating were solved
        std::vector<int64_t> sb(h->nseg + 1);
        ck(cudaMemcpy(sb.data(), h->seg_begin_d, (h->nseg + 1) * sizeof(int64_t),
                      cudaMemcpyDeviceToHost), "model bounds");
        double U = 0.0;
        for (int64_t g = 0; g < h->nseg; g++)
            if (h->h_seg_active[g])
                for (int64_t o = sb[g]; o < sb[g + 1]; o++) U += h->upd_origin[o];
        h->last_updates = U;
    }
    h->last_patched = patched;
}

void do_solve(mgr_handle *h, int precision, bool use_graph) {
    solve_prepare(h, precision);
    bool timing = false;
    const int variant = solve_variant(h, precision, &timing);
    const bool cache = bcache_needed(h, precision);
    if (h->stored && cache) {
        ensure_bcache(h, h->N);
        if (h->bc_stamp != h->bc_serial) {   // once per trace, grid and boundary table
            reset_flags(h);
            TraceView t{0, h->N, h->nrays, h->off_all, h->len_all, h->tcell, h->tshift, h->tdz, h->tmp_};
            enqueue_bcache(h, t, h->o_begin, h->o_end);
            ck(cudaStreamSynchronize(h->stream), "boundary cache");
            check_flags(h, "boundary cache");
            h->bc_stamp = h->bc_serial;
        }
    }
    if (h->stored) {
        // the events stay outside the graph (a captured record only orders work)
        ck(cudaEventRecord(h->ev0, h->stream), "event");
        if (use_graph && !timing) {
            const int key = precision * 16 + (variant + 1) * 2 + (h->keep_J ? 1 : 0);
            h->launches += graph_run(h, h->g_solve, key,
                                     [&] { return enqueue_stored_solve(h, precision, variant); });
        } else {
            h->launches += enqueue_stored_solve(h, precision, variant);
        }
        ck(cudaEventRecord(h->ev1, h->stream), "event");
        ck(cudaStreamSynchronize(h->stream), "solve sync");
        finish_solve(h, precision, variant, timing,
                     precision == MGR_MIXED ? (int64_t)*h->h_patch : 0);
        h->last_trace_ms = 0.0;
        if (h->noff >= 2) {
            TraceView t{0, h->N, h->nrays, h->off_all, h->len_all, h->tcell, h->tshift, h->tdz, h->tmp_};
            enqueue_offdiag(h, t, h->o_begin, h->o_end);
            ck(cudaStreamSynchronize(h->stream), "off-diagonal ALO");
            check_flags(h, "off-diagonal ALO");
        }
        return;
    }
    // traces in batches of origins, rebuilt for every solve
    if (cache) ensure_bcache(h, h->batch_origins);
    const SolveArgs a = solve_args(h);
    reset_flags(h);
    unsigned long long patched = 0;
    int64_t redo_done = 0;
    ck(cudaEventRecord(h->ev0, h->stream), "event");
    const int64_t nbatches = (h->o_end - h->o_begin + h->batch_origins - 1) / h->batch_origins;
    while ((int64_t)h->batch_ev.size() < 2 * nbatches) {
        cudaEvent_t e;
        ck(cudaEventCreate(&e), "event");
        h->batch_ev.push_back(e);
    }
    int64_t bi = 0;
    for (int64_t o0 = h->o_begin; o0 < h->o_end; o0 += h->batch_origins, bi++) {
        const int64_t cnt = std::min(h->batch_origins, h->o_end - o0);
        ck(cudaEventRecord(h->batch_ev[2 * bi], h->stream), "event");
        TraceView t = build_batch(h, o0, cnt);
        if (cache) enqueue_bcache(h, t, 0, cnt);
        ck(cudaEventRecord(h->batch_ev[2 * bi + 1], h->stream), "event");
        SolveArgs ab = a;   // a batch's store holds exactly the origins it solves
        ab.s_begin = 0;
        ab.s_end = cnt;
        if (precision == MGR_MIXED)
            ck(cudaMemsetAsync(h->patch_count, 0, sizeof(unsigned long long), h->stream), "patch reset");
        int kind = 0;
        ck(launch_formal_solve(h->mv, t, ab, precision, variant, h->flags, h->stream, &kind),
           "formal solve");
        h->tune[precision == MGR_MIXED].kind = kind;
        h->launches += precision == MGR_MIXED ? 2 : 1;
        if (h->noff >= 2) enqueue_offdiag(h, t, 0, cnt);
        if (precision == MGR_MIXED) {
            ck(cudaMemcpyAsync(h->h_patch, h->patch_count, sizeof(unsigned long long),
                               cudaMemcpyDeviceToHost, h->stream), "d2h");
            ck(cudaMemcpyAsync(h->h_flags, h->flags, sizeof(DevFlags), cudaMemcpyDeviceToHost,
                               h->stream), "flags");
            ck(cudaStreamSynchronize(h->stream), "patch count");
            patched += *h->h_patch;
            // overflowing origins of this batch, in double, while its traces exist
            const int64_t listed = (int64_t)h->h_flags->redo_count;
            if (listed > redo_done) {
                enqueue_redo(h, t, redo_done, listed);
                redo_done = listed;
            }
        }
    }
    if (redo_done > 0)
        ck(cudaMemsetAsync(h->redo_flag, 0, h->N * sizeof(int32_t), h->stream), "redo reset");
    ck(cudaEventRecord(h->ev1, h->stream), "event");
    ck(cudaMemcpyAsync(h->h_flags, h->flags, sizeof(DevFlags), cudaMemcpyDeviceToHost, h->stream), "flags");
    ck(cudaStreamSynchronize(h->stream), "solve sync");
    double trace_ms = 0.0;
    for (int64_t b = 0; b < bi; b++) {
        float ms = 0.f;
        ck(cudaEventElapsedTime(&ms, h->batch_ev[2 * b], h->batch_ev[2 * b + 1]), "elapsed");
        trace_ms += ms;
    }
    finish_solve(h, precision, variant, timing, (int64_t)patched);
    h->last_trace_ms = trace_ms;
}

void read_stats(mgr_handle *h) {
    ck(cudaMemcpyAsync(h->h_stats, h->stats, 8 * sizeof(double), cudaMemcpyDeviceToHost, h->stream), "stats");
    ck(cudaStreamSynchronize(h->stream), "stats sync");
}

// Convergence statistics (and per-model ones for a batch) and the error
// counters, copied to pinned host memory.  Stream work only.
int enqueue_stats(mgr_handle *h, const LevelArgs &a) {
    int n = 0;
    if (h->nseg > 0) {
        ck(launch_seg_convergence(h->mv, a, h->seg_stats_d, h->stream), "model convergence");
        ck(cudaMemcpyAsync(h->h_seg_stats, h->seg_stats_d, 3 * h->nseg * sizeof(double),
                           cudaMemcpyDeviceToHost, h->stream), "model stats");
        n = 1;
    }
    ck(cudaMemcpyAsync(h->h_stats, h->stats, 8 * sizeof(double), cudaMemcpyDeviceToHost, h->stream),
       "stats");
    ck(cudaMemcpyAsync(h->h_flags, h->flags, sizeof(DevFlags), cudaMemcpyDeviceToHost, h->stream),
       "flags");
    return n;
}

NonlocalArgs nonlocal_args(mgr_handle *h) {
    return NonlocalArgs{h->Loff, h->Loff_nr, h->noff - 1, h->nl_x[0], h->nl_x[1], h->nl_change};
}

// Statistical equilibrium with the non-local ALO: the rate equations of all
// cells as one system, solved by block-Jacobi sweeps from the populations
// before the solve until no population changes by more than 1e-14 of
// itself (of 1e-10 of its cell's total below that), or, once below 1e-6,
// the change sets no new low for five sweeps (the rounding floor of the
// cell solves); then the statistics and emissivities/opacities.  The host
// reads each sweep's change, so this step is not graph-captured.
int stateq_nonlocal(mgr_handle *h) {
    const LevelArgs a = level_args(h);
    reset_flags(h);
    const int64_t NL = h->N * h->nlev;
    ck(launch_history_shift(h->mv, a, h->stream), "history");
    ck(cudaMemcpyAsync(h->nl_x[0], h->prev1, NL * sizeof(double), cudaMemcpyDeviceToDevice,
                       h->stream), "iterate");
    NonlocalArgs nl = nonlocal_args(h);
    const int nb = nonlocal_sweep_blocks(h->mv);
    int cur = 0, launches = 2, best_sweep = 0;
    double best = INFINITY, last = INFINITY;
    bool ok = false;
    int64_t sweep = 0;
    for (; sweep < 1000; sweep++) {
        nl.x_in = h->nl_x[cur];
        nl.x_out = h->nl_x[1 - cur];
        ck(launch_stateq_nonlocal_sweep(h->mv, a, nl, h->flags, h->stream), "stateq sweep");
        ck(cudaMemcpyAsync(h->h_nl_change, h->nl_change + nb, sizeof(double),
                           cudaMemcpyDeviceToHost, h->stream), "change");
        ck(cudaStreamSynchronize(h->stream), "stateq sweep");
        launches += 2;
        cur = 1 - cur;
        last = *h->h_nl_change;
        if (!(last == last)) break;   // NaN: a singular block (lu_err is set)
        if (last <= 1.0E-14) { ok = true; break; }
        if (last < best) {
            best = last;
            best_sweep = (int)sweep;
        } else if (best < 1.0E-6 && sweep >= best_sweep + 5) {
            ok = true;   // the rounding floor of the cell solves
            break;
        }
    }
    h->nl_sweeps = sweep + 1;
    h->nl_best_change = best;
    ck(cudaMemcpyAsync(h->pop, h->nl_x[cur], NL * sizeof(double), cudaMemcpyDeviceToDevice,
                       h->stream), "populations");
    ck(launch_convergence(h->mv, a, h->stream), "convergence");
    ck(launch_emissivity_opacity(h->mv, a, h->stream), "emissivity");
    launches += 3;
    const int n = enqueue_stats(h, a);
    if (!ok) {
        ck(cudaStreamSynchronize(h->stream), "stats");
        if (h->h_flags->lu_err == 0)
            fail(MGR_ERR_LU_SINGULAR,
                 "non-local rate equations: block Jacobi did not converge (" +
                     std::to_string(h->nl_sweeps) + " sweeps, smallest change " +
                     std::to_string(best) + " at sweep " + std::to_string(best_sweep) +
                     ", last " + std::to_string(last) + ")");
    }
    return launches + n;
}

// Statistical equilibrium (+ statistics); returns the kernels launched.
int enqueue_stateq(mgr_handle *h) {
    if (h->noff >= 2) return stateq_nonlocal(h);
    const LevelArgs a = level_args(h);
    reset_flags(h);
    ck(launch_stateq(h->mv, a, h->flags, h->stream), "stateq");
    return 2 + enqueue_stats(h, a);
}

// Jeff, statistical equilibrium and statistics after a formal solve.
int enqueue_level(mgr_handle *h) {
    if (h->noff >= 2) ck(launch_jeff_nonlocal(h->mv, level_args(h), nonlocal_args(h), h->stream), "jeff");
    else ck(launch_jeff(h->mv, level_args(h), h->stream), "jeff");
    return 1 + enqueue_stateq(h);
}

// Ng step, its convergence statistics and the new emissivities/opacities.
int enqueue_ng(mgr_handle *h) {
    const LevelArgs a = level_args(h);
    reset_flags(h);
    int n = 0;
    if (h->nseg > 0) {
        ck(launch_seg_ng(h->mv, a, h->stream), "model ng");
        n += 1;
    } else {
        ck(launch_ng(h->mv, a, h->stream), "ng");
        n += 3;
    }
    ck(launch_convergence(h->mv, a, h->stream), "convergence");
    ck(launch_emissivity_opacity(h->mv, a, h->stream), "emissivity");
    return n + 3 + enqueue_stats(h, a);
}

void do_stateq(mgr_handle *h) {
    need(h->pops_valid, MGR_ERR_STATE, "no level populations yet");
    h->launches += enqueue_stateq(h);
    ck(cudaStreamSynchronize(h->stream), "statistical equilibrium");
    check_flags_copied(h, "statistical equilibrium");
}

void do_ng(mgr_handle *h) {
    need(h->pops_valid, MGR_ERR_STATE, "no level populations yet");
    h->launches += enqueue_ng(h);
    ck(cudaStreamSynchronize(h->stream), "ng");
}

}  // namespace

// ======================================================================= C ABI

namespace {
mgr_status run(mgr_handle *h, const std::function<void()> &fn) {
    if (!h) return MGR_ERR_INVALID_ARG;
    try {
        fn();
        h->err.clear();
        return MGR_OK;
    } catch (const Failure &f) {
        h->err = f.msg;
        return f.code;
    } catch (const std::exception &e) {
        h->err = e.what();
        return MGR_ERR_INVALID_ARG;
    } catch (...) {
        h->err = "unknown error";
        return MGR_ERR_INVALID_ARG;
    }
}
}  // namespace

extern "C" {

const char *mgr_version(void) { return "magritte_b200 0.1 (sm_100a)"; }

mgr_status mgr_create(int device, mgr_handle **out) {
    if (!out) return MGR_ERR_INVALID_ARG;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) return MGR_ERR_CUDA;
    mgr_handle *h = new (std::nothrow) mgr_handle();
    if (!h) return MGR_ERR_NO_MEMORY;
    h->device = device;
    const mgr_status s = run(h, [&] {
        set_device(h);
        ck(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "stream");
        ck(cudaEventCreate(&h->ev0), "event");
        ck(cudaEventCreate(&h->ev1), "event");
        ck(cudaEventCreate(&h->tev0), "event");
        ck(cudaEventCreate(&h->tev1), "event");
        ck(cudaMallocHost(&h->h_stats, 8 * sizeof(double)), "pinned");
        ck(cudaMallocHost(&h->h_flags, sizeof(DevFlags)), "pinned");
        ck(cudaMallocHost(&h->h_patch, sizeof(unsigned long long)), "pinned");
    });
    if (s != MGR_OK) {
        mgr_destroy(h);
        return s;
    }
    *out = h;
    return MGR_OK;
}

mgr_status mgr_destroy(mgr_handle *h) {
    if (!h) return MGR_ERR_INVALID_ARG;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    free_model(h);
    if (h->h_stats) cudaFreeHost(h->h_stats);
    if (h->h_flags) cudaFreeHost(h->h_flags);
    if (h->h_patch) cudaFreeHost(h->h_patch);
    if (h->h_tstats) cudaFreeHost(h->h_tstats);
    if (h->h_nl_change) cudaFreeHost(h->h_nl_change);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->tev0) cudaEventDestroy(h->tev0);
    if (h->tev1) cudaEventDestroy(h->tev1);
    for (cudaEvent_t e : h->batch_ev) cudaEventDestroy(e);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return MGR_OK;
}

const char *mgr_last_error(const mgr_handle *h) { return h ? h->err.c_str() : "NULL handle"; }

mgr_status mgr_upload_model(mgr_handle *h, const mgr_model_desc *model) {
    return run(h, [&] { do_upload(h, model); });
}

mgr_status mgr_set_trace_budget(mgr_handle *h, int64_t bytes) {
    return run(h, [&] {
        need(bytes >= 0, MGR_ERR_INVALID_ARG, "negative budget");
        h->trace_budget = bytes;
        free_traces(h);
    });
}

mgr_status mgr_compute_spectral_discretisation(mgr_handle *h) {
    return run(h, [&] {
        need(h->model_loaded, MGR_ERR_STATE, "no model uploaded");
        // identity check of the reference's per-cell sort: within a line the
        // roots ascend; consecutive lines must not interleave in any cell
        std::vector<double> pw(h->N), line(h->nrad), roots(h->nquads);
        ck(cudaMemcpy(pw.data(), h->mv.pw, h->N * sizeof(double), cudaMemcpyDeviceToHost), "d2h");
        ck(cudaMemcpy(line.data(), h->mv.line, h->nrad * sizeof(double), cudaMemcpyDeviceToHost), "d2h");
        ck(cudaMemcpy(roots.data(), h->mv.roots, h->nquads * sizeof(double), cudaMemcpyDeviceToHost), "d2h");
        for (int64_t p = 0; p < h->N; p++)
            for (int k = 0; k + 1 < h->nrad; k++) {
                volatile double w0 = line[k] * pw[p], w1 = line[k + 1] * pw[p];
                volatile double a0 = w0 * roots[h->nquads - 1], a1 = w1 * roots[0];
                const double top = line[k] + a0, bot = line[k + 1] + a1;
                if (!(top < bot))
                    fail(MGR_ERR_UNSUPPORTED,
                         "line profiles interleave in cell " + std::to_string(p) +
                             " (frequency grid not ascending); the device path needs separated lines");
            }
        h->line_set = true;
        h->bc_serial++;
    });
}

mgr_status mgr_compute_boundary_intensities(mgr_handle *h) {
    return run(h, [&] {
        need(h->line_set, MGR_ERR_STATE, "compute_spectral_discretisation first");
        set_device(h);
        boundary_table(h);
    });
}

mgr_status mgr_compute_LTE_level_populations(mgr_handle *h) {
    return run(h, [&] {
        need(h->model_loaded, MGR_ERR_STATE, "no model uploaded");
        set_device(h);
        const LevelArgs a = level_args(h);
        ck(launch_lte(h->mv, a, h->stream), "lte");
        ck(launch_emissivity_opacity(h->mv, a, h->stream), "emissivity");
        h->launches += 2;
        ck(cudaStreamSynchronize(h->stream), "lte sync");
        h->pops_valid = true;
    });
}

mgr_status mgr_trace(mgr_handle *h) {
    return run(h, [&] { do_trace(h); });
}

mgr_status mgr_get_npoints_on_rays(mgr_handle *h, int64_t *npoints) {
    return run(h, [&] {
        need(npoints != nullptr, MGR_ERR_INVALID_ARG, "NULL output");
        if (!h->traced) do_trace(h);
        host_lens(h);
        const int64_t N = h->N;
        for (int r = 0; r < h->npairs; r++) {
            const int64_t ar = h->antipod[r];
            for (int64_t o = 0; o < N; o++)
                npoints[r * N + o] = (int64_t)h->h_len[r * N + o] + h->h_len[ar * N + o] + 1;
        }
    });
}

mgr_status mgr_get_trace(mgr_handle *h, int64_t o, int64_t r, int64_t cap, int64_t *cell,
                         double *shift, double *dZ, int64_t *n) {
    return run(h, [&] {
        need(n != nullptr, MGR_ERR_INVALID_ARG, "NULL n");
        need(h->model_loaded, MGR_ERR_STATE, "no model uploaded");
        need(o >= 0 && o < h->N && r >= 0 && r < h->nrays, MGR_ERR_INVALID_ARG, "origin/ray out of range");
        set_device(h);
        if (!h->traced) do_trace(h);
        host_lens(h);
        const int64_t len = h->h_len[r * h->N + o];
        *n = len;
        const int64_t m = std::min(len, cap);
        if (m <= 0) return;
        need(cell && shift && dZ, MGR_ERR_INVALID_ARG, "NULL output arrays");
        int64_t base = 0;
        const int32_t *tc;
        const double *ts, *tz;
        if (h->stored) {
            ck(cudaMemcpy(&base, h->off_all + r * h->N + o, sizeof(int64_t), cudaMemcpyDeviceToHost), "d2h");
            tc = h->tcell; ts = h->tshift; tz = h->tdz;
        } else {
            TraceView t = build_batch(h, o, 1);
            ck(cudaMemcpyAsync(&base, t.off + r, sizeof(int64_t), cudaMemcpyDeviceToHost, h->stream), "d2h");
            ck(cudaStreamSynchronize(h->stream), "sync");
            tc = h->tcell; ts = h->tshift; tz = h->tdz;
        }
        std::vector<int32_t> c(m);
        ck(cudaMemcpy(c.data(), tc + base, m * sizeof(int32_t), cudaMemcpyDeviceToHost), "d2h");
        ck(cudaMemcpy(shift, ts + base, m * sizeof(double), cudaMemcpyDeviceToHost), "d2h");
        ck(cudaMemcpy(dZ, tz + base, m * sizeof(double), cudaMemcpyDeviceToHost), "d2h");
        for (int64_t i = 0; i < m; i++) cell[i] = c[i];
    });
}

mgr_status mgr_set_keep_J(mgr_handle *h, int32_t keep) {
    return run(h, [&] { h->keep_J = keep != 0; });
}

mgr_status mgr_compute_radiation_field(mgr_handle *h, int32_t precision) {
    return run(h, [&] { do_solve(h, precision, false); });
}

mgr_status mgr_compute_Jeff(mgr_handle *h) {
    return run(h, [&] {
        need(h->pops_valid, MGR_ERR_STATE, "no level populations yet");
        if (h->noff >= 2)
            ck(launch_jeff_nonlocal(h->mv, level_args(h), nonlocal_args(h), h->stream), "jeff");
        else
            ck(launch_jeff(h->mv, level_args(h), h->stream), "jeff");
        h->launches += 1;
        ck(cudaStreamSynchronize(h->stream), "jeff sync");
    });
}

mgr_status mgr_compute_level_populations_from_stateq(mgr_handle *h) {
    return run(h, [&] {
        need(h->whole(), MGR_ERR_STATE,
             "a shard (origin range) updates its cells with mgr_stateq_local and mgr_stateq_finish");
        do_stateq(h);
    });
}

mgr_status mgr_set_origin_range(mgr_handle *h, int64_t o_begin, int64_t o_end) {
    return run(h, [&] {
        need(h->model_loaded, MGR_ERR_STATE, "no model uploaded");
        need(h->nseg == 0, MGR_ERR_UNSUPPORTED, "a batch of models is not partitioned");
        need(h->noff < 2, MGR_ERR_UNSUPPORTED, "a non-local ALO run is not partitioned");
        need(0 <= o_begin && o_begin < o_end && o_end <= h->N, MGR_ERR_INVALID_ARG,
             "origin range outside [0, ncells)");
        need(o_begin % kCellsPerPartial == 0 && (o_end % kCellsPerPartial == 0 || o_end == h->N),
             MGR_ERR_INVALID_ARG, "origin range bounds must be multiples of 4 (or ncells)");
        set_device(h);
        ck(cudaStreamSynchronize(h->stream), "sync");
        h->o_begin = o_begin;
        h->o_end = o_end;
        h->traced = false;   // the next trace counts the updates of this range
        h->gen++;
    });
}

mgr_status mgr_stateq_local(mgr_handle *h) {
    return run(h, [&] {
        need(h->pops_valid, MGR_ERR_STATE, "no level populations yet");
        set_device(h);
        const LevelArgs a = level_args(h);
        reset_flags(h);
        ck(launch_jeff(h->mv, a, h->stream), "jeff");
        ck(launch_stateq(h->mv, a, h->flags, h->stream), "stateq");
        h->launches += 3;
        check_flags(h, "statistical equilibrium");
    });
}

mgr_status mgr_stateq_finish(mgr_handle *h) {
    return run(h, [&] {
        set_device(h);
        const LevelArgs a = level_args(h);
        ck(launch_emissivity_opacity(h->mv, a, h->stream), "emissivity");
        ck(launch_convergence_final(h->mv, a, h->stream), "convergence");
        h->launches += 2;
        read_stats(h);
    });
}

mgr_status mgr_get_device_buffer(mgr_handle *h, int32_t which, void **ptr, int64_t *count) {
    return run(h, [&] {
        need(h->model_loaded && ptr && count, MGR_ERR_INVALID_ARG, "no model or NULL output");
        switch (which) {
            case MGR_BUF_POPULATION: *ptr = h->pop; *count = h->N * h->nlev; break;
            case MGR_BUF_PREV1: *ptr = h->prev1; *count = h->N * h->nlev; break;
            case MGR_BUF_PREV2: *ptr = h->prev2; *count = h->N * h->nlev; break;
            case MGR_BUF_PREV3: *ptr = h->prev3; *count = h->N * h->nlev; break;
            case MGR_BUF_JLIN: *ptr = h->Jlin; *count = h->N * h->nrad; break;
            case MGR_BUF_LAMBDA: *ptr = h->Lam; *count = h->N * h->nrad; break;
            case MGR_BUF_CONVERGENCE_PARTIALS:
                *ptr = h->partials;
                *count = 3 * ((h->N + kCellsPerPartial - 1) / kCellsPerPartial);
                break;
            default: fail(MGR_ERR_INVALID_ARG, "unknown buffer");
        }
    });
}

mgr_status mgr_ng_acceleration(mgr_handle *h) {
    return run(h, [&] { do_ng(h); });
}

mgr_status mgr_get_convergence(mgr_handle *h, double *fnc, double *rcm, double *max_rel) {
    return run(h, [&] {
        read_stats(h);
        if (fnc) *fnc = h->h_stats[0];
        if (rcm) *rcm = h->h_stats[1];
        if (max_rel) *max_rel = h->h_stats[2];
    });
}

mgr_status mgr_compute_level_populations(mgr_handle *h, const mgr_ali_opts *opts,
                                         int64_t *iterations, double *err_max_hist) {
    bool not_converged = false;
    const mgr_status s = run(h, [&] {
        need(opts != nullptr, MGR_ERR_INVALID_ARG, "NULL options");
        need(opts->max_iter >= 1, MGR_ERR_INVALID_ARG, "max_iter must be >= 1");
        need(opts->ng_every == 0 || opts->ng_every >= 3, MGR_ERR_INVALID_ARG,
             "ng_every must be 0 (the reference's 4) or >= 3");
        const int64_t ng_every = opts->ng_every > 0 ? opts->ng_every : 4;
        need(h->line_set, MGR_ERR_STATE, "compute_spectral_discretisation first");
        need(h->pops_valid, MGR_ERR_STATE, "no level populations yet");
        need(h->whole(), MGR_ERR_STATE,
             "a shard (origin range) iterates through a partitioned driver, not this loop");
        const bool graph = opts->use_graph != 0 && h->noff < 2;   // non-local: host-driven sweeps
        auto converged = [&](double fnc, double mx) {
            return opts->tol_max_rel > 0.0 ? mx < opts->tol_max_rel : !(fnc > 0.005);
        };
        if (h->nseg > 0) {
            for (int64_t g = 0; g < h->nseg; g++) h->h_seg_active[g] = 1;
            std::fill(h->seg_iters.begin(), h->seg_iters.end(), (int64_t)0);
            ck(cudaMemcpyAsync(h->seg_active_d, h->h_seg_active, h->nseg * sizeof(int32_t),
                               cudaMemcpyHostToDevice, h->stream), "model mask");
        }
        int64_t iteration = 0, normal = 0;
        bool more = true;
        while (more && iteration < opts->max_iter) {
            iteration++;
            if (opts->use_ng && normal == ng_every) {
                h->launches += graph ? graph_run(h, h->g_ng, 0, [&] { return enqueue_ng(h); })
                                     : enqueue_ng(h);
                ck(cudaStreamSynchronize(h->stream), "ng");
                normal = 0;
            } else {
                do_solve(h, opts->precision, graph);
                h->launches += graph ? graph_run(h, h->g_level, 0, [&] { return enqueue_level(h); })
                                     : enqueue_level(h);
                ck(cudaStreamSynchronize(h->stream), "statistical equilibrium");
                check_flags_copied(h, "statistical equilibrium");
                normal++;
            }
            double mx = h->h_stats[2];
            if (h->nseg > 0) {
                bool any = false, changed = false;
                mx = 0.0;
                for (int64_t g = 0; g < h->nseg; g++) {
                    if (!h->h_seg_active[g]) continue;
                    const double *st = h->h_seg_stats + 3 * g;
                    mx = std::max(mx, st[2]);
                    if (converged(st[0], st[2])) {
                        h->h_seg_active[g] = 0;
                        h->seg_iters[g] = iteration;
                        changed = true;
                    } else {
                        any = true;
                    }
                }
                if (changed)
                    ck(cudaMemcpyAsync(h->seg_active_d, h->h_seg_active, h->nseg * sizeof(int32_t),
                                       cudaMemcpyHostToDevice, h->stream), "model mask");
                more = any;
            } else {
                more = !converged(h->h_stats[0], mx);
            }
            if (err_max_hist) err_max_hist[iteration - 1] = mx;
        }
        if (h->nseg > 0) {
            for (int64_t g = 0; g < h->nseg; g++)
                if (h->h_seg_active[g]) h->seg_iters[g] = iteration;
            // leave every model active for later single steps
            for (int64_t g = 0; g < h->nseg; g++) h->h_seg_active[g] = 1;
            ck(cudaMemcpyAsync(h->seg_active_d, h->h_seg_active, h->nseg * sizeof(int32_t),
                               cudaMemcpyHostToDevice, h->stream), "model mask");
            ck(cudaStreamSynchronize(h->stream), "model mask");
        }
        if (iterations) *iterations = iteration;
        not_converged = more;
        if (more) h->err = "maximum number of iterations reached";
    });
    if (s == MGR_OK && not_converged) return MGR_ERR_NOT_CONVERGED;
    return s;
}

mgr_status mgr_set_segments(mgr_handle *h, int64_t nseg, const int64_t *seg_begin) {
    return run(h, [&] {
        need(h->model_loaded, MGR_ERR_STATE, "no model uploaded");
        need(nseg >= 1 && seg_begin != nullptr, MGR_ERR_INVALID_ARG, "need nseg >= 1 and bounds");
        need(seg_begin[0] == 0 && seg_begin[nseg] == h->N, MGR_ERR_INVALID_ARG,
             "model bounds must start at 0 and end at ncells");
        need(h->noff < 2 || nseg == 1, MGR_ERR_UNSUPPORTED,
             "a batch of models runs with the local ALO (n_off_diag 0 or 1)");
        for (int64_t g = 0; g < nseg; g++)
            need(seg_begin[g + 1] > seg_begin[g], MGR_ERR_INVALID_ARG, "empty or unordered model");
        set_device(h);
        ck(cudaStreamSynchronize(h->stream), "sync");
        free_segments(h);
        if (nseg == 1) return;
        std::vector<int32_t> cs(h->N);
        for (int64_t g = 0; g < nseg; g++)
            for (int64_t c = seg_begin[g]; c < seg_begin[g + 1]; c++) cs[c] = (int32_t)g;
        h->seg_begin_d = upload<int64_t>(h, seg_begin, nseg + 1, nullptr);
        h->cell_seg_d = upload<int32_t>(h, cs.data(), h->N, nullptr);
        h->seg_active_d = dalloc<int32_t>(h, nseg, nullptr);
        h->seg_stats_d = dalloc<double>(h, 3 * nseg, nullptr);
        ck(cudaMemset(h->seg_stats_d, 0, 3 * nseg * sizeof(double)), "memset");
        ck(cudaMallocHost(&h->h_seg_stats, 3 * nseg * sizeof(double)), "pinned");
        ck(cudaMallocHost(&h->h_seg_active, nseg * sizeof(int32_t)), "pinned");
        for (int64_t g = 0; g < nseg; g++) h->h_seg_active[g] = 1;
        ck(cudaMemcpy(h->seg_active_d, h->h_seg_active, nseg * sizeof(int32_t),
                      cudaMemcpyHostToDevice), "upload");
        h->nseg = nseg;
        h->seg_iters.assign(nseg, 0);
        h->traced = false;   // the next trace also counts each model's updates
        h->mv.nseg = nseg;
        h->mv.seg_begin = h->seg_begin_d;
        h->mv.cell_seg = h->cell_seg_d;
        h->mv.seg_active = h->seg_active_d;
    });
}

mgr_status mgr_get_segment_results(mgr_handle *h, double *stats, int64_t *iterations) {
    return run(h, [&] {
        need(h->nseg > 0, MGR_ERR_STATE, "no model batch set");
        ck(cudaStreamSynchronize(h->stream), "sync");
        if (stats)
            ck(cudaMemcpy(stats, h->seg_stats_d, 3 * h->nseg * sizeof(double),
                          cudaMemcpyDeviceToHost), "d2h");
        if (iterations)
            for (int64_t g = 0; g < h->nseg; g++) iterations[g] = h->seg_iters[g];
    });
}

mgr_status mgr_set_autotune(mgr_handle *h, int32_t enable) {
    return run(h, [&] {
        need(enable >= 0 && enable <= 2, MGR_ERR_INVALID_ARG, "autotune mode is 0, 1 or 2");
        h->autotune = enable;
        h->tune[0] = mgr_handle::Tune{};
        h->tune[1] = mgr_handle::Tune{};
    });
}

mgr_status mgr_get_tuning(mgr_handle *h, int32_t precision, mgr_tuning *out) {
    return run(h, [&] {
        need(out != nullptr, MGR_ERR_INVALID_ARG, "NULL output");
        need(precision == MGR_FP64 || precision == MGR_MIXED, MGR_ERR_INVALID_ARG, "bad precision");
        const mgr_handle::Tune &tu = h->tune[precision == MGR_MIXED];
        *out = mgr_tuning{};
        out->kernel = tu.kind;
        const int v = tu.best >= 0 ? tu.best : (tu.kind == 1 && precision == MGR_MIXED ? 2 : 1);
        out->min_blocks = solve_variant_blocks(v);
        out->warps_per_block = 4;
        out->tuned = tu.best >= 0 ? 1 : 0;
        for (int i = 0; i < kSolveVariants && i < 8; i++) out->ms[i] = tu.ms[i];
    });
}

mgr_status mgr_set_populations(mgr_handle *h, const double *pop) {
    return run(h, [&] {
        need(h->model_loaded && pop, MGR_ERR_INVALID_ARG, "no model or NULL input");
        ck(cudaMemcpy(h->pop, pop, h->N * h->nlev * sizeof(double), cudaMemcpyHostToDevice), "h2d");
        ck(launch_emissivity_opacity(h->mv, level_args(h), h->stream), "emissivity");
        h->launches += 1;
        ck(cudaStreamSynchronize(h->stream), "sync");
        h->pops_valid = true;
    });
}

#define MGR_GETTER(NAME, PTR, COUNT)                                                          \
    mgr_status NAME(mgr_handle *h, double *out) {                                             \
        return run(h, [&] {                                                                   \
            need(h->model_loaded && out, MGR_ERR_INVALID_ARG, "no model or NULL output");     \
            need(PTR != nullptr, MGR_ERR_STATE, "not computed");                              \
            ck(cudaStreamSynchronize(h->stream), "sync");                                     \
            ck(cudaMemcpy(out, PTR, (size_t)(COUNT) * sizeof(double), cudaMemcpyDeviceToHost), \
               "d2h");                                                                        \
        });                                                                                   \
    }

MGR_GETTER(mgr_get_populations, h->pop, h->N * h->nlev)
MGR_GETTER(mgr_get_J, h->J, h->N * (int64_t)h->nfreqs)
MGR_GETTER(mgr_get_Jlin, h->Jlin, h->N * h->nrad)
MGR_GETTER(mgr_get_Jeff, h->Jeff, h->N * h->nrad)
MGR_GETTER(mgr_get_lambda, h->Lam, h->N * h->nrad)

mgr_status mgr_get_population_history(mgr_handle *h, double *prev1, double *prev2, double *prev3) {
    return run(h, [&] {
        need(h->model_loaded, MGR_ERR_INVALID_ARG, "no model uploaded");
        set_device(h);
        ck(cudaStreamSynchronize(h->stream), "sync");
        const size_t bytes = (size_t)h->N * h->nlev * sizeof(double);
        if (prev1) ck(cudaMemcpy(prev1, h->prev1, bytes, cudaMemcpyDeviceToHost), "d2h");
        if (prev2) ck(cudaMemcpy(prev2, h->prev2, bytes, cudaMemcpyDeviceToHost), "d2h");
        if (prev3) ck(cudaMemcpy(prev3, h->prev3, bytes, cudaMemcpyDeviceToHost), "d2h");
    });
}

mgr_status mgr_set_population_history(mgr_handle *h, const double *pop, const double *prev1,
                                      const double *prev2, const double *prev3) {
    return run(h, [&] {
        need(h->model_loaded && pop, MGR_ERR_INVALID_ARG, "no model or NULL populations");
        set_device(h);
        ck(cudaStreamSynchronize(h->stream), "sync");
        const size_t bytes = (size_t)h->N * h->nlev * sizeof(double);
        ck(cudaMemcpy(h->pop, pop, bytes, cudaMemcpyHostToDevice), "h2d");
        double *dst[3] = {h->prev1, h->prev2, h->prev3};
        const double *src[3] = {prev1, prev2, prev3};
        for (int i = 0; i < 3; i++) {
            if (src[i]) ck(cudaMemcpy(dst[i], src[i], bytes, cudaMemcpyHostToDevice), "h2d");
            else ck(cudaMemset(dst[i], 0, bytes), "memset");
        }
        ck(launch_emissivity_opacity(h->mv, level_args(h), h->stream), "emissivity");
        h->launches += 1;
        ck(cudaStreamSynchronize(h->stream), "sync");
        h->pops_valid = true;
    });
}

mgr_status mgr_get_emissivity_opacity(mgr_handle *h, double *eta, double *chi) {
    return run(h, [&] {
        need(h->model_loaded && eta && chi, MGR_ERR_INVALID_ARG, "no model or NULL output");
        ck(cudaStreamSynchronize(h->stream), "sync");
        ck(cudaMemcpy(eta, h->eps, h->N * h->nrad * sizeof(double), cudaMemcpyDeviceToHost), "d2h");
        ck(cudaMemcpy(chi, h->kap, h->N * h->nrad * sizeof(double), cudaMemcpyDeviceToHost), "d2h");
    });
}

mgr_status mgr_get_frequencies(mgr_handle *h, double *nu) {
    return run(h, [&] {
        need(h->model_loaded && nu, MGR_ERR_INVALID_ARG, "no model or NULL output");
        std::vector<double> pw(h->N), line(h->nrad), roots(h->nquads);
        ck(cudaMemcpy(pw.data(), h->mv.pw, h->N * sizeof(double), cudaMemcpyDeviceToHost), "d2h");
        ck(cudaMemcpy(line.data(), h->mv.line, h->nrad * sizeof(double), cudaMemcpyDeviceToHost), "d2h");
        ck(cudaMemcpy(roots.data(), h->mv.roots, h->nquads * sizeof(double), cudaMemcpyDeviceToHost), "d2h");
        for (int64_t p = 0; p < h->N; p++)
            for (int k = 0; k < h->nrad; k++) {
                volatile double w = line[k] * pw[p];
                for (int z = 0; z < h->nquads; z++) {
                    volatile double a = w * roots[z];
                    nu[(p * h->nrad + k) * h->nquads + z] = line[k] + a;
                }
            }
    });
}

mgr_status mgr_get_patch_stats(mgr_handle *h, int64_t *patched, int64_t *fallbacks) {
    return run(h, [&] {
        if (patched) *patched = h->last_patched;
        if (fallbacks) *fallbacks = h->fp64_fallbacks;
    });
}

mgr_status mgr_set_patch_capacity(mgr_handle *h, int64_t entries) {
    return run(h, [&] {
        need(entries >= 0, MGR_ERR_INVALID_ARG, "negative capacity");
        set_device(h);
        ck(cudaStreamSynchronize(h->stream), "sync");
        free_ptr((void *&)h->patch);
        free_ptr((void *&)h->patch_count);
        free_ptr((void *&)h->redo_flag);
        free_ptr((void *&)h->redo_list);
        h->patch_cap_set = entries;
        h->gen++;
    });
}

mgr_status mgr_set_n_off_diag(mgr_handle *h, int32_t n_off_diag) {
    return run(h, [&] {
        need(h->model_loaded, MGR_ERR_STATE, "no model uploaded");
        need(n_off_diag >= 0 && n_off_diag <= kMaxOffDiag, MGR_ERR_INVALID_ARG,
             "n_off_diag outside 0 .. 8");
        need(n_off_diag < 2 || (h->whole() && h->nseg == 0), MGR_ERR_UNSUPPORTED,
             "the non-local ALO runs on one whole model (no batch, no origin range)");
        need(h->nlev <= kMaxLevels, MGR_ERR_UNSUPPORTED, "too many levels");
        set_device(h);
        ck(cudaStreamSynchronize(h->stream), "sync");
        void **bufs[] = {(void **)&h->Loff, (void **)&h->Loff_nr, (void **)&h->nl_x[0],
                         (void **)&h->nl_x[1], (void **)&h->nl_change};
        for (void **b : bufs) free_ptr(*b);
        h->noff = n_off_diag;
        if (n_off_diag >= 2) {
            const int64_t ne = (int64_t)h->npairs * 2 * (n_off_diag - 1);
            h->Loff = dalloc<double>(h, h->N * h->nrad * ne, nullptr);
            h->Loff_nr = dalloc<int32_t>(h, h->N * ne, nullptr);
            ck(cudaMemsetAsync(h->Loff, 0, h->N * h->nrad * ne * sizeof(double), h->stream), "zero");
            ck(cudaMemsetAsync(h->Loff_nr, 0xff, h->N * ne * sizeof(int32_t), h->stream), "zero");
            h->nl_x[0] = dalloc<double>(h, h->N * h->nlev, nullptr);
            h->nl_x[1] = dalloc<double>(h, h->N * h->nlev, nullptr);
            h->nl_change = dalloc<double>(h, nonlocal_sweep_blocks(h->mv) + 1, nullptr);
            if (!h->h_nl_change) ck(cudaMallocHost(&h->h_nl_change, sizeof(double)), "pinned");
            ck(cudaStreamSynchronize(h->stream), "sync");
        }
        h->gen++;
    });
}

mgr_status mgr_get_alo_nonlocal(mgr_handle *h, double *Loff, int64_t *Loff_nr) {
    return run(h, [&] {
        need(h->noff >= 2, MGR_ERR_STATE, "n_off_diag < 2: the ALO is diagonal");
        set_device(h);
        ck(cudaStreamSynchronize(h->stream), "sync");
        const int64_t ne = (int64_t)h->npairs * 2 * (h->noff - 1);
        if (Loff)
            ck(cudaMemcpy(Loff, h->Loff, h->N * h->nrad * ne * sizeof(double),
                          cudaMemcpyDeviceToHost), "d2h");
        if (Loff_nr) {
            std::vector<int32_t> tmp(h->N * ne);
            ck(cudaMemcpy(tmp.data(), h->Loff_nr, tmp.size() * sizeof(int32_t),
                          cudaMemcpyDeviceToHost), "d2h");
            for (size_t i = 0; i < tmp.size(); i++) Loff_nr[i] = tmp[i];
        }
    });
}

mgr_status mgr_get_nonlocal_sweeps(mgr_handle *h, int64_t *sweeps) {
    return run(h, [&] {
        need(sweeps != nullptr, MGR_ERR_INVALID_ARG, "NULL output");
        *sweeps = h->nl_sweeps;
    });
}

mgr_status mgr_get_solve_breakdown(mgr_handle *h, double *trace_ms) {
    return run(h, [&] {
        if (trace_ms) *trace_ms = h->last_trace_ms;
    });
}

mgr_status mgr_get_solve_stats(mgr_handle *h, double *ms, double *updates) {
    return run(h, [&] {
        if (ms) *ms = h->last_solve_ms;
        if (updates) *updates = h->last_updates;
    });
}

mgr_status mgr_synchronize(mgr_handle *h) {
    return run(h, [&] { ck(cudaStreamSynchronize(h->stream), "sync"); });
}

mgr_status mgr_timer_start(mgr_handle *h) {
    return run(h, [&] { ck(cudaEventRecord(h->tev0, h->stream), "timer start"); });
}

mgr_status mgr_timer_stop(mgr_handle *h, double *ms) {
    return run(h, [&] {
        need(ms != nullptr, MGR_ERR_INVALID_ARG, "NULL output");
        ck(cudaEventRecord(h->tev1, h->stream), "timer stop");
        ck(cudaEventSynchronize(h->tev1), "timer sync");
        float f = 0.f;
        ck(cudaEventElapsedTime(&f, h->tev0, h->tev1), "elapsed");
        *ms = f;
    });
}

// Features of every origin into a device buffer [N*MGR_MLP_FEATURES].
static void device_features(mgr_handle *h, float *dF) {
    if (!h->traced) do_trace(h);
    if (h->stored) {
        TraceView t{0, h->N, h->nrays, h->off_all, h->len_all, h->tcell, h->tshift, h->tdz, h->tmp_};
        ck(launch_features(h->mv, t, dF, h->stream), "features");
        h->launches += 1;
    } else {
        for (int64_t o0 = 0; o0 < h->N; o0 += h->batch_origins) {
            const int64_t cnt = std::min(h->batch_origins, h->N - o0);
            TraceView t = build_batch(h, o0, cnt);
            ck(launch_features(h->mv, t, dF + o0 * MGR_MLP_FEATURES, h->stream), "features");
            h->launches += 2;
        }
    }
}

mgr_status mgr_get_features(mgr_handle *h, float *features) {
    return run(h, [&] {
        need(h->model_loaded && features, MGR_ERR_INVALID_ARG, "no model or NULL output");
        set_device(h);
        float *dF = dalloc<float>(h, h->N * MGR_MLP_FEATURES, nullptr);
        std::unique_ptr<void, decltype(&cudaFree)> guard(dF, &cudaFree);
        device_features(h, dF);
        ck(cudaMemcpyAsync(features, dF, h->N * MGR_MLP_FEATURES * sizeof(float),
                           cudaMemcpyDeviceToHost, h->stream), "d2h");
        ck(cudaStreamSynchronize(h->stream), "features sync");
    });
}

mgr_status mgr_get_lte_logfrac(mgr_handle *h, float *logfrac) {
    return run(h, [&] {
        need(h->model_loaded && logfrac, MGR_ERR_INVALID_ARG, "no model or NULL output");
        set_device(h);
        float *dL = dalloc<float>(h, h->N * h->nlev, nullptr);
        std::unique_ptr<void, decltype(&cudaFree)> guard(dL, &cudaFree);
        ck(launch_lte_logfrac(h->mv, 0, h->N, dL, h->stream), "lte logfrac");
        h->launches += 1;
        ck(cudaMemcpyAsync(logfrac, dL, h->N * h->nlev * sizeof(float), cudaMemcpyDeviceToHost,
                           h->stream), "d2h");
        ck(cudaStreamSynchronize(h->stream), "sync");
    });
}

mgr_status mgr_warm_start(mgr_handle *h, const mgr_mlp *net) {
    return run(h, [&] {
        need(h->model_loaded, MGR_ERR_STATE, "no model uploaded");
        need(net && net->params && net->feat_mean && net->feat_istd, MGR_ERR_INVALID_ARG, "bad network");
        need(net->nin == MGR_MLP_FEATURES && net->nout == h->nlev, MGR_ERR_INVALID_ARG,
             "network shape does not match the model (features, levels)");
        set_device(h);
        const int64_t N = h->N, np = mlp_param_count(net->nin, net->nout);
        if (!h->ws_F) {
            h->ws_F = dalloc<float>(h, N * MGR_MLP_FEATURES, nullptr);
            h->ws_L = dalloc<float>(h, N * h->nlev, nullptr);
            h->ws_D = dalloc<float>(h, N * h->nlev, nullptr);
            h->ws_mean = dalloc<float>(h, MGR_MLP_FEATURES, nullptr);
            h->ws_istd = dalloc<float>(h, MGR_MLP_FEATURES, nullptr);
        }
        if (h->ws_np != np) {
            free_ptr((void *&)h->ws_P);
            h->ws_P = dalloc<float>(h, np, nullptr);
            h->ws_np = np;
        }
        float *dF = h->ws_F, *dL = h->ws_L, *dD = h->ws_D, *P = h->ws_P;
        MlpDevice d;
        d.nin = net->nin;
        d.nout = net->nout;
        ck(cudaMemcpyAsync(P, net->params, np * sizeof(float), cudaMemcpyHostToDevice, h->stream),
           "network parameters");
        ck(cudaMemcpyAsync(h->ws_mean, net->feat_mean, net->nin * sizeof(float),
                           cudaMemcpyHostToDevice, h->stream), "feature mean");
        ck(cudaMemcpyAsync(h->ws_istd, net->feat_istd, net->nin * sizeof(float),
                           cudaMemcpyHostToDevice, h->stream), "feature scale");
        d.mean = h->ws_mean;
        d.istd = h->ws_istd;
        mlp_bind(P, d.nin, d.nout, d.W, d.b);
        ck(mlp_prepare(), "mlp attributes");
        device_features(h, dF);
        ck(launch_lte_logfrac(h->mv, 0, N, dL, h->stream), "lte logfrac");
        ck(launch_mlp_forward(d, dF, N, dD, h->stream), "mlp forward");
        ck(launch_warm_populations(h->mv, 0, N, dL, dD, h->pop, h->stream), "warm populations");
        ck(launch_emissivity_opacity(h->mv, level_args(h), h->stream), "emissivity");
        h->launches += 4;
        ck(cudaStreamSynchronize(h->stream), "warm start sync");
        h->pops_valid = true;
    });
}

mgr_status mgr_compute_image(mgr_handle *h, int64_t ray, double width, double *nu, double *I_m,
                             double *I_p, double *ImX, double *ImY) {
    return run(h, [&] {
        need(h->model_loaded && h->pops_valid, MGR_ERR_STATE, "model and populations first");
        need(ray >= 0 && ray < h->nrays, MGR_ERR_INVALID_ARG, "ray out of range");
        need(width > 0.0 && std::isfinite(width), MGR_ERR_INVALID_ARG, "width must be positive");
        set_device(h);
        const int64_t N = h->N;
        const int K = h->nrad, nq = h->nquads, nf = h->nfreqs;
        // the image grid (Simulation::compute_spectral_discretisation_image,
        // sim_spectrum.tpp:200-250): line + line*width*root, sorted
        std::vector<double> line(K), roots(nq), grid(nf);
        ck(cudaMemcpy(line.data(), h->mv.line, K * sizeof(double), cudaMemcpyDeviceToHost), "d2h");
        ck(cudaMemcpy(roots.data(), h->mv.roots, nq * sizeof(double), cudaMemcpyDeviceToHost), "d2h");
        for (int k = 0; k < K; k++)
            for (int z = 0; z < nq; z++) {
                volatile double lw = line[k] * width;
                volatile double a = lw * roots[z];
                grid[k * nq + z] = line[k] + a;
            }
        std::sort(grid.begin(), grid.end());
        // lines each bin can reach: a traced point sees shift * nu with
        // |shift - 1| <= vmax, the origin nu itself; +-11 widths
        std::vector<int32_t> lo(nf), hi(nf);
        const double sd = h->vmax * (1.0 + 1e-9) + 1e-15;
        for (int f = 0; f < nf; f++) {
            const double flo = grid[f] * (1.0 - sd) * (1.0 - 1e-12);
            const double fhi = grid[f] * (1.0 + sd) * (1.0 + 1e-12);
            int l0 = K, l1 = -1;
            for (int l = 0; l < K; l++) {
                const double wl = line[l] * (1.0 - 11.0 * h->pw_max) * (1.0 - 1e-12);
                const double wh = line[l] * (1.0 + 11.0 * h->pw_max) * (1.0 + 1e-12);
                if (fhi >= wl && flo <= wh) { l0 = std::min(l0, l); l1 = std::max(l1, l); }
            }
            lo[f] = l0 < K ? l0 : 0;
            hi[f] = l1;
        }
        // the two rest-frame traces of every origin: the antipode in front
        const int64_t ar = h->antipod[ray];
        need(ar >= 0, MGR_ERR_INVALID_ARG, "the ray has no antipode");
        auto ray_correct = [&](int64_t r) { return r >= h->nrays / 2 ? h->antipod[r] : r; };
        std::vector<void *> tmp;
        struct Free {
            std::vector<void *> &v;
            ~Free() { for (void *p : v) cudaFree(p); }
        } fr{tmp};
        int32_t *len = dalloc<int32_t>(h, 2 * N, &tmp);
        int64_t *off = dalloc<int64_t>(h, 2 * N, &tmp);
        reset_flags(h);
        ck(launch_image_trace_count(h->mv, (int)ar, (int)ray, (int)ray_correct(ar),
                                    (int)ray_correct(ray), len, h->flags, h->stream), "image trace");
        h->launches += 1;
        check_flags(h, "image trace");
        const int64_t total = scan_lengths(h, len, off, 2 * N);
        int32_t *cell = dalloc<int32_t>(h, total, &tmp);
        double *shift = dalloc<double>(h, total, &tmp);
        double *dZ = dalloc<double>(h, total, &tmp);
        ck(launch_image_trace_fill(h->mv, (int)ar, (int)ray, (int)ray_correct(ar),
                                   (int)ray_correct(ray), len, off, cell, shift, dZ, h->flags,
                                   h->stream), "image trace fill");
        h->launches += 1;
        check_flags(h, "image trace fill");
        ImageArgs a{};
        double *dgrid = upload(h, grid.data(), nf, &tmp);
        a.grid = dgrid;
        a.lo = upload(h, lo.data(), nf, &tmp);
        a.hi = upload(h, hi.data(), nf, &tmp);
        double *table = dalloc<double>(h, h->nboundary * (int64_t)nf, &tmp);
        ck(launch_image_table(h->mv, h->nboundary, h->b2c_dev, dgrid, nf, table, h->stream),
           "image boundary");
        a.table = table;
        a.len = len;
        a.off = off;
        a.cell = cell;
        a.shift = shift;
        a.dZ = dZ;
        a.eps = h->eps;
        a.kap = h->kap;
        a.I_m = dalloc<double>(h, N * nf, &tmp);
        a.I_p = dalloc<double>(h, N * nf, &tmp);
        a.nf = nf;
        reset_flags(h);
        ck(launch_image(h->mv, a, h->flags, h->stream), "image");
        h->launches += 2;
        check_flags(h, "image");
        if (I_m) ck(cudaMemcpy(I_m, a.I_m, N * nf * sizeof(double), cudaMemcpyDeviceToHost), "d2h");
        if (I_p) ck(cudaMemcpy(I_p, a.I_p, N * nf * sizeof(double), cudaMemcpyDeviceToHost), "d2h");
        if (nu) std::copy(grid.begin(), grid.end(), nu);
        // Image::set_coordinates (Simulation/Image/image.cpp:86-127)
        if (ImX || ImY) {
            std::vector<double> pos(3 * N), rr(3);
            ck(cudaMemcpy(pos.data(), h->mv.pos, 3 * N * sizeof(double), cudaMemcpyDeviceToHost), "d2h");
            ck(cudaMemcpy(rr.data(), h->mv.rays + 3 * ray, 3 * sizeof(double), cudaMemcpyDeviceToHost),
               "d2h");
            const double rx = rr[0], ry = rr[1], rz = rr[2];
            const double den = std::sqrt(rx * rx + ry * ry);
            for (int64_t p = 0; p < N; p++) {
                const double x = pos[3 * p], y = pos[3 * p + 1], zz = pos[3 * p + 2];
                double X = x, Y = y;
                if (den != 0.0) {
                    const double iden = 1.0 / den;
                    const double ix = ry * iden, iy = -rx * iden;
                    const double jx = rx * rz * iden, jy = ry * rz * iden, jz = -den;
                    X = ix * x + iy * y;
                    Y = jx * x + jy * y + jz * zz;
                }
                if (ImX) ImX[p] = X;
                if (ImY) ImY[p] = Y;
            }
        }
    });
}

static int64_t scat_count(const mgr_handle *h) {
    return (int64_t)h->npairs * h->N * h->nfreqs;
}

mgr_status mgr_set_scattering_terms(mgr_handle *h, const double *U, const double *V) {
    return run(h, [&] {
        need(h->model_loaded, MGR_ERR_STATE, "no model uploaded");
        set_device(h);
        const int64_t n = scat_count(h);
        if (!h->scat_U) {
            h->scat_U = dalloc<double>(h, n, nullptr);
            h->scat_V = dalloc<double>(h, n, nullptr);
        }
        if (U) ck(cudaMemcpy(h->scat_U, U, n * sizeof(double), cudaMemcpyHostToDevice), "h2d");
        else ck(cudaMemset(h->scat_U, 0, n * sizeof(double)), "memset");
        if (V) ck(cudaMemcpy(h->scat_V, V, n * sizeof(double), cudaMemcpyHostToDevice), "h2d");
        else ck(cudaMemset(h->scat_V, 0, n * sizeof(double)), "memset");
    });
}

mgr_status mgr_get_scattering_terms(mgr_handle *h, double *U, double *V) {
    return run(h, [&] {
        need(h->scat_U != nullptr, MGR_ERR_STATE, "no scattering terms yet");
        set_device(h);
        ck(cudaStreamSynchronize(h->stream), "sync");
        const int64_t n = scat_count(h);
        if (U) ck(cudaMemcpy(U, h->scat_U, n * sizeof(double), cudaMemcpyDeviceToHost), "d2h");
        if (V) ck(cudaMemcpy(V, h->scat_V, n * sizeof(double), cudaMemcpyDeviceToHost), "d2h");
    });
}

mgr_status mgr_compute_radiation_field_scattering(mgr_handle *h) {
    return run(h, [&] {
        need(h->line_set, MGR_ERR_STATE, "compute_spectral_discretisation first");
        need(h->pops_valid, MGR_ERR_STATE, "no level populations yet");
        need(h->scat_U != nullptr, MGR_ERR_STATE, "set the scattering terms first");
        need(h->whole(), MGR_ERR_UNSUPPORTED, "the scattering solve runs on a whole model");
        set_device(h);
        if (!h->traced) do_trace(h);
        need(h->stored, MGR_ERR_UNSUPPORTED,
             "the scattering solve needs the traces stored (raise the trace budget)");
        if (!h->bdy_set) boundary_table(h);
        const int64_t n = scat_count(h);
        if (!h->scat_u) {
            h->scat_u = dalloc<double>(h, n, nullptr);
            h->scat_v = dalloc<double>(h, n, nullptr);
        }
        if (h->keep_J && !h->J) h->J = dalloc<double>(h, h->N * (int64_t)h->nfreqs, nullptr);
        ScatterArgs a{};
        a.eps = h->eps;
        a.kap = h->kap;
        a.U = h->scat_U;
        a.V = h->scat_V;
        a.u = h->scat_u;
        a.v = h->scat_v;
        a.J = h->keep_J ? h->J : nullptr;
        a.Jlin = h->Jlin;
        a.Lam = h->Lam;
        TraceView t{0, h->N, h->nrays, h->off_all, h->len_all, h->tcell, h->tshift, h->tdz, h->tmp_};
        reset_flags(h);
        ck(cudaEventRecord(h->ev0, h->stream), "event");
        ck(launch_scatter(h->mv, t, a, h->flags, h->stream), "scattering solve");
        ck(cudaEventRecord(h->ev1, h->stream), "event");
        h->launches += 1;
        check_flags(h, "scattering solve");
        float ms = 0.f;
        ck(cudaEventElapsedTime(&ms, h->ev0, h->ev1), "elapsed");
        h->last_solve_ms = ms;
        h->last_updates = h->updates_per_solve;
    });
}

mgr_status mgr_get_scattering_uv(mgr_handle *h, double *u, double *v) {
    return run(h, [&] {
        need(h->scat_u != nullptr, MGR_ERR_STATE, "no scattering solve yet");
        set_device(h);
        ck(cudaStreamSynchronize(h->stream), "sync");
        const int64_t n = scat_count(h);
        if (u) ck(cudaMemcpy(u, h->scat_u, n * sizeof(double), cudaMemcpyDeviceToHost), "d2h");
        if (v) ck(cudaMemcpy(v, h->scat_v, n * sizeof(double), cudaMemcpyDeviceToHost), "d2h");
    });
}

mgr_status mgr_calc_U_and_V(mgr_handle *h) {
    return run(h, [&] {
        need(h->scat_u != nullptr && h->scat_U != nullptr, MGR_ERR_STATE, "no scattering solve yet");
        set_device(h);
        ck(launch_calc_uv(h->mv, h->scat_u, h->scat_v, h->scat_U, h->scat_V, h->stream), "U and V");
        h->launches += 1;
        ck(cudaStreamSynchronize(h->stream), "sync");
    });
}

mgr_status mgr_get_launch_count(mgr_handle *h, int64_t *count) {
    return run(h, [&] {
        need(count != nullptr, MGR_ERR_INVALID_ARG, "NULL output");
        *count = h->launches;
    });
}

}  // extern "C"
