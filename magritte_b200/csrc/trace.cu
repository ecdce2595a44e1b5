// trace.cu -- ray tracing through the neighbour graph on the device.
//
// One thread walks one (direction, origin) ray, as Geometry::trace_ray
// <CoMoving> does (Model/Geometry/geometry.tpp:21-95): at each step it picks,
// among the current cell's neighbours that lie further along the ray, the
// one closest to the ray (get_next_general, :328-421), then records the
// projected point, inserting Doppler interpolation points where the shift
// jump exceeds dshift_max (set_data, :100-207).  Every double operation is
// separately rounded (__dmul_rn/__dadd_rn/...) so the traced cell sequence,
// shifts and increments are bit-identical to the oracle's.
//
// Two passes over the same walk: a counting pass sizes each trace, a prefix
// sum places it, a filling pass writes it.  Threads of a warp take 32
// consecutive origins of one direction, which on a lattice walk in step.
// The walk is bounded by the cell count (Z grows strictly, so no cell can
// repeat); failures are counted in DevFlags, never trapped.
#include "mgr_internal.cuh"

namespace mgr {

namespace {

struct Walker {
    const ModelView &m;
    int64_t origin;
    double rx, ry, rz;       // direction of the walk
    double sx, sy, sz;       // direction the Doppler shift is projected on
    double ox, oy, oz;       // origin position
    double vox, voy, voz;    // origin velocity (zero in the rest frame)

    // shift_dir < 0: co-moving frame; otherwise the rest frame with the
    // shift projected on ray shift_dir (Geometry::get_doppler_shift<Rest>
    // fixes it "up the ray": the first-half ray of the pair)
    __device__ Walker(const ModelView &mv, int64_t o, int d, int shift_dir = -1) : m(mv), origin(o) {
        rx = m.rays[3 * d + 0]; ry = m.rays[3 * d + 1]; rz = m.rays[3 * d + 2];
        ox = m.pos[3 * o + 0]; oy = m.pos[3 * o + 1]; oz = m.pos[3 * o + 2];
        if (shift_dir < 0) {
            sx = rx; sy = ry; sz = rz;
            vox = m.vel[3 * o + 0]; voy = m.vel[3 * o + 1]; voz = m.vel[3 * o + 2];
        } else {
            sx = m.rays[3 * shift_dir + 0]; sy = m.rays[3 * shift_dir + 1];
            sz = m.rays[3 * shift_dir + 2];
            vox = voy = voz = 0.0;   // v - 0 is v exactly
        }
    }

    // Geometry::get_doppler_shift<CoMoving> and <Rest> (geometry.tpp:433-465)
    __device__ __forceinline__ double shift(int64_t c) const {
        const double dx = rsub(m.vel[3 * c + 0], vox);
        const double dy = rsub(m.vel[3 * c + 1], voy);
        const double dz = rsub(m.vel[3 * c + 2], voz);
        return rsub(1.0, rdot3(dx, dy, dz, sx, sy, sz));
    }

    // Geometry::get_next_general (geometry.tpp:328-421)
    __device__ __forceinline__ int64_t next(int64_t current, double &Z, double &dZ) const {
        double dmin = 1.7976931348623157e308;   // numeric_limits<double>::max()
        int64_t nxt = -1;
        const int32_t b = m.nbr_off[current], e = m.nbr_off[current + 1];
        for (int32_t k = b; k < e; k++) {
            const int32_t nb = __ldg(m.nbr + k);
            const double Rx = rsub(__ldg(m.pos + 3 * nb + 0), ox);
            const double Ry = rsub(__ldg(m.pos + 3 * nb + 1), oy);
            const double Rz = rsub(__ldg(m.pos + 3 * nb + 2), oz);
            const double Z_new = rdot3(Rx, Ry, Rz, rx, ry, rz);
            if (Z_new > Z) {
                const double d2 = rsub(rdot3(Rx, Ry, Rz, Rx, Ry, Rz), rmul(Z_new, Z_new));
                if (d2 < dmin) {
                    dmin = d2;
                    nxt = nb;
                    dZ = rsub(Z_new, Z);
                }
            }
        }
        Z = radd(Z, dZ);
        return nxt;
    }

    // The same step along a known next cell nb (the one next() chose): its
    // projection and increment by the same operations.
    __device__ __forceinline__ double advance(int64_t nb, double &Z) const {
        const double Rx = rsub(__ldg(m.pos + 3 * nb + 0), ox);
        const double Ry = rsub(__ldg(m.pos + 3 * nb + 1), oy);
        const double Rz = rsub(__ldg(m.pos + 3 * nb + 2), oz);
        const double dZ = rsub(rdot3(Rx, Ry, Rz, rx, ry, rz), Z);
        Z = radd(Z, dZ);
        return dZ;
    }
};

// Sink that only counts points.
struct CountSink {
    int64_t n = 0;
    __device__ __forceinline__ void push(int64_t, double, double) { n++; }
};

// Sink that writes points into the slot [base, base+cap), in both the
// double format and the 16-byte mixed-precision record.
struct WriteSink {
    int64_t n = 0, cap, base;
    int32_t *cell;
    double *shift, *dZ;
    MixedPoint *mp;
    const double *inv_pw;
    double half_inv_scale;
    bool over = false;
    __device__ __forceinline__ void push(int64_t c, double s, double z) {
        if (n < cap) {
            cell[base + n] = (int32_t)c;
            shift[base + n] = s;
            dZ[base + n] = z;
            if (mp) {
                MixedPoint q;
                q.cell = (int32_t)c;
                q.delta = (float)(s - 1.0);
                q.dzs = (float)(z * half_inv_scale);
                q.ipw = (float)inv_pw[c];
                mp[base + n] = q;
            }
        } else {
            over = true;
        }
        n++;
    }
};

// Geometry::set_data (geometry.tpp:100-207); returns false on > 10000
// interpolation points.
template <class Sink>
__device__ __forceinline__ bool set_data(int64_t crt, int64_t nxt, double shift_crt,
                                         double shift_nxt, double dZ_loc, double dshift_max,
                                         Sink &sink) {
    const double dshift = rsub(shift_nxt, shift_crt);
    const double dshift_abs = fabs(dshift);
    if (dshift_abs > dshift_max) {
        const double q = radd(rdiv(dshift_abs, dshift_max), 1.0);
        if (!(q < 10001.0)) return false;           // n_interpl > 10000, or NaN
        const long long n_interpl = (long long)q;
        const long long half_n_interpl = (long long)rmul(0.5, (double)n_interpl);
        const double dZ_interpl = rdiv(dZ_loc, (double)n_interpl);
        const double dshift_interpl = rdiv(dshift, (double)n_interpl);
        if (n_interpl > 10000 || n_interpl < 0) return false;
        for (long long k = 1; k < half_n_interpl; k++)
            sink.push(crt, radd(shift_crt, rmul((double)k, dshift_interpl)), dZ_interpl);
        for (long long k = half_n_interpl; k <= n_interpl; k++)
            sink.push(nxt, radd(shift_crt, rmul((double)k, dshift_interpl)), dZ_interpl);
    } else {
        sink.push(nxt, shift_nxt, dZ_loc);
    }
    return true;
}

// Geometry::trace_ray<CoMoving> (geometry.tpp:21-95).  Returns 0 or an
// error code: 1 no neighbour ahead, 2 too many interpolation points,
// 3 step limit.
// With a hop log (log, stride = the rays of the log, idx = this ray), each
// hop's cell is recorded while it fits the log's capacity, and the hop
// count (or -1 beyond it) at the end of a walk without error.
template <class Sink>
__device__ int walk(const ModelView &m, int64_t o, int d, Sink &sink, int shift_dir = -1,
                    const HopLog *log = nullptr, int64_t stride = 0, int64_t idx = 0) {
    const Walker w(m, o, d, shift_dir);
    const double dsm = m.dshift_max[o];
    double Z = 0.0, dZ = 0.0;
    int hops = 0;
    auto record = [&](int64_t c) {
        if (log && hops < log->cap) log->cell[(int64_t)hops * stride + idx] = (int32_t)c;
        hops++;
    };
    auto finish = [&]() {
        if (log) log->n[idx] = hops <= log->cap ? hops : -1;
        return 0;
    };
    int64_t nxt = w.next(o, Z, dZ);
    if (nxt == -1) return finish();
    record(nxt);
    int64_t crt = o;
    double shift_crt = w.shift(crt);
    double shift_nxt = w.shift(nxt);
    if (!set_data(crt, nxt, shift_crt, shift_nxt, dZ, dsm, sink)) return 2;
    int64_t steps = 0;
    while (!m.boundary[nxt]) {
        if (++steps > m.N) return 3;
        shift_crt = shift_nxt;
        crt = nxt;
        nxt = w.next(nxt, Z, dZ);
        if (nxt < 0) return 1;
        record(nxt);
        shift_nxt = w.shift(nxt);
        if (!set_data(crt, nxt, shift_crt, shift_nxt, dZ, dsm, sink)) return 2;
    }
    return finish();
}

// The walk of a ray whose hops the counting pass logged: the same points
// from the logged cells, without the neighbour search.  Returns 0, or 2 if
// set_data fails (it cannot where the counting pass succeeded).
template <class Sink>
__device__ int replay(const ModelView &m, int64_t o, int d, const HopLog &log, int64_t stride,
                      int64_t idx, int nh, Sink &sink) {
    const Walker w(m, o, d, -1);
    const double dsm = m.dshift_max[o];
    double Z = 0.0;
    int64_t crt = o;
    double shift_crt = w.shift(crt);
    for (int k = 0; k < nh; k++) {
        const int64_t nxt = __ldg(log.cell + (int64_t)k * stride + idx);
        const double dZ = w.advance(nxt, Z);
        const double shift_nxt = w.shift(nxt);
        if (!set_data(crt, nxt, shift_crt, shift_nxt, dZ, dsm, sink)) return 2;
        crt = nxt;
        shift_crt = shift_nxt;
    }
    return 0;
}

__device__ __forceinline__ void count_error(DevFlags *f, int code) {
    if (code == 1) atomicAdd(&f->trace_err, 1ull);
    else if (code == 2) atomicAdd(&f->interp_err, 1ull);
    else if (code == 3) atomicAdd(&f->stuck_err, 1ull);
}

__global__ void __launch_bounds__(128) trace_count_kernel(ModelView m, int64_t o_begin,
                                                          int64_t o_count, int32_t *len,
                                                          DevFlags *flags, HopLog log,
                                                          bool logged) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t total = (int64_t)m.nrays * o_count;
    if (idx >= total) return;
    const int d = (int)(idx / o_count);
    const int64_t o = o_begin + idx % o_count;
    CountSink sink;
    const int code = walk(m, o, d, sink, -1, logged ? &log : nullptr, total, idx);
    if (code) count_error(flags, code);
    len[idx] = code ? 0 : (int32_t)sink.n;
}

__global__ void __launch_bounds__(128) trace_fill_kernel(ModelView m, TraceView t,
                                                         int32_t *cell, double *shift,
                                                         double *dZ, MixedPoint *mp,
                                                         DevFlags *flags, HopLog log,
                                                         bool logged) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t total = (int64_t)t.ndir * t.o_count;
    if (idx >= total) return;
    const int d = (int)(idx / t.o_count);
    const int64_t o = t.o_begin + idx % t.o_count;
    WriteSink sink;
    sink.cap = t.len[idx];
    sink.base = t.off[idx];
    sink.cell = cell;
    sink.shift = shift;
    sink.dZ = dZ;
    sink.mp = mp;
    sink.inv_pw = m.inv_pw;
    sink.half_inv_scale = 0.5 / m.mixed_scale;
    const int nh = logged ? log.n[idx] : -1;
    const int code = nh >= 0 ? replay(m, o, d, log, total, idx, nh, sink) : walk(m, o, d, sink);
    if (code) count_error(flags, code);
    if (sink.over || (code == 0 && sink.n != sink.cap)) atomicAdd(&flags->cap_err, 1ull);
}

// Rest-frame traces of the two rays of one image (Simulation::
// compute_and_write_image, sim_radiation.tpp:398-399): direction slot d of
// origin o walks ray dirs[d]; idx = d * N + o.
__global__ void __launch_bounds__(128) image_trace_count_kernel(ModelView m, int2 dirs,
                                                                int2 sdirs, int32_t *len,
                                                                DevFlags *flags) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= 2 * m.N) return;
    const int d = (int)(idx / m.N);
    const int64_t o = idx % m.N;
    CountSink sink;
    const int code = walk(m, o, d == 0 ? dirs.x : dirs.y, sink, d == 0 ? sdirs.x : sdirs.y);
    if (code) count_error(flags, code);
    len[idx] = code ? 0 : (int32_t)sink.n;
}

__global__ void __launch_bounds__(128) image_trace_fill_kernel(ModelView m, int2 dirs,
                                                               int2 sdirs, const int32_t *len,
                                                               const int64_t *off, int32_t *cell,
                                                               double *shift, double *dZ,
                                                               DevFlags *flags) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= 2 * m.N) return;
    const int d = (int)(idx / m.N);
    const int64_t o = idx % m.N;
    WriteSink sink;
    sink.cap = len[idx];
    sink.base = off[idx];
    sink.cell = cell;
    sink.shift = shift;
    sink.dZ = dZ;
    sink.mp = nullptr;
    sink.inv_pw = m.inv_pw;
    sink.half_inv_scale = 0.0;
    const int code = walk(m, o, d == 0 ? dirs.x : dirs.y, sink, d == 0 ? sdirs.x : sdirs.y);
    if (code) count_error(flags, code);
    if (sink.over || (code == 0 && sink.n != sink.cap)) atomicAdd(&flags->cap_err, 1ull);
}

// Statistics of a counted trace, one thread per origin: the points of every
// direction, the ray-point sum of the formal solve's update count
// (sum over pairs of ndep = n_r + n_ar + 1 where ndep > 1, as
// get_npoints_on_rays counts them, simulation.tpp:540-552), the longest ray
// pair, and optionally each origin's points and updates.
__global__ void __launch_bounds__(256) trace_stats_kernel(const int32_t *__restrict__ len,
                                                          const int32_t *__restrict__ antipod,
                                                          int64_t N, int R, int npairs, int nfreqs,
                                                          unsigned long long *acc,
                                                          int32_t *pts_origin, float *upd_origin,
                                                          int64_t u_begin, int64_t u_end) {
    const int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long pts = 0, U = 0, mx = 0;
    if (o < N) {
        for (int d = 0; d < R; d++) pts += (unsigned)len[(int64_t)d * N + o];
        for (int r = 0; r < npairs; r++) {
            const unsigned long long ndep =
                (unsigned)len[(int64_t)r * N + o] + (unsigned)len[(int64_t)antipod[r] * N + o] + 1ull;
            if (ndep > 1 && o >= u_begin && o < u_end) U += ndep;
            mx = ndep - 1 > mx ? ndep - 1 : mx;
        }
        if (pts_origin) pts_origin[o] = (int32_t)pts;
        if (upd_origin) upd_origin[o] = (float)((double)U * nfreqs);
    }
#pragma unroll
    for (int sh = 16; sh > 0; sh >>= 1) {
        pts += __shfl_xor_sync(0xffffffffu, pts, sh);
        U += __shfl_xor_sync(0xffffffffu, U, sh);
        const unsigned long long m2 = __shfl_xor_sync(0xffffffffu, mx, sh);
        mx = m2 > mx ? m2 : mx;
    }
    if ((threadIdx.x & 31) == 0 && (pts | U | mx)) {
        atomicAdd(acc + 0, pts);
        atomicAdd(acc + 1, U);
        atomicMax(acc + 2, mx);
    }
}

}  // namespace

cudaError_t launch_trace_stats(const ModelView &m, const int32_t *len, unsigned long long *acc,
                               int32_t *pts_origin, float *upd_origin, int64_t u_begin,
                               int64_t u_end, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(acc, 0, 3 * sizeof(unsigned long long), s);
    if (e != cudaSuccess) return e;
    const int64_t blocks = (m.N + 255) / 256;
    trace_stats_kernel<<<(unsigned)blocks, 256, 0, s>>>(len, m.antipod, m.N, m.nrays, m.npairs,
                                                        m.nfreqs, acc, pts_origin, upd_origin,
                                                        u_begin, u_end);
    return cudaGetLastError();
}

cudaError_t launch_image_trace_count(const ModelView &m, int ray_front, int ray_back,
                                     int shift_front, int shift_back, int32_t *len,
                                     DevFlags *flags, cudaStream_t s) {
    const int64_t blocks = (2 * m.N + 127) / 128;
    image_trace_count_kernel<<<(unsigned)blocks, 128, 0, s>>>(
        m, make_int2(ray_front, ray_back), make_int2(shift_front, shift_back), len, flags);
    return cudaGetLastError();
}

cudaError_t launch_image_trace_fill(const ModelView &m, int ray_front, int ray_back,
                                    int shift_front, int shift_back, const int32_t *len,
                                    const int64_t *off, int32_t *cell, double *shift, double *dZ,
                                    DevFlags *flags, cudaStream_t s) {
    const int64_t blocks = (2 * m.N + 127) / 128;
    image_trace_fill_kernel<<<(unsigned)blocks, 128, 0, s>>>(
        m, make_int2(ray_front, ray_back), make_int2(shift_front, shift_back), len, off, cell,
        shift, dZ, flags);
    return cudaGetLastError();
}

cudaError_t launch_trace_count(const ModelView &m, int64_t o_begin, int64_t o_count,
                               int32_t *len, DevFlags *flags, cudaStream_t s,
                               const HopLog *hops) {
    const int64_t total = (int64_t)m.nrays * o_count;
    if (total == 0) return cudaSuccess;
    const int threads = 128;
    const int64_t blocks = (total + threads - 1) / threads;
    trace_count_kernel<<<(unsigned)blocks, threads, 0, s>>>(
        m, o_begin, o_count, len, flags, hops ? *hops : HopLog{nullptr, nullptr, 0}, hops != nullptr);
    return cudaGetLastError();
}

cudaError_t launch_trace_fill(const ModelView &m, const TraceView &t, int32_t *cell,
                              double *shift, double *dZ, MixedPoint *mp, DevFlags *flags,
                              cudaStream_t s, const HopLog *hops) {
    const int64_t total = (int64_t)t.ndir * t.o_count;
    if (total == 0) return cudaSuccess;
    // a log indexes the rays of all origins: usable for a store of all of them
    if (hops && (t.o_begin != 0 || t.o_count != m.N)) return cudaErrorInvalidValue;
    const int threads = 128;
    const int64_t blocks = (total + threads - 1) / threads;
    trace_fill_kernel<<<(unsigned)blocks, threads, 0, s>>>(
        m, t, cell, shift, dZ, mp, flags, hops ? *hops : HopLog{nullptr, nullptr, 0}, hops != nullptr);
    return cudaGetLastError();
}

}  // namespace mgr
