// runtime.hpp -- internals of the host runtime shared by the C ABI (bsar_api.cpp) and the
// serving engine (bsar_serve.cpp): the context, budget-charged device buffers, DEM and
// scene staging, pulse compression and the mixed form's per-request device record.
#pragma once

#include "bsar.h"

#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "kernels.hpp"

using namespace bsar;

namespace bsar_rt {

constexpr double kPi = 3.14159265358979323846;
constexpr double kDefaultSearchRadius = 1.5;   // m, Newton node-scan radius
constexpr int64_t kDefaultTileWaitPolls = int64_t(1) << 24;

struct Error {
    bsar_status status;
    std::string msg;
};

[[noreturn]] inline void fail(bsar_status s, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    throw Error{s, buf};
}

inline void cuda_check(cudaError_t e, const char* what)
{
    if (e != cudaSuccess) fail(BSAR_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

inline bool is_pow2(int64_t n) { return n > 0 && (n & (n - 1)) == 0; }
inline int64_t next_pow2(int64_t n)
{
    int64_t p = 1;
    while (p < n) p *= 2;
    return p;
}
inline int ilog2(int64_t n)
{
    int l = 0;
    while ((int64_t(1) << l) < n) l++;
    return l;
}

}  // namespace bsar_rt

using namespace bsar_rt;

// ------------------------------------------------------------------------------------
// Context and device buffers
// ------------------------------------------------------------------------------------
struct DevBuf;

struct bsar_ctx {
    uint64_t serial = 0;   // unique per context in the process
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    uint64_t budget = 0;
    uint64_t used = 0;
    uint64_t launches = 0;
    std::mutex mu;
    uint64_t next_scene = 1;
    std::map<uint64_t, std::unique_ptr<struct Scene>> scenes;
    std::map<std::pair<int64_t, int>, std::unique_ptr<DevBuf>> twiddles;   // (P, real bytes; -4: rf_twiddles)
    // cached grid axes for the asynchronous entry point
    std::vector<double> grid_host;
    std::unique_ptr<DevBuf> grid_dev;
    // device status word raised by bounded device-side waits
    std::unique_ptr<DevBuf> status;
    // one-request mixed launch: request record and work counter
    std::unique_ptr<DevBuf> mixed_req, mixed_counter;
    // stream-ordered pool: while `use_pool` is set (the default), buffers come from it,
    // allocated and released on the context's current stream without the device-wide
    // synchronisation of cudaMalloc / cudaFree; freed blocks stay in the pool until
    // bsar_destroy.  Buffers that other streams use (the server's batch records) are
    // taken with `use_pool` cleared.
    cudaMemPool_t pool = nullptr;
    bool use_pool = false;
    // polls of the mixed kernel's bounded DEM-tile wait (bsar_set_tile_wait_limit)
    int64_t tile_wait_polls = kDefaultTileWaitPolls;
};

struct DevBuf {
    bsar_ctx* ctx = nullptr;
    void* p = nullptr;
    size_t bytes = 0;
    bool pooled = false;
    DevBuf() = default;
    DevBuf(bsar_ctx* c, size_t n) : ctx(c), bytes(n)
    {
        if (n == 0) return;
        if (ctx->used + n > ctx->budget)
            fail(BSAR_ERR_OOM_BUDGET, "request of %zu bytes exceeds the HBM budget (%llu of %llu bytes in use)", n,
                 (unsigned long long)ctx->used, (unsigned long long)ctx->budget);
        pooled = ctx->use_pool && ctx->pool;
        cudaError_t e = pooled ? cudaMallocFromPoolAsync(&p, n, ctx->pool, ctx->stream) : cudaMalloc(&p, n);
        if (e != cudaSuccess) {
            p = nullptr;
            cudaGetLastError();
            fail(e == cudaErrorMemoryAllocation ? BSAR_ERR_OOM_BUDGET : BSAR_ERR_CUDA, "device allocation (%zu): %s",
                 n, cudaGetErrorString(e));
        }
        ctx->used += n;
    }
    // A pooled buffer is released on the context's current stream: every use of it has
    // finished (the owner synchronised, or saw the using work complete) before release.
    ~DevBuf()
    {
        if (p) {
            if (pooled)
                cudaFreeAsync(p, ctx->stream);
            else
                cudaFree(p);
            ctx->used -= bytes;
        }
    }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    template <typename T> T* as() const { return static_cast<T*>(p); }
};

inline std::unique_ptr<DevBuf> dev_alloc(bsar_ctx* ctx, size_t n) { return std::make_unique<DevBuf>(ctx, n); }

inline std::unique_ptr<DevBuf> dev_upload(bsar_ctx* ctx, const void* host, size_t n)
{
    auto b = dev_alloc(ctx, n);
    if (n) cuda_check(cudaMemcpyAsync(b->p, host, n, cudaMemcpyHostToDevice, ctx->stream), "upload");
    return b;
}

inline void launched(bsar_ctx* ctx, cudaError_t e, const char* what)
{
    cuda_check(e, what);
    ctx->launches++;
}

inline void sync(bsar_ctx* ctx) { cuda_check(cudaStreamSynchronize(ctx->stream), "stream synchronize"); }

// Last error messages, kept per calling thread and per context: bsar_last_error returns
// the message of the calling thread's latest call on that context, so threads sharing a
// context (the reference calls its Fermat solver from up to 12 OpenMP threads) never read
// a string another thread is rewriting.  A successful call clears the thread's entry.
// Entries carry the context's serial number, so a context created later at the address
// of a destroyed one never shows an entry another thread left for the old one.
struct ThreadError {
    uint64_t serial;
    std::string msg;
};
inline std::map<const bsar_ctx*, ThreadError>& thread_errors()
{
    thread_local std::map<const bsar_ctx*, ThreadError> m;
    return m;
}
inline void set_error(const bsar_ctx* ctx, const std::string& msg) { thread_errors()[ctx] = {ctx->serial, msg}; }
inline void clear_error(const bsar_ctx* ctx) { thread_errors().erase(ctx); }
inline const char* thread_error_message(const bsar_ctx* ctx)
{
    auto& m = thread_errors();
    auto it = m.find(ctx);
    return (it == m.end() || it->second.serial != ctx->serial) ? "" : it->second.msg.c_str();
}

// Runs an entry point's body with the context locked and its device current, turning
// errors into a status and the calling thread's last error.
template <typename F> inline bsar_status guarded(bsar_ctx* ctx, F&& f)
{
    if (!ctx) return BSAR_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(ctx->mu);
    try {
        cuda_check(cudaSetDevice(ctx->device), "cudaSetDevice");
        f();
        clear_error(ctx);
        return BSAR_OK;
    } catch (const Error& e) {
        set_error(ctx, e.msg);
        return e.status;
    } catch (const std::bad_alloc&) {
        set_error(ctx, "host allocation failed");
        return BSAR_ERR_OOM_BUDGET;
    }
}

// A bounded device-side wait that ran out raises the context's status word.
inline void check_device_status(bsar_ctx* ctx)
{
    if (!ctx->status) return;
    int h = 0;
    cuda_check(cudaMemcpy(&h, ctx->status->p, sizeof(int), cudaMemcpyDeviceToHost), "status read");
    if (h) {
        cuda_check(cudaMemset(ctx->status->p, 0, sizeof(int)), "status reset");
        fail(BSAR_ERR_TIMEOUT, "a device-side DEM tile copy did not complete within its wait limit");
    }
}


// ------------------------------------------------------------------------------------
// DEM staging
// ------------------------------------------------------------------------------------
struct DemDev {
    std::unique_ptr<DevBuf> xv, yv, z, z32;
    DemView view{};
    int pitch = 0;                                  // row pitch of z32 (floats, multiple of 4)
    float zmin32 = 0.0f;                            // lowest FP32 height of the DEM
    alignas(64) unsigned char tmap[sizeof(CUtensorMap)] = {};
    bool has_tmap = false;
};

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link to libcuda).
inline PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        cudaGetLastError();
    }
    return fn;
}

// Tensor map of the FP32 DEM for the mixed kernel's TMA tile loads.
inline bool make_dem_tmap(DemDev& r)
{
    auto enc = tensor_map_encoder();
    if (!enc || !r.z32) return false;
    cuuint64_t dims[2] = {(cuuint64_t)r.view.nx, (cuuint64_t)r.view.ny};
    cuuint64_t strides[1] = {(cuuint64_t)r.pitch * sizeof(float)};
    cuuint32_t box[2] = {(cuuint32_t)kMixedTileI, (cuuint32_t)kMixedTileJ};
    cuuint32_t estr[2] = {1, 1};
    CUresult e = enc(reinterpret_cast<CUtensorMap*>(r.tmap), CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, r.z32->p, dims,
                     strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return e == CUDA_SUCCESS;
}

inline void check_dem(const bsar_dem* d)
{
    if (!d) fail(BSAR_ERR_INVALID_ARG, "dem is NULL");
    if (d->nx < 0 || d->ny < 0) fail(BSAR_ERR_INVALID_ARG, "negative DEM size");
    if (d->nx > (1 << 20) || d->ny > (1 << 20)) fail(BSAR_ERR_INVALID_ARG, "DEM axis longer than 2^20 nodes");
    if (d->nx > 0 && d->ny > 0 && (!d->x_vec || !d->y_vec || !d->z))
        fail(BSAR_ERR_INVALID_ARG, "DEM arrays are NULL");
}

inline bool non_decreasing(const double* v, int64_t n)
{
    for (int64_t i = 0; i + 1 < n; i++)
        if (!(v[i] <= v[i + 1])) return false;
    return true;
}

inline bool strictly_ascending(const double* v, int64_t n)
{
    for (int64_t i = 0; i + 1 < n; i++)
        if (!(v[i] < v[i + 1])) return false;
    return true;
}

// Strictly ascending and equally spaced: every node within 1e-6 of a step of
// v[0] + k * step (the node index of a coordinate is then a rounding away).
inline bool equally_spaced(const double* v, int64_t n)
{
    if (!strictly_ascending(v, n)) return false;
    if (n < 3) return true;
    const double step = (v[n - 1] - v[0]) / (double)(n - 1);
    for (int64_t k = 1; k + 1 < n; k++)
        if (!(std::fabs(v[k] - (v[0] + (double)k * step)) <= 1e-6 * step)) return false;
    return true;
}

inline DemDev stage_dem(bsar_ctx* ctx, const bsar_dem* d, bool want_z32)
{
    check_dem(d);
    DemDev r;
    DemView& v = r.view;
    v.nx = (int)d->nx;
    v.ny = (int)d->ny;
    v.empty = (d->nx == 0 || d->ny == 0) ? 1 : 0;
    if (v.empty) {
        // keep valid pointers for kernels that never dereference them
        r.xv = dev_alloc(ctx, 16);
        r.yv = dev_alloc(ctx, 16);
        r.z = dev_alloc(ctx, 16);
        cuda_check(cudaMemsetAsync(r.z->p, 0, 16, ctx->stream), "memset");
        v.xv = r.xv->as<double>();
        v.yv = r.yv->as<double>();
        v.z = r.z->as<double>();
        v.z32 = nullptr;
        return r;
    }
    r.xv = dev_upload(ctx, d->x_vec, sizeof(double) * d->nx);
    r.yv = dev_upload(ctx, d->y_vec, sizeof(double) * d->ny);
    r.z = dev_upload(ctx, d->z, sizeof(double) * d->nx * d->ny);
    v.xv = r.xv->as<double>();
    v.yv = r.yv->as<double>();
    v.z = r.z->as<double>();
    v.asc_x = non_decreasing(d->x_vec, d->nx) ? 1 : 0;
    v.asc_y = non_decreasing(d->y_vec, d->ny) ? 1 : 0;
    v.uniform = (equally_spaced(d->x_vec, d->nx) && equally_spaced(d->y_vec, d->ny)) ? 1 : 0;
    v.x0 = d->x_vec[0];
    v.y0 = d->y_vec[0];
    v.stepx = d->nx > 1 ? (d->x_vec[d->nx - 1] - d->x_vec[0]) / (double)(d->nx - 1) : 1.0;
    v.stepy = d->ny > 1 ? (d->y_vec[d->ny - 1] - d->y_vec[0]) / (double)(d->ny - 1) : 1.0;
    if (want_z32) {
        // rows padded to a multiple of 4 floats: 16-byte tensor-map strides
        r.pitch = (int)((d->nx + 3) & ~int64_t(3));
        std::vector<float> zf((size_t)r.pitch * d->ny, 0.0f);
        float zmin = INFINITY;
        for (int64_t j = 0; j < d->ny; j++)
            for (int64_t i = 0; i < d->nx; i++) {
                zf[j * r.pitch + i] = (float)d->z[j * d->nx + i];
                zmin = std::min(zmin, zf[j * r.pitch + i]);
            }
        r.zmin32 = zmin;
        r.z32 = dev_upload(ctx, zf.data(), sizeof(float) * zf.size());
        sync(ctx);   // zf goes out of scope
        v.z32 = r.z32->as<float>();
        if (d->nx >= 2 && d->ny >= 2) r.has_tmap = make_dem_tmap(r);
    }
    return r;
}

// Node-scan half width for a radius in metres.
inline int search_nodes(const DemView& v, double radius)
{
    if (!(radius > 0)) radius = kDefaultSearchRadius;
    if (v.empty || v.nx < 2 || v.ny < 2) return 1;
    double step = std::min(std::fabs(v.stepx), std::fabs(v.stepy));
    int W = (int)std::ceil(radius / step - 1e-9);
    return std::max(1, std::min(W, 256));
}

inline void check_newton_dem(const DemView& v)
{
    if (!v.empty && v.nx >= 2 && v.ny >= 2 && !v.uniform)
        fail(BSAR_ERR_INVALID_ARG, "the Newton solver needs strictly ascending, equally spaced DEM axes");
}

// ------------------------------------------------------------------------------------
// FFT twiddles
// ------------------------------------------------------------------------------------
inline const void* twiddles(bsar_ctx* ctx, int64_t P, int real_bytes)
{
    auto key = std::make_pair(P, real_bytes);
    auto it = ctx->twiddles.find(key);
    if (it != ctx->twiddles.end()) return it->second->p;
    int64_t h = std::max<int64_t>(P / 2, 1);
    std::unique_ptr<DevBuf> b;
    if (real_bytes == 8) {
        std::vector<double> w(2 * h);
        for (int64_t k = 0; k < h; k++) {
            double a = -2.0 * kPi * (double)k / (double)P;
            w[2 * k] = std::cos(a);
            w[2 * k + 1] = std::sin(a);
        }
        b = dev_upload(ctx, w.data(), sizeof(double) * w.size());
        sync(ctx);
    } else {
        std::vector<float> w(2 * h);
        for (int64_t k = 0; k < h; k++) {
            double a = -2.0 * kPi * (double)k / (double)P;
            w[2 * k] = (float)std::cos(a);
            w[2 * k + 1] = (float)std::sin(a);
        }
        b = dev_upload(ctx, w.data(), sizeof(float) * w.size());
        sync(ctx);
    }
    const void* p = b->p;
    ctx->twiddles[key] = std::move(b);
    return p;
}

// The FP32 register transforms' second-pass twiddles in lane order (rf_twiddle_source):
// the same FP32 values as twiddles(ctx, P, 4), rearranged.
inline const void* rf_twiddles(bsar_ctx* ctx, int64_t P)
{
    const int logP = ilog2(P);
    auto key = std::make_pair(P, -4);
    auto it = ctx->twiddles.find(key);
    if (it != ctx->twiddles.end()) return it->second->p;
    const int64_t n = rf_twiddle_count(logP);
    std::vector<float> w(2 * n);
    for (int64_t e = 0; e < n; e++) {
        const int64_t k = rf_twiddle_source(logP, e);
        double a = -2.0 * kPi * (double)k / (double)P;
        w[2 * e] = (float)std::cos(a);
        w[2 * e + 1] = (float)std::sin(a);
    }
    auto b = dev_upload(ctx, w.data(), sizeof(float) * w.size());
    sync(ctx);
    const void* p = b->p;
    ctx->twiddles[key] = std::move(b);
    return p;
}

// longest FFT: one CTA up to 8192 (FP64) / 16384 (FP32) points, a cluster of up to 8 CTAs beyond
inline int64_t max_fft_len(int real_bytes) { return fft_max_len(real_bytes); }

// ------------------------------------------------------------------------------------
// Scenes
// ------------------------------------------------------------------------------------
struct RcBuf {
    std::unique_ptr<DevBuf> data;   // np x nr samples in the precision's storage type
    std::unique_ptr<DevBuf> scale;  // FP16 per-pulse scales
};

struct Scene {
    DemDev dem;
    int64_t np = 0, ns = 0, nr = 0;
    int upsample = 4;
    int kind = 0;
    double n1 = 1, n2 = 1, c = 3e8, fc = 1e9, fs = 1e9, f0 = 0, f1 = 0, T = 0;
    std::unique_ptr<DevBuf> tx, rx, samples;
    std::vector<double> reference;     // matched-filter reference (Ns complex), RAW scenes
    std::unique_ptr<DevBuf> reference_dev;   // the reference on the device (stage_reference)
    RcBuf rc[3];                       // per bsar_precision
    std::unique_ptr<DevBuf> spec[3];   // matched-filter spectrum per precision (bit-reversed)
    // mixed-form anchors (per grid centre and node-scan width)
    std::unique_ptr<DevBuf> anchors;
    double anchor_key[4] = {NAN, NAN, NAN, NAN};
    float off_x = 0.f, off_y = 0.f;    // mean crossing offset from the grid centre
};

inline Scene* get_scene(bsar_ctx* ctx, bsar_scene_id id)
{
    auto it = ctx->scenes.find(id);
    if (it == ctx->scenes.end()) fail(BSAR_ERR_NOT_FOUND, "unknown scene id %llu", (unsigned long long)id);
    return it->second.get();
}

inline bool all_finite(const double* p, int64_t n)
{
    for (int64_t i = 0; i < n; i++)
        if (!std::isfinite(p[i])) return false;
    return true;
}

// Largest imaging grid (voxels) a call takes.
constexpr int64_t kMaxGridVoxels = (int64_t)1 << 34;

// Checks an imaging grid and returns its voxel count.  Every axis must fit an int (the
// kernels index axes with 32-bit integers) and the product is bounded one factor at a
// time, so nx * ny * nz cannot wrap.
inline int64_t check_grid(const bsar_grid* g)
{
    if (!g) fail(BSAR_ERR_INVALID_ARG, "grid is NULL");
    if (g->nx < 1 || g->ny < 1 || g->nz < 1 || !g->x_axis || !g->y_axis || !g->z_axis)
        fail(BSAR_ERR_INVALID_ARG, "empty grid");
    constexpr int64_t kMaxAxis = 0x7fffffff;
    if (g->nx > kMaxAxis || g->ny > kMaxAxis || g->nz > kMaxAxis || g->nx > kMaxGridVoxels / g->ny ||
        g->nx * g->ny > kMaxGridVoxels / g->nz)
        fail(BSAR_ERR_INVALID_ARG, "grid too large (%lld x %lld x %lld voxels; at most 2^34)", (long long)g->nx,
             (long long)g->ny, (long long)g->nz);
    if (!all_finite(g->x_axis, g->nx) || !all_finite(g->y_axis, g->ny) || !all_finite(g->z_axis, g->nz))
        fail(BSAR_ERR_INVALID_ARG, "non-finite grid axis");
    return g->nx * g->ny * g->nz;
}

// createCHIRP (src/raw_data_processing.cpp:257-290) and the fftshifted reference
// (:371-394) of length n.
inline std::vector<double> matched_reference(double f0, double f1, double T, double fs, int64_t n)
{
    double k = (f1 - f0) / T;
    int nc = (int)(T * fs) + 1;
    if (nc > n) fail(BSAR_ERR_INVALID_ARG, "chirp of %d samples is longer than the %lld-sample pulse", nc, (long long)n);
    std::vector<double> chirp(2 * (size_t)nc);
    for (int i = 0; i < nc; i++) {
        double t = i / fs;
        double ph = 2.0 * kPi * (f0 * t + (k / 2.0) * t * t);
        chirp[2 * i] = std::cos(ph);
        chirp[2 * i + 1] = std::sin(ph);
    }
    std::vector<double> ref(2 * (size_t)n, 0.0);
    int half = nc / 2;
    for (int i = 0; i < nc - half; i++) {
        ref[2 * i] = chirp[2 * (half + i)];
        ref[2 * i + 1] = chirp[2 * (half + i) + 1];
    }
    int64_t start = n - half;
    for (int i = 0; i < half; i++) {
        ref[2 * (start + i)] = chirp[2 * i];
        ref[2 * (start + i) + 1] = chirp[2 * i + 1];
    }
    return ref;
}

// Copies the scene's matched-filter reference to the device now, so that a later
// compress_scene enqueues no upload from pageable memory (which would first drain the
// stream).
inline void stage_reference(bsar_ctx* ctx, Scene* s)
{
    if (!s->reference.empty() && !s->reference_dev)
        s->reference_dev = dev_upload(ctx, s->reference.data(), sizeof(double) * s->reference.size());
}

// Device buffers come from the stream-ordered pool: a temporary released at the end of an
// enqueuing function is freed in stream order, so the function need not wait for its
// kernels.
inline bool stream_ordered(const bsar_ctx* ctx) { return ctx->use_pool && ctx->pool; }

// Enqueues the compression; with wait = true (or without pooled buffers) it first waits
// for the reference spectrum it had to build.
inline void compress_scene(bsar_ctx* ctx, Scene* s, int precision, bool wait = true)
{
    RcBuf& rb = s->rc[precision];
    const int64_t nr = s->nr;
    const size_t elem = precision == BSAR_FP64 ? sizeof(double2) : (precision == BSAR_MIXED ? sizeof(float2) : sizeof(__half2));
    if (!rb.data) rb.data = dev_alloc(ctx, elem * (size_t)s->np * nr);
    if (precision == BSAR_MIXED_FP16 && !rb.scale) rb.scale = dev_alloc(ctx, sizeof(float) * s->np);
    PulseArgs a{};
    a.in = s->samples->as<double2>();
    a.batch = s->np;
    a.ns = (int)s->ns;
    a.P = (int)s->ns;
    a.logP = ilog2(s->ns);
    a.real_bytes = precision == BSAR_FP64 ? 8 : 4;
    a.n_keep = (int)s->ns;
    a.factor = s->upsample;
    a.out_kind = precision;
    a.out64 = precision == BSAR_FP64 ? rb.data->as<double2>() : nullptr;
    a.out32 = precision == BSAR_MIXED ? rb.data->as<float2>() : nullptr;
    a.out16 = precision == BSAR_MIXED_FP16 ? rb.data->as<__half2>() : nullptr;
    a.scale16 = rb.scale ? rb.scale->as<float>() : nullptr;
    if (s->kind == BSAR_SAMPLES_COMPRESSED) {
        // already range-compressed: upsampling only (splineInterpolation)
        if (precision == BSAR_FP64)
            launched(ctx, launch_spline(a.in, s->ns, s->np, s->upsample, a.out64, ctx->stream), "spline");
        else
            launched(ctx, launch_upsample_store(a.in, s->ns, s->np, s->upsample, precision, a.out32, a.out16, a.scale16,
                                                ctx->stream),
                     "upsample");
        return;
    }
    if (s->ns > max_fft_len(a.real_bytes))
        fail(BSAR_ERR_UNSUPPORTED, "pulse length %lld exceeds the longest FFT (%lld for this precision)",
             (long long)s->ns, (long long)max_fft_len(a.real_bytes));
    a.tw = twiddles(ctx, a.P, a.real_bytes);
    a.tw_rf = rf_length(a.real_bytes, a.logP) ? rf_twiddles(ctx, a.P) : nullptr;
    std::unique_ptr<DevBuf>& spec = s->spec[precision];
    if (!spec) {
        // the reference's spectrum once per scene and precision (the reference recomputes
        // it for every pulse, src/fft_utils.cpp:81-82)
        spec = dev_alloc(ctx, (size_t)a.P * (a.real_bytes == 8 ? sizeof(double2) : sizeof(float2)));
        std::unique_ptr<DevBuf> tmp;
        if (!s->reference_dev) tmp = dev_upload(ctx, s->reference.data(), sizeof(double) * s->reference.size());
        const DevBuf* dref = s->reference_dev ? s->reference_dev.get() : tmp.get();
        launched(ctx, launch_ref_spectrum(dref->as<double2>(), (int)s->ns, a.P, a.logP, a.tw, 1, spec->p,
                                          a.real_bytes, ctx->stream),
                 "reference spectrum");
        if (wait || !stream_ordered(ctx)) sync(ctx);
    }
    a.spec = spec->p;
    launched(ctx, launch_pulse_compress(a, ctx->stream), "pulse compression");
}


// Validates a scene description and creates the scene (samples copied when `copy`).
inline std::unique_ptr<Scene> make_scene(bsar_ctx* ctx, const bsar_scene_desc& s, bool copy)
{
    {
        if (s.n_pulses < 1 || !s.tx || !s.rx) fail(BSAR_ERR_INVALID_ARG, "no pulses / trajectories");
        if (s.n_samples < 2 || (copy && !s.samples)) fail(BSAR_ERR_INVALID_ARG, "no samples");
        if (s.samples_kind == BSAR_SAMPLES_RAW && !is_pow2(s.n_samples))
            fail(BSAR_ERR_INVALID_ARG, "raw pulses must have a power-of-two length");
        if (s.upsample < 1 || s.upsample > 64) fail(BSAR_ERR_INVALID_ARG, "upsample factor out of range");
        if (s.samples_kind != BSAR_SAMPLES_RAW && s.samples_kind != BSAR_SAMPLES_COMPRESSED)
            fail(BSAR_ERR_INVALID_ARG, "unknown samples kind");
        if (!all_finite(s.tx, 3 * s.n_pulses) || !all_finite(s.rx, 3 * s.n_pulses))
            fail(BSAR_ERR_INVALID_ARG, "non-finite trajectory");
        if (!(s.c > 0) || !(s.fc > 0) || !(s.fs > 0) || !std::isfinite(s.n1) || !std::isfinite(s.n2))
            fail(BSAR_ERR_INVALID_ARG, "bad physical constants");
        if (s.n_pulses > (1 << 24) || s.n_samples * s.upsample > ((int64_t)1 << 30))
            fail(BSAR_ERR_INVALID_ARG, "scene too large");
        check_dem(&s.dem);
        if (s.dem.nx > 0 && s.dem.ny > 0 && !all_finite(s.dem.z, s.dem.nx * s.dem.ny))
            fail(BSAR_ERR_INVALID_ARG, "non-finite DEM height");
        // admission: the raw scene plus one FP64 upsampled copy must fit the budget
        uint64_t need = sizeof(double2) * (uint64_t)s.n_pulses * s.n_samples * (1 + (uint64_t)s.upsample) +
                        sizeof(double) * 2 * (uint64_t)std::max<int64_t>(s.dem.nx, 1) * std::max<int64_t>(s.dem.ny, 1);
        if (ctx->used + need > ctx->budget)
            fail(BSAR_ERR_OOM_BUDGET, "scene needs %llu bytes; %llu of %llu in use", (unsigned long long)need,
                 (unsigned long long)ctx->used, (unsigned long long)ctx->budget);
        auto sc = std::make_unique<Scene>();
        sc->np = s.n_pulses;
        sc->ns = s.n_samples;
        sc->upsample = s.upsample;
        sc->nr = s.n_samples * s.upsample;
        sc->kind = s.samples_kind;
        sc->n1 = s.n1;
        sc->n2 = s.n2;
        sc->c = s.c;
        sc->fc = s.fc;
        sc->fs = s.fs;
        sc->f0 = s.chirp_f0;
        sc->f1 = s.chirp_f1;
        sc->T = s.chirp_T;
        if (s.samples_kind == BSAR_SAMPLES_RAW) {
            if (!(s.chirp_T > 0)) fail(BSAR_ERR_INVALID_ARG, "raw scenes need the chirp parameters");
            sc->reference = matched_reference(s.chirp_f0, s.chirp_f1, s.chirp_T, s.fs, s.n_samples);
        }
        sc->dem = stage_dem(ctx, &s.dem, true);
        sc->tx = dev_upload(ctx, s.tx, sizeof(double) * 3 * s.n_pulses);
        sc->rx = dev_upload(ctx, s.rx, sizeof(double) * 3 * s.n_pulses);
        if (copy)
            sc->samples = dev_upload(ctx, s.samples, sizeof(double2) * s.n_pulses * s.n_samples);
        else
            sc->samples = dev_alloc(ctx, sizeof(double2) * s.n_pulses * s.n_samples);
        sync(ctx);
        return sc;
    }
}


// Echo synthesis into a scene's raw pulses (bsar_scene_synthesize), on ctx->stream.
// wait = false (pooled buffers only): return once the work is enqueued; the scatterer
// arrays are read before the call returns either way.
inline void synthesize_samples(bsar_ctx* ctx, Scene* sc, const double* scat_pos, const double* scat_amp, int64_t n_scat,
                               double snr_db, uint64_t seed, int flags = 0, bool wait = true)
{
    check_newton_dem(sc->dem.view);
    const int W = search_nodes(sc->dem.view, 0.0);
    const int64_t np = sc->np, ns = std::max<int64_t>(n_scat, 1);
    auto pos = dev_alloc(ctx, sizeof(double) * 3 * ns);
    auto amp = dev_alloc(ctx, sizeof(double) * ns);
    if (n_scat > 0) {
        cuda_check(cudaMemcpyAsync(pos->p, scat_pos, sizeof(double) * 3 * n_scat, cudaMemcpyHostToDevice, ctx->stream),
                   "h2d");
        cuda_check(cudaMemcpyAsync(amp->p, scat_amp, sizeof(double) * n_scat, cudaMemcpyHostToDevice, ctx->stream), "h2d");
    }
    auto tau = dev_alloc(ctx, sizeof(double) * np * ns);
    auto car = dev_alloc(ctx, sizeof(double2) * np * ns);
    const int nc = (int)(sc->T * sc->fs) + 1;
    const double sigma = std::isfinite(snr_db) ? std::sqrt(nc / std::pow(10.0, snr_db / 10.0)) : 0.0;
    launched(ctx, launch_echo_synth(sc->dem.view, sc->tx->as<double>(), sc->rx->as<double>(), (int)np,
                                    pos->as<double>(), amp->as<double>(), (int)n_scat, sc->n1, sc->n2, W, sc->c, sc->fc,
                                    sc->fs, sc->f0, sc->f1, sc->T, (int)sc->ns, sigma, seed,
                                    (flags & BSAR_SYNTH_REFERENCE_BINS) ? 1 : 0, tau->as<double>(),
                                    car->as<double2>(), sc->samples->as<double2>(), ctx->stream),
             "echo synthesis");
    if (wait || !stream_ordered(ctx)) sync(ctx);   // the work buffers are released on return
}

// Per-pulse anchors of the mixed form at the grid centre (FP64 reference path, reduced
// phase, integer bin + fraction) and the mean crossing offset used to place DEM tiles;
// cached per scene, grid centre and node-scan width.  Fills a.ref_*.
inline void set_anchors(bsar_ctx* ctx, Scene* s, const bsar_grid* g, BpArgs& a)
{
    double centre[3] = {0.5 * (g->x_axis[0] + g->x_axis[g->nx - 1]), 0.5 * (g->y_axis[0] + g->y_axis[g->ny - 1]),
                        0.5 * (g->z_axis[0] + g->z_axis[g->nz - 1])};
    double key[4] = {centre[0], centre[1], centre[2], (double)a.W};
    int64_t np = s->np;
    if (!s->anchors || std::memcmp(key, s->anchor_key, sizeof key) != 0) {
        s->anchors = dev_alloc(ctx, (sizeof(double) + sizeof(float) + sizeof(int) + sizeof(float)) * np);
        auto offs = dev_alloc(ctx, sizeof(double) * 4 * np);
        char* base = s->anchors->as<char>();
        launched(ctx, launch_ref_ranges(s->dem.view, a.tx, a.rx, (int)np, centre, s->n1, s->n2, a.W, a.lambda,
                                        a.fs_eff / s->c, (double*)base, (float*)(base + 8 * np),
                                        (int*)(base + 12 * np), (float*)(base + 16 * np), offs->as<double>(),
                                        ctx->stream),
                 "reference ranges");
        std::vector<double> h(4 * np);
        cuda_check(cudaMemcpyAsync(h.data(), offs->p, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, ctx->stream),
                   "d2h");
        sync(ctx);
        double ox = 0, oy = 0;
        for (int64_t i = 0; i < np; i++) {
            ox += h[4 * i] + h[4 * i + 2];
            oy += h[4 * i + 1] + h[4 * i + 3];
        }
        s->off_x = (float)(ox / (2.0 * np));
        s->off_y = (float)(oy / (2.0 * np));
        std::memcpy(s->anchor_key, key, sizeof key);
    }
    char* base = s->anchors->as<char>();
    a.ref_L = (const double*)base;
    a.ref_phase = (const float*)(base + 8 * np);
    a.ref_bin_i = (const int*)(base + 12 * np);
    a.ref_bin_f = (const float*)(base + 16 * np);
}

// Device buffers of the one-request mixed launch: request record, work counter, status.
inline void ensure_mixed_buffers(bsar_ctx* ctx)
{
    if (!ctx->status) {
        // the status word is shared with the server's batch streams: a plain allocation,
        // cleared before any stream can use it
        const bool pooled = ctx->use_pool;
        ctx->use_pool = false;
        try {
            ctx->status = dev_alloc(ctx, sizeof(int));
        } catch (...) {
            ctx->use_pool = pooled;
            throw;
        }
        ctx->use_pool = pooled;
        cuda_check(cudaMemsetAsync(ctx->status->p, 0, sizeof(int), ctx->stream), "memset");
        sync(ctx);
    }
    if (!ctx->mixed_req) ctx->mixed_req = dev_alloc(ctx, sizeof(MixedReq));
    if (!ctx->mixed_counter) ctx->mixed_counter = dev_alloc(ctx, sizeof(int));
}

// The device record of one mixed-form request.
inline MixedReq mixed_request(const Scene* s, const BpArgs& a, bool fp16, int32_t flags)
{
    MixedReq r;
    std::memset(&r, 0, sizeof r);
    if (s->dem.has_tmap) std::memcpy(r.tmap, s->dem.tmap, sizeof(r.tmap));
    r.a = a;
    r.z32 = s->dem.view.z32;
    r.pitch = s->dem.pitch;
    r.use_tile = s->dem.has_tmap ? 1 : 0;
    r.fp16 = fp16 ? 1 : 0;
    r.exhaustive = (flags & BSAR_BP_EXHAUSTIVE_SCAN) ? 1 : 0;
    r.stepx = (float)s->dem.view.stepx;
    r.stepy = (float)s->dem.view.stepy;
    r.istepx = (float)(1.0 / s->dem.view.stepx);
    r.istepy = (float)(1.0 / s->dem.view.stepy);
    r.ox = s->dem.view.x0;
    r.oy = s->dem.view.y0;
    r.idx64 = 1.0 / s->dem.view.stepx;
    r.idy64 = 1.0 / s->dem.view.stepy;
    r.off_x = s->off_x;
    r.off_y = s->off_y;
    r.start_band = mixed_start_band(s->dem.view);
    r.zmin = s->dem.zmin32;
    return r;
}

