// bsar_api.cpp -- host runtime behind the C ABI of include/bsar.h.
//
// A context owns a CUDA stream, a device-memory budget and the resident scenes.  Each
// entry point validates its arguments, stages host data into device buffers charged to
// the budget, launches the kernels of k_plain.cu / k_mixed.cu / k_pulse.cu and copies the
// results back.  There is no host-side compute path: every result comes from a kernel.
#include "bsar.h"

#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "kernels.hpp"

using namespace bsar;

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kDefaultSearchRadius = 1.5;   // m, Newton node-scan radius

struct Error {
    bsar_status status;
    std::string msg;
};

[[noreturn]] void fail(bsar_status s, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    throw Error{s, buf};
}

void cuda_check(cudaError_t e, const char* what)
{
    if (e != cudaSuccess) fail(BSAR_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

bool is_pow2(int64_t n) { return n > 0 && (n & (n - 1)) == 0; }
int64_t next_pow2(int64_t n)
{
    int64_t p = 1;
    while (p < n) p *= 2;
    return p;
}
int ilog2(int64_t n)
{
    int l = 0;
    while ((int64_t(1) << l) < n) l++;
    return l;
}

}  // namespace

// ------------------------------------------------------------------------------------
// Context and device buffers
// ------------------------------------------------------------------------------------
struct DevBuf;

struct bsar_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    uint64_t budget = 0;
    uint64_t used = 0;
    uint64_t launches = 0;
    std::mutex mu;
    std::string last_error;
    uint64_t next_scene = 1;
    std::map<uint64_t, std::unique_ptr<struct Scene>> scenes;
    std::map<std::pair<int64_t, int>, std::unique_ptr<DevBuf>> twiddles;   // (P, real bytes)
    // cached grid axes for the asynchronous entry point
    std::vector<double> grid_host;
    std::unique_ptr<DevBuf> grid_dev;
    // device status word raised by bounded device-side waits
    std::unique_ptr<DevBuf> status;
};

struct DevBuf {
    bsar_ctx* ctx = nullptr;
    void* p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(bsar_ctx* c, size_t n) : ctx(c), bytes(n)
    {
        if (n == 0) return;
        if (ctx->used + n > ctx->budget)
            fail(BSAR_ERR_OOM_BUDGET, "request of %zu bytes exceeds the HBM budget (%llu of %llu bytes in use)", n,
                 (unsigned long long)ctx->used, (unsigned long long)ctx->budget);
        cudaError_t e = cudaMalloc(&p, n);
        if (e != cudaSuccess) {
            p = nullptr;
            cudaGetLastError();
            fail(e == cudaErrorMemoryAllocation ? BSAR_ERR_OOM_BUDGET : BSAR_ERR_CUDA, "cudaMalloc(%zu): %s", n,
                 cudaGetErrorString(e));
        }
        ctx->used += n;
    }
    ~DevBuf()
    {
        if (p) {
            cudaFree(p);
            ctx->used -= bytes;
        }
    }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    template <typename T> T* as() const { return static_cast<T*>(p); }
};

static std::unique_ptr<DevBuf> dev_alloc(bsar_ctx* ctx, size_t n) { return std::make_unique<DevBuf>(ctx, n); }

static std::unique_ptr<DevBuf> dev_upload(bsar_ctx* ctx, const void* host, size_t n)
{
    auto b = dev_alloc(ctx, n);
    if (n) cuda_check(cudaMemcpyAsync(b->p, host, n, cudaMemcpyHostToDevice, ctx->stream), "upload");
    return b;
}

static void launched(bsar_ctx* ctx, cudaError_t e, const char* what)
{
    cuda_check(e, what);
    ctx->launches++;
}

static void sync(bsar_ctx* ctx) { cuda_check(cudaStreamSynchronize(ctx->stream), "stream synchronize"); }

// A bounded device-side wait that ran out raises the context's status word.
static void check_device_status(bsar_ctx* ctx)
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
    alignas(64) unsigned char tmap[sizeof(CUtensorMap)] = {};
    bool has_tmap = false;
};

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link to libcuda).
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
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
static bool make_dem_tmap(DemDev& r)
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

static void check_dem(const bsar_dem* d)
{
    if (!d) fail(BSAR_ERR_INVALID_ARG, "dem is NULL");
    if (d->nx < 0 || d->ny < 0) fail(BSAR_ERR_INVALID_ARG, "negative DEM size");
    if (d->nx > (1 << 20) || d->ny > (1 << 20)) fail(BSAR_ERR_INVALID_ARG, "DEM axis longer than 2^20 nodes");
    if (d->nx > 0 && d->ny > 0 && (!d->x_vec || !d->y_vec || !d->z))
        fail(BSAR_ERR_INVALID_ARG, "DEM arrays are NULL");
}

static bool non_decreasing(const double* v, int64_t n)
{
    for (int64_t i = 0; i + 1 < n; i++)
        if (!(v[i] <= v[i + 1])) return false;
    return true;
}

static bool strictly_ascending(const double* v, int64_t n)
{
    for (int64_t i = 0; i + 1 < n; i++)
        if (!(v[i] < v[i + 1])) return false;
    return true;
}

static DemDev stage_dem(bsar_ctx* ctx, const bsar_dem* d, bool want_z32)
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
    v.uniform = (strictly_ascending(d->x_vec, d->nx) && strictly_ascending(d->y_vec, d->ny)) ? 1 : 0;
    v.x0 = d->x_vec[0];
    v.y0 = d->y_vec[0];
    v.stepx = d->nx > 1 ? (d->x_vec[d->nx - 1] - d->x_vec[0]) / (double)(d->nx - 1) : 1.0;
    v.stepy = d->ny > 1 ? (d->y_vec[d->ny - 1] - d->y_vec[0]) / (double)(d->ny - 1) : 1.0;
    if (want_z32) {
        // rows padded to a multiple of 4 floats: 16-byte tensor-map strides
        r.pitch = (int)((d->nx + 3) & ~int64_t(3));
        std::vector<float> zf((size_t)r.pitch * d->ny, 0.0f);
        for (int64_t j = 0; j < d->ny; j++)
            for (int64_t i = 0; i < d->nx; i++) zf[j * r.pitch + i] = (float)d->z[j * d->nx + i];
        r.z32 = dev_upload(ctx, zf.data(), sizeof(float) * zf.size());
        sync(ctx);   // zf goes out of scope
        v.z32 = r.z32->as<float>();
        if (d->nx >= 2 && d->ny >= 2) r.has_tmap = make_dem_tmap(r);
    }
    return r;
}

// Node-scan half width for a radius in metres.
static int search_nodes(const DemView& v, double radius)
{
    if (!(radius > 0)) radius = kDefaultSearchRadius;
    if (v.empty || v.nx < 2 || v.ny < 2) return 1;
    double step = std::min(std::fabs(v.stepx), std::fabs(v.stepy));
    int W = (int)std::ceil(radius / step - 1e-9);
    return std::max(1, std::min(W, 256));
}

static void check_newton_dem(const DemView& v)
{
    if (!v.empty && v.nx >= 2 && v.ny >= 2 && !v.uniform)
        fail(BSAR_ERR_INVALID_ARG, "the Newton solver needs strictly ascending DEM axes");
}

// ------------------------------------------------------------------------------------
// FFT twiddles
// ------------------------------------------------------------------------------------
static const void* twiddles(bsar_ctx* ctx, int64_t P, int real_bytes)
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

// largest FFT one CTA holds in shared memory (227 KB usable)
static int64_t max_fft_len(int real_bytes) { return real_bytes == 8 ? 8192 : 16384; }

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
    RcBuf rc[3];                       // per bsar_precision
    std::unique_ptr<DevBuf> spec[3];   // matched-filter spectrum per precision (bit-reversed)
    // mixed-form anchors (per grid centre and node-scan width)
    std::unique_ptr<DevBuf> anchors;
    double anchor_key[4] = {NAN, NAN, NAN, NAN};
    float off_x = 0.f, off_y = 0.f;    // mean crossing offset from the grid centre
};

static Scene* get_scene(bsar_ctx* ctx, bsar_scene_id id)
{
    auto it = ctx->scenes.find(id);
    if (it == ctx->scenes.end()) fail(BSAR_ERR_NOT_FOUND, "unknown scene id %llu", (unsigned long long)id);
    return it->second.get();
}

static bool all_finite(const double* p, int64_t n)
{
    for (int64_t i = 0; i < n; i++)
        if (!std::isfinite(p[i])) return false;
    return true;
}

// createCHIRP (src/raw_data_processing.cpp:257-290) and the fftshifted reference
// (:371-394) of length n.
static std::vector<double> matched_reference(double f0, double f1, double T, double fs, int64_t n)
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

static void compress_scene(bsar_ctx* ctx, Scene* s, int precision)
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
        fail(BSAR_ERR_UNSUPPORTED, "pulse length %lld exceeds the single-CTA FFT (%lld for this precision)",
             (long long)s->ns, (long long)max_fft_len(a.real_bytes));
    a.tw = twiddles(ctx, a.P, a.real_bytes);
    std::unique_ptr<DevBuf>& spec = s->spec[precision];
    if (!spec) {
        // the reference's spectrum once per scene and precision (the reference recomputes
        // it for every pulse, src/fft_utils.cpp:81-82)
        spec = dev_alloc(ctx, (size_t)a.P * (a.real_bytes == 8 ? sizeof(double2) : sizeof(float2)));
        const std::vector<double>& ref = s->reference;
        auto dref = dev_upload(ctx, ref.data(), sizeof(double) * ref.size());
        launched(ctx, launch_ref_spectrum(dref->as<double2>(), (int)s->ns, a.P, a.logP, a.tw, 1, spec->p,
                                          a.real_bytes, ctx->stream),
                 "reference spectrum");
        sync(ctx);
    }
    a.spec = spec->p;
    launched(ctx, launch_pulse_compress(a, ctx->stream), "pulse compression");
}

// ------------------------------------------------------------------------------------
// API glue
// ------------------------------------------------------------------------------------
template <typename F> static bsar_status guarded(bsar_ctx* ctx, F&& f)
{
    if (!ctx) return BSAR_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(ctx->mu);
    try {
        cuda_check(cudaSetDevice(ctx->device), "cudaSetDevice");
        f();
        ctx->last_error.clear();
        return BSAR_OK;
    } catch (const Error& e) {
        ctx->last_error = e.msg;
        return e.status;
    } catch (const std::bad_alloc&) {
        ctx->last_error = "host allocation failed";
        return BSAR_ERR_OOM_BUDGET;
    }
}

extern "C" {

const char* bsar_status_string(bsar_status s)
{
    switch (s) {
    case BSAR_OK: return "ok";
    case BSAR_ERR_INVALID_ARG: return "invalid argument";
    case BSAR_ERR_OOM_BUDGET: return "HBM budget exceeded";
    case BSAR_ERR_TIMEOUT: return "device wait timed out";
    case BSAR_ERR_CUDA: return "CUDA error";
    case BSAR_ERR_NOT_FOUND: return "not found";
    case BSAR_ERR_UNSUPPORTED: return "unsupported";
    case BSAR_ERR_QUEUE_FULL: return "queue full";
    }
    return "unknown status";
}

bsar_status bsar_create(bsar_ctx** out, const bsar_opts* opts)
{
    if (!out) return BSAR_ERR_INVALID_ARG;
    *out = nullptr;
    int dev = opts ? opts->device : 0;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return BSAR_ERR_CUDA;
    }
    if (dev < 0 || dev >= count) return BSAR_ERR_INVALID_ARG;
    if (opts && opts->flags != 0) return BSAR_ERR_INVALID_ARG;
    if (cudaSetDevice(dev) != cudaSuccess) return BSAR_ERR_CUDA;
    auto* ctx = new bsar_ctx();
    ctx->device = dev;
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete ctx;
        return BSAR_ERR_CUDA;
    }
    ctx->own_stream = true;
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    ctx->budget = (opts && opts->hbm_budget_bytes) ? opts->hbm_budget_bytes : (uint64_t)(0.9 * (double)fr);
    *out = ctx;
    return BSAR_OK;
}

void bsar_destroy(bsar_ctx* ctx)
{
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    ctx->scenes.clear();
    ctx->twiddles.clear();
    ctx->grid_dev.reset();
    if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char* bsar_last_error(const bsar_ctx* ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

bsar_status bsar_set_stream(bsar_ctx* ctx, void* stream)
{
    return guarded(ctx, [&] {
        sync(ctx);
        if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
        if (stream) {
            ctx->stream = (cudaStream_t)stream;
            ctx->own_stream = false;
        } else {
            cuda_check(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking), "stream create");
            ctx->own_stream = true;
        }
    });
}

bsar_status bsar_synchronize(bsar_ctx* ctx)
{
    return guarded(ctx, [&] {
        sync(ctx);
        check_device_status(ctx);
    });
}

uint64_t bsar_launch_count(const bsar_ctx* ctx) { return ctx ? ctx->launches : 0; }
uint64_t bsar_bytes_in_use(const bsar_ctx* ctx) { return ctx ? ctx->used : 0; }

bsar_status bsar_dem_elevation(bsar_ctx* ctx, const bsar_dem* dem, const double* xy, int64_t n, double* z_out)
{
    return guarded(ctx, [&] {
        if (n < 0 || (n > 0 && (!xy || !z_out))) fail(BSAR_ERR_INVALID_ARG, "bad point buffers");
        if (n == 0) return;
        DemDev d = stage_dem(ctx, dem, false);
        auto dxy = dev_upload(ctx, xy, sizeof(double) * 2 * n);
        auto dz = dev_alloc(ctx, sizeof(double) * n);
        launched(ctx, launch_dem_elevation(d.view, dxy->as<double>(), n, dz->as<double>(), ctx->stream), "elevation");
        cuda_check(cudaMemcpyAsync(z_out, dz->p, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream), "download");
        sync(ctx);
    });
}

static int fermat_solver(const bsar_fermat_opts* f) { return f ? f->solver : BSAR_SOLVER_GRID; }

bsar_status bsar_refraction_points(bsar_ctx* ctx, const bsar_dem* dem, const double* p1, const double* p2, int64_t n,
                                   double n1, double n2, const bsar_fermat_opts* fopts, double* out)
{
    return guarded(ctx, [&] {
        if (n < 0 || (n > 0 && (!p1 || !p2 || !out))) fail(BSAR_ERR_INVALID_ARG, "bad point buffers");
        int solver = fermat_solver(fopts);
        if (solver != BSAR_SOLVER_GRID && solver != BSAR_SOLVER_NEWTON) fail(BSAR_ERR_INVALID_ARG, "unknown solver");
        const int prec = fopts ? fopts->precision : BSAR_FP64;
        if (prec != BSAR_FP64 && prec != BSAR_MIXED) fail(BSAR_ERR_INVALID_ARG, "unknown precision");
        if (prec == BSAR_MIXED && solver != BSAR_SOLVER_NEWTON)
            fail(BSAR_ERR_UNSUPPORTED, "the mixed solver is the Newton solver");
        if (n == 0) return;
        DemDev d = stage_dem(ctx, dem, prec == BSAR_MIXED);
        if (solver == BSAR_SOLVER_NEWTON) check_newton_dem(d.view);
        if (prec == BSAR_MIXED && (d.view.empty || d.view.nx < 2 || d.view.ny < 2))
            fail(BSAR_ERR_UNSUPPORTED, "the mixed solver needs a DEM of at least 2 x 2 nodes");
        int W = search_nodes(d.view, fopts ? fopts->search_radius_m : 0.0);
        auto a = dev_upload(ctx, p1, sizeof(double) * 3 * n);
        auto b = dev_upload(ctx, p2, sizeof(double) * 3 * n);
        auto o = dev_alloc(ctx, sizeof(double) * 3 * n);
        if (prec == BSAR_MIXED)
            launched(ctx, launch_refraction_mixed(d.view, d.pitch, a->as<double>(), b->as<double>(), n, n1, n2, W,
                                                  o->as<double>(), ctx->stream),
                     "refraction points (mixed)");
        else
            launched(ctx, launch_refraction_points(d.view, a->as<double>(), b->as<double>(), n, n1, n2, solver, W,
                                                   o->as<double>(), ctx->stream),
                     "refraction points");
        cuda_check(cudaMemcpyAsync(out, o->p, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, ctx->stream), "download");
        sync(ctx);
    });
}

bsar_status bsar_slant_range_fermat(bsar_ctx* ctx, const bsar_dem* dem, const double* tx, const double* rx,
                                    int64_t np, const double* target, double n1, double n2,
                                    const bsar_fermat_opts* fopts, double* ranges, double* ida, double* volta,
                                    double* refl)
{
    return guarded(ctx, [&] {
        if (np < 0 || (np > 0 && (!tx || !rx || !target || !ranges || !ida || !volta)))
            fail(BSAR_ERR_INVALID_ARG, "bad buffers");
        int solver = fermat_solver(fopts);
        if (solver != BSAR_SOLVER_GRID && solver != BSAR_SOLVER_NEWTON) fail(BSAR_ERR_INVALID_ARG, "unknown solver");
        if (fopts && fopts->precision != BSAR_FP64)
            fail(BSAR_ERR_UNSUPPORTED, "ranges are returned by the FP64 solvers");
        if (np == 0) return;
        DemDev d = stage_dem(ctx, dem, false);
        if (solver == BSAR_SOLVER_NEWTON) check_newton_dem(d.view);
        int W = search_nodes(d.view, fopts ? fopts->search_radius_m : 0.0);
        auto dtx = dev_upload(ctx, tx, sizeof(double) * 3 * np);
        auto drx = dev_upload(ctx, rx, sizeof(double) * 3 * np);
        auto dr = dev_alloc(ctx, sizeof(double) * 4 * np);
        auto di = dev_alloc(ctx, sizeof(double) * 3 * np);
        auto dv = dev_alloc(ctx, sizeof(double) * 3 * np);
        std::unique_ptr<DevBuf> dl;
        if (refl) dl = dev_alloc(ctx, sizeof(double) * 3 * np);
        launched(ctx, launch_slant_range(d.view, dtx->as<double>(), drx->as<double>(), np, target, n1, n2, solver, W,
                                         dr->as<double>(), di->as<double>(), dv->as<double>(),
                                         dl ? dl->as<double>() : nullptr, ctx->stream),
                 "slant range");
        cuda_check(cudaMemcpyAsync(ranges, dr->p, sizeof(double) * 4 * np, cudaMemcpyDeviceToHost, ctx->stream), "d2h");
        cuda_check(cudaMemcpyAsync(ida, di->p, sizeof(double) * 3 * np, cudaMemcpyDeviceToHost, ctx->stream), "d2h");
        cuda_check(cudaMemcpyAsync(volta, dv->p, sizeof(double) * 3 * np, cudaMemcpyDeviceToHost, ctx->stream), "d2h");
        if (refl)
            cuda_check(cudaMemcpyAsync(refl, dl->p, sizeof(double) * 3 * np, cudaMemcpyDeviceToHost, ctx->stream), "d2h");
        sync(ctx);
    });
}

bsar_status bsar_spline_upsample(bsar_ctx* ctx, const double* in, int64_t n, int64_t batch, int32_t factor, double* out)
{
    return guarded(ctx, [&] {
        if (n < 0 || batch < 0 || factor < 1) fail(BSAR_ERR_INVALID_ARG, "bad sizes");
        if (n == 0 || batch == 0) return;
        // the reference indexes p[n-2] for every output (src/interpolation.cpp:22-25)
        if (n < 2) fail(BSAR_ERR_INVALID_ARG, "splineInterpolation needs at least 2 samples");
        if (!in || !out) fail(BSAR_ERR_INVALID_ARG, "NULL buffer");
        auto di = dev_upload(ctx, in, sizeof(double2) * n * batch);
        auto dout = dev_alloc(ctx, sizeof(double2) * n * factor * batch);
        launched(ctx, launch_spline(di->as<double2>(), n, batch, factor, dout->as<double2>(), ctx->stream), "spline");
        cuda_check(cudaMemcpyAsync(out, dout->p, sizeof(double2) * n * factor * batch, cudaMemcpyDeviceToHost,
                                   ctx->stream),
                   "download");
        sync(ctx);
    });
}

bsar_status bsar_fft(bsar_ctx* ctx, double* data, int64_t n, int64_t batch, int32_t inverse)
{
    return guarded(ctx, [&] {
        if (n < 0 || batch < 0) fail(BSAR_ERR_INVALID_ARG, "bad sizes");
        if (n <= 1 || batch == 0) return;   // src/fft_utils.cpp:14
        if (!data) fail(BSAR_ERR_INVALID_ARG, "NULL buffer");
        if (!is_pow2(n)) {
            // src/fft_utils.cpp:17-20: warning, data unchanged
            throw Error{BSAR_OK, "FFT input size is not a power of 2; data left unchanged"};
        }
        if (n > max_fft_len(8)) fail(BSAR_ERR_UNSUPPORTED, "FP64 FFT longer than %lld", (long long)max_fft_len(8));
        const void* tw = twiddles(ctx, n, 8);
        auto d = dev_upload(ctx, data, sizeof(double2) * n * batch);
        launched(ctx, launch_fft_rows(d->as<double2>(), batch, (int)n, ilog2(n), (const double2*)tw, inverse, ctx->stream),
                 "fft");
        cuda_check(cudaMemcpyAsync(data, d->p, sizeof(double2) * n * batch, cudaMemcpyDeviceToHost, ctx->stream), "d2h");
        sync(ctx);
    });
}

bsar_status bsar_fft_correlate(bsar_ctx* ctx, const double* signal, int64_t ns, int64_t batch, const double* reference,
                               int64_t nref, int32_t conjugate, double* out)
{
    return guarded(ctx, [&] {
        if (ns < 0 || nref < 0 || batch < 0) fail(BSAR_ERR_INVALID_ARG, "bad sizes");
        int64_t N = std::max(ns, nref);
        if (N == 0 || batch == 0) return;
        if ((ns > 0 && !signal) || (nref > 0 && !reference) || !out) fail(BSAR_ERR_INVALID_ARG, "NULL buffer");
        int64_t P = next_pow2(N);
        if (P > max_fft_len(8)) fail(BSAR_ERR_UNSUPPORTED, "FP64 FFT longer than %lld", (long long)max_fft_len(8));
        const void* tw = twiddles(ctx, P, 8);
        auto ds = dev_alloc(ctx, sizeof(double2) * std::max<int64_t>(ns, 1) * batch);
        if (ns > 0)
            cuda_check(cudaMemcpyAsync(ds->p, signal, sizeof(double2) * ns * batch, cudaMemcpyHostToDevice, ctx->stream),
                       "upload");
        auto dr = dev_alloc(ctx, sizeof(double2) * std::max<int64_t>(nref, 1));
        if (nref > 0)
            cuda_check(cudaMemcpyAsync(dr->p, reference, sizeof(double2) * nref, cudaMemcpyHostToDevice, ctx->stream),
                       "upload");
        auto spec = dev_alloc(ctx, sizeof(double2) * P);
        auto dout = dev_alloc(ctx, sizeof(double2) * N * batch);
        launched(ctx, launch_ref_spectrum(dr->as<double2>(), (int)nref, (int)P, ilog2(P), tw, conjugate ? 1 : 0, spec->p,
                                          8, ctx->stream),
                 "reference spectrum");
        PulseArgs a{};
        a.in = ds->as<double2>();
        a.batch = batch;
        a.ns = (int)ns;
        a.P = (int)P;
        a.logP = ilog2(P);
        a.tw = tw;
        a.spec = spec->p;
        a.real_bytes = 8;
        a.n_keep = (int)N;
        a.factor = 0;
        a.out64 = dout->as<double2>();
        launched(ctx, launch_pulse_compress(a, ctx->stream), "correlate");
        cuda_check(cudaMemcpyAsync(out, dout->p, sizeof(double2) * N * batch, cudaMemcpyDeviceToHost, ctx->stream), "d2h");
        sync(ctx);
    });
}

bsar_status bsar_scene_upload(bsar_ctx* ctx, const bsar_scene_desc* desc, bsar_scene_id* out)
{
    return guarded(ctx, [&] {
        if (!desc || !out) fail(BSAR_ERR_INVALID_ARG, "NULL argument");
        const bsar_scene_desc& s = *desc;
        if (s.n_pulses < 1 || !s.tx || !s.rx) fail(BSAR_ERR_INVALID_ARG, "no pulses / trajectories");
        if (s.n_samples < 2 || !s.samples) fail(BSAR_ERR_INVALID_ARG, "no samples");
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
        sc->samples = dev_upload(ctx, s.samples, sizeof(double2) * s.n_pulses * s.n_samples);
        sync(ctx);
        uint64_t id = ctx->next_scene++;
        ctx->scenes[id] = std::move(sc);
        *out = id;
    });
}

bsar_status bsar_scene_release(bsar_ctx* ctx, bsar_scene_id id)
{
    return guarded(ctx, [&] {
        get_scene(ctx, id);
        sync(ctx);
        ctx->scenes.erase(id);
    });
}

bsar_status bsar_scene_compress(bsar_ctx* ctx, bsar_scene_id id, int32_t precision)
{
    return guarded(ctx, [&] {
        if (precision < BSAR_FP64 || precision > BSAR_MIXED_FP16) fail(BSAR_ERR_INVALID_ARG, "unknown precision");
        compress_scene(ctx, get_scene(ctx, id), precision);
    });
}

bsar_status bsar_scene_read_upsampled(bsar_ctx* ctx, bsar_scene_id id, double* out)
{
    return guarded(ctx, [&] {
        Scene* s = get_scene(ctx, id);
        if (!out) fail(BSAR_ERR_INVALID_ARG, "NULL buffer");
        if (!s->rc[BSAR_FP64].data) compress_scene(ctx, s, BSAR_FP64);
        cuda_check(cudaMemcpyAsync(out, s->rc[BSAR_FP64].data->p, sizeof(double2) * s->np * s->nr,
                                   cudaMemcpyDeviceToHost, ctx->stream),
                   "download");
        sync(ctx);
    });
}

static void check_grid(const bsar_grid* g)
{
    if (!g) fail(BSAR_ERR_INVALID_ARG, "grid is NULL");
    if (g->nx < 1 || g->ny < 1 || g->nz < 1 || !g->x_axis || !g->y_axis || !g->z_axis)
        fail(BSAR_ERR_INVALID_ARG, "empty grid");
    if (g->nx * g->ny * g->nz > ((int64_t)1 << 34)) fail(BSAR_ERR_INVALID_ARG, "grid too large");
    if (!all_finite(g->x_axis, g->nx) || !all_finite(g->y_axis, g->ny) || !all_finite(g->z_axis, g->nz))
        fail(BSAR_ERR_INVALID_ARG, "non-finite grid axis");
}

// Stage the grid axes; reuse the device copy when the axes did not change.
static const double* stage_grid(bsar_ctx* ctx, const bsar_grid* g)
{
    std::vector<double> h;
    h.reserve(g->nx + g->ny + g->nz);
    h.insert(h.end(), g->x_axis, g->x_axis + g->nx);
    h.insert(h.end(), g->y_axis, g->y_axis + g->ny);
    h.insert(h.end(), g->z_axis, g->z_axis + g->nz);
    if (!(ctx->grid_dev && h == ctx->grid_host)) {
        sync(ctx);
        ctx->grid_dev = dev_upload(ctx, h.data(), sizeof(double) * h.size());
        sync(ctx);
        ctx->grid_host.swap(h);
    }
    return ctx->grid_dev->as<double>();
}

static void backproject(bsar_ctx* ctx, bsar_scene_id id, const bsar_grid* g, const bsar_bp_opts* o, double2* d_out)
{
    Scene* s = get_scene(ctx, id);
    check_grid(g);
    if (!o) fail(BSAR_ERR_INVALID_ARG, "options are NULL");
    if (o->solver != BSAR_SOLVER_GRID && o->solver != BSAR_SOLVER_NEWTON) fail(BSAR_ERR_INVALID_ARG, "unknown solver");
    if (o->legs != BSAR_LEGS_MEAN && o->legs != BSAR_LEGS_PER_PULSE) fail(BSAR_ERR_INVALID_ARG, "unknown legs mode");
    if (o->precision < BSAR_FP64 || o->precision > BSAR_MIXED_FP16) fail(BSAR_ERR_INVALID_ARG, "unknown precision");
    if (o->precision != BSAR_FP64 && o->solver != BSAR_SOLVER_NEWTON)
        fail(BSAR_ERR_UNSUPPORTED, "the mixed forms use the Newton solver");
    if (o->precision != BSAR_FP64 && o->legs != BSAR_LEGS_PER_PULSE)
        fail(BSAR_ERR_UNSUPPORTED, "the mixed forms use per-pulse legs");
    if (o->solver == BSAR_SOLVER_NEWTON) check_newton_dem(s->dem.view);
    if (o->precision != BSAR_FP64 && (s->dem.view.empty || s->dem.view.nx < 2 || s->dem.view.ny < 2))
        fail(BSAR_ERR_UNSUPPORTED, "the mixed forms need a DEM of at least 2 x 2 nodes");
    if (!s->rc[o->precision].data) compress_scene(ctx, s, o->precision);
    const double* axes = stage_grid(ctx, g);
    BpArgs a{};
    a.dem = s->dem.view;
    a.tx = s->tx->as<double>();
    a.rx = s->rx->as<double>();
    a.np = (int)s->np;
    a.nr = s->nr;
    a.rc64 = s->rc[BSAR_FP64].data ? s->rc[BSAR_FP64].data->as<double2>() : nullptr;
    a.rc32 = s->rc[BSAR_MIXED].data ? s->rc[BSAR_MIXED].data->as<float2>() : nullptr;
    a.rc16 = s->rc[BSAR_MIXED_FP16].data ? s->rc[BSAR_MIXED_FP16].data->as<__half2>() : nullptr;
    a.scale16 = s->rc[BSAR_MIXED_FP16].scale ? s->rc[BSAR_MIXED_FP16].scale->as<float>() : nullptr;
    a.gx = axes;
    a.gy = axes + g->nx;
    a.gz = axes + g->nx + g->ny;
    a.nx = (int)g->nx;
    a.ny = (int)g->ny;
    a.nz = (int)g->nz;
    a.n1 = s->n1;
    a.n2 = s->n2;
    a.c = s->c;
    a.fs_eff = s->fs * s->upsample;          // proc_test_script.cpp:220-223
    a.lambda = s->c / s->fc;                  // proc_test_script.cpp:213
    a.W = search_nodes(s->dem.view, o->search_radius_m);
    a.v_begin = 0;
    a.v_count = g->nx * g->ny * g->nz;
    a.out = d_out;
    if (o->precision == BSAR_FP64) {
        launched(ctx, launch_bp_plain(a, o->solver, o->legs, ctx->stream), "back-projection (FP64)");
        return;
    }
    // per-pulse anchors at the grid centre
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
    if (!ctx->status) {
        ctx->status = dev_alloc(ctx, sizeof(int));
        cuda_check(cudaMemsetAsync(ctx->status->p, 0, sizeof(int), ctx->stream), "memset");
    }
    MixedLaunch ml{s->dem.pitch, s->dem.has_tmap ? (const void*)s->dem.tmap : nullptr, s->off_x, s->off_y,
                   ctx->status->as<int>()};
    cudaError_t e = launch_bp_mixed(a, ml, o->legs, o->precision == BSAR_MIXED_FP16 ? 1 : 0, ctx->stream);
    if (e == cudaErrorNotSupported) {
        cudaGetLastError();
        fail(BSAR_ERR_UNSUPPORTED, "mixed back-projection mode not supported");
    }
    launched(ctx, e, "back-projection (mixed)");
}

bsar_status bsar_backproject(bsar_ctx* ctx, bsar_scene_id id, const bsar_grid* g, const bsar_bp_opts* o,
                             double* image_out)
{
    return guarded(ctx, [&] {
        if (!image_out) fail(BSAR_ERR_INVALID_ARG, "image_out is NULL");
        check_grid(g);
        int64_t nv = g->nx * g->ny * g->nz;
        auto img = dev_alloc(ctx, sizeof(double2) * nv);
        backproject(ctx, id, g, o, img->as<double2>());
        cuda_check(cudaMemcpyAsync(image_out, img->p, sizeof(double2) * nv, cudaMemcpyDeviceToHost, ctx->stream), "d2h");
        sync(ctx);
        check_device_status(ctx);
    });
}

bsar_status bsar_backproject_device(bsar_ctx* ctx, bsar_scene_id id, const bsar_grid* g, const bsar_bp_opts* o,
                                    void* d_image)
{
    return guarded(ctx, [&] {
        if (!d_image) fail(BSAR_ERR_INVALID_ARG, "d_image is NULL");
        backproject(ctx, id, g, o, static_cast<double2*>(d_image));
    });
}

}  // extern "C"
