// bsar_api.cpp -- host runtime behind the C ABI of include/bsar.h.
//
// A context owns a CUDA stream, a device-memory budget and the resident scenes.  Each
// entry point validates its arguments, stages host data into device buffers charged to
// the budget, launches the kernels of k_plain.cu / k_mixed.cu / k_pulse.cu and copies the
// results back.  There is no host-side compute path: every result comes from a kernel.
#include "runtime.hpp"

// ------------------------------------------------------------------------------------
// API glue
// ------------------------------------------------------------------------------------
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
    case BSAR_ERR_CANCELLED: return "cancelled";
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
    static std::atomic<uint64_t> serials{0};
    auto* ctx = new bsar_ctx();
    ctx->serial = ++serials;
    ctx->device = dev;
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete ctx;
        return BSAR_ERR_CUDA;
    }
    ctx->own_stream = true;
    // the context's device buffers come from its own stream-ordered pool, which keeps
    // freed blocks for the next call: a cudaMalloc / cudaFree per call costs a
    // device-wide synchronisation each and, now and then, hundreds of milliseconds
    {
        cudaMemPoolProps pp = {};
        pp.allocType = cudaMemAllocationTypePinned;
        pp.location.type = cudaMemLocationTypeDevice;
        pp.location.id = dev;
        uint64_t keep = ~0ull;
        if (cudaMemPoolCreate(&ctx->pool, &pp) != cudaSuccess ||
            cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess) {
            if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
            ctx->pool = nullptr;
            cudaGetLastError();
        }
        ctx->use_pool = ctx->pool != nullptr;
    }
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
    ctx->status.reset();
    ctx->mixed_req.reset();
    ctx->mixed_counter.reset();
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
    if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
    clear_error(ctx);   // the destroying thread's entry (others' carry the old serial)
    delete ctx;
}

const char* bsar_last_error(const bsar_ctx* ctx)
{
    if (!ctx) return "null context";
    return thread_error_message(ctx);
}

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

static bsar_scene_id add_scene(bsar_ctx* ctx, std::unique_ptr<Scene> sc)
{
    uint64_t id = ctx->next_scene++;
    ctx->scenes[id] = std::move(sc);
    return id;
}

bsar_status bsar_scene_upload(bsar_ctx* ctx, const bsar_scene_desc* desc, bsar_scene_id* out)
{
    return guarded(ctx, [&] {
        if (!desc || !out) fail(BSAR_ERR_INVALID_ARG, "NULL argument");
        *out = add_scene(ctx, make_scene(ctx, *desc, true));
    });
}

bsar_status bsar_scene_synthesize_ex(bsar_ctx* ctx, const bsar_scene_desc* desc, const double* scat_pos,
                                     const double* scat_amp, int64_t n_scat, double snr_db, uint64_t seed, int32_t flags,
                                     bsar_scene_id* out)
{
    return guarded(ctx, [&] {
        if (!desc || !out) fail(BSAR_ERR_INVALID_ARG, "NULL argument");
        if (desc->samples_kind != BSAR_SAMPLES_RAW) fail(BSAR_ERR_INVALID_ARG, "synthesis makes raw scenes");
        if (n_scat < 0 || (n_scat > 0 && (!scat_pos || !scat_amp))) fail(BSAR_ERR_INVALID_ARG, "bad scatterers");
        if (!all_finite(scat_pos, 3 * n_scat) || !all_finite(scat_amp, n_scat))
            fail(BSAR_ERR_INVALID_ARG, "non-finite scatterer");
        auto sc = make_scene(ctx, *desc, false);
        if (flags & ~BSAR_SYNTH_REFERENCE_BINS) fail(BSAR_ERR_INVALID_ARG, "unknown synthesis flags");
        synthesize_samples(ctx, sc.get(), scat_pos, scat_amp, n_scat, snr_db, seed, flags);
        sync(ctx);
        *out = add_scene(ctx, std::move(sc));
    });
}

bsar_status bsar_scene_synthesize(bsar_ctx* ctx, const bsar_scene_desc* desc, const double* scat_pos,
                                  const double* scat_amp, int64_t n_scat, double snr_db, uint64_t seed,
                                  bsar_scene_id* out)
{
    return bsar_scene_synthesize_ex(ctx, desc, scat_pos, scat_amp, n_scat, snr_db, seed, 0, out);
}

bsar_status bsar_scene_read_samples(bsar_ctx* ctx, bsar_scene_id id, double* out)
{
    return guarded(ctx, [&] {
        Scene* s = get_scene(ctx, id);
        if (!out) fail(BSAR_ERR_INVALID_ARG, "NULL buffer");
        cuda_check(cudaMemcpyAsync(out, s->samples->p, sizeof(double2) * s->np * s->ns, cudaMemcpyDeviceToHost,
                                   ctx->stream),
                   "download");
        sync(ctx);
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

bsar_status bsar_scene_read_stored(bsar_ctx* ctx, bsar_scene_id id, int32_t precision, double* out)
{
    return guarded(ctx, [&] {
        Scene* s = get_scene(ctx, id);
        if (!out) fail(BSAR_ERR_INVALID_ARG, "NULL buffer");
        if (precision < BSAR_FP64 || precision > BSAR_MIXED_FP16) fail(BSAR_ERR_INVALID_ARG, "unknown precision");
        RcBuf& rb = s->rc[precision];
        if (!rb.data) compress_scene(ctx, s, precision);
        const size_t n = (size_t)s->np * s->nr;
        if (precision == BSAR_FP64) {
            cuda_check(cudaMemcpyAsync(out, rb.data->p, sizeof(double2) * n, cudaMemcpyDeviceToHost, ctx->stream),
                       "download");
            sync(ctx);
            return;
        }
        if (precision == BSAR_MIXED) {
            std::vector<float2> h(n);
            cuda_check(cudaMemcpyAsync(h.data(), rb.data->p, sizeof(float2) * n, cudaMemcpyDeviceToHost, ctx->stream),
                       "download");
            sync(ctx);
            for (size_t i = 0; i < n; i++) {
                out[2 * i] = h[i].x;
                out[2 * i + 1] = h[i].y;
            }
            return;
        }
        std::vector<__half2> h(n);
        std::vector<float> sc(s->np);
        cuda_check(cudaMemcpyAsync(h.data(), rb.data->p, sizeof(__half2) * n, cudaMemcpyDeviceToHost, ctx->stream),
                   "download");
        cuda_check(cudaMemcpyAsync(sc.data(), rb.scale->p, sizeof(float) * s->np, cudaMemcpyDeviceToHost, ctx->stream),
                   "download");
        sync(ctx);
        for (size_t i = 0; i < n; i++) {
            const double f = sc[i / s->nr];
            out[2 * i] = (double)__low2float(h[i]) * f;
            out[2 * i + 1] = (double)__high2float(h[i]) * f;
        }
    });
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

// The voxels [v_begin, v_begin + v_count) of the grid's flat order (v_count < 0: all) into
// d_out, the full [x][y][z] image; per-pulse anchors and pulse chunks are those of the
// whole grid, so a voxel's value does not depend on the range it is computed in.
static void backproject(bsar_ctx* ctx, bsar_scene_id id, const bsar_grid* g, const bsar_bp_opts* o, double2* d_out,
                        int64_t v_begin = 0, int64_t v_count = -1)
{
    Scene* s = get_scene(ctx, id);
    const int64_t nv_grid = check_grid(g);
    if (v_count < 0) v_count = nv_grid - v_begin;
    if (v_begin < 0 || v_count < 1 || v_begin > nv_grid - v_count)
        fail(BSAR_ERR_INVALID_ARG, "voxel range [%lld, %lld) outside the grid's %lld voxels", (long long)v_begin,
             (long long)(v_begin + v_count), (long long)nv_grid);
    if (!o) fail(BSAR_ERR_INVALID_ARG, "options are NULL");
    if (o->solver != BSAR_SOLVER_GRID && o->solver != BSAR_SOLVER_NEWTON) fail(BSAR_ERR_INVALID_ARG, "unknown solver");
    if (o->legs != BSAR_LEGS_MEAN && o->legs != BSAR_LEGS_PER_PULSE) fail(BSAR_ERR_INVALID_ARG, "unknown legs mode");
    if (o->precision < BSAR_FP64 || o->precision > BSAR_MIXED_FP16) fail(BSAR_ERR_INVALID_ARG, "unknown precision");
    if (o->flags & ~BSAR_BP_EXHAUSTIVE_SCAN) fail(BSAR_ERR_INVALID_ARG, "unknown back-projection flags");
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
    a.v_begin = v_begin;
    a.v_count = v_count;
    a.out = d_out;
    if (o->precision == BSAR_FP64) {
        launched(ctx, launch_bp_plain(a, o->solver, o->legs, ctx->stream), "back-projection (FP64)");
        return;
    }
    set_anchors(ctx, s, g, a);
    if (o->legs != BSAR_LEGS_PER_PULSE) fail(BSAR_ERR_UNSUPPORTED, "the mixed forms use per-pulse legs");
    ensure_mixed_buffers(ctx);
    MixedReq r = mixed_request(s, a, o->precision == BSAR_MIXED_FP16, o->flags);
    // small grids: each tile's pulses in K chunks, so the work items fill the GPU
    const int64_t vtiles = (a.v_count + 127) / 128;
    const int K = mixed_chunks(nv_grid, a.np);
    std::unique_ptr<DevBuf> partial, tile_done, chunks;
    if (K > 1) {
        partial = dev_alloc(ctx, sizeof(double2) * (size_t)K * (size_t)(g->nx * g->ny * g->nz));
        tile_done = dev_alloc(ctx, sizeof(int) * (size_t)vtiles);
        cuda_check(cudaMemsetAsync(tile_done->p, 0, sizeof(int) * (size_t)vtiles, ctx->stream), "memset");
        const MixedChunks c{K, 0, partial->as<double2>(), tile_done->as<int>()};
        chunks = dev_upload(ctx, &c, sizeof c);
    }
    cuda_check(cudaMemcpyAsync(ctx->mixed_req->p, &r, sizeof r, cudaMemcpyHostToDevice, ctx->stream), "h2d");
    cuda_check(cudaMemsetAsync(ctx->mixed_counter->p, 0, sizeof(int), ctx->stream), "memset");
    MixedBatch b{ctx->mixed_req->as<MixedReq>(), nullptr, nullptr, (int)(vtiles * K),
                 ctx->mixed_counter->as<int>(), ctx->status->as<int>(), chunks ? chunks->as<MixedChunks>() : nullptr,
                 (long long)ctx->tile_wait_polls};
    const int grid = (int)std::min<int64_t>(b.ntiles, mixed_grid_ctas());
    cudaError_t e = launch_bp_mixed(b, a.W, grid, ctx->stream, K > 1);
    launched(ctx, e, "back-projection (mixed)");
}

bsar_status bsar_set_tile_wait_limit(bsar_ctx* ctx, int64_t polls)
{
    return guarded(ctx, [&] { ctx->tile_wait_polls = polls < 0 ? kDefaultTileWaitPolls : polls; });
}

bsar_status bsar_backproject(bsar_ctx* ctx, bsar_scene_id id, const bsar_grid* g, const bsar_bp_opts* o,
                             double* image_out)
{
    return guarded(ctx, [&] {
        if (!image_out) fail(BSAR_ERR_INVALID_ARG, "image_out is NULL");
        const int64_t nv = check_grid(g);
        auto img = dev_alloc(ctx, sizeof(double2) * nv);
        backproject(ctx, id, g, o, img->as<double2>());
        cuda_check(cudaMemcpyAsync(image_out, img->p, sizeof(double2) * nv, cudaMemcpyDeviceToHost, ctx->stream), "d2h");
        sync(ctx);
        check_device_status(ctx);
    });
}

bsar_status bsar_backproject_range(bsar_ctx* ctx, bsar_scene_id id, const bsar_grid* g, const bsar_bp_opts* o,
                                   int64_t v_begin, int64_t v_count, double* image_out)
{
    return guarded(ctx, [&] {
        if (!image_out) fail(BSAR_ERR_INVALID_ARG, "image_out is NULL");
        const int64_t nv = check_grid(g);
        auto img = dev_alloc(ctx, sizeof(double2) * nv);
        cuda_check(cudaMemsetAsync(img->p, 0, sizeof(double2) * nv, ctx->stream), "clear image");
        backproject(ctx, id, g, o, img->as<double2>(), v_begin, v_count);
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
