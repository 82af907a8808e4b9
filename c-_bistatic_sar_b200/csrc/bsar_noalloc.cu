// bsar_noalloc.cu -- bsar_backproject_mixed_noalloc: the one-request mixed back-projection
// with every per-call device buffer carved out of one file-scope scratch array, so a call
// makes no device allocation (no cudaMalloc / cudaFree, no pool, no library workspace).
//
// Who needs it: programs whose device memory is owned by another allocator -- a
// framework's caching allocator that has reserved most of the GPU, or a client held to a
// fixed memory limit -- where a cudaMalloc from this library fails or forces that
// allocator to give memory back; and latency-critical loops that cannot take the
// device-wide wait a cudaFree implies, which stalls every other stream on the GPU.
//
// Scratch layout (each region 256-byte aligned):
//   request record (MixedReq, holds the DEM tensor map)
//   work counter + status word        -- must start at zero: cleared every call
//   per-pulse anchors (ref_L, ref_phase, ref_bin_i, ref_bin_f) and crossing offsets
//   grid axes
//   image (complex128, copied to the caller's buffer at the end)
//   small grids only: the chunk record, pulse-chunk sums and per-tile chunk counts
//   (cleared every call); the same chunking as the allocating entry point, so both
//   give the same image
//
// The array is 64 MiB.  A device commits it when this file's module is loaded there:
// under CUDA's default lazy module loading that is the first call on the device (its
// cudaGetSymbolAddress), with CUDA_MODULE_LOADING=EAGER it is when the library's first
// CUDA call initialises the device.  Either way the device holds it until the process
// exits.  So that first call is the one moment this entry point asks the driver for
// memory: make it before another allocator (a framework's caching allocator) reserves
// the device's memory, and before any stream capture -- or set
// CUDA_MODULE_LOADING=EAGER.  The array is one per device and per process and keeps
// the previous call's contents: calls that overlap in time on one device (two threads,
// two contexts, or an earlier call's work still on another stream) race on it.
#include <mutex>

#include "runtime.hpp"

namespace {

constexpr size_t kScratchBytes = size_t(64) << 20;
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_addr_mu;
void* g_addr[kMaxDevices] = {};

// Device address of the scratch array on `dev` (the current device), looked up once.
unsigned char* scratch_on(int dev)
{
    std::lock_guard<std::mutex> lk(g_addr_mu);
    if (dev < 0 || dev >= kMaxDevices) fail(BSAR_ERR_INVALID_ARG, "device index %d out of range", dev);
    if (!g_addr[dev]) cuda_check(cudaGetSymbolAddress(&g_addr[dev], g_scratch), "scratch symbol address");
    return static_cast<unsigned char*>(g_addr[dev]);
}

size_t up256(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace

extern "C" bsar_status bsar_backproject_mixed_noalloc(bsar_ctx* ctx, bsar_scene_id id, const bsar_grid* g,
                                                      const bsar_bp_opts* o, double* image_out)
{
    return guarded(ctx, [&] {
        if (!image_out || !o) fail(BSAR_ERR_INVALID_ARG, "NULL argument");
        // axes bounded one factor at a time: the voxel count below cannot wrap
        const int64_t nv = check_grid(g);
        if (o->flags & ~BSAR_BP_EXHAUSTIVE_SCAN) fail(BSAR_ERR_INVALID_ARG, "unknown back-projection flags");
        if (o->solver != BSAR_SOLVER_NEWTON || o->legs != BSAR_LEGS_PER_PULSE ||
            (o->precision != BSAR_MIXED && o->precision != BSAR_MIXED_FP16))
            fail(BSAR_ERR_UNSUPPORTED, "this entry point runs the mixed forms (Newton, per-pulse legs)");
        Scene* s = get_scene(ctx, id);
        check_newton_dem(s->dem.view);
        if (s->dem.view.empty || s->dem.view.nx < 2 || s->dem.view.ny < 2)
            fail(BSAR_ERR_UNSUPPORTED, "the mixed forms need a DEM of at least 2 x 2 nodes");
        if (!s->rc[o->precision].data)
            fail(BSAR_ERR_INVALID_ARG, "the scene has no samples for this precision: call bsar_scene_compress first");
        const int64_t np = s->np;
        // scratch layout and its limit
        const size_t o_req = 0;
        const size_t o_cnt = o_req + up256(sizeof(MixedReq));
        const size_t o_anc = o_cnt + 256;
        const size_t o_off = o_anc + up256(20 * (size_t)np);
        const size_t o_axes = o_off + up256(32 * (size_t)np);
        const size_t o_img = o_axes + up256(8 * (size_t)(g->nx + g->ny + g->nz));
        const int64_t vtiles = (nv + 127) / 128;
        const int K = mixed_chunks(nv, (int)np);
        const size_t o_chk = o_img + up256(16 * (size_t)nv);
        const size_t o_part = o_chk + (K > 1 ? up256(sizeof(MixedChunks)) : 0);
        const size_t o_done = o_part + (K > 1 ? up256(16 * (size_t)K * (size_t)nv) : 0);
        const size_t need = o_done + (K > 1 ? up256(4 * (size_t)vtiles) : 0);
        if (need > kScratchBytes)
            fail(BSAR_ERR_INVALID_ARG, "the call needs %zu bytes of scratch; the fixed scratch holds %zu", need,
                 kScratchBytes);
        unsigned char* S = scratch_on(ctx->device);
        cudaStream_t st = ctx->stream;
        double* axes = reinterpret_cast<double*>(S + o_axes);
        cuda_check(cudaMemcpyAsync(axes, g->x_axis, 8 * g->nx, cudaMemcpyHostToDevice, st), "axes");
        cuda_check(cudaMemcpyAsync(axes + g->nx, g->y_axis, 8 * g->ny, cudaMemcpyHostToDevice, st), "axes");
        cuda_check(cudaMemcpyAsync(axes + g->nx + g->ny, g->z_axis, 8 * g->nz, cudaMemcpyHostToDevice, st), "axes");
        int* counter = reinterpret_cast<int*>(S + o_cnt);
        int* status = counter + 1;
        cuda_check(cudaMemsetAsync(counter, 0, 2 * sizeof(int), st), "clear counter and status");
        BpArgs a{};
        a.dem = s->dem.view;
        a.tx = s->tx->as<double>();
        a.rx = s->rx->as<double>();
        a.np = (int)np;
        a.nr = s->nr;
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
        a.fs_eff = s->fs * s->upsample;
        a.lambda = s->c / s->fc;
        a.W = search_nodes(s->dem.view, o->search_radius_m);
        a.v_begin = 0;
        a.v_count = nv;
        a.out = reinterpret_cast<double2*>(S + o_img);
        // per-pulse anchors about the grid centre, as the allocating entry point makes them
        const double centre[3] = {0.5 * (g->x_axis[0] + g->x_axis[g->nx - 1]),
                                  0.5 * (g->y_axis[0] + g->y_axis[g->ny - 1]),
                                  0.5 * (g->z_axis[0] + g->z_axis[g->nz - 1])};
        unsigned char* anc = S + o_anc;
        double* offs = reinterpret_cast<double*>(S + o_off);
        launched(ctx, launch_ref_ranges(s->dem.view, a.tx, a.rx, (int)np, centre, s->n1, s->n2, a.W, a.lambda,
                                        a.fs_eff / s->c, (double*)anc, (float*)(anc + 8 * np), (int*)(anc + 12 * np),
                                        (float*)(anc + 16 * np), offs, st),
                 "reference ranges");
        a.ref_L = (const double*)anc;
        a.ref_phase = (const float*)(anc + 8 * np);
        a.ref_bin_i = (const int*)(anc + 12 * np);
        a.ref_bin_f = (const float*)(anc + 16 * np);
        // mean crossing offset (DEM tile centring), summed in pulse order through a fixed
        // host buffer
        double ox = 0.0, oy = 0.0;
        {
            constexpr int64_t kChunk = 1024;
            double h[4 * kChunk];
            for (int64_t p0 = 0; p0 < np; p0 += kChunk) {
                const int64_t n = std::min(kChunk, np - p0);
                cuda_check(cudaMemcpyAsync(h, offs + 4 * p0, sizeof(double) * 4 * n, cudaMemcpyDeviceToHost, st),
                           "offsets");
                sync(ctx);
                for (int64_t i = 0; i < n; i++) {
                    ox += h[4 * i] + h[4 * i + 2];
                    oy += h[4 * i + 1] + h[4 * i + 3];
                }
            }
        }
        MixedReq r = mixed_request(s, a, o->precision == BSAR_MIXED_FP16, o->flags);
        r.off_x = (float)(ox / (2.0 * np));
        r.off_y = (float)(oy / (2.0 * np));
        MixedChunks* d_chunks = nullptr;
        if (K > 1) {
            const MixedChunks c{K, 0, reinterpret_cast<double2*>(S + o_part), reinterpret_cast<int*>(S + o_done)};
            d_chunks = reinterpret_cast<MixedChunks*>(S + o_chk);
            cuda_check(cudaMemcpyAsync(d_chunks, &c, sizeof c, cudaMemcpyHostToDevice, st), "chunk record");
            cuda_check(cudaMemsetAsync(c.tile_done, 0, 4 * (size_t)vtiles, st), "clear chunk counts");
        }
        MixedReq* d_req = reinterpret_cast<MixedReq*>(S + o_req);
        cuda_check(cudaMemcpyAsync(d_req, &r, sizeof r, cudaMemcpyHostToDevice, st), "request record");
        MixedBatch b{d_req, nullptr, nullptr, (int)(vtiles * K), counter, status, d_chunks,
                     (long long)ctx->tile_wait_polls};
        const int grid = (int)std::min<int64_t>(b.ntiles, mixed_grid_ctas());
        launched(ctx, launch_bp_mixed(b, a.W, grid, st, K > 1), "back-projection (mixed, scratch)");
        cuda_check(cudaMemcpyAsync(image_out, a.out, 16 * (size_t)nv, cudaMemcpyDeviceToHost, st), "image");
        int hstat = 0;
        cuda_check(cudaMemcpyAsync(&hstat, status, sizeof(int), cudaMemcpyDeviceToHost, st), "status");
        sync(ctx);
        if (hstat) fail(BSAR_ERR_TIMEOUT, "a device-side DEM tile copy did not complete within its wait limit");
    });
}
