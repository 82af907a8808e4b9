// bsar_serve.cpp -- continuous-batching image-formation server (bsar_server_* of bsar.h).
//
// Two threads per server.  The worker owns the batches: two batch slots, each with its
// own stream, pinned staging and device copies, keep up to two batches in flight:
//
//   loop:
//     fill every idle batch slot: a list of (request, work item) pairs -- a 128-voxel
//       tile, or one pulse chunk of a tile for small grids -- of the admitted requests in
//       earliest-deadline order (arrival + twice the request's own service time), most
//       costly items first, launched as a replay of a captured CUDA graph (request
//       records and tile list copied from pinned staging, work counter zeroed,
//       persistent mixed kernel); no context lock
//     wait for the older batch (bounded)
//     retire requests whose tiles are all done (image to the caller's buffer on the
//       `ret` stream, latency recorded; the buffers go to the I/O thread)
//
// The I/O thread frees finished requests' buffers (which returns their budget) and admits
// pending requests FIFO as the HBM budget and the in-flight slots allow: scene upload or
// on-device echo synthesis, pulse compression + upsampling, per-pulse anchors, on the
// high-priority `io` stream with stream-ordered allocations.  Every upload comes before
// the first kernel, so an admission waits on the device once (the anchors' read-back),
// and its kernels take SM slots as the running batch's CTAs free them.
//
// The second batch's CTAs take the SMs the first batch's tail leaves idle.  Work items
// are the same 128-voxel groups (and pulse chunks) a one-request launch uses, so every
// voxel's arithmetic is independent of the batch it runs in.
#include "runtime.hpp"

#include <chrono>
#include <condition_variable>
#include <deque>
#include <thread>

namespace {

using Clock = std::chrono::steady_clock;
// batch key bit: the batch holds a request whose tiles run in pulse chunks
constexpr int kChunkedKey = 1 << 16;

constexpr int kMaxSlots = 256;
constexpr double kBatchTimeoutS = 300.0;   // default bound on the wait for one batch

enum class St { Pending, Active, Done, Failed };

struct Req {
    uint64_t id = 0;
    St state = St::Pending;
    bsar_status status = BSAR_OK;
    std::string error;
    // copies of the request's small arrays
    std::vector<double> dem_x, dem_y, dem_z, tx, rx, gx, gy, gz, spos, samp;
    bsar_scene_desc desc{};
    bsar_grid grid{};
    bsar_bp_opts opts{};
    int64_t n_scat = 0;
    double snr_db = 0;
    uint64_t seed = 0;
    double* image_out = nullptr;
    bool cancelled = false;                         // bsar_server_cancel: no further work items
    // device state while admitted
    int slot = -1;
    uint64_t reserved = 0;
    std::unique_ptr<Scene> scene;
    std::unique_ptr<DevBuf> axes, image;
    std::unique_ptr<DevBuf> partial, tile_done;     // pulse-chunk sums of small grids
    MixedReq rec{};
    MixedChunks chunks{};
    int64_t ntiles = 0, next_tile = 0, done_tiles = 0;
    Clock::time_point t_submit, t_done;
    double voxel_pulses = 0;
    double deadline_s = 0;          // scheduling deadline, seconds after the server started
};

// Upper bound of the pulse-chunk buffers of a grid of nv voxels: at most 8 chunks per
// 128-voxel tile, and chunks only while the tiles leave resident CTAs idle (fewer than
// 4096 tiles on any device).  Host-only, so it does not ask the device.
uint64_t chunk_bytes(uint64_t nv)
{
    const uint64_t tiles = (nv + 127) / 128;
    return tiles < 4096 ? 16 * 8 * nv + 4 * tiles : 0;
}

uint64_t estimate_bytes(const Req& r)
{
    const uint64_t np = r.desc.n_pulses, ns = r.desc.n_samples, up = r.desc.upsample;
    const uint64_t nd = (uint64_t)std::max<int64_t>(r.desc.dem.nx, 1) * std::max<int64_t>(r.desc.dem.ny, 1);
    const uint64_t nv = (uint64_t)r.grid.nx * r.grid.ny * r.grid.nz;
    const uint64_t sample = r.opts.precision == BSAR_MIXED_FP16 ? 4 : 8;
    return 16 * np * ns                              // raw pulses
           + sample * np * ns * up                   // upsampled pulses
           + 16 * ns + 16 * nv                       // spectrum, image
           + 12 * nd + 48 * np + 52 * np             // DEM, trajectories, anchors
           + 24 * np * (uint64_t)std::max<int64_t>(r.n_scat, 1)   // synthesis work buffers
           + chunk_bytes(nv)                         // pulse-chunk sums of a small grid
           + (1u << 20);
}

}  // namespace

struct ServeBatch {
    MixedReq* h_reqs = nullptr;                     // pinned staging
    MixedChunks* h_chunks = nullptr;
    int2* h_tiles = nullptr;
    int* h_ntiles = nullptr;
    std::unique_ptr<DevBuf> d_reqs, d_chunks, d_tiles, d_ntiles, d_counter;
    cudaStream_t st = nullptr;
    cudaEvent_t ev = nullptr;
    std::map<int, cudaGraphExec_t> graphs;          // per node-scan width W (| kChunkedKey)
    std::vector<std::pair<Req*, int64_t>> items;    // requests in the batch, tiles each
    double voxel_pulses = 0;                        // work of the batch
    Clock::time_point t_launch;
    bool inflight = false;
    uint64_t seq = 0;
};

struct bsar_server {
    bsar_ctx* ctx = nullptr;
    bsar_server_opts opts{};
    uint64_t budget = 0, reserved = 0;
    std::thread worker;                             // builds, launches and retires batches
    std::thread io_thread;                          // admits requests, releases their buffers
    std::mutex mu;
    std::condition_variable cv_work, cv_done, cv_io;
    std::vector<Req*> to_free;                      // finished requests whose buffers await release
    bool stop = false;
    uint64_t next_id = 1;
    std::deque<Req*> pending;
    std::vector<Req*> active;                       // admission order
    std::map<uint64_t, std::unique_ptr<Req>> reqs;
    bool slot_used[kMaxSlots] = {};
    ServeBatch batch[2];
    Clock::time_point t_start = Clock::now();
    double rate_est = 1e9;                          // voxel-pulses/s of recent batches
    Clock::time_point t_last_batch_done = Clock::now();
    double batch_busy_s = 0.0;                      // time with a batch on the device
    uint64_t batch_seq = 0;
    cudaStream_t io = nullptr;                      // admission and buffer release
    cudaStream_t ret = nullptr;                     // image read-back of finished requests
    int grid_ctas = 0, max_tiles = 0;
    // statistics
    std::vector<double> latencies;
    uint64_t submitted = 0, completed = 0, failed = 0, launches = 0, tiles = 0;
    uint64_t peak_inflight = 0, peak_reserved = 0;
    double vp_done = 0;
    bool any_submit = false;
    Clock::time_point t_first, t_last;
    std::string fatal;
    bsar_status fatal_status = BSAR_ERR_CUDA;       // what the requests left at a stop fail with
    double batch_timeout_s = kBatchTimeoutS;
};

namespace {

// Runs `f` with the context locked, its stream switched to `st` and (when `pooled`)
// device buffers taken from the stream-ordered pool.
template <typename F> void with_ctx(bsar_server* s, cudaStream_t st, bool pooled, F&& f)
{
    std::lock_guard<std::mutex> lk(s->ctx->mu);
    cudaStream_t saved = s->ctx->stream;
    s->ctx->stream = st;
    const bool saved_pool = s->ctx->use_pool;
    s->ctx->use_pool = pooled;
    try {
        f();
    } catch (...) {
        s->ctx->stream = saved;
        s->ctx->use_pool = saved_pool;
        throw;
    }
    s->ctx->stream = saved;
    s->ctx->use_pool = saved_pool;
}

// Completes a request (server lock held).  keep_reserved: its device buffers are not
// released yet, so its share of the budget stays reserved until the I/O thread frees them.
void finish(bsar_server* s, Req* r, bsar_status st, const std::string& err, bool keep_reserved = false)
{
    r->status = st;
    r->error = err;
    r->state = st == BSAR_OK ? St::Done : St::Failed;
    r->t_done = Clock::now();
    if (r->slot >= 0) s->slot_used[r->slot] = false;
    r->slot = -1;
    if (!keep_reserved) {
        s->reserved -= r->reserved;
        r->reserved = 0;
    }
    if (st == BSAR_OK) {
        s->completed++;
        s->vp_done += r->voxel_pulses;
        s->latencies.push_back(std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count());
        s->t_last = r->t_done;
    } else {
        s->failed++;
    }
}

void release(bsar_server* s, Req* r)
{
    with_ctx(s, s->io, true, [&] {
        r->scene.reset();
        r->axes.reset();
        r->image.reset();
        r->partial.reset();
        r->tile_done.reset();
    });
}

// Admission of one request (I/O thread, server lock NOT held): scene upload or
// synthesis, pulse compression + upsampling, anchors, device image.
void admit(bsar_server* s, Req* r)
{
    with_ctx(s, s->io, true, [&] {
        bsar_ctx* ctx = s->ctx;
        bsar_scene_desc d = r->desc;
        const bool synth = d.samples == nullptr;
        r->scene = make_scene(ctx, d, !synth);
        check_newton_dem(r->scene->dem.view);
        if (r->scene->dem.view.empty || r->scene->dem.view.nx < 2 || r->scene->dem.view.ny < 2)
            fail(BSAR_ERR_UNSUPPORTED, "the mixed forms need a DEM of at least 2 x 2 nodes");
        // every upload from pageable memory before the first kernel (such a copy first
        // drains the stream, whose kernels wait for SM slots behind the running batch), so
        // the admission waits on the device once, for the anchors below
        std::vector<double> ax;
        ax.insert(ax.end(), r->gx.begin(), r->gx.end());
        ax.insert(ax.end(), r->gy.begin(), r->gy.end());
        ax.insert(ax.end(), r->gz.begin(), r->gz.end());
        r->axes = dev_upload(ctx, ax.data(), sizeof(double) * ax.size());
        stage_reference(ctx, r->scene.get());
        if (synth)
            synthesize_samples(ctx, r->scene.get(), r->spos.data(), r->samp.data(), r->n_scat, r->snr_db, r->seed, 0,
                               false);
        compress_scene(ctx, r->scene.get(), r->opts.precision, false);
        r->scene->samples.reset();        // only the upsampled pulses are needed from here (freed in stream order)
        r->scene->reference_dev.reset();
        const int64_t nv = r->grid.nx * r->grid.ny * r->grid.nz;
        r->image = dev_alloc(ctx, sizeof(double2) * nv);
        Scene* sc = r->scene.get();
        BpArgs a{};
        a.dem = sc->dem.view;
        a.tx = sc->tx->as<double>();
        a.rx = sc->rx->as<double>();
        a.np = (int)sc->np;
        a.nr = sc->nr;
        a.rc32 = sc->rc[BSAR_MIXED].data ? sc->rc[BSAR_MIXED].data->as<float2>() : nullptr;
        a.rc16 = sc->rc[BSAR_MIXED_FP16].data ? sc->rc[BSAR_MIXED_FP16].data->as<__half2>() : nullptr;
        a.scale16 = sc->rc[BSAR_MIXED_FP16].scale ? sc->rc[BSAR_MIXED_FP16].scale->as<float>() : nullptr;
        a.gx = r->axes->as<double>();
        a.gy = a.gx + r->grid.nx;
        a.gz = a.gy + r->grid.ny;
        a.nx = (int)r->grid.nx;
        a.ny = (int)r->grid.ny;
        a.nz = (int)r->grid.nz;
        a.n1 = sc->n1;
        a.n2 = sc->n2;
        a.c = sc->c;
        a.fs_eff = sc->fs * sc->upsample;
        a.lambda = sc->c / sc->fc;
        a.W = search_nodes(sc->dem.view, r->opts.search_radius_m);
        a.v_begin = 0;
        a.v_count = nv;
        a.out = r->image->as<double2>();
        // small grids: each tile's pulses in K chunks (the rule every path applies)
        const int64_t vtiles = (nv + 127) / 128;
        const int K = mixed_chunks(nv, (int)sc->np);
        if (K > 1) {
            r->partial = dev_alloc(ctx, sizeof(double2) * (size_t)K * (size_t)nv);
            r->tile_done = dev_alloc(ctx, sizeof(int) * (size_t)vtiles);
            cuda_check(cudaMemsetAsync(r->tile_done->p, 0, sizeof(int) * (size_t)vtiles, ctx->stream), "memset");
        }
        bsar_grid g = r->grid;
        g.x_axis = r->gx.data();
        g.y_axis = r->gy.data();
        g.z_axis = r->gz.data();
        set_anchors(ctx, sc, &g, a);
        sync(ctx);
        r->rec = mixed_request(sc, a, r->opts.precision == BSAR_MIXED_FP16, r->opts.flags);
        if (K > 1) r->chunks = MixedChunks{K, 0, r->partial->as<double2>(), r->tile_done->as<int>()};
        r->ntiles = vtiles * K;             // work items: (tile, chunk) pairs
        r->voxel_pulses = (double)nv * (double)sc->np;
    });
}

// Deadline of a request for the batch scheduler: its arrival plus twice its own service
// time at the server's recent throughput (earliest deadline first).  Small requests thus
// pass a large one that arrived shortly before them, and a large one is not starved by a
// stream of small ones: it gets the whole GPU once its deadline is the earliest.  Against
// equal shares for every admitted request this cut the modelled p99 latency of the served
// mix by a third and its p50 by an eighth.
constexpr double kDeadlineServiceFactor = 2.0;

double request_deadline(const bsar_server* s, const Req* r)
{
    const double arrival = std::chrono::duration<double>(r->t_submit - s->t_start).count();
    return arrival + kDeadlineServiceFactor * r->voxel_pulses / std::max(s->rate_est, 1.0);
}

// Batch into slot `b`: the admitted requests' remaining work items in deadline order,
// then ordered longest first (a tile's cost follows its request's pulse count) so the
// persistent kernel's dynamic work counter ends the batch evenly.
int build_batch(bsar_server* s, ServeBatch& b, int* W_out)
{
    int n = 0, W = -1;
    std::vector<Req*> live;
    for (Req* r : s->active)
        if (r->next_tile < r->ntiles) live.push_back(r);
    b.items.clear();
    if (live.empty()) return 0;
    struct Item {
        int np, slot, tile;
    };
    std::vector<Item> list;
    std::map<Req*, int64_t> per_req;
    std::stable_sort(live.begin(), live.end(), [](const Req* x, const Req* y) { return x->deadline_s < y->deadline_s; });
    // one node-scan width per batch, the earliest deadline's: each width runs its own kernel
    // instantiation (the per-warp table scan), so a request's image does not depend on the
    // widths of the requests it is batched with; other widths go to the next batch
    const int W0 = live.front()->rec.a.W;
    for (Req* r : live) {
        if (r->rec.a.W != W0) continue;
        const int64_t take = std::min<int64_t>(r->ntiles - r->next_tile, (int64_t)(s->max_tiles - n));
        // a work item's cost follows the pulses of its chunk
        const int cost = r->rec.a.np / std::max(1, r->chunks.nchunk);
        for (int64_t t = 0; t < take; t++) list.push_back({cost, r->slot, (int)(r->next_tile + t)});
        if (take > 0) {
            n += (int)take;
            r->next_tile += take;
            per_req[r] += take;
            W = W0;
        }
        if (n >= s->max_tiles) break;
    }
    b.voxel_pulses = 0;
    for (const auto& it : per_req)
        b.voxel_pulses += (double)it.second * 128.0 * it.first->rec.a.np / std::max(1, it.first->chunks.nchunk);
    std::stable_sort(list.begin(), list.end(), [](const Item& x, const Item& y) { return x.np > y.np; });
    for (int k = 0; k < n; k++) b.h_tiles[k] = make_int2(list[k].slot, list[k].tile);
    for (Req* r : s->active) {
        b.h_reqs[r->slot] = r->rec;
        b.h_chunks[r->slot] = r->chunks;
    }
    *b.h_ntiles = n;
    for (Req* r : s->active)
        if (per_req.count(r)) b.items.push_back({r, per_req[r]});
    bool chunked = false;
    for (const auto& it : b.items) chunked = chunked || it.first->chunks.nchunk > 1;
    *W_out = W | (chunked ? kChunkedKey : 0);
    return n;
}

// Captured graph of one batch launch: staging copies, counter reset, persistent kernel.
cudaGraphExec_t batch_graph(bsar_server* s, ServeBatch& bt, int W)
{
    auto it = bt.graphs.find(W);
    if (it != bt.graphs.end()) return it->second;
    MixedBatch b{bt.d_reqs->as<MixedReq>(), bt.d_tiles->as<int2>(), bt.d_ntiles->as<int>(), 0,
                 bt.d_counter->as<int>(), s->ctx->status->as<int>(), bt.d_chunks->as<MixedChunks>(),
                 (long long)s->ctx->tile_wait_polls};
    cudaGraph_t g = nullptr;
    cuda_check(cudaStreamBeginCapture(bt.st, cudaStreamCaptureModeThreadLocal), "begin capture");
    cudaMemcpyAsync(bt.d_reqs->p, bt.h_reqs, sizeof(MixedReq) * kMaxSlots, cudaMemcpyHostToDevice, bt.st);
    cudaMemcpyAsync(bt.d_chunks->p, bt.h_chunks, sizeof(MixedChunks) * kMaxSlots, cudaMemcpyHostToDevice, bt.st);
    cudaMemcpyAsync(bt.d_tiles->p, bt.h_tiles, sizeof(int2) * s->max_tiles, cudaMemcpyHostToDevice, bt.st);
    cudaMemcpyAsync(bt.d_ntiles->p, bt.h_ntiles, sizeof(int), cudaMemcpyHostToDevice, bt.st);
    cudaMemsetAsync(bt.d_counter->p, 0, sizeof(int), bt.st);
    cudaError_t le = launch_bp_mixed(b, W & ~kChunkedKey, s->grid_ctas, bt.st, (W & kChunkedKey) != 0);
    cudaError_t ce = cudaStreamEndCapture(bt.st, &g);
    cuda_check(le, "batch launch (capture)");
    cuda_check(ce, "end capture");
    cudaGraphExec_t exec = nullptr;
    cuda_check(cudaGraphInstantiate(&exec, g, 0), "graph instantiate");
    cudaGraphDestroy(g);
    bt.graphs[W] = exec;
    return exec;
}

void launch_batch(bsar_server* s, ServeBatch& bt, int W, int n)
{
    if (s->opts.use_graph) {
        cuda_check(cudaGraphLaunch(batch_graph(s, bt, W), bt.st), "graph launch");
    } else {
        MixedBatch b{bt.d_reqs->as<MixedReq>(), bt.d_tiles->as<int2>(), nullptr, n, bt.d_counter->as<int>(),
                     s->ctx->status->as<int>(), bt.d_chunks->as<MixedChunks>(), (long long)s->ctx->tile_wait_polls};
        cuda_check(cudaMemcpyAsync(bt.d_reqs->p, bt.h_reqs, sizeof(MixedReq) * kMaxSlots, cudaMemcpyHostToDevice, bt.st),
                   "h2d");
        cuda_check(cudaMemcpyAsync(bt.d_chunks->p, bt.h_chunks, sizeof(MixedChunks) * kMaxSlots, cudaMemcpyHostToDevice,
                                   bt.st),
                   "h2d");
        cuda_check(cudaMemcpyAsync(bt.d_tiles->p, bt.h_tiles, sizeof(int2) * n, cudaMemcpyHostToDevice, bt.st), "h2d");
        cuda_check(cudaMemsetAsync(bt.d_counter->p, 0, sizeof(int), bt.st), "memset");
        cuda_check(launch_bp_mixed(b, W & ~kChunkedKey, std::min(n, s->grid_ctas), bt.st, (W & kChunkedKey) != 0),
                   "batch launch");
    }
    cuda_check(cudaEventRecord(bt.ev, bt.st), "event");
    bt.t_launch = Clock::now();
    bt.inflight = true;
    bt.seq = ++s->batch_seq;
    s->launches++;
    s->tiles += n;
}

// Admits the oldest pending request if budget and slots allow (I/O thread; server lock
// held on entry and exit, released around the device work).  Returns true if it took a
// request.
bool admit_one(bsar_server* s, std::unique_lock<std::mutex>& lk)
{
    if (s->pending.empty() || s->stop || !s->fatal.empty()) return false;
    Req* r = s->pending.front();
    const uint64_t need = estimate_bytes(*r);
    int slot = -1;
    for (int k = 0; k < s->opts.max_inflight; k++)
        if (!s->slot_used[k]) {
            slot = k;
            break;
        }
    if (slot < 0) return false;
    if (s->reserved + need > s->budget && !s->active.empty()) return false;
    s->pending.pop_front();
    s->slot_used[slot] = true;
    r->slot = slot;
    r->reserved = need;
    s->reserved += need;
    s->peak_reserved = std::max(s->peak_reserved, s->reserved);
    lk.unlock();
    bsar_status st = BSAR_OK;
    std::string err;
    try {
        if (need > s->budget)
            fail(BSAR_ERR_OOM_BUDGET, "request needs %llu bytes, the server budget is %llu", (unsigned long long)need,
                 (unsigned long long)s->budget);
        admit(s, r);
    } catch (const Error& e) {
        st = e.status;
        err = e.msg;
    } catch (const std::bad_alloc&) {
        st = BSAR_ERR_OOM_BUDGET;
        err = "host allocation failed";
    }
    if (st != BSAR_OK) release(s, r);
    lk.lock();
    if (st == BSAR_OK && (r->cancelled || !s->fatal.empty())) {   // cancelled, or the server stopped,
        lk.unlock();                                                // while it was being admitted
        release(s, r);
        lk.lock();
        st = r->cancelled ? BSAR_ERR_CANCELLED : s->fatal_status;
        err = r->cancelled ? "cancelled" : s->fatal;
    }
    if (st == BSAR_OK) {
        r->state = St::Active;
        r->deadline_s = request_deadline(s, r);
        s->active.push_back(r);
        s->peak_inflight = std::max<uint64_t>(s->peak_inflight, s->active.size());
    } else {
        finish(s, r, st, err);
        s->cv_done.notify_all();
    }
    return true;
}

// Waits (bounded) for batch `bt`.  Lock held on entry and exit, released while it polls.
// Returns an empty string, or why the batch failed.
std::string wait_batch(bsar_server* s, ServeBatch& bt, std::unique_lock<std::mutex>& lk)
{
    const auto t0 = Clock::now();
    for (;;) {
        cudaError_t e = cudaEventQuery(bt.ev);
        if (e == cudaSuccess) return std::string();
        if (e != cudaErrorNotReady) return std::string("batch: ") + cudaGetErrorString(e);
        if (std::chrono::duration<double>(Clock::now() - t0).count() > s->batch_timeout_s) {
            s->fatal_status = BSAR_ERR_TIMEOUT;
            return "a batch did not finish within its time limit";
        }
        lk.unlock();
        std::this_thread::sleep_for(std::chrono::microseconds(50));
        lk.lock();
    }
}

// Completes the admitted requests that need no more work (worker thread; server lock held
// on entry and exit): each image is read back on the server's own stream, without the
// context lock, so a running admission does not hold it up; the request completes at
// once and its device buffers go to the I/O thread for release.
void retire_finished(bsar_server* s, std::unique_lock<std::mutex>& lk)
{
    std::vector<Req*> done;
    for (Req* r : s->active)
        if (r->done_tiles >= r->ntiles) done.push_back(r);
    if (done.empty()) return;
    for (Req* r : done) s->active.erase(std::find(s->active.begin(), s->active.end(), r));
    lk.unlock();
    std::vector<std::pair<bsar_status, std::string>> out(done.size(), {BSAR_OK, std::string()});
    for (size_t k = 0; k < done.size(); k++) {
        Req* r = done[k];
        if (r->cancelled) {
            out[k] = {BSAR_ERR_CANCELLED, "cancelled"};
            continue;
        }
        cudaError_t e = cudaMemcpyAsync(r->image_out, r->image->p, r->image->bytes, cudaMemcpyDeviceToHost, s->ret);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s->ret);
        if (e != cudaSuccess) out[k] = {BSAR_ERR_CUDA, std::string("image d2h: ") + cudaGetErrorString(e)};
    }
    lk.lock();
    for (size_t k = 0; k < done.size(); k++) {
        finish(s, done[k], out[k].first, out[k].second, true);
        s->to_free.push_back(done[k]);
    }
    s->cv_done.notify_all();
    s->cv_io.notify_all();
}

// Releases the device buffers of finished requests and returns their budget (I/O thread;
// server lock held on entry and exit).  Returns true if there were any.
bool free_finished(bsar_server* s, std::unique_lock<std::mutex>& lk)
{
    if (s->to_free.empty()) return false;
    std::vector<Req*> v;
    v.swap(s->to_free);
    lk.unlock();
    for (Req* r : v) release(s, r);
    lk.lock();
    for (Req* r : v) {
        s->reserved -= r->reserved;
        r->reserved = 0;
    }
    return true;
}

// The I/O thread: releases finished requests' buffers first (they return budget), then
// admits the oldest pending request; admission's device work waits for SM slots behind
// the running batch, and the worker keeps launching batches meanwhile.
void io_main(bsar_server* s)
{
    cudaSetDevice(s->ctx->device);
    std::unique_lock<std::mutex> lk(s->mu);
    while (!s->stop) {
        const bool freed = free_finished(s, lk);
        const bool took = admit_one(s, lk);
        if (took) s->cv_work.notify_all();
        if (!freed && !took) s->cv_io.wait_for(lk, std::chrono::milliseconds(2));
    }
}

void worker_main(bsar_server* s)
{
    cudaSetDevice(s->ctx->device);
    std::unique_lock<std::mutex> lk(s->mu);
    while (!s->stop) {
        // 1. fill the idle batch slots
        try {
            for (ServeBatch& bt : s->batch) {
                if (bt.inflight) continue;
                int W = 0;
                const int n = build_batch(s, bt, &W);
                // no context lock: the launch touches only the server's own buffers and
                // streams, so it does not wait for an admission that holds the context
                if (n > 0) launch_batch(s, bt, W, n);
            }
        } catch (const Error& e) {
            s->fatal = e.msg;
            break;
        }
        ServeBatch* old = nullptr;
        for (ServeBatch& bt : s->batch)
            if (bt.inflight && (!old || bt.seq < old->seq)) old = &bt;
        if (!old) {
            // nothing on the device: retire what needs no more work (cancelled requests),
            // or sleep until the I/O thread admits work
            retire_finished(s, lk);
            s->cv_work.wait_for(lk, std::chrono::milliseconds(2));
            continue;
        }
        // 2. wait for the older batch (the I/O thread admits meanwhile)
        std::string err = wait_batch(s, *old, lk);
        if (!err.empty()) {
            s->fatal = err;
            break;
        }
        old->inflight = false;
        // a bounded device wait that ran out: drain the other batch, fail both batches' requests
        std::string serr;
        try {
            check_device_status(s->ctx);     // synchronous copies of the context's status word
        } catch (const Error& e) {
            serr = e.msg;
        }
        if (!serr.empty()) {
            std::vector<Req*> bad;
            for (auto& p : old->items) bad.push_back(p.first);
            for (ServeBatch& bt : s->batch)
                if (bt.inflight) {
                    std::string e2 = wait_batch(s, bt, lk);
                    if (!e2.empty()) s->fatal = e2;
                    bt.inflight = false;
                    for (auto& p : bt.items) bad.push_back(p.first);
                }
            if (!s->fatal.empty()) break;
            std::sort(bad.begin(), bad.end());
            bad.erase(std::unique(bad.begin(), bad.end()), bad.end());
            for (Req* r : bad) {
                s->active.erase(std::find(s->active.begin(), s->active.end(), r));
                lk.unlock();
                release(s, r);
                lk.lock();
                finish(s, r, BSAR_ERR_TIMEOUT, serr);
            }
            s->cv_done.notify_all();
            continue;
        }
        {
            // throughput of the batch just finished: its work over the time since it started
            // or since the previous batch finished, whichever is later
            const auto now = Clock::now();
            const auto from = std::max(old->t_launch, s->t_last_batch_done);
            const double dt = std::chrono::duration<double>(now - from).count();
            if (dt > 1e-4 && old->voxel_pulses > 0) s->rate_est = 0.8 * s->rate_est + 0.2 * (old->voxel_pulses / dt);
            if (dt > 0) s->batch_busy_s += dt;    // the intervals [from, now] do not overlap
            s->t_last_batch_done = now;
        }
        for (auto& p : old->items) p.first->done_tiles += p.second;
        old->items.clear();
        retire_finished(s, lk);
    }
    // fail whatever is left (device buffers are released by bsar_server_destroy after
    // the batch streams are synchronised)
    const std::string why = s->fatal.empty() ? "server stopped" : s->fatal;
    const bsar_status st = s->fatal.empty() ? BSAR_ERR_CUDA : s->fatal_status;
    for (Req* r : s->active) finish(s, r, st, why);
    s->active.clear();
    for (Req* r : s->pending) finish(s, r, st, why);
    s->pending.clear();
    s->cv_done.notify_all();
}

double percentile(std::vector<double> v, double p)
{
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    double idx = p * (double)(v.size() - 1);
    size_t lo = (size_t)idx;
    size_t hi = std::min(lo + 1, v.size() - 1);
    return v[lo] + (idx - (double)lo) * (v[hi] - v[lo]);
}

}  // namespace

extern "C" {

bsar_status bsar_server_create(bsar_ctx* ctx, const bsar_server_opts* opts, bsar_server** out)
{
    if (!ctx || !out) return BSAR_ERR_INVALID_ARG;
    *out = nullptr;
    auto s = std::make_unique<bsar_server>();
    s->ctx = ctx;
    if (opts) s->opts = *opts;
    if (s->opts.max_inflight <= 0) s->opts.max_inflight = 64;
    if (s->opts.max_inflight > kMaxSlots) return BSAR_ERR_INVALID_ARG;
    if (!(s->opts.batch_timeout_s >= 0.0)) return BSAR_ERR_INVALID_ARG;
    if (s->opts.batch_timeout_s > 0.0) s->batch_timeout_s = s->opts.batch_timeout_s;
    std::lock_guard<std::mutex> lk(ctx->mu);
    try {
        cuda_check(cudaSetDevice(ctx->device), "cudaSetDevice");
        s->grid_ctas = mixed_grid_ctas();
        s->max_tiles = s->opts.tiles_per_launch > 0 ? s->opts.tiles_per_launch : 2 * s->grid_ctas;
        const uint64_t free_budget = ctx->budget > ctx->used ? ctx->budget - ctx->used : 0;
        s->budget = s->opts.hbm_budget_bytes ? s->opts.hbm_budget_bytes : (uint64_t)(0.9 * (double)free_budget);
        if (!ctx->pool) {
            cudaMemPoolProps pp = {};
            pp.allocType = cudaMemAllocationTypePinned;
            pp.location.type = cudaMemLocationTypeDevice;
            pp.location.id = ctx->device;
            cuda_check(cudaMemPoolCreate(&ctx->pool, &pp), "memory pool");
            uint64_t keep = ~0ull;     // keep freed blocks for the next admission
            cuda_check(cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &keep), "pool attribute");
        }
        // the batch records and the status word are used from the batch streams: plain
        // device allocations, not stream-ordered ones on the context's stream
        const bool saved_pool = ctx->use_pool;
        ctx->use_pool = false;
        struct RestorePool {
            bsar_ctx* c;
            bool v;
            ~RestorePool() { c->use_pool = v; }
        } restore_pool{ctx, saved_pool};
        // admission outranks the batches: its kernels take the SM slots the batch CTAs
        // free before the queued batch does, so a request is ready for the next batch
        int least = 0, greatest = 0;
        cuda_check(cudaDeviceGetStreamPriorityRange(&least, &greatest), "stream priorities");
        cuda_check(cudaStreamCreateWithPriority(&s->io, cudaStreamNonBlocking, greatest), "stream");
        cuda_check(cudaStreamCreateWithPriority(&s->ret, cudaStreamNonBlocking, greatest), "stream");
        for (ServeBatch& bt : s->batch) {
            cuda_check(cudaStreamCreateWithPriority(&bt.st, cudaStreamNonBlocking, least), "stream");
            cuda_check(cudaEventCreateWithFlags(&bt.ev, cudaEventDisableTiming), "event");
            cuda_check(cudaMallocHost((void**)&bt.h_reqs, sizeof(MixedReq) * kMaxSlots), "pinned");
            cuda_check(cudaMallocHost((void**)&bt.h_chunks, sizeof(MixedChunks) * kMaxSlots), "pinned");
            std::memset(bt.h_chunks, 0, sizeof(MixedChunks) * kMaxSlots);
            cuda_check(cudaMallocHost((void**)&bt.h_tiles, sizeof(int2) * s->max_tiles), "pinned");
            cuda_check(cudaMallocHost((void**)&bt.h_ntiles, sizeof(int)), "pinned");
            std::memset(bt.h_reqs, 0, sizeof(MixedReq) * kMaxSlots);
            bt.d_reqs = dev_alloc(ctx, sizeof(MixedReq) * kMaxSlots);
            bt.d_chunks = dev_alloc(ctx, sizeof(MixedChunks) * kMaxSlots);
            bt.d_tiles = dev_alloc(ctx, sizeof(int2) * s->max_tiles);
            bt.d_ntiles = dev_alloc(ctx, sizeof(int));
            bt.d_counter = dev_alloc(ctx, sizeof(int));
        }
        if (!ctx->status) {
            ctx->status = dev_alloc(ctx, sizeof(int));
            cuda_check(cudaMemset(ctx->status->p, 0, sizeof(int)), "memset");
        }
    } catch (const Error& e) {
        set_error(ctx, e.msg);
        return e.status;
    }
    bsar_server* raw = s.release();
    raw->worker = std::thread(worker_main, raw);
    raw->io_thread = std::thread(io_main, raw);
    *out = raw;
    return BSAR_OK;
}

bsar_status bsar_server_submit(bsar_server* s, const bsar_request* q, bsar_request_id* out)
{
    if (!s || !q || !out) return BSAR_ERR_INVALID_ARG;
    auto r = std::make_unique<Req>();
    const bsar_scene_desc& d = q->scene;
    const int64_t np = d.n_pulses;
    if (np < 1 || !d.tx || !d.rx || d.dem.nx < 2 || d.dem.ny < 2 || !d.dem.x_vec || !d.dem.y_vec || !d.dem.z)
        return BSAR_ERR_INVALID_ARG;
    if (!q->image_out) return BSAR_ERR_INVALID_ARG;
    try {
        check_grid(&q->grid);          // sizes bounded before any product is formed
    } catch (const Error&) {
        return BSAR_ERR_INVALID_ARG;
    }
    if (q->opts.flags & ~BSAR_BP_EXHAUSTIVE_SCAN) return BSAR_ERR_INVALID_ARG;
    if (q->opts.solver != BSAR_SOLVER_NEWTON || q->opts.legs != BSAR_LEGS_PER_PULSE ||
        (q->opts.precision != BSAR_MIXED && q->opts.precision != BSAR_MIXED_FP16))
        return BSAR_ERR_UNSUPPORTED;
    if (!d.samples && (q->n_scat < 0 || (q->n_scat > 0 && (!q->scat_pos || !q->scat_amp))))
        return BSAR_ERR_INVALID_ARG;
    r->dem_x.assign(d.dem.x_vec, d.dem.x_vec + d.dem.nx);
    r->dem_y.assign(d.dem.y_vec, d.dem.y_vec + d.dem.ny);
    r->dem_z.assign(d.dem.z, d.dem.z + d.dem.nx * d.dem.ny);
    r->tx.assign(d.tx, d.tx + 3 * np);
    r->rx.assign(d.rx, d.rx + 3 * np);
    r->gx.assign(q->grid.x_axis, q->grid.x_axis + q->grid.nx);
    r->gy.assign(q->grid.y_axis, q->grid.y_axis + q->grid.ny);
    r->gz.assign(q->grid.z_axis, q->grid.z_axis + q->grid.nz);
    if (!d.samples && q->n_scat > 0) {
        r->spos.assign(q->scat_pos, q->scat_pos + 3 * q->n_scat);
        r->samp.assign(q->scat_amp, q->scat_amp + q->n_scat);
    }
    r->desc = d;
    r->desc.dem.x_vec = r->dem_x.data();
    r->desc.dem.y_vec = r->dem_y.data();
    r->desc.dem.z = r->dem_z.data();
    r->desc.tx = r->tx.data();
    r->desc.rx = r->rx.data();
    r->grid = q->grid;
    r->opts = q->opts;
    r->n_scat = d.samples ? 0 : q->n_scat;
    r->snr_db = q->snr_db;
    r->seed = q->seed;
    r->image_out = q->image_out;
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return BSAR_ERR_CUDA;
    if (!s->fatal.empty()) return s->fatal_status;
    r->id = s->next_id++;
    r->t_submit = Clock::now();
    if (!s->any_submit) {
        s->any_submit = true;
        s->t_first = r->t_submit;
    }
    s->submitted++;
    *out = r->id;
    s->pending.push_back(r.get());
    s->reqs[r->id] = std::move(r);
    s->cv_io.notify_all();
    return BSAR_OK;
}

bsar_status bsar_server_estimate(const bsar_request* q, uint64_t* bytes)
{
    if (!q || !bytes) return BSAR_ERR_INVALID_ARG;
    Req r;
    r.desc = q->scene;
    r.grid = q->grid;
    r.opts = q->opts;
    r.n_scat = q->scene.samples ? 0 : q->n_scat;
    *bytes = estimate_bytes(r);
    return BSAR_OK;
}

bsar_status bsar_server_poll(bsar_server* s, bsar_request_id id, int32_t* done, double* latency_ms)
{
    if (!s || !done) return BSAR_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return BSAR_ERR_NOT_FOUND;
    Req* r = it->second.get();
    *done = (r->state == St::Done || r->state == St::Failed) ? 1 : 0;
    if (!*done) return BSAR_OK;
    if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
    return r->status;
}

bsar_status bsar_server_wait(bsar_server* s, bsar_request_id id, double timeout_s, double* latency_ms)
{
    if (!s) return BSAR_ERR_INVALID_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return BSAR_ERR_NOT_FOUND;
    Req* r = it->second.get();
    const auto deadline = Clock::now() + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(timeout_s));
    while (r->state != St::Done && r->state != St::Failed) {
        if (s->cv_done.wait_until(lk, deadline) == std::cv_status::timeout &&
            r->state != St::Done && r->state != St::Failed)
            return BSAR_ERR_TIMEOUT;
    }
    if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
    return r->status;
}

bsar_status bsar_server_cancel(bsar_server* s, bsar_request_id id)
{
    if (!s) return BSAR_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return BSAR_ERR_NOT_FOUND;
    Req* r = it->second.get();
    if (r->state == St::Done || r->state == St::Failed) return BSAR_ERR_NOT_FOUND;
    r->cancelled = true;
    auto p = std::find(s->pending.begin(), s->pending.end(), r);
    if (p != s->pending.end()) {
        s->pending.erase(p);
        finish(s, r, BSAR_ERR_CANCELLED, "cancelled");
        s->cv_done.notify_all();
        return BSAR_OK;
    }
    // admitted (or being admitted): no further work items; the worker completes it when the
    // items already on the device are done
    if (r->state == St::Active) r->ntiles = r->next_tile;
    s->cv_work.notify_all();
    s->cv_io.notify_all();
    return BSAR_OK;
}

bsar_status bsar_server_get_stats(bsar_server* s, bsar_server_stats* o)
{
    if (!s || !o) return BSAR_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    o->submitted = s->submitted;
    o->completed = s->completed;
    o->failed = s->failed;
    o->launches = s->launches;
    o->tiles = s->tiles;
    o->p50_ms = percentile(s->latencies, 0.50);
    o->p99_ms = percentile(s->latencies, 0.99);
    double sum = 0, mx = 0;
    for (double v : s->latencies) {
        sum += v;
        mx = std::max(mx, v);
    }
    o->mean_ms = s->latencies.empty() ? 0.0 : sum / s->latencies.size();
    o->max_ms = mx;
    o->voxel_pulses = s->vp_done;
    o->busy_s = s->completed ? std::chrono::duration<double>(s->t_last - s->t_first).count() : 0.0;
    o->peak_inflight = s->peak_inflight;
    o->peak_reserved_bytes = s->peak_reserved;
    o->batch_busy_s = s->batch_busy_s;
    return BSAR_OK;
}

void bsar_server_destroy(bsar_server* s)
{
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->cv_work.notify_all();
        s->cv_io.notify_all();
    }
    if (s->worker.joinable()) s->worker.join();
    if (s->io_thread.joinable()) s->io_thread.join();
    {
        std::lock_guard<std::mutex> lk(s->ctx->mu);
        cudaSetDevice(s->ctx->device);
        for (ServeBatch& bt : s->batch)
            if (bt.st) cudaStreamSynchronize(bt.st);
        if (s->io) cudaStreamSynchronize(s->io);
        cudaStream_t saved = s->ctx->stream;
        s->ctx->stream = s->io ? s->io : saved;     // pooled request buffers are released on `io`
        for (auto& kv : s->reqs) {
            kv.second->scene.reset();
            kv.second->axes.reset();
            kv.second->image.reset();
            kv.second->partial.reset();
            kv.second->tile_done.reset();
        }
        if (s->io) cudaStreamSynchronize(s->io);
        s->ctx->stream = saved;
        for (ServeBatch& bt : s->batch) {
            for (auto& kv : bt.graphs) cudaGraphExecDestroy(kv.second);
            bt.d_reqs.reset();
            bt.d_chunks.reset();
            bt.d_tiles.reset();
            bt.d_ntiles.reset();
            bt.d_counter.reset();
            if (bt.h_reqs) cudaFreeHost(bt.h_reqs);
            if (bt.h_chunks) cudaFreeHost(bt.h_chunks);
            if (bt.h_tiles) cudaFreeHost(bt.h_tiles);
            if (bt.h_ntiles) cudaFreeHost(bt.h_ntiles);
            if (bt.ev) cudaEventDestroy(bt.ev);
            if (bt.st) cudaStreamDestroy(bt.st);
        }
        if (s->io) cudaStreamDestroy(s->io);
        if (s->ret) {
            cudaStreamSynchronize(s->ret);
            cudaStreamDestroy(s->ret);
        }
    }
    delete s;
}

}  // extern "C"
