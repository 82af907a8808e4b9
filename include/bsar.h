/*
 * bsar.h -- C ABI of the B200 bistatic SAR back-projection library (libbsar.so).
 *
 * Drop-in boundary for the hot path of DavidAtenciaMondragon/c-_bistatic_sar:
 * pulse compression (fft_utils) -> x4 Hermite fast-time upsampling (interpolation)
 * -> Fermat refraction solve (raw_data_processing) -> back-projection (the voxel
 * loop inline in proc_test_script.cpp).  Each entry point below names the reference
 * function or code block it replaces (path:line inside the reference project).
 *
 * Conventions
 *   - Plain pointers and sizes only.  Complex arrays are interleaved (re, im) double
 *     pairs; point arrays are n x 3 row-major (x, y, z); pulses are pulse-major
 *     (sample s of pulse p at [p * n + s]).
 *   - Host buffers are caller-owned and only read / written during the call; device
 *     memory is owned by the context.  The context takes it from its own stream-ordered
 *     pool (cudaMallocFromPoolAsync on the context's stream), which keeps freed blocks
 *     for later calls until bsar_destroy; bsar_bytes_in_use counts the live buffers.
 *     Every call is synchronous unless its name ends in _device.
 *   - Every entry point returns a bsar_status; bsar_last_error(ctx) gives the message of
 *     the calling thread's latest call on ctx (empty after a success), so threads that
 *     share a context each read their own failure.  The string stays valid until that
 *     thread's next call on ctx.
 *     There is no CPU fallback: without a usable CUDA device bsar_create fails.
 *   - A context is internally locked; calls from several threads are serialised.
 */
#ifndef BSAR_H
#define BSAR_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BSAR_ABI_VERSION 1

typedef enum bsar_status {
    BSAR_OK = 0,
    BSAR_ERR_INVALID_ARG = 1,  /* malformed sizes, null pointers, non-finite geometry */
    BSAR_ERR_OOM_BUDGET = 2,   /* the request does not fit the context's HBM budget  */
    BSAR_ERR_TIMEOUT = 3,      /* a bounded device-side wait ran out                 */
    BSAR_ERR_CUDA = 4,         /* a CUDA runtime error (message in bsar_last_error)  */
    BSAR_ERR_NOT_FOUND = 5,    /* unknown scene or request id                        */
    BSAR_ERR_UNSUPPORTED = 6,  /* a valid request outside what this build implements */
    BSAR_ERR_QUEUE_FULL = 7,   /* serving: no admission slot right now               */
    BSAR_ERR_CANCELLED = 8     /* serving: the request was cancelled                 */
} bsar_status;

/* Fermat crossing-point solver. */
typedef enum bsar_solver {
    BSAR_SOLVER_GRID = 0,   /* the reference's 5-level 709-point grid search,
                               src/raw_data_processing.cpp:455-572 (bit-exact in FP64) */
    BSAR_SOLVER_NEWTON = 1  /* node scan + Newton on the bilinear DEM facets           */
} bsar_solver;

/* Leg distances R1t / R1r used by back-projection. */
typedef enum bsar_legs {
    BSAR_LEGS_MEAN = 0,      /* mean over all pulses, as shipped (proc_test_script.cpp:518-548) */
    BSAR_LEGS_PER_PULSE = 1  /* r1Tx / r1Rx of the pulse itself (src/raw_data_processing.cpp:197-215) */
} bsar_legs;

typedef enum bsar_precision {
    BSAR_FP64 = 0,        /* plain: FP64 delays, FP64 complex samples and sums            */
    BSAR_MIXED = 1,       /* FP32 differential delays vs an FP64 per-pulse reference range,
                             complex64 samples, Kahan-compensated FP32 sums               */
    BSAR_MIXED_FP16 = 2   /* as MIXED, samples stored FP16 complex with an FP32 pulse scale */
} bsar_precision;

typedef struct bsar_ctx bsar_ctx;
typedef uint64_t bsar_scene_id;

typedef struct bsar_opts {
    int32_t device;             /* CUDA device ordinal                                  */
    int32_t flags;              /* reserved, must be 0                                  */
    uint64_t hbm_budget_bytes;  /* device bytes the context may hold; 0 = 90 % of free */
} bsar_opts;

/* ProcessedDEM (reference include/radar_params.h:75-79): X_vec, Y_vec, Z_DEM[y][x].
 * nx == 0 or ny == 0 is an empty DEM (flat surface z = 0, src/raw_data_processing.cpp:616-618).
 * z holds ny * nx heights, z[j * nx + i] = Z_DEM[j][i]; pack a ragged Z_DEM with 0.0
 * where the reference would find no entry (:649-652). */
typedef struct bsar_dem {
    int64_t nx, ny;
    const double* x_vec;
    const double* y_vec;
    const double* z;
} bsar_dem;

typedef struct bsar_fermat_opts {
    int32_t solver;          /* bsar_solver                                                */
    int32_t precision;       /* BSAR_FP64, or BSAR_MIXED (FP32 scan + FP64 final step)     */
    double search_radius_m;  /* Newton node-scan radius around the flat-interface start;
                                <= 0 selects 1.5 m                                         */
} bsar_fermat_opts;

/* ---------------------------------------------------------------------------------
 * Context
 * ------------------------------------------------------------------------------- */
bsar_status bsar_create(bsar_ctx** out, const bsar_opts* opts);
void bsar_destroy(bsar_ctx* ctx);
const char* bsar_status_string(bsar_status status);
const char* bsar_last_error(const bsar_ctx* ctx);
/* Use a caller-owned cudaStream_t for all work of this context (NULL = own stream). */
bsar_status bsar_set_stream(bsar_ctx* ctx, void* cuda_stream);
bsar_status bsar_synchronize(bsar_ctx* ctx);
/* Bounded wait of the mixed kernel for its DEM tile copies (TMA).  Node scans of half
 * width 12, and of widths without a kernel of their own, stage a tile; the 3 and 6 scans
 * read the DEM from global memory.  polls: polls of the copy's barrier before a CTA gives
 * up on the tile, reads the heights from global memory instead (the same values, so the
 * same image) and raises the context's status word, which the call then reports as
 * BSAR_ERR_TIMEOUT.  polls < 0 restores the default (2^24); 0 makes every wait run out
 * at once, with no fault and no hang (the copy that was started is still waited for
 * before the CTA exits).  Read when a launch is issued (a server reads it when it records
 * a batch launch). */
bsar_status bsar_set_tile_wait_limit(bsar_ctx* ctx, int64_t polls);
/* Number of this library's kernel launches issued by the context so far. */
uint64_t bsar_launch_count(const bsar_ctx* ctx);
/* Device bytes currently held by the context (scenes, work buffers). */
uint64_t bsar_bytes_in_use(const bsar_ctx* ctx);

/* ---------------------------------------------------------------------------------
 * Functional entry points: the reference functions, batched.
 * ------------------------------------------------------------------------------- */

/* interpolateDEMElevation, src/raw_data_processing.cpp:615-680, for n points (x, y)
 * (xy: n x 2) -> z_out[n].  Bit-exact with the reference. */
bsar_status bsar_dem_elevation(bsar_ctx* ctx, const bsar_dem* dem, const double* xy, int64_t n,
                               double* z_out);

/* calculateRefractionPoint, src/raw_data_processing.cpp:455-572, for n (start, end)
 * pairs (n x 3 each) with indices n1 (start side) and n2 (end side) -> points_out (n x 3).
 * fopts->precision BSAR_MIXED (Newton only) returns the mixed form's crossing points. */
bsar_status bsar_refraction_points(bsar_ctx* ctx, const bsar_dem* dem, const double* p_start,
                                   const double* p_end, int64_t n, double n1, double n2,
                                   const bsar_fermat_opts* fopts, double* points_out);

/* calculaSlantRangeFermat, src/raw_data_processing.cpp:112-255, for one target over
 * n_pulses Tx/Rx positions (n x 3).  ranges: 4 x n (r1Tx, r2Tx, r1Rx, r2Rx); refr_ida /
 * refr_volta: n x 3; reflection (n x 3, may be NULL): calculateReflectionPoint (:575-612). */
bsar_status bsar_slant_range_fermat(bsar_ctx* ctx, const bsar_dem* dem, const double* tx,
                                    const double* rx, int64_t n_pulses, const double* target,
                                    double n1, double n2, const bsar_fermat_opts* fopts,
                                    double* ranges, double* refr_ida, double* refr_volta,
                                    double* reflection);

/* splineInterpolation, src/interpolation.cpp:4-51, on `batch` pulses of n complex
 * samples -> batch x (n * factor).  Bit-exact with the reference; n must be >= 2. */
bsar_status bsar_spline_upsample(bsar_ctx* ctx, const double* in, int64_t n, int64_t batch,
                                 int32_t factor, double* out);

/* FFTProcessor::fft / ::ifft, src/fft_utils.cpp:11-61, in place on `batch` rows of n
 * complex samples.  As in the reference, a row whose length is not a power of two is
 * left unchanged (the call still returns BSAR_OK and records a message). */
bsar_status bsar_fft(bsar_ctx* ctx, double* data, int64_t n, int64_t batch, int32_t inverse);

/* FFTProcessor::fftCorrelation (conjugate = 1, src/fft_utils.cpp:63-101) or
 * ::fftConvolution (conjugate = 0, :103-138) of `batch` rows of n_signal samples against
 * one reference of n_reference samples; out: batch x max(n_signal, n_reference). */
bsar_status bsar_fft_correlate(bsar_ctx* ctx, const double* signal, int64_t n_signal,
                               int64_t batch, const double* reference, int64_t n_reference,
                               int32_t conjugate, double* out);

/* ---------------------------------------------------------------------------------
 * Resident scenes: DEM, trajectories and pulses stay in HBM between calls.
 * ------------------------------------------------------------------------------- */
typedef enum bsar_samples_kind {
    BSAR_SAMPLES_RAW = 0,        /* raw echoes: bsar_scene_compress runs pulse compression */
    BSAR_SAMPLES_COMPRESSED = 1  /* already range-compressed (rootData), not upsampled     */
} bsar_samples_kind;

typedef struct bsar_scene_desc {
    bsar_dem dem;
    int64_t n_pulses;          /* Np */
    const double* tx;          /* Np x 3 transmitter positions (Tx_positions.csv) */
    const double* rx;          /* Np x 3 receiver positions    (Rx_positions.csv) */
    int64_t n_samples;         /* Ns fast-time samples per pulse (a power of two for
                                  raw pulses)                                       */
    const double* samples;     /* Np x Ns complex, pulse-major                       */
    int32_t samples_kind;      /* bsar_samples_kind                                 */
    int32_t upsample;          /* fast-time factor (the reference uses 4,
                                  proc_test_script.cpp:220)                          */
    double n1, n2;             /* refractive indices above / below the surface      */
    double c;                  /* propagation speed (reference: 3e8)                */
    double fc;                 /* carrier frequency; lambda = c / fc                 */
    double fs;                 /* raw sampling rate; back-projection uses fs*upsample */
    double chirp_f0, chirp_f1; /* LFM chirp start / stop frequency (baseband)        */
    double chirp_T;            /* pulse duration                                    */
} bsar_scene_desc;

bsar_status bsar_scene_upload(bsar_ctx* ctx, const bsar_scene_desc* desc, bsar_scene_id* out);
bsar_status bsar_scene_release(bsar_ctx* ctx, bsar_scene_id scene);

/* Echo synthesis on the device (the simulator's processRawData, src/raw_data_processing.cpp:
 * 292-421, at the exact fractional delay): a resident raw scene is made from desc (whose
 * `samples` is ignored) and n_scat point scatterers (positions n x 3, amplitudes n).  Per
 * pulse and scatterer the FP64 Newton Fermat solve gives the two-way optical path L; the
 * pulse is sum_s a_s exp(-j 2 pi fc L/c) chirp(t - L/c) with the chirp centred on the
 * delay, plus complex Gaussian noise of variance Nc / 10^(snr_db/10) per sample (Nc the
 * chirp length; a non-finite snr_db adds none) drawn from a counter-based generator
 * seeded by `seed`. */
bsar_status bsar_scene_synthesize(bsar_ctx* ctx, const bsar_scene_desc* desc, const double* scat_pos,
                                  const double* scat_amp, int64_t n_scat, double snr_db, uint64_t seed,
                                  bsar_scene_id* out);
/* The same with flags.  BSAR_SYNTH_REFERENCE_BINS reproduces the simulator's envelope
 * placement: each echo's chirp is centred on sample 1 + round(t*fs)
 * (src/raw_data_processing.cpp:329) and wraps around the pulse like the simulator's
 * circular convolution with the fftshifted chirp (:371-406); the phase stays exact. */
enum { BSAR_SYNTH_REFERENCE_BINS = 1 };
bsar_status bsar_scene_synthesize_ex(bsar_ctx* ctx, const bsar_scene_desc* desc, const double* scat_pos,
                                     const double* scat_amp, int64_t n_scat, double snr_db, uint64_t seed,
                                     int32_t flags, bsar_scene_id* out);

/* Copy a scene's raw (or given compressed) pulses, Np x Ns complex, to the host. */
bsar_status bsar_scene_read_samples(bsar_ctx* ctx, bsar_scene_id scene, double* out);

/* Pulse compression + upsampling of a resident scene, one launch over all pulses:
 * rootData = IFFT(FFT(raw) . conj(FFT(reference))) per pulse (processRawData,
 * src/raw_data_processing.cpp:371-446) followed by the x`upsample` Hermite interpolation
 * (proc_test_script.cpp:326-350), stored for `precision` (FP64 / complex64 / FP16 +
 * scale).  For BSAR_SAMPLES_COMPRESSED scenes only the upsampling runs. */
bsar_status bsar_scene_compress(bsar_ctx* ctx, bsar_scene_id scene, int32_t precision);

/* Copy the scene's upsampled FP64 pulses (Np x Ns*upsample) to the host (diagnostics). */
bsar_status bsar_scene_read_upsampled(bsar_ctx* ctx, bsar_scene_id scene, double* out);

/* Copy the upsampled pulses as stored for `precision` (complex64, or FP16 complex times
 * the per-pulse scale), widened to complex128 (diagnostics; compresses when needed). */
bsar_status bsar_scene_read_stored(bsar_ctx* ctx, bsar_scene_id scene, int32_t precision, double* out);

typedef struct bsar_grid {
    int64_t nx, ny, nz;
    const double* x_axis;   /* grid_xAxis */
    const double* y_axis;   /* grid_yAxis */
    const double* z_axis;   /* grid_zAxis */
} bsar_grid;

typedef struct bsar_bp_opts {
    int32_t solver;          /* bsar_solver    */
    int32_t legs;            /* bsar_legs      */
    int32_t precision;       /* bsar_precision */
    int32_t flags;           /* 0 or BSAR_BP_EXHAUSTIVE_SCAN */
    double search_radius_m;  /* Newton node-scan radius (<= 0: 1.5 m) */
} bsar_bp_opts;

/* bsar_bp_opts.flags.  BSAR_BP_EXHAUSTIVE_SCAN: the mixed forms rank every node of each
 * Fermat node-scan window instead of skipping the rows and column groups that a lower
 * bound proves cannot hold the minimum.  The image is bit-identical either way; the flag
 * exists to verify that, at the cost of speed.  The FP64 forms always scan every node. */
enum { BSAR_BP_EXHAUSTIVE_SCAN = 1 };

/* The imager's voxel loop, proc_test_script.cpp:451-767: for every voxel the Fermat
 * solves of all pulses, the delays / phases (:559-577) and the interpolated, phase-
 * corrected sum (:583-669).  image_out: complex nx x ny x nz, z fastest -- the layout
 * of output[x][y][z] (:761-767).  Runs bsar_scene_compress first if the scene has not
 * been compressed for this precision. */
bsar_status bsar_backproject(bsar_ctx* ctx, bsar_scene_id scene, const bsar_grid* grid,
                             const bsar_bp_opts* opts, double* image_out);

/* A range of the imager's voxel loop: the voxels [v_begin, v_begin + v_count) of the
 * grid's flat order (z -> x -> y, y fastest; proc_test_script.cpp:132-151, the index the
 * OpenMP loop of :451 splits), written at their places in image_out, the full complex
 * nx x ny x nz image [x][y][z]; every other voxel is set to 0.  Per-pulse anchors and
 * pulse chunks are the whole grid's, so every voxel's value equals bsar_backproject's,
 * bit for bit: ranges computed on several devices add up to the one-device image (a
 * z-slab is one contiguous range). */
bsar_status bsar_backproject_range(bsar_ctx* ctx, bsar_scene_id scene, const bsar_grid* grid,
                                   const bsar_bp_opts* opts, int64_t v_begin, int64_t v_count, double* image_out);

/* As bsar_backproject, but asynchronous on the context stream with the image written to
 * device memory d_image (complex128, same layout); the grid axes are read at the call. */
bsar_status bsar_backproject_device(bsar_ctx* ctx, bsar_scene_id scene, const bsar_grid* grid,
                                    const bsar_bp_opts* opts, void* d_image);

/* No counterpart in the reference.  The mixed back-projection of bsar_backproject
 * (Newton, per-pulse legs, precision BSAR_MIXED or BSAR_MIXED_FP16) with no device
 * allocation, for callers that cannot allocate: programs whose GPU memory is owned by
 * another allocator (a framework's caching allocator, a client held to a memory limit),
 * where a cudaMalloc fails or makes that allocator release memory, and latency-critical
 * loops that cannot take the device-wide wait of a cudaFree.  Request record, work
 * counter, status word, anchors, grid axes and image live in one fixed 64 MiB scratch
 * array per device (a call that does not fit, beyond about 4M voxels, fails with
 * BSAR_ERR_INVALID_ARG).  The device commits the array when the module holding it
 * loads -- under CUDA's default lazy loading at the first call on that device, with
 * CUDA_MODULE_LOADING=EAGER at the library's first CUDA call -- and holds it until the
 * process exits.  That first call is therefore the one moment memory is taken: make it
 * before another allocator reserves the device's memory and before any stream capture,
 * or set CUDA_MODULE_LOADING=EAGER.  The scene must already hold samples for the
 * precision (bsar_scene_compress).  Calls that overlap in time on one device race on the
 * scratch. */
bsar_status bsar_backproject_mixed_noalloc(bsar_ctx* ctx, bsar_scene_id scene, const bsar_grid* grid,
                                           const bsar_bp_opts* opts, double* image_out);

/* ---------------------------------------------------------------------------------
 * Files around the path.
 * Matrix files use the reference's binary format (src/binary_reader.cpp:8-99, the
 * writers of src/data_export.cpp:71-138 and 180-309): uint32 dimension count, uint32
 * complex flag (1 = complex), uint32 type-name length, char[16] type name, uint64
 * dimensions, then doubles, real and imaginary interleaved for complex data.
 * ------------------------------------------------------------------------------- */
typedef struct bsar_matrix_header {
    uint32_t ndims;
    uint32_t is_complex;
    uint32_t dtype_len;         /* bytes of the type name kept (at most 16) */
    char dtype[17];             /* type name as stored (not interpreted: values are doubles) */
    uint64_t dims[8];
    uint64_t total;             /* product of the dimensions */
} bsar_matrix_header;

/* readBinary's header (binary_reader.cpp:18-60); BSAR_ERR_NOT_FOUND if the file does not
 * open, BSAR_ERR_INVALID_ARG if it is truncated. */
bsar_status bsar_matrix_read_header(const char* path, bsar_matrix_header* out);
/* readBinary<double> (binary_reader.cpp:8-95): `total` complex128 values into `out`
 * (real files get a zero imaginary part); fails when capacity < total or the file is short. */
bsar_status bsar_matrix_read(const char* path, double* out, uint64_t capacity);
/* exportComplexMatrix (data_export.cpp:71-138) for any rank: header with type "double",
 * then the values (complex128 when is_complex, else doubles).  Empty matrices are refused. */
bsar_status bsar_matrix_write(const char* path, uint32_t ndims, const uint64_t* dims, int32_t is_complex,
                              const double* data);

/* Pulse file -> resident scene.  The file is the 2-D matrix the simulator exports
 * (dims[0] fast-time samples, dims[1] pulses; the imager's reading,
 * proc_test_script.cpp:303-331).  desc supplies everything but the samples and
 * n_samples; desc->n_pulses must equal dims[1].  The values are streamed through pinned
 * memory to the device; BSAR_FILE_ROW_MAJOR transposes them there. */
enum { BSAR_FILE_AS_IMAGER = 0,   /* element (sample r, pulse p) at p*dims[0] + r, as the imager indexes it */
       BSAR_FILE_ROW_MAJOR = 1 }; /* element (r, p) at r*dims[1] + p, the matrix's own row-major layout */
bsar_status bsar_scene_upload_file(bsar_ctx* ctx, const bsar_scene_desc* desc, const char* path, int32_t layout,
                                   bsar_scene_id* out);

/* export3DComplexMatrix (data_export.cpp:180-309): image [x][y][z] (z fastest, the layout
 * bsar_backproject returns) written with x fastest, then y, then z; with all three axes
 * given, <path without extension>_grid_{x,y,z}.csv beside it as exportVector writes them. */
bsar_status bsar_image_export(const char* path, const double* image, int64_t nx, int64_t ny, int64_t nz,
                              const double* gx, const double* gy, const double* gz);
/* The same from a device image (bsar_backproject_device): permuted on the device. */
bsar_status bsar_image_export_device(bsar_ctx* ctx, const char* path, const void* d_image, int64_t nx, int64_t ny,
                                     int64_t nz, const double* gx, const double* gy, const double* gz);

/* loadDEM's ESRI ASCII grid (src/load_dem_simple.cpp:9-224): header keywords ncols,
 * nrows, xllcorner, yllcorner, cellsize, NODATA_value; the first other line starts the
 * grid; file row j gives y_vec[j] = yllcorner + j*cellsize (no north-up flip); missing
 * values read as NODATA.  A .tif name or an unreadable file gives the reference's
 * stand-in DEM (32 x 32 nodes over [-500, 500]^2 m, height 0) and a flag.  Call with
 * x_vec = y_vec = z = NULL to get nx, ny; then with buffers of that size (z ny x nx). */
enum { BSAR_DEM_FALLBACK_TIF = 1, BSAR_DEM_FALLBACK_UNREADABLE = 2, BSAR_DEM_ROWS_MISMATCH = 4 };
bsar_status bsar_dem_load_esri(const char* path, int64_t* nx, int64_t* ny, double* x_vec, double* y_vec, double* z,
                               int32_t* flags);

/* ---------------------------------------------------------------------------------
 * Serving: image-formation requests of different grids, pulse counts and DEMs are
 * admitted as they arrive (FIFO) against an HBM budget, by a thread of their own while
 * the batches run; each admitted request's scene stays resident while its voxel tiles
 * (128 voxels each) are packed with other requests' tiles into one persistent
 * mixed-kernel launch per batch (optionally a replayed CUDA graph), earliest deadline
 * first (arrival plus twice the request's own service time at the server's recent
 * throughput).  Requests that arrive while others run join the next batch.  A voxel's
 * result does not depend on what else shares its batch.
 * ------------------------------------------------------------------------------- */
typedef struct bsar_server bsar_server;
typedef uint64_t bsar_request_id;

typedef struct bsar_server_opts {
    uint64_t hbm_budget_bytes;  /* device bytes admitted requests may hold; 0 = 90 % of the
                                   context's remaining budget                              */
    int32_t max_inflight;       /* admitted requests at once (1..256; 0 = 64)             */
    int32_t tiles_per_launch;   /* work items per launch (0 = two waves of resident CTAs) */
    int32_t use_graph;          /* 1: every launch replays a captured CUDA graph           */
    int32_t reserved;
    double batch_timeout_s;     /* host-side limit on one batch's device time (0 = 300 s);
                                   when it runs out the server stops: the requests it holds
                                   fail with BSAR_ERR_TIMEOUT and later submissions are
                                   refused, and bsar_server_destroy still waits for the
                                   batches on the device before it frees their memory     */
} bsar_server_opts;

typedef struct bsar_request {
    bsar_scene_desc scene;      /* scene.samples == NULL: echoes synthesised on the device
                                   from the scatterers below (bsar_scene_synthesize)       */
    const double* scat_pos;     /* n_scat x 3 */
    const double* scat_amp;     /* n_scat     */
    int64_t n_scat;
    double snr_db;
    uint64_t seed;
    bsar_grid grid;
    bsar_bp_opts opts;          /* precision BSAR_MIXED or BSAR_MIXED_FP16 (Newton, per-pulse) */
    double* image_out;          /* nx*ny*nz complex128 [x][y][z], written on completion    */
} bsar_request;

typedef struct bsar_server_stats {
    uint64_t submitted, completed, failed, launches, tiles;
    double p50_ms, p99_ms, mean_ms, max_ms;   /* submission -> image on the host */
    double voxel_pulses;                      /* work of the completed requests   */
    double busy_s;                            /* first submission -> last completion */
    uint64_t peak_inflight;                   /* most requests admitted at once  */
    uint64_t peak_reserved_bytes;             /* most HBM reserved at once       */
    double batch_busy_s;                      /* time with a batch on the device, as the
                                                 server thread sees launches and completions */
} bsar_server_stats;

/* The server keeps `ctx` for itself until bsar_server_destroy (other calls on the same
 * context wait for its lock).  Small request arrays (DEM, trajectories, grid, scatterers)
 * are copied at submission; scene.samples and image_out must stay valid until the
 * request completes. */
bsar_status bsar_server_create(bsar_ctx* ctx, const bsar_server_opts* opts, bsar_server** out);
bsar_status bsar_server_submit(bsar_server* srv, const bsar_request* req, bsar_request_id* out);
/* Device bytes a request reserves against the server's budget while admitted (an upper
 * bound: it includes the pulse-chunk sums a small grid may use, computed without asking
 * the device).  A request above the whole budget fails with BSAR_ERR_OOM_BUDGET; smaller
 * ones wait. */
bsar_status bsar_server_estimate(const bsar_request* req, uint64_t* bytes);
/* done = 1 when the request finished; its status is the return value once done. */
bsar_status bsar_server_poll(bsar_server* srv, bsar_request_id id, int32_t* done, double* latency_ms);
/* Waits up to timeout_s (BSAR_ERR_TIMEOUT when it runs out). */
bsar_status bsar_server_wait(bsar_server* srv, bsar_request_id id, double timeout_s, double* latency_ms);
bsar_status bsar_server_get_stats(bsar_server* srv, bsar_server_stats* out);
/* Cancels a request: a queued one is dropped at once, an admitted one gets no further
 * work items and is released when the ones already on the device finish.  Either way it
 * completes with BSAR_ERR_CANCELLED, its image_out untouched, and the other requests are
 * unaffected.  BSAR_ERR_NOT_FOUND for unknown or already finished requests. */
bsar_status bsar_server_cancel(bsar_server* srv, bsar_request_id id);
void bsar_server_destroy(bsar_server* srv);

#ifdef __cplusplus
}
#endif

#endif /* BSAR_H */
