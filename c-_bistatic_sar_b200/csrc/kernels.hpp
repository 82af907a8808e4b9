// kernels.hpp -- launch interface between the host runtime (bsar_api.cpp) and the
// CUDA translation units.  Plain structs of device pointers and sizes.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "dev_view.hpp"

namespace bsar {

// ------------------------------- pulse / FFT ----------------------------------------
struct PulseArgs {
    const double2* in;   // batch x ns raw samples (complex128)
    int64_t batch;
    int ns;
    int P, logP;         // padded FFT length
    const void* tw;      // P/2 twiddles, real_bytes precision
    const void* tw_rf;   // FP32 register transforms (4096..16384 points): the twiddles of their
                         // second pass in lane order (rf_twiddle_count(P) entries, rf_twiddles)
    const void* spec;    // P reference-spectrum entries, bit-reversed order (FP32 register
                         // transforms: in the order their third pass reads, rf_spectrum_index)
    int real_bytes;      // 8: FP64 transform, 4: FP32 transform
    int n_keep;          // compressed samples kept per pulse
    int factor;          // 0: keep compressed (complex128 -> out64); >0 upsample
    int out_kind;        // 0 complex128, 1 complex64, 2 FP16 complex + per-pulse scale
    double2* out64;
    float2* out32;
    __half2* out16;
    float* scale16;
};

cudaError_t launch_ref_spectrum(const double2* ref, int nref, int P, int logP, const void* tw, int correlate,
                                void* spec, int real_bytes, cudaStream_t st);

// FP32 pulse compression of P = 2^L points, 12 <= L <= 14, runs as register transforms
// (k_pulse_compress_rf).  A P-point transform there is 16 elements a thread over T = P/16
// threads in five passes; the second (and fourth) pass works on blocks of B = 16 TB
// elements, TB = 2^(L-12), and the third on groups of TB.
inline bool rf_length(int real_bytes, int logP) { return real_bytes == 4 && logP >= 12 && logP <= 14; }
// Twiddles of the second / fourth pass in the order the lanes read them: for the stage of
// span d (8, 4, 2, 1), entry B (16 - 2d) + B k + r holds twiddle (r + B k) P / (2 B d),
// k < d, r < B; 15 B entries.
inline int64_t rf_twiddle_count(int logP) { return 15LL * (16LL << (logP - 12)); }
inline int64_t rf_twiddle_source(int logP, int64_t e)
{
    const int64_t P = 1LL << logP, B = 16LL << (logP - 12);
    const int64_t blk = e / B, r = e % B;                 // blk in [0, 15): stage and k
    const int64_t d = blk < 8 ? 8 : (blk < 12 ? 4 : (blk < 14 ? 2 : 1));
    const int64_t k = blk - (16 - 2 * d);
    return (r + B * k) * (P / (2 * B * d));
}
// Spectrum index that thread t reads for its element m in the third pass, stored at
// m T + t: the element of group t / TB at offset t mod TB + TB m.
inline __host__ __device__ int rf_spectrum_index(int logP, int o)
{
    const int T = 1 << (logP - 4), TB = 1 << (logP - 12), B = 16 * TB;
    const int m = o / T, t = o % T;
    return (t / TB) * B + t % TB + TB * m;
}
cudaError_t launch_pulse_compress(const PulseArgs& a, cudaStream_t st);
// longest transform the FFT launchers take (a cluster of up to 8 CTAs)
int64_t fft_max_len(int real_bytes);
cudaError_t launch_fft_rows(double2* data, int64_t batch, int P, int logP, const double2* tw, int inverse,
                            cudaStream_t st);
cudaError_t launch_spline(const double2* in, int64_t n, int64_t batch, int factor, double2* out,
                          cudaStream_t st);
cudaError_t launch_upsample_store(const double2* in, int64_t n, int64_t batch, int factor, int out_kind, float2* out32,
                                  __half2* out16, float* scale16, cudaStream_t st);

cudaError_t launch_echo_synth(const DemView& d, const double* tx, const double* rx, int np, const double* spos,
                              const double* samp, int nscat, double n1, double n2, int W, double c, double fc,
                              double fs, double f0, double f1, double T, int nsamp, double sigma, uint64_t seed,
                              int ref_bins,
                              double* tau, double2* carrier, double2* raw, cudaStream_t st);

// ------------------------------- Fermat (FP64) ---------------------------------------
cudaError_t launch_dem_elevation(const DemView& d, const double* xy, int64_t n, double* z, cudaStream_t st);
cudaError_t launch_refraction_points(const DemView& d, const double* p1, const double* p2, int64_t n, double n1,
                                     double n2, int solver, int W, double* out, cudaStream_t st);
cudaError_t launch_slant_range(const DemView& d, const double* tx, const double* rx, int64_t np,
                               const double* target, double n1, double n2, int solver, int W, double* ranges,
                               double* ida, double* volta, double* refl, cudaStream_t st);

// ------------------------------- back-projection -------------------------------------
struct BpArgs {
    DemView dem;
    const double* tx;     // np x 3
    const double* rx;     // np x 3
    int np;
    int64_t nr;           // upsampled samples per pulse
    const double2* rc64;  // np x nr (FP64 form)
    const float2* rc32;   // np x nr (mixed)
    const __half2* rc16;  // np x nr (mixed FP16)
    const float* scale16; // np per-pulse scales (mixed FP16)
    const double* gx;
    const double* gy;
    const double* gz;
    int nx, ny, nz;
    double n1, n2, c, fs_eff, lambda;
    int W;                // Newton node-scan half width
    int64_t v_begin, v_count;  // voxel range, reference flat order (z -> x -> y)
    double2* out;         // image [x][y][z]
    // mixed form: per-pulse FP64 reference optical path and reduced carrier phase
    const double* ref_L;    // np
    const float* ref_phase; // np, (2 pi / lambda) * ref_L reduced to [-pi, pi)
    const int* ref_bin_i;   // np, floor(ref_L * fs_eff / c)
    const float* ref_bin_f; // np, ref_L * fs_eff / c - ref_bin_i
};

// DEM tile of the mixed kernel (nodes): TMA box dims.  The x extent is a multiple of
// 4 floats so every tiled copy row is a multiple of 16 bytes.
constexpr int kMixedTileI = 68;
constexpr int kMixedTileJ = 64;

// One image-formation request of the mixed kernel, as it sits in device memory: the
// back-projection arguments, the FP32 DEM view and the tensor map of that DEM.
struct alignas(64) MixedReq {
    alignas(64) unsigned char tmap[128];   // CUtensorMap of the FP32 DEM (box kMixedTileI x kMixedTileJ)
    BpArgs a;
    const float* z32;     // pitch-padded FP32 heights, z32[j * pitch + i]
    int pitch;            // row pitch (floats), a multiple of 4
    int use_tile;         // tmap valid: stage DEM tiles with TMA
    int fp16;             // samples stored FP16 complex + scale (else complex64)
    int exhaustive;       // 1: node scans rank every node (no pruning); the image is the same
    float stepx, stepy, istepx, istepy;
    double ox, oy;        // origin of the FP32 frame (first DEM node)
    double idx64, idy64;  // 1 / spacing
    float off_x, off_y;   // mean crossing offset from the voxel, metres (tile centring)
    float start_band;     // node units: FP32 flat starts this close to a cell boundary are redone in FP64
    float zmin;           // lowest FP32 height of the DEM (bounds of the pruned node scan)
};

// Pulse chunks of a request (kept beside MixedReq, read only by the chunked kernel).
// nchunk > 1: work item t of the request is chunk t % nchunk of tile t / nchunk; each
// chunk writes its voxels' sums to partial[chunk * (nx ny nz) + image index], and the last
// of a tile's chunks to finish (counted in tile_done[tile], zero before the request's first
// launch) adds the chunks, in chunk order, into the image.
struct MixedChunks {
    int nchunk;           // <= 1: the whole pulse range in one work item
    int pad;
    double2* partial;
    int* tile_done;
};

// A batch of the persistent mixed kernel: `ntiles` work items (request index, tile of 128
// voxels in the request's flat voxel order); tiles == null means request 0, tiles 0..n-1.
struct MixedBatch {
    const MixedReq* reqs;
    const int2* tiles;
    const int* ntiles_dev;   // if non-null, the tile count is read on the device
    int ntiles;
    int* counter;            // zeroed before the launch
    int* status;             // device status word (1 = a tile copy timed out)
    const MixedChunks* chunks;   // per request, indexed as reqs (the chunked kernel only)
    long long wait_polls;        // polls of the bounded DEM-tile wait before giving up on a tile
};

cudaError_t launch_bp_plain(const BpArgs& a, int solver, int legs, cudaStream_t st);
cudaError_t launch_refraction_mixed(const DemView& d, int pitch, const double* p1, const double* p2, int64_t n,
                                    double n1, double n2, int W, double* out, cudaStream_t st);
// chunked: some request of the batch has nchunk > 1 (the kernel with the chunk sums)
cudaError_t launch_bp_mixed(const MixedBatch& b, int W, int grid, cudaStream_t st, bool chunked);
float mixed_start_band(const DemView& d);
// batched tiled transpose: out[b][c][r] = in[b][r][c] (complex128), and real -> complex128
cudaError_t launch_transpose_c128(const double2* in, double2* out, int64_t R, int64_t C, int64_t in_ld, int64_t out_ld,
                                  int64_t in_bs, int64_t out_bs, int64_t batch, cudaStream_t st);
cudaError_t launch_real_to_c128(const double* in, double2* out, int64_t n, cudaStream_t st);
int mixed_grid_ctas();   // persistent grid size (SMs x resident CTAs)
// Pulse chunks per 128-voxel tile for a request of `voxels` voxels and `pulses` pulses:
// as many as keep the request's work items within one wave of resident CTAs, at most 8
// and with at least 128 pulses each; 1 for grids that already fill the GPU.  A property of the
// request and the device only, so every path gives the same request the same image.
int mixed_chunks(int64_t voxels, int pulses);
cudaError_t launch_ref_ranges(const DemView& d, const double* tx, const double* rx, int np, const double* center,
                              double n1, double n2, int W, double lambda, double bin_per_m, double* ref_L,
                              float* ref_phase, int* ref_bin_i, float* ref_bin_f, double* offsets, cudaStream_t st);

}  // namespace bsar
