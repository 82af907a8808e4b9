// k_layout.cu -- layout changes of complex128 arrays between the reference's files and
// the device layouts (the file hand-off around the hot path).
//
//   k_transpose_c128  batched tiled transpose through shared memory:
//                     out[b][c][r] = in[b][r][c] with independent row and batch strides.
//                     Used for the simulator's [range row][pulse column] matrix -> the
//                     pulse-major samples the scene holds, and for the [x][y][z] image ->
//                     the x-fastest order of the reference's image file (one transpose of
//                     the (x, z) plane per y).
//   k_real_to_c128    real samples -> complex128 with zero imaginary part.
//
// Both are HBM-bound byte moves: 32 x 32 tiles staged in shared memory so that reads and
// writes are both coalesced (16-byte elements, 512 bytes per warp row), grid sized to a
// few waves of the SMs with grid-stride loops over tiles and batches.
#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.hpp"

namespace bsar {

namespace {

constexpr int kT = 32;      // tile edge
constexpr int kRows = 8;    // thread rows per block (block = 32 x 8)

__global__ void __launch_bounds__(kT * kRows) k_transpose_c128(const double2* __restrict__ in, double2* __restrict__ out,
                                                               int64_t R, int64_t C, int64_t in_ld, int64_t out_ld,
                                                               int64_t in_bs, int64_t out_bs, int64_t batch)
{
    __shared__ double2 tile[kT][kT + 1];
    const int64_t tr = (R + kT - 1) / kT, tc = (C + kT - 1) / kT;
    const int64_t ntiles = tr * tc * batch;
    for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int64_t b = t / (tr * tc);
        const int64_t rem = t - b * tr * tc;
        const int64_t r0 = (rem / tc) * kT, c0 = (rem % tc) * kT;
        const double2* src = in + b * in_bs;
        double2* dst = out + b * out_bs;
        for (int i = threadIdx.y; i < kT; i += kRows) {
            const int64_t r = r0 + i, c = c0 + threadIdx.x;
            if (r < R && c < C) tile[i][threadIdx.x] = src[r * in_ld + c];
        }
        __syncthreads();
        for (int i = threadIdx.y; i < kT; i += kRows) {
            const int64_t c = c0 + i, r = r0 + threadIdx.x;
            if (r < R && c < C) dst[c * out_ld + r] = tile[threadIdx.x][i];
        }
        __syncthreads();
    }
}

__global__ void k_real_to_c128(const double* __restrict__ in, double2* __restrict__ out, int64_t n)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        out[k] = make_double2(in[k], 0.0);
}

int blocks_for(int64_t work, int per_block_work, int cap)
{
    int64_t b = (work + per_block_work - 1) / per_block_work;
    if (b < 1) b = 1;
    if (b > cap) b = cap;
    return (int)b;
}

}  // namespace

cudaError_t launch_transpose_c128(const double2* in, double2* out, int64_t R, int64_t C, int64_t in_ld, int64_t out_ld,
                                  int64_t in_bs, int64_t out_bs, int64_t batch, cudaStream_t st)
{
    if (R <= 0 || C <= 0 || batch <= 0) return cudaSuccess;
    const int64_t tiles = ((R + kT - 1) / kT) * ((C + kT - 1) / kT) * batch;
    k_transpose_c128<<<blocks_for(tiles, 1, 148 * 16), dim3(kT, kRows), 0, st>>>(in, out, R, C, in_ld, out_ld, in_bs,
                                                                                 out_bs, batch);
    return cudaGetLastError();
}

cudaError_t launch_real_to_c128(const double* in, double2* out, int64_t n, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    k_real_to_c128<<<blocks_for(n, 256, 148 * 32), 256, 0, st>>>(in, out, n);
    return cudaGetLastError();
}

}  // namespace bsar
