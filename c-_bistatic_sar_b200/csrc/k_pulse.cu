// k_pulse.cu -- batched FFT, pulse compression and fast-time upsampling.
//
// One CTA per pulse holds the whole padded pulse (P complex samples) in shared
// memory and runs, in place:
//   forward radix-2 DIF FFT (natural order in -> bit-reversed order out)
//   matched-filter multiply with the reference spectrum, stored bit-reversed
//   radix-2 DIT FFT (bit-reversed in -> natural order out)
// so no bit-reversal pass and no second buffer are needed.  The inverse transform is
// taken as conj(FFT(conj(.)))/P, the same identity the reference's ifft uses
// (src/fft_utils.cpp:46-61).  The x`factor` Hermite upsampling of
// src/interpolation.cpp:4-51 runs as the epilogue, reading neighbours from shared
// memory and writing the upsampled pulse in the requested storage type.
//
// Pulses longer than one CTA's shared memory holds (FP64 above 8192, FP32 above 16384
// samples) run on a thread-block cluster of C = 2..8 CTAs: CTA r holds elements
// [r*M, (r+1)*M), M = P/C.  The radix-2 stages whose span reaches M pair elements of two
// CTAs and exchange them through distributed shared memory; every butterfly performs
// the same operations as the one-CTA transform, so both give identical bits.
//
// Compiled with --fmad=false: the Hermite epilogue (and the standalone spline kernel)
// reproduce the reference's FP64 results bit for bit.
#include <cooperative_groups.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.hpp"

namespace bsar {

template <typename R> struct C2;
template <> struct C2<double> { using T = double2; };
template <> struct C2<float> { using T = float2; };

template <typename V> __device__ __forceinline__ V cmul(V a, V b)
{
    V r;
    r.x = a.x * b.x - a.y * b.y;
    r.y = a.x * b.y + a.y * b.x;
    return r;
}
template <typename V> __device__ __forceinline__ V cadd(V a, V b) { V r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <typename V> __device__ __forceinline__ V csub(V a, V b) { V r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }
template <typename V> __device__ __forceinline__ V cconj(V a) { a.y = -a.y; return a; }

// In-place radix-2 DIF over smem x[0..P): natural order in, bit-reversed order out.
// tw[k] = exp(-2 pi i k / P), k < P/2.  Stages run in pairs: each thread takes the four
// elements two consecutive stages combine and does both stages' butterflies in
// registers (the same operations, so the same bits, as two radix-2 passes), halving the
// shared-memory round trips and barriers.
template <typename V>
__device__ __forceinline__ void fft_dif(V* x, int P, int logP, const V* __restrict__ tw)
{
    int s = logP - 1;
    for (; s >= 1; s -= 2) {
        const int h2 = 1 << (s - 1), h = h2 << 1;
        const int ts = P >> (s + 1), ts2 = ts << 1;
        for (int q = threadIdx.x; q < (P >> 2); q += blockDim.x) {
            const int k2 = q & (h2 - 1);
            const int e0 = ((q >> (s - 1)) << (s + 1)) + k2;
            V a0 = x[e0], a1 = x[e0 + h2], a2 = x[e0 + h], a3 = x[e0 + h + h2];
            // stage s: (e0, e2) with twiddle k2, (e1, e3) with twiddle k2 + h2
            V b0 = cadd(a0, a2), b2 = cmul(csub(a0, a2), __ldg(tw + k2 * ts));
            V b1 = cadd(a1, a3), b3 = cmul(csub(a1, a3), __ldg(tw + (k2 + h2) * ts));
            // stage s - 1: (e0, e1) and (e2, e3), twiddle k2
            const V w = __ldg(tw + k2 * ts2);
            x[e0] = cadd(b0, b1);
            x[e0 + h2] = cmul(csub(b0, b1), w);
            x[e0 + h] = cadd(b2, b3);
            x[e0 + h + h2] = cmul(csub(b2, b3), w);
        }
        __syncthreads();
    }
    if (s == 0) {
        for (int b = threadIdx.x; b < (P >> 1); b += blockDim.x) {
            V a = x[2 * b], c = x[2 * b + 1];
            x[2 * b] = cadd(a, c);
            x[2 * b + 1] = cmul(csub(a, c), __ldg(tw));
        }
        __syncthreads();
    }
}

// In-place radix-2 DIT over smem x[0..P): bit-reversed order in, natural order out,
// stages paired in registers as in fft_dif.
template <typename V>
__device__ __forceinline__ void fft_dit(V* x, int P, int logP, const V* __restrict__ tw)
{
    int s = 0;
    for (; s + 1 < logP; s += 2) {
        const int h = 1 << s;
        const int ts = P >> (s + 1), ts2 = ts >> 1;
        for (int q = threadIdx.x; q < (P >> 2); q += blockDim.x) {
            const int k = q & (h - 1);
            const int e0 = ((q >> s) << (s + 2)) + k;
            V a0 = x[e0], a1 = x[e0 + h], a2 = x[e0 + 2 * h], a3 = x[e0 + 3 * h];
            // stage s: (e0, e1) and (e2, e3), twiddle k
            const V w = __ldg(tw + k * ts);
            V t = cmul(a1, w);
            V b0 = cadd(a0, t), b1 = csub(a0, t);
            t = cmul(a3, w);
            V b2 = cadd(a2, t), b3 = csub(a2, t);
            // stage s + 1: (e0, e2) with twiddle k, (e1, e3) with twiddle k + h
            t = cmul(b2, __ldg(tw + k * ts2));
            x[e0] = cadd(b0, t);
            x[e0 + 2 * h] = csub(b0, t);
            t = cmul(b3, __ldg(tw + (k + h) * ts2));
            x[e0 + h] = cadd(b1, t);
            x[e0 + 3 * h] = csub(b1, t);
        }
        __syncthreads();
    }
    if (s < logP) {
        const int h = 1 << s;
        const int tstride = P >> (s + 1);
        for (int b = threadIdx.x; b < (P >> 1); b += blockDim.x) {
            int k = b & (h - 1);
            int i0 = ((b >> s) << (s + 1)) + k;
            int i1 = i0 + h;
            V t = cmul(x[i1], __ldg(tw + k * tstride));
            V a = x[i0];
            x[i0] = cadd(a, t);
            x[i1] = csub(a, t);
        }
        __syncthreads();
    }
}

__device__ __forceinline__ unsigned brev_n(unsigned j, int logP) { return __brev(j) >> (32 - logP); }

// ---------------------------------------------------------------------------------
// Reference spectrum: spec[j] = FFT(ref)[brev(j)] (conj when `conjugate` == 0 so that
// the pulse kernel's conj(X) * spec is conj(X * G) for G = conj(H) or H).
// ---------------------------------------------------------------------------------
template <typename R>
__global__ void k_ref_spectrum(const double2* __restrict__ ref, int nref, int P, int logP,
                               const typename C2<R>::T* __restrict__ tw, int correlate,
                               typename C2<R>::T* __restrict__ spec)
{
    using V = typename C2<R>::T;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* x = reinterpret_cast<V*>(smem_raw);
    for (int i = threadIdx.x; i < P; i += blockDim.x) {
        V v;
        if (i < nref) { double2 d = ref[i]; v.x = (R)d.x; v.y = (R)d.y; } else { v.x = 0; v.y = 0; }
        x[i] = v;
    }
    __syncthreads();
    fft_dif(x, P, logP, tw);
    for (int i = threadIdx.x; i < P; i += blockDim.x) {
        V v = x[i];
        // correlation: G = conj(H) -> conj(G) = H ; convolution: G = H -> conj(G) = conj(H)
        spec[i] = correlate ? v : cconj(v);
    }
}

// Hermite weights of splineInterpolation for output index o (src/interpolation.cpp:18-36).
struct Hermite {
    int64_t idx;
    double h1, h2, h3, h4;
};

__device__ __forceinline__ Hermite hermite_at(int64_t o, int64_t n, int factor)
{
    Hermite H;
    double pos = (double)o / factor;
    int64_t idx = (int64_t)pos;
    double frac = pos - (double)idx;
    if (idx >= n - 1) {
        idx = n - 2;
        frac = 1.0;
    }
    double t = frac, t2 = t * t, t3 = t2 * t;
    H.idx = idx;
    H.h1 = 2 * t3 - 3 * t2 + 1;
    H.h2 = -2 * t3 + 3 * t2;
    H.h3 = t3 - 2 * t2 + t;
    H.h4 = t3 - t2;
    return H;
}

// One component of the Hermite interpolation given p[idx-1..idx+2] (:39-46).
__device__ __forceinline__ double hermite_comp(const Hermite& H, int64_t n, double pm1, double p0,
                                               double p1, double p2)
{
    double dPrev = (H.idx > 0) ? (p0 - pm1) : 0;
    double dNext = (H.idx < n - 2) ? (p2 - p1) : 0;
    return H.h1 * p0 + H.h2 * p1 + H.h3 * dPrev + H.h4 * dNext;
}

// Hermite upsampling into FP32 storage (complex64, or FP16 complex x 1/scale): one
// thread per input interval computes the interval's `factor` outputs from one read of
// its four neighbours, with the weights of t = k / factor (FP64 formula rounded to FP32).
// The last interval repeats the last sample, as splineInterpolation's clamp to interval
// n - 2 with t = 1 does.  `ld(i)` returns sample i as float2.
template <typename Load>
__device__ __forceinline__ void hermite_store32(Load ld, int64_t n, int factor, int out_kind, float inv_scale,
                                                float2* __restrict__ out32, __half2* __restrict__ out16)
{
    __shared__ float4 wt[64];                       // weights of t = k / factor (factor <= 64)
    if (threadIdx.x < factor) {
        const double t = (double)threadIdx.x / factor, t2 = t * t, t3 = t2 * t;
        wt[threadIdx.x] = make_float4((float)(2 * t3 - 3 * t2 + 1), (float)(-2 * t3 + 3 * t2),
                                      (float)(t3 - 2 * t2 + t), (float)(t3 - t2));
    }
    __syncthreads();
    for (int64_t iv = threadIdx.x; iv < n; iv += blockDim.x) {
        const int64_t o0 = iv * factor;
        if (iv >= n - 1) {
            const float2 v = ld(n - 1);
            for (int k = 0; k < factor; k++) {
                if (out_kind == 1) out32[o0 + k] = v;
                else out16[o0 + k] = __floats2half2_rn(v.x * inv_scale, v.y * inv_scale);
            }
            continue;
        }
        const float2 pm1 = ld(iv > 0 ? iv - 1 : 0), p0 = ld(iv), p1 = ld(iv + 1), p2 = ld(iv + 2 < n ? iv + 2 : n - 1);
        const float dpx = iv > 0 ? p0.x - pm1.x : 0.f, dpy = iv > 0 ? p0.y - pm1.y : 0.f;
        const float dnx = iv < n - 2 ? p2.x - p1.x : 0.f, dny = iv < n - 2 ? p2.y - p1.y : 0.f;
        for (int k = 0; k < factor; k++) {
            const float4 w = wt[k];
            const float h1 = w.x, h2 = w.y, h3 = w.z, h4 = w.w;
            const float re = fmaf(h1, p0.x, fmaf(h2, p1.x, fmaf(h3, dpx, h4 * dnx)));
            const float im = fmaf(h1, p0.y, fmaf(h2, p1.y, fmaf(h3, dpy, h4 * dny)));
            if (out_kind == 1) out32[o0 + k] = make_float2(re, im);
            else out16[o0 + k] = __floats2half2_rn(re * inv_scale, im * inv_scale);
        }
    }
}

// ---------------------------------------------------------------------------------
// Pulse compression (+ optional upsampling) of `batch` pulses, one CTA per pulse.
//   in        batch x ns complex128 (raw echoes), zero-padded to P
//   spec      P entries from k_ref_spectrum
//   n_keep    compressed samples kept per pulse (max(ns, nref))
//   factor    0: store the n_keep compressed samples as complex128 to out64
//             >0: store the upsampled pulse (n_keep*factor samples) as out_kind
// ---------------------------------------------------------------------------------
template <typename R>
__global__ void k_pulse_compress(const double2* __restrict__ in, int ns, int P, int logP,
                                 const typename C2<R>::T* __restrict__ tw,
                                 const typename C2<R>::T* __restrict__ spec, int n_keep, int factor,
                                 int out_kind, double2* __restrict__ out64, float2* __restrict__ out32,
                                 __half2* __restrict__ out16, float* __restrict__ scale16)
{
    using V = typename C2<R>::T;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* x = reinterpret_cast<V*>(smem_raw);
    __shared__ float red[32];
    const int64_t p = blockIdx.x;
    const double2* __restrict__ src = in + p * (int64_t)ns;
    // four loads in flight per thread before the shared-memory stores
    for (int i0 = threadIdx.x; i0 < P; i0 += 4 * blockDim.x) {
        double2 d[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int i = i0 + u * blockDim.x;
            d[u] = (i < ns) ? __ldg(src + i) : make_double2(0.0, 0.0);
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int i = i0 + u * blockDim.x;
            if (i < P) {
                V v;
                v.x = (R)d[u].x;
                v.y = (R)d[u].y;
                x[i] = v;
            }
        }
    }
    __syncthreads();
    fft_dif(x, P, logP, tw);
    for (int i = threadIdx.x; i < P; i += blockDim.x) x[i] = cmul(cconj(x[i]), __ldg(spec + i));
    __syncthreads();
    fft_dit(x, P, logP, tw);
    const R invP = (R)1 / (R)P;
    for (int i = threadIdx.x; i < P; i += blockDim.x) {
        V v = x[i];
        v.x = v.x * invP;
        v.y = -v.y * invP;
        x[i] = v;
    }
    __syncthreads();
    if (factor <= 0) {
        double2* dst = out64 + p * (int64_t)n_keep;
        for (int i = threadIdx.x; i < n_keep; i += blockDim.x) dst[i] = make_double2((double)x[i].x, (double)x[i].y);
        return;
    }
    const int64_t n = n_keep;
    const int64_t nout = n * factor;
    float scale = 1.0f;
    if (out_kind == 2) {
        float m = 0.0f;
        for (int i = threadIdx.x; i < n; i += blockDim.x) m = fmaxf(m, fmaxf(fabsf((float)x[i].x), fabsf((float)x[i].y)));
        for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
        __syncthreads();
        if (threadIdx.x < 32) {
            m = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0.0f;
            for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
            if (threadIdx.x == 0) red[0] = m;
        }
        __syncthreads();
        m = red[0];
        // the Hermite overshoot stays well inside 2x the sample maximum
        scale = (m > 0.0f) ? m / 16384.0f : 1.0f;
        if (threadIdx.x == 0) scale16[p] = scale;
    }
    const float inv_scale = 1.0f / scale;
    if (out_kind != 0) {
        hermite_store32([&](int64_t i) { const V v = x[i]; return make_float2((float)v.x, (float)v.y); }, n, factor,
                        out_kind, inv_scale, out32 ? out32 + p * nout : nullptr, out16 ? out16 + p * nout : nullptr);
        return;
    }
    for (int64_t o = threadIdx.x; o < nout; o += blockDim.x) {
        Hermite H = hermite_at(o, n, factor);
        int64_t i = H.idx;
        V pm1 = x[i > 0 ? i - 1 : 0], p0 = x[i], p1 = x[i + 1], p2 = x[i + 2 < n ? i + 2 : n - 1];
        double re = hermite_comp(H, n, (double)pm1.x, (double)p0.x, (double)p1.x, (double)p2.x);
        double im = hermite_comp(H, n, (double)pm1.y, (double)p0.y, (double)p1.y, (double)p2.y);
        int64_t dst = p * nout + o;
        if (out_kind == 0)
            out64[dst] = make_double2(re, im);
        else if (out_kind == 1)
            out32[dst] = make_float2((float)re, (float)im);
        else
            out16[dst] = __floats2half2_rn((float)re * inv_scale, (float)im * inv_scale);
    }
}

// Upsampling of already-compressed pulses into the mixed forms' storage (complex64, or
// FP16 complex with a per-pulse scale): one CTA per pulse, Hermite weights as above.
__global__ void k_upsample_store(const double2* __restrict__ in, int64_t n, int factor, int out_kind,
                                 float2* __restrict__ out32, __half2* __restrict__ out16, float* __restrict__ scale16)
{
    __shared__ float red[32];
    const int64_t p = blockIdx.x;
    const double2* src = in + p * n;
    const int64_t nout = n * factor;
    float scale = 1.0f;
    if (out_kind == 2) {
        float m = 0.0f;
        for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
            double2 v = __ldg(src + i);
            m = fmaxf(m, fmaxf(fabsf((float)v.x), fabsf((float)v.y)));
        }
        for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
        __syncthreads();
        if (threadIdx.x < 32) {
            m = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0.0f;
            for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
            if (threadIdx.x == 0) red[0] = m;
        }
        __syncthreads();
        m = red[0];
        scale = (m > 0.0f) ? m / 16384.0f : 1.0f;
        if (threadIdx.x == 0) scale16[p] = scale;
    }
    const float inv_scale = 1.0f / scale;
    hermite_store32([&](int64_t i) { const double2 v = __ldg(src + i); return make_float2((float)v.x, (float)v.y); }, n,
                    factor, out_kind, inv_scale, out32 ? out32 + p * nout : nullptr, out16 ? out16 + p * nout : nullptr);
}

// Plain batched FFT rows (natural order in and out) -- FFTProcessor::fft / ::ifft.
__global__ void k_fft_rows(double2* __restrict__ data, int P, int logP, const double2* __restrict__ tw,
                           int inverse)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* x = reinterpret_cast<double2*>(smem_raw);
    double2* row = data + (int64_t)blockIdx.x * P;
    for (int i = threadIdx.x; i < P; i += blockDim.x) {
        double2 v = row[i];
        if (inverse) v.y = -v.y;
        x[i] = v;
    }
    __syncthreads();
    fft_dif(x, P, logP, tw);
    for (int i = threadIdx.x; i < P; i += blockDim.x) {
        double2 v = x[brev_n((unsigned)i, logP)];
        if (inverse) {
            v.x = v.x / (double)P;
            v.y = -v.y / (double)P;
        }
        row[i] = v;
    }
}

// splineInterpolation over a batch (src/interpolation.cpp:4-51), bit-exact FP64.
__global__ void k_spline(const double2* __restrict__ in, int64_t n, int64_t batch, int factor,
                         double2* __restrict__ out)
{
    const int64_t nout = n * factor;
    const int64_t total = nout * batch;
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < total;
         g += (int64_t)gridDim.x * blockDim.x) {
        int64_t p = g / nout, o = g - p * nout;
        const double2* src = in + p * n;
        Hermite H = hermite_at(o, n, factor);
        int64_t i = H.idx;
        double2 pm1 = __ldg(src + (i > 0 ? i - 1 : 0)), p0 = __ldg(src + i), p1 = __ldg(src + i + 1);
        double2 p2 = __ldg(src + (i + 2 < n ? i + 2 : n - 1));
        out[g] = make_double2(hermite_comp(H, n, pm1.x, p0.x, p1.x, p2.x),
                              hermite_comp(H, n, pm1.y, p0.y, p1.y, p2.y));
    }
}


// ---------------------------------------------------------------------------------
// Cluster-split transforms (P = C * M, CTA r of the cluster holds x[r*M .. r*M+M)).
// ---------------------------------------------------------------------------------
namespace cg = cooperative_groups;

constexpr int kClThreads = 1024;
template <typename R> struct ClPer;                       // elements per thread at M max
template <> struct ClPer<double> { static constexpr int v = 8; };    // M <= 8192  (128 KB)
template <> struct ClPer<float> { static constexpr int v = 16; };    // M <= 16384 (128 KB)

// One radix-2 stage of span h >= M: each CTA updates its own M elements from their
// partners in CTA r ^ (h / M).  dit = 0: DIF butterfly, dit = 1: DIT butterfly.
template <typename R, typename V>
__device__ __forceinline__ void cl_stage(V* x, int P, int s, int logM, const V* __restrict__ tw, int dit,
                                         const cg::cluster_group& cl)
{
    constexpr int kPer = ClPer<R>::v;
    const int M = 1 << logM;
    const unsigned r = cl.block_rank();
    const int base = (int)(r << logM);
    const int h = 1 << s;
    const int tstride = P >> (s + 1);
    const V* peer = cl.map_shared_rank(x, r ^ (unsigned)(h >> logM));
    V nv[kPer];
    cl.sync();                                    // every CTA's previous stage is written
#pragma unroll
    for (int j = 0; j < kPer; j++) {
        const int l = threadIdx.x + j * kClThreads;
        if (l < M) {
            const int i = base + l;
            const V a = x[l], c = peer[l];            // own element, partner element
            const V w = __ldg(tw + (i & (h - 1)) * tstride);
            const bool lo = (i & h) == 0;             // i is the butterfly's first index
            if (!dit)
                nv[j] = lo ? cadd(a, c) : cmul(csub(c, a), w);
            else
                nv[j] = lo ? cadd(a, cmul(c, w)) : csub(c, cmul(a, w));
        }
    }
    cl.sync();                                    // all partner reads are done
#pragma unroll
    for (int j = 0; j < kPer; j++) {
        const int l = threadIdx.x + j * kClThreads;
        if (l < M) x[l] = nv[j];
    }
}

// DIF over the whole cluster: natural order in, bit-reversed order out (global indices).
template <typename R, typename V>
__device__ void fft_dif_cl(V* x, int P, int logP, int logM, const V* __restrict__ tw, const cg::cluster_group& cl)
{
    for (int s = logP - 1; s >= logM; s--) cl_stage<R>(x, P, s, logM, tw, 0, cl);
    __syncthreads();
    const int M = 1 << logM;
    for (int s = logM - 1; s >= 0; s--) {
        const int h = 1 << s;
        const int tstride = P >> (s + 1);
        for (int b = threadIdx.x; b < (M >> 1); b += blockDim.x) {
            int k = b & (h - 1);
            int i0 = ((b >> s) << (s + 1)) + k;
            int i1 = i0 + h;
            V a = x[i0], c = x[i1];
            x[i0] = cadd(a, c);
            x[i1] = cmul(csub(a, c), __ldg(tw + k * tstride));
        }
        __syncthreads();
    }
}

// DIT over the whole cluster: bit-reversed order in, natural order out.  Ends with a
// cluster barrier, so every CTA may read any element afterwards.
template <typename R, typename V>
__device__ void fft_dit_cl(V* x, int P, int logP, int logM, const V* __restrict__ tw, const cg::cluster_group& cl)
{
    const int M = 1 << logM;
    for (int s = 0; s < logM; s++) {
        const int h = 1 << s;
        const int tstride = P >> (s + 1);
        for (int b = threadIdx.x; b < (M >> 1); b += blockDim.x) {
            int k = b & (h - 1);
            int i0 = ((b >> s) << (s + 1)) + k;
            int i1 = i0 + h;
            V t = cmul(x[i1], __ldg(tw + k * tstride));
            V a = x[i0];
            x[i0] = cadd(a, t);
            x[i1] = csub(a, t);
        }
        __syncthreads();
    }
    for (int s = logM; s < logP; s++) cl_stage<R>(x, P, s, logM, tw, 1, cl);
    cl.sync();
}

template <typename V>
__device__ __forceinline__ V cl_load(V* x, int j, int logM, const cg::cluster_group& cl)
{
    const V* q = cl.map_shared_rank(x, (unsigned)(j >> logM));
    return q[j & ((1 << logM) - 1)];
}

template <typename R>
__global__ void __launch_bounds__(kClThreads, 1)
    k_ref_spectrum_cl(const double2* __restrict__ ref, int nref, int P, int logP, int logM,
                      const typename C2<R>::T* __restrict__ tw, int correlate, typename C2<R>::T* __restrict__ spec)
{
    using V = typename C2<R>::T;
    cg::cluster_group cl = cg::this_cluster();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* x = reinterpret_cast<V*>(smem_raw);
    const int M = 1 << logM;
    const int base = (int)(cl.block_rank() << logM);
    for (int l = threadIdx.x; l < M; l += blockDim.x) {
        V v;
        const int i = base + l;
        if (i < nref) { double2 d = ref[i]; v.x = (R)d.x; v.y = (R)d.y; } else { v.x = 0; v.y = 0; }
        x[l] = v;
    }
    fft_dif_cl<R>(x, P, logP, logM, tw, cl);
    for (int l = threadIdx.x; l < M; l += blockDim.x) spec[base + l] = correlate ? x[l] : cconj(x[l]);
    cl.sync();
}

template <typename R>
__global__ void __launch_bounds__(kClThreads, 1)
    k_pulse_compress_cl(const double2* __restrict__ in, int ns, int P, int logP, int logM,
                        const typename C2<R>::T* __restrict__ tw, const typename C2<R>::T* __restrict__ spec,
                        int n_keep, int factor, int out_kind, double2* __restrict__ out64, float2* __restrict__ out32,
                        __half2* __restrict__ out16, float* __restrict__ scale16)
{
    using V = typename C2<R>::T;
    cg::cluster_group cl = cg::this_cluster();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* x = reinterpret_cast<V*>(smem_raw);
    __shared__ float red[32];
    const int C = (int)cl.num_blocks();
    const unsigned r = cl.block_rank();
    const int M = 1 << logM;
    const int base = (int)(r << logM);
    const int64_t p = blockIdx.x / C;
    const double2* __restrict__ src = in + p * (int64_t)ns;
    for (int l = threadIdx.x; l < M; l += blockDim.x) {
        V v;
        const int i = base + l;
        if (i < ns) { double2 d = __ldg(src + i); v.x = (R)d.x; v.y = (R)d.y; } else { v.x = 0; v.y = 0; }
        x[l] = v;
    }
    fft_dif_cl<R>(x, P, logP, logM, tw, cl);
    for (int l = threadIdx.x; l < M; l += blockDim.x) x[l] = cmul(cconj(x[l]), __ldg(spec + base + l));
    __syncthreads();
    fft_dit_cl<R>(x, P, logP, logM, tw, cl);
    const R invP = (R)1 / (R)P;
    for (int l = threadIdx.x; l < M; l += blockDim.x) {
        V v = x[l];
        v.x = v.x * invP;
        v.y = -v.y * invP;
        x[l] = v;
    }
    cl.sync();
    if (factor <= 0) {
        double2* dst = out64 + p * (int64_t)n_keep;
        for (int l = threadIdx.x; l < M; l += blockDim.x)
            if (base + l < n_keep) dst[base + l] = make_double2((double)x[l].x, (double)x[l].y);
        cl.sync();
        return;
    }
    const int64_t n = n_keep;
    const int64_t nout = n * factor;
    float scale = 1.0f;
    if (out_kind == 2) {
        float m = 0.0f;
        for (int l = threadIdx.x; l < M; l += blockDim.x)
            if (base + l < n) m = fmaxf(m, fmaxf(fabsf((float)x[l].x), fabsf((float)x[l].y)));
        for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
        __syncthreads();
        if (threadIdx.x < 32) {
            m = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0.0f;
            for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
            if (threadIdx.x == 0) red[0] = m;
        }
        cl.sync();
        m = 0.0f;
        for (int q = 0; q < C; q++) m = fmaxf(m, *cl.map_shared_rank(&red[0], (unsigned)q));
        scale = (m > 0.0f) ? m / 16384.0f : 1.0f;
        if (r == 0 && threadIdx.x == 0) scale16[p] = scale;
    }
    const float inv_scale = 1.0f / scale;
    const int64_t chunk = (nout + C - 1) / C;
    const int64_t o_end = min(nout, (int64_t)(r + 1) * chunk);
    for (int64_t o = (int64_t)r * chunk + threadIdx.x; o < o_end; o += blockDim.x) {
        Hermite H = hermite_at(o, n, factor);
        const int i = (int)H.idx;
        V pm1 = cl_load(x, i > 0 ? i - 1 : 0, logM, cl), p0 = cl_load(x, i, logM, cl), p1 = cl_load(x, i + 1, logM, cl);
        V p2 = cl_load(x, i + 2 < n ? i + 2 : (int)n - 1, logM, cl);
        double re = hermite_comp(H, n, (double)pm1.x, (double)p0.x, (double)p1.x, (double)p2.x);
        double im = hermite_comp(H, n, (double)pm1.y, (double)p0.y, (double)p1.y, (double)p2.y);
        int64_t dst = p * nout + o;
        if (out_kind == 0)
            out64[dst] = make_double2(re, im);
        else if (out_kind == 1)
            out32[dst] = make_float2((float)re, (float)im);
        else
            out16[dst] = __floats2half2_rn((float)re * inv_scale, (float)im * inv_scale);
    }
    cl.sync();                                    // peers may still read this CTA's samples
}

__global__ void __launch_bounds__(kClThreads, 1)
    k_fft_rows_cl(double2* __restrict__ data, int P, int logP, int logM, const double2* __restrict__ tw, int inverse)
{
    cg::cluster_group cl = cg::this_cluster();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* x = reinterpret_cast<double2*>(smem_raw);
    const int C = (int)cl.num_blocks();
    const int M = 1 << logM;
    const int base = (int)(cl.block_rank() << logM);
    double2* row = data + (int64_t)(blockIdx.x / C) * P;
    for (int l = threadIdx.x; l < M; l += blockDim.x) {
        double2 v = row[base + l];
        if (inverse) v.y = -v.y;
        x[l] = v;
    }
    fft_dif_cl<double>(x, P, logP, logM, tw, cl);
    cl.sync();
    for (int l = threadIdx.x; l < M; l += blockDim.x) {
        double2 v = cl_load(x, (int)brev_n((unsigned)(base + l), logP), logM, cl);
        if (inverse) {
            v.x = v.x / (double)P;
            v.y = -v.y / (double)P;
        }
        row[base + l] = v;
    }
    cl.sync();
}

// ------------------------------- launchers ------------------------------------------
static int fft_threads(int P) { return P >= 1024 ? 512 : (P >= 64 ? P / 2 : 32); }

template <typename R>
size_t fft_smem_bytes(int P) { return (size_t)P * sizeof(typename C2<R>::T); }

// Cluster size for a P-point transform: 1 while one CTA holds it, else the smallest
// power of two whose per-CTA share fits (ClPer * kClThreads elements).
static int cluster_size(int P, int real_bytes)
{
    const int mmax = real_bytes == 8 ? ClPer<double>::v * kClThreads : ClPer<float>::v * kClThreads;
    int C = 1;
    while (P / C > mmax) C *= 2;
    return C;
}

int64_t fft_max_len(int real_bytes) { return 8LL * (real_bytes == 8 ? ClPer<double>::v : ClPer<float>::v) * kClThreads; }

template <typename K, typename... Args>
static cudaError_t launch_cluster(K kernel, int64_t clusters, int C, size_t smem, cudaStream_t st, Args... args)
{
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(clusters * C), 1, 1);
    cfg.blockDim = dim3(kClThreads, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)C;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

cudaError_t launch_ref_spectrum(const double2* ref, int nref, int P, int logP, const void* tw,
                                int correlate, void* spec, int real_bytes, cudaStream_t st)
{
    const int C = cluster_size(P, real_bytes);
    if (C > 1) {
        const int logM = logP - __builtin_ctz(C);
        if (real_bytes == 8)
            return launch_cluster(k_ref_spectrum_cl<double>, 1, C, fft_smem_bytes<double>(P >> (logP - logM)), st,
                                  ref, nref, P, logP, logM, (const double2*)tw, correlate, (double2*)spec);
        return launch_cluster(k_ref_spectrum_cl<float>, 1, C, fft_smem_bytes<float>(P >> (logP - logM)), st, ref,
                              nref, P, logP, logM, (const float2*)tw, correlate, (float2*)spec);
    }
    if (real_bytes == 8) {
        size_t sm = fft_smem_bytes<double>(P);
        cudaFuncSetAttribute(k_ref_spectrum<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        k_ref_spectrum<double><<<1, fft_threads(P), sm, st>>>(ref, nref, P, logP, (const double2*)tw, correlate,
                                                            (double2*)spec);
    } else {
        size_t sm = fft_smem_bytes<float>(P);
        cudaFuncSetAttribute(k_ref_spectrum<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        k_ref_spectrum<float><<<1, fft_threads(P), sm, st>>>(ref, nref, P, logP, (const float2*)tw, correlate,
                                                           (float2*)spec);
    }
    return cudaGetLastError();
}

cudaError_t launch_pulse_compress(const PulseArgs& a, cudaStream_t st)
{
    const int C = cluster_size(a.P, a.real_bytes);
    if (C > 1) {
        const int logM = a.logP - __builtin_ctz(C);
        const int M = 1 << logM;
        if (a.real_bytes == 8)
            return launch_cluster(k_pulse_compress_cl<double>, a.batch, C, fft_smem_bytes<double>(M), st, a.in, a.ns,
                                  a.P, a.logP, logM, (const double2*)a.tw, (const double2*)a.spec, a.n_keep, a.factor,
                                  a.out_kind, a.out64, a.out32, a.out16, a.scale16);
        return launch_cluster(k_pulse_compress_cl<float>, a.batch, C, fft_smem_bytes<float>(M), st, a.in, a.ns, a.P,
                              a.logP, logM, (const float2*)a.tw, (const float2*)a.spec, a.n_keep, a.factor,
                              a.out_kind, a.out64, a.out32, a.out16, a.scale16);
    }
    if (a.real_bytes == 8) {
        size_t sm = fft_smem_bytes<double>(a.P);
        cudaFuncSetAttribute(k_pulse_compress<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        cudaFuncSetAttribute(k_pulse_compress<double>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        k_pulse_compress<double><<<(unsigned)a.batch, fft_threads(a.P), sm, st>>>(
            a.in, a.ns, a.P, a.logP, (const double2*)a.tw, (const double2*)a.spec, a.n_keep, a.factor,
            a.out_kind, a.out64, a.out32, a.out16, a.scale16);
    } else {
        size_t sm = fft_smem_bytes<float>(a.P);
        cudaFuncSetAttribute(k_pulse_compress<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        cudaFuncSetAttribute(k_pulse_compress<float>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        k_pulse_compress<float><<<(unsigned)a.batch, fft_threads(a.P), sm, st>>>(
            a.in, a.ns, a.P, a.logP, (const float2*)a.tw, (const float2*)a.spec, a.n_keep, a.factor,
            a.out_kind, a.out64, a.out32, a.out16, a.scale16);
    }
    return cudaGetLastError();
}

cudaError_t launch_fft_rows(double2* data, int64_t batch, int P, int logP, const double2* tw, int inverse,
                            cudaStream_t st)
{
    const int C = cluster_size(P, 8);
    if (C > 1) {
        const int logM = logP - __builtin_ctz(C);
        return launch_cluster(k_fft_rows_cl, batch, C, fft_smem_bytes<double>(1 << logM), st, data, P, logP, logM, tw,
                              inverse);
    }
    size_t sm = (size_t)P * sizeof(double2);
    cudaFuncSetAttribute(k_fft_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_fft_rows<<<(unsigned)batch, fft_threads(P), sm, st>>>(data, P, logP, tw, inverse);
    return cudaGetLastError();
}

cudaError_t launch_upsample_store(const double2* in, int64_t n, int64_t batch, int factor, int out_kind, float2* out32,
                                  __half2* out16, float* scale16, cudaStream_t st)
{
    k_upsample_store<<<(unsigned)batch, 256, 0, st>>>(in, n, factor, out_kind, out32, out16, scale16);
    return cudaGetLastError();
}

cudaError_t launch_spline(const double2* in, int64_t n, int64_t batch, int factor, double2* out, cudaStream_t st)
{
    int64_t total = n * factor * batch;
    int blocks = (int)((total + 255) / 256);
    if (blocks > 148 * 64) blocks = 148 * 64;
    if (blocks < 1) blocks = 1;
    k_spline<<<blocks, 256, 0, st>>>(in, n, batch, factor, out);
    return cudaGetLastError();
}

}  // namespace bsar
