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
// FP32 pulses of 4096..16384 samples into FP32 storage take k_pulse_compress_rf instead:
// the same butterflies with the transforms held in registers, 16 elements per thread, and
// 5 shared-memory exchanges per pulse instead of one per pair of stages.
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
// rf_logP > 0: the spectrum of a register transform, stored in the order its third pass
// reads (rf_spectrum_index); 0: bit-reversed order.
template <typename R>
__global__ void k_ref_spectrum(const double2* __restrict__ ref, int nref, int P, int logP,
                               const typename C2<R>::T* __restrict__ tw, int correlate,
                               typename C2<R>::T* __restrict__ spec, int rf_logP)
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
        V v = x[rf_logP ? rf_spectrum_index(rf_logP, i) : i];
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
    // x4 (the imager's factor) into 16-byte aligned storage: the interval's four outputs
    // leave as two 16-byte stores (complex64) or one (FP16 complex), same values
    const void* out_base = out_kind == 1 ? (const void*)out32 : (const void*)out16;
    if (factor == 4 && (reinterpret_cast<uintptr_t>(out_base) & 15) == 0) {
        const float4 ws[4] = {wt[0], wt[1], wt[2], wt[3]};
        for (int64_t iv = threadIdx.x; iv < n; iv += blockDim.x) {
            float2 o[4];
            if (iv >= n - 1) {
                o[0] = o[1] = o[2] = o[3] = ld(n - 1);
            } else {
                const float2 pm1 = ld(iv > 0 ? iv - 1 : 0), p0 = ld(iv), p1 = ld(iv + 1),
                             p2 = ld(iv + 2 < n ? iv + 2 : n - 1);
                const float dpx = iv > 0 ? p0.x - pm1.x : 0.f, dpy = iv > 0 ? p0.y - pm1.y : 0.f;
                const float dnx = iv < n - 2 ? p2.x - p1.x : 0.f, dny = iv < n - 2 ? p2.y - p1.y : 0.f;
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    const float4 w = ws[k];
                    o[k].x = fmaf(w.x, p0.x, fmaf(w.y, p1.x, fmaf(w.z, dpx, w.w * dnx)));
                    o[k].y = fmaf(w.x, p0.y, fmaf(w.y, p1.y, fmaf(w.z, dpy, w.w * dny)));
                }
            }
            if (out_kind == 1) {
                float4* d = reinterpret_cast<float4*>(out32 + iv * 4);
                d[0] = make_float4(o[0].x, o[0].y, o[1].x, o[1].y);
                d[1] = make_float4(o[2].x, o[2].y, o[3].x, o[3].y);
            } else {
                unsigned u[4];
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    const __half2 h = __floats2half2_rn(o[k].x * inv_scale, o[k].y * inv_scale);
                    u[k] = *reinterpret_cast<const unsigned*>(&h);
                }
                *reinterpret_cast<uint4*>(out16 + iv * 4) = make_uint4(u[0], u[1], u[2], u[3]);
            }
        }
        return;
    }
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

// ---------------------------------------------------------------------------------
// FP32 pulse compression with the transforms held in registers, P = 2^L, L = 12..14.
//
// P/16 threads, 16 elements each.  A pass loads one group of 16 elements per thread,
// runs four radix-2 stages on it in registers and stores it back; the stages of a
// transform fall into three passes (spans P/2..P/16, P/32..P/256, then the rest), and
// the middle pass of the pair of transforms does the forward transform's last stages,
// the matched-filter multiply and the inverse transform's first stages together:
//   pass 1   elements t + (P/16) m      from global memory (the raw pulse)
//   pass 2   elements b (P/16) + o + B m,         B = 16 TB
//   pass 3   elements c B + s + TB m,             TB = 2^(L-12) threads share a block
// Stages whose span is below TB pair elements of neighbouring lanes and run through warp
// shuffles.  Every butterfly, twiddle and operation order is that of fft_dif / fft_dit,
// so the result is the same, bit for bit, as k_pulse_compress<float>; only the grouping
// of stages into shared-memory round trips changes (5 instead of 16).
//
// Shared memory holds the P elements unpadded, at x[swz(e)]: the XOR swizzle permutes
// elements inside blocks of 16 TB, keyed by the block index, so that the 16 lanes of a
// half-warp hit 16 different bank pairs in every pass (passes 1 and 2 read consecutive
// elements of one block; pass 3 reads one element of each of several blocks).
// ---------------------------------------------------------------------------------
template <int L> __device__ __forceinline__ int swz(int e)
{
    constexpr int lt = L - 12;
    return e ^ (((e >> (4 + lt)) & (15 >> lt)) << lt);
}

// swz(base + STRIDE m) for the bases the passes use, from one swizzle of the base: the
// first and fifth pass (STRIDE = T, base = t) add T m above the swizzled bits; the second
// and fourth (STRIDE = B, base = (t / B) T + t mod B) take m's low bits as the swizzle
// key, a constant for each m; the third (STRIDE = TB, base = (t / TB) B + t mod TB) flips
// m into the swizzled field.  One or no instruction per element instead of five.
template <int L, int STRIDE> __device__ __forceinline__ int rf_sbase(int base)
{
    constexpr int B = 16 << (L - 12);
    return STRIDE == B ? base : swz<L>(base);
}

template <int L, int STRIDE> __device__ __forceinline__ int rf_index(int sb, int m)
{
    constexpr int T = 1 << (L - 4), B = 16 << (L - 12), lt = L - 12;
    static_assert(STRIDE == T || STRIDE == B || STRIDE == (1 << lt), "a pass stride");
    if constexpr (STRIDE == T) return sb + T * m;
    else if constexpr (STRIDE == B) return (sb ^ ((m & (15 >> lt)) << lt)) + B * m;
    else return sb ^ (m << lt);
}

// The opaque copy of `base` makes each call compute its 16 addresses afresh, instead of
// the compiler keeping a pass's addresses live until the inverse pass reuses them.
template <int L, int STRIDE>
__device__ __forceinline__ void rf_load(const float2* x, float2 (&v)[16], int base)
{
    asm volatile("" : "+r"(base));
    const int sb = rf_sbase<L, STRIDE>(base);
#pragma unroll
    for (int m = 0; m < 16; m++) v[m] = x[rf_index<L, STRIDE>(sb, m)];
}

template <int L, int STRIDE>
__device__ __forceinline__ void rf_store(float2* x, const float2 (&v)[16], int base)
{
    asm volatile("" : "+r"(base));
    const int sb = rf_sbase<L, STRIDE>(base);
#pragma unroll
    for (int m = 0; m < 16; m++) x[rf_index<L, STRIDE>(sb, m)] = v[m];
}

// Four DIF stages (spans 8, 4, 2, 1 x STRIDE) on elements base + STRIDE m; r = base mod
// STRIDE, so element e of a pair (e, e + h) has twiddle index (e mod h) P / (2h) =
// (r + STRIDE (m mod d)) P / (2 STRIDE d).
template <int L, int STRIDE>
__device__ __forceinline__ void rf_dif4(float2 (&v)[16], int r, const float2* __restrict__ tw)
{
    constexpr int P = 1 << L;
#pragma unroll
    for (int d = 8; d >= 1; d >>= 1) {
        const int tstep = P / (2 * STRIDE * d);
        asm volatile("" ::: "memory");     // keep later stages' twiddle loads after this stage
#pragma unroll
        for (int m = 0; m < 16; m++) {
            if (m & d) continue;
            const float2 a = v[m], b = v[m + d];
            v[m] = cadd(a, b);
            v[m + d] = cmul(csub(a, b), __ldg(tw + (r + STRIDE * (m & (d - 1))) * tstep));
        }
    }
}

// Four DIT stages (spans 1, 2, 4, 8 x STRIDE), twiddles as in rf_dif4.
template <int L, int STRIDE>
__device__ __forceinline__ void rf_dit4(float2 (&v)[16], int r, const float2* __restrict__ tw)
{
    constexpr int P = 1 << L;
#pragma unroll
    for (int d = 1; d <= 8; d <<= 1) {
        const int tstep = P / (2 * STRIDE * d);
        asm volatile("" ::: "memory");
#pragma unroll
        for (int m = 0; m < 16; m++) {
            if (m & d) continue;
            const float2 a = v[m], t = cmul(v[m + d], __ldg(tw + (r + STRIDE * (m & (d - 1))) * tstep));
            v[m] = cadd(a, t);
            v[m + d] = csub(a, t);
        }
    }
}

// The same four stages on the second / fourth pass's blocks (STRIDE = B), twiddles from
// the lane-ordered table (rf_twiddle_source): entry B (16 - 2d) + B (m mod d) + r.
template <int L>
__device__ __forceinline__ void rf_dif4b(float2 (&v)[16], int r, const float2* __restrict__ twb)
{
    constexpr int B = 16 << (L - 12);
#pragma unroll
    for (int d = 8; d >= 1; d >>= 1) {
        asm volatile("" ::: "memory");
#pragma unroll
        for (int m = 0; m < 16; m++) {
            if (m & d) continue;
            const float2 a = v[m], b = v[m + d];
            v[m] = cadd(a, b);
            v[m + d] = cmul(csub(a, b), __ldg(twb + B * (16 - 2 * d) + B * (m & (d - 1)) + r));
        }
    }
}

template <int L>
__device__ __forceinline__ void rf_dit4b(float2 (&v)[16], int r, const float2* __restrict__ twb)
{
    constexpr int B = 16 << (L - 12);
#pragma unroll
    for (int d = 1; d <= 8; d <<= 1) {
        asm volatile("" ::: "memory");
#pragma unroll
        for (int m = 0; m < 16; m++) {
            if (m & d) continue;
            const float2 a = v[m], t = cmul(v[m + d], __ldg(twb + B * (16 - 2 * d) + B * (m & (d - 1)) + r));
            v[m] = cadd(a, t);
            v[m + d] = csub(a, t);
        }
    }
}

__device__ __forceinline__ float2 shfl_xor2(float2 a, int s)
{
    a.x = __shfl_xor_sync(0xffffffffu, a.x, s);
    a.y = __shfl_xor_sync(0xffffffffu, a.y, s);
    return a;
}

// DIF stage of span s < TB across lanes (lane ^ s holds the partner): the lane whose
// element has bit s clear keeps a + b, its partner (a - b) w, w = tw[(sub mod s) P/(2s)].
template <int L>
__device__ __forceinline__ void rf_dif_lanes(float2 (&v)[16], int sub, int s, const float2* __restrict__ tw)
{
    constexpr int P = 1 << L;
    const bool hi = sub & s;
    const float2 w = __ldg(tw + (sub & (s - 1)) * (P / (2 * s)));
#pragma unroll
    for (int m = 0; m < 16; m++) {
        const float2 o = shfl_xor2(v[m], s);
        v[m] = hi ? cmul(csub(o, v[m]), w) : cadd(v[m], o);
    }
}

// DIT stage of span s < TB across lanes: t = b w, a + t to the lane holding a, a - t
// to the lane holding b.
template <int L>
__device__ __forceinline__ void rf_dit_lanes(float2 (&v)[16], int sub, int s, const float2* __restrict__ tw)
{
    constexpr int P = 1 << L;
    const bool hi = sub & s;
    const float2 w = __ldg(tw + (sub & (s - 1)) * (P / (2 * s)));
#pragma unroll
    for (int m = 0; m < 16; m++) {
        const float2 o = shfl_xor2(v[m], s);
        v[m] = hi ? csub(o, cmul(v[m], w)) : cadd(v[m], cmul(o, w));
    }
}

// x4 Hermite epilogue of the register transforms when all P samples are kept: thread t
// takes the intervals iv = t + k T, k < 16, whose neighbours t - 1 .. t + 2 lie k T
// further on, so their swizzled indices are the thread's four swizzled neighbours plus
// k T (the first pass's identity, also across the ends of a block of T).  The values,
// weights and clamps are hermite_store32's (splineInterpolation's one-sided tangents, the
// last interval repeating the last sample); only the indexing differs.  out_kind 1:
// complex64, 2: FP16 complex x inv_scale (the one the kernel uses it for: 12-14 % faster
// than hermite_store32 there); 16-byte aligned outputs.
template <int L>
__device__ __forceinline__ void rf_hermite4(const float2* x, int t, int out_kind, float inv_scale,
                                            float2* __restrict__ out32, __half2* __restrict__ out16)
{
    constexpr int P = 1 << L, T = P / 16;
    float4 ws[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const double u = (double)q / 4, u2 = u * u, u3 = u2 * u;
        ws[q] = make_float4((float)(2 * u3 - 3 * u2 + 1), (float)(-2 * u3 + 3 * u2), (float)(u3 - 2 * u2 + u),
                            (float)(u3 - u2));
    }
    auto sidx = [](int j) { return j < 0 ? swz<L>(j + T) - T : (j >= T ? swz<L>(j - T) + T : swz<L>(j)); };
    const int sm1 = sidx(t - 1), s0 = sidx(t), s1 = sidx(t + 1), s2 = sidx(t + 2);
#pragma unroll
    for (int k = 0; k < 16; k++) {
        const int iv = t + k * T;
        float2 o[4];
        if (iv >= P - 1) {
            o[0] = o[1] = o[2] = o[3] = x[s0 + k * T];
        } else {
            // indices selected, never out of range: element 0 for iv = 0 (its tangent is
            // zero) and element P - 1 = iv + 1 for iv = P - 2
            const float2 pm1 = x[iv > 0 ? sm1 + k * T : 0], p0 = x[s0 + k * T], p1 = x[s1 + k * T],
                         p2 = x[iv + 2 < P ? s2 + k * T : s1 + k * T];
            const float dpx = iv > 0 ? p0.x - pm1.x : 0.f, dpy = iv > 0 ? p0.y - pm1.y : 0.f;
            const float dnx = iv < P - 2 ? p2.x - p1.x : 0.f, dny = iv < P - 2 ? p2.y - p1.y : 0.f;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const float4 w = ws[q];
                o[q].x = fmaf(w.x, p0.x, fmaf(w.y, p1.x, fmaf(w.z, dpx, w.w * dnx)));
                o[q].y = fmaf(w.x, p0.y, fmaf(w.y, p1.y, fmaf(w.z, dpy, w.w * dny)));
            }
        }
        if (out_kind == 1) {
            float4* d = reinterpret_cast<float4*>(out32 + (int64_t)iv * 4);
            d[0] = make_float4(o[0].x, o[0].y, o[1].x, o[1].y);
            d[1] = make_float4(o[2].x, o[2].y, o[3].x, o[3].y);
        } else {
            unsigned u[4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const __half2 h = __floats2half2_rn(o[q].x * inv_scale, o[q].y * inv_scale);
                u[q] = *reinterpret_cast<const unsigned*>(&h);
            }
            *reinterpret_cast<uint4*>(out16 + (int64_t)iv * 4) = make_uint4(u[0], u[1], u[2], u[3]);
        }
    }
}

// CTAs per SM the register budget is sized for: two (64 registers a thread at 512 threads,
// 128 at 256); one at 1024 threads.
template <int L> struct RfOcc { static constexpr int v = L == 14 ? 1 : 2; };

template <int L>
__global__ void __launch_bounds__((1 << L) / 16, RfOcc<L>::v)
    k_pulse_compress_rf(const double2* __restrict__ in, int ns, const float2* __restrict__ tw,
                        const float2* __restrict__ twb, const float2* __restrict__ spec, int n_keep, int factor,
                        int out_kind,
                        double2* __restrict__ out64, float2* __restrict__ out32, __half2* __restrict__ out16,
                        float* __restrict__ scale16)
{
    constexpr int P = 1 << L, T = P / 16, TB = 1 << (L - 12), B = 16 * TB;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* x = reinterpret_cast<float2*>(smem_raw);
    __shared__ float red[32];
    const int t = threadIdx.x;
    const int64_t p = blockIdx.x;
    const double2* __restrict__ src = in + p * (int64_t)ns;
    float2 v[16];
    // pass 1: the raw pulse (zero-padded to P) straight into registers, eight FP64 loads
    // in flight at a time
#pragma unroll
    for (int h = 0; h < 2; h++) {
#pragma unroll
        for (int m = 8 * h; m < 8 * h + 8; m++) {
            const int i = t + T * m;
            const double2 d = i < ns ? __ldg(src + i) : make_double2(0.0, 0.0);
            v[m] = make_float2((float)d.x, (float)d.y);
        }
        asm volatile("" ::: "memory");
    }
    rf_dif4<L, T>(v, t, tw);
    rf_store<L, T>(x, v, t);
    __syncthreads();
    // pass 2
    const int o2 = t % B, b2 = (t / B) * T + o2;
    rf_load<L, B>(x, v, b2);
    rf_dif4b<L>(v, o2, twb);
    rf_store<L, B>(x, v, b2);
    __syncthreads();
    // pass 3: last forward stages, matched filter, first inverse stages
    const int sub = t % TB, b3 = (t / TB) * B + sub;
    rf_load<L, TB>(x, v, b3);
    rf_dif4<L, TB>(v, sub, tw);
#pragma unroll
    for (int s = TB / 2; s >= 1; s >>= 1) rf_dif_lanes<L>(v, sub, s, tw);
#pragma unroll
    for (int h = 0; h < 2; h++) {
        asm volatile("" ::: "memory");
#pragma unroll
        for (int m = 8 * h; m < 8 * h + 8; m++) v[m] = cmul(cconj(v[m]), __ldg(spec + T * m + t));
    }
#pragma unroll
    for (int s = 1; s < TB; s <<= 1) rf_dit_lanes<L>(v, sub, s, tw);
    rf_dit4<L, TB>(v, sub, tw);
    rf_store<L, TB>(x, v, b3);
    __syncthreads();
    // passes 2 and 1 of the inverse transform, then conj / P
    rf_load<L, B>(x, v, b2);
    rf_dit4b<L>(v, o2, twb);
    rf_store<L, B>(x, v, b2);
    __syncthreads();
    rf_load<L, T>(x, v, t);
    rf_dit4<L, T>(v, t, tw);
    const float invP = 1.0f / (float)P;
#pragma unroll
    for (int m = 0; m < 16; m++) {
        v[m].x = v[m].x * invP;
        v[m].y = -v[m].y * invP;
    }
    rf_store<L, T>(x, v, t);
    __syncthreads();
    auto ld = [&](int64_t i) { return x[swz<L>((int)i)]; };
    if (factor <= 0) {
        double2* dst = out64 + p * (int64_t)n_keep;
        for (int i = t; i < n_keep; i += T) {
            const float2 c = ld(i);
            dst[i] = make_double2((double)c.x, (double)c.y);
        }
        return;
    }
    const int64_t n = n_keep, nout = n * factor;
    float scale = 1.0f;
    if (out_kind == 2) {
        float mx = 0.0f;
        for (int i = t; i < n; i += T) {
            const float2 c = ld(i);
            mx = fmaxf(mx, fmaxf(fabsf(c.x), fabsf(c.y)));
        }
        for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        if ((t & 31) == 0) red[t >> 5] = mx;
        __syncthreads();
        if (t < 32) {
            mx = (t < (T >> 5)) ? red[t] : 0.0f;
            for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
            if (t == 0) red[0] = mx;
        }
        __syncthreads();
        mx = red[0];
        // the Hermite overshoot stays well inside 2x the sample maximum
        scale = (mx > 0.0f) ? mx / 16384.0f : 1.0f;
        if (t == 0) scale16[p] = scale;
    }
    float2* o32 = out32 ? out32 + p * nout : nullptr;
    __half2* o16 = out16 ? out16 + p * nout : nullptr;
    const void* ob = out_kind == 1 ? (const void*)o32 : (const void*)o16;
    // FP16 storage only: for complex64 the generic loop's two 16-byte stores per interval
    // ran faster than this unrolled one (125 against 134 us at 8192 points)
    if (factor == 4 && n == P && out_kind == 2 && ob && (reinterpret_cast<uintptr_t>(ob) & 15) == 0) {
        rf_hermite4<L>(x, t, out_kind, 1.0f / scale, o32, o16);
        return;
    }
    hermite_store32(ld, n, factor, out_kind, 1.0f / scale, o32, o16);
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
                                                            (double2*)spec, 0);
    } else {
        size_t sm = fft_smem_bytes<float>(P);
        cudaFuncSetAttribute(k_ref_spectrum<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        const int rf_logP = (rf_length(4, logP) && P == (1 << logP)) ? logP : 0;
        k_ref_spectrum<float><<<1, fft_threads(P), sm, st>>>(ref, nref, P, logP, (const float2*)tw, correlate,
                                                           (float2*)spec, rf_logP);
    }
    return cudaGetLastError();
}

template <int L> static cudaError_t launch_pulse_rf(const PulseArgs& a, cudaStream_t st)
{
    const size_t sm = (size_t)(1 << L) * sizeof(float2);
    cudaFuncSetAttribute(k_pulse_compress_rf<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    // 60 % of the unified memory as shared memory holds two CTAs' pulses; the rest stays
    // L1 for the twiddles, the reference spectrum and register spills
    cudaFuncSetAttribute(k_pulse_compress_rf<L>, cudaFuncAttributePreferredSharedMemoryCarveout, 60);
    if (!a.tw_rf) return cudaErrorInvalidValue;
    k_pulse_compress_rf<L><<<(unsigned)a.batch, (1 << L) / 16, sm, st>>>(
        a.in, a.ns, (const float2*)a.tw, (const float2*)a.tw_rf, (const float2*)a.spec, a.n_keep, a.factor,
        a.out_kind, a.out64, a.out32, a.out16, a.scale16);
    return cudaGetLastError();
}

cudaError_t launch_pulse_compress(const PulseArgs& a, cudaStream_t st)
{
    // FP32 transforms of 4096..16384 points into FP32 storage (or none): registers
    if (rf_length(a.real_bytes, a.logP) && a.P == (1 << a.logP)) {
        // the spectrum of these lengths is stored in the register transforms' order
        if (a.factor > 0 && a.out_kind == 0) return cudaErrorInvalidValue;
        if (a.logP == 12) return launch_pulse_rf<12>(a, st);
        if (a.logP == 13) return launch_pulse_rf<13>(a, st);
        return launch_pulse_rf<14>(a, st);
    }
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
