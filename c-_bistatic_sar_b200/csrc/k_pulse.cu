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
// Compiled with --fmad=false: the Hermite epilogue (and the standalone spline kernel)
// reproduce the reference's FP64 results bit for bit.
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
// tw[k] = exp(-2 pi i k / P), k < P/2.
template <typename V>
__device__ __forceinline__ void fft_dif(V* x, int P, int logP, const V* __restrict__ tw)
{
    for (int s = logP - 1; s >= 0; s--) {
        const int h = 1 << s;            // half span
        const int tstride = P >> (s + 1); // twiddle index step
        for (int b = threadIdx.x; b < (P >> 1); b += blockDim.x) {
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

// In-place radix-2 DIT over smem x[0..P): bit-reversed order in, natural order out.
template <typename V>
__device__ __forceinline__ void fft_dit(V* x, int P, int logP, const V* __restrict__ tw)
{
    for (int s = 0; s < logP; s++) {
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
    for (int i = threadIdx.x; i < P; i += blockDim.x) {
        V v;
        if (i < ns) { double2 d = __ldg(src + i); v.x = (R)d.x; v.y = (R)d.y; } else { v.x = 0; v.y = 0; }
        x[i] = v;
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
    for (int64_t o = threadIdx.x; o < nout; o += blockDim.x) {
        Hermite H = hermite_at(o, n, factor);
        int64_t i = H.idx;
        double2 pm1 = __ldg(src + (i > 0 ? i - 1 : 0)), p0 = __ldg(src + i), p1 = __ldg(src + i + 1);
        double2 p2 = __ldg(src + (i + 2 < n ? i + 2 : n - 1));
        double re = hermite_comp(H, n, pm1.x, p0.x, p1.x, p2.x);
        double im = hermite_comp(H, n, pm1.y, p0.y, p1.y, p2.y);
        if (out_kind == 1)
            out32[p * nout + o] = make_float2((float)re, (float)im);
        else
            out16[p * nout + o] = __floats2half2_rn((float)re * inv_scale, (float)im * inv_scale);
    }
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

// ------------------------------- launchers ------------------------------------------
static int fft_threads(int P) { return P >= 1024 ? 512 : (P >= 64 ? P / 2 : 32); }

template <typename R>
size_t fft_smem_bytes(int P) { return (size_t)P * sizeof(typename C2<R>::T); }

cudaError_t launch_ref_spectrum(const double2* ref, int nref, int P, int logP, const void* tw,
                                int correlate, void* spec, int real_bytes, cudaStream_t st)
{
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
    if (a.real_bytes == 8) {
        size_t sm = fft_smem_bytes<double>(a.P);
        cudaFuncSetAttribute(k_pulse_compress<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        k_pulse_compress<double><<<(unsigned)a.batch, fft_threads(a.P), sm, st>>>(
            a.in, a.ns, a.P, a.logP, (const double2*)a.tw, (const double2*)a.spec, a.n_keep, a.factor,
            a.out_kind, a.out64, a.out32, a.out16, a.scale16);
    } else {
        size_t sm = fft_smem_bytes<float>(a.P);
        cudaFuncSetAttribute(k_pulse_compress<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        k_pulse_compress<float><<<(unsigned)a.batch, fft_threads(a.P), sm, st>>>(
            a.in, a.ns, a.P, a.logP, (const float2*)a.tw, (const float2*)a.spec, a.n_keep, a.factor,
            a.out_kind, a.out64, a.out32, a.out16, a.scale16);
    }
    return cudaGetLastError();
}

cudaError_t launch_fft_rows(double2* data, int64_t batch, int P, int logP, const double2* tw, int inverse,
                            cudaStream_t st)
{
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
