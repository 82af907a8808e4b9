// k_mixed.cu -- the mixed-precision back-projection kernel.
//
// One thread per voxel, voxels of a warp consecutive in the reference's flat order
// (y fastest), every thread walking the pulses in order.  Lanes of a warp solve the same
// pulse for neighbouring voxels, so their DEM windows, Tx/Rx loads and sample gathers
// coincide or sit next to each other.
//
// Per (voxel, pulse):
//   Fermat, twice (Tx -> voxel, voxel -> Rx):
//     FP32  flat-interface start, node scan of +-W DEM nodes, active-set Newton polish
//           on the 4 facets around the best node (coordinates relative to the DEM origin)
//     FP64  one final Newton step on the winning facet; its leg lengths give the
//           bistatic optical path L in FP64
//   delay / phase: dL = L - L_ref(pulse) rounded to FP32; the fast-time bin and carrier
//           phase are FP32 offsets from per-pulse FP64 anchors (integer bin + fraction,
//           phase reduced to [-pi, pi) in FP64)
//   gather: two complex64 (or FP16 complex x pulse scale) samples, linear interpolation
//           (proc_test_script.cpp:589-636), times exp(j phi), Kahan-compensated FP32 sum.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "dev_common.cuh"
#include "kernels.hpp"

namespace bsar {

namespace {

struct Facet32 {
    float x0, y0, dx, dy, z00, b, c, e;
};

struct MixedCtx {
    const float* __restrict__ z32;
    int nx, ny;
    float stepx, stepy;      // uniform node spacing
    double ox, oy;           // origin of the FP32 frame (first DEM node)
};

__device__ __forceinline__ float zf(const MixedCtx& m, int i, int j) { return __ldg(m.z32 + (int64_t)j * m.nx + i); }

// FP32 bilinear height (clamped to the DEM) for the flat-interface start.
__device__ __forceinline__ float height32(const MixedCtx& m, float x, float y)
{
    float fx = x / m.stepx, fy = y / m.stepy;
    int i = min(max((int)floorf(fx), 0), m.nx - 2);
    int j = min(max((int)floorf(fy), 0), m.ny - 2);
    float u = fminf(fmaxf(fx - (float)i, 0.f), 1.f), v = fminf(fmaxf(fy - (float)j, 0.f), 1.f);
    float z00 = zf(m, i, j), z01 = zf(m, i + 1, j), z10 = zf(m, i, j + 1), z11 = zf(m, i + 1, j + 1);
    return z00 + (z01 - z00) * u + (z10 - z00) * v + (z11 - z01 - z10 + z00) * u * v;
}

__device__ __forceinline__ bool facet_step32(const Facet32& F, const float A[3], const float B[3], float na,
                                             float nb, float& u, float& v)
{
    float x = fmaf(u, F.dx, F.x0), y = fmaf(v, F.dy, F.y0);
    float h = F.z00 + F.b * u + F.c * v + F.e * u * v;
    float idx_ = 1.0f / F.dx, idy = 1.0f / F.dy;
    float zx = (F.b + F.e * v) * idx_;
    float zy = (F.c + F.e * u) * idy;
    float zxy = F.e * idx_ * idy;
    float r1x = x - A[0], r1y = y - A[1], r1z = h - A[2];
    float r2x = x - B[0], r2y = y - B[1], r2z = h - B[2];
    float q1 = r1x * r1x + r1y * r1y + r1z * r1z;
    float q2 = r2x * r2x + r2y * r2y + r2z * r2z;
    float s1 = rsqrtf(q1), s2 = rsqrtf(q2);
    float g1 = na * s1, g2 = nb * s2;
    float iq1 = s1 * s1, iq2 = s2 * s2;
    float a1x = r1x + r1z * zx, a1y = r1y + r1z * zy;
    float a2x = r2x + r2z * zx, a2y = r2y + r2z * zy;
    float gx = g1 * a1x + g2 * a2x;
    float gy = g1 * a1y + g2 * a2y;
    float txx = 1.0f + zx * zx, tyy = 1.0f + zy * zy, txy = zx * zy;
    float hxx = g1 * (txx - a1x * a1x * iq1) + g2 * (txx - a2x * a2x * iq2);
    float hyy = g1 * (tyy - a1y * a1y * iq1) + g2 * (tyy - a2y * a2y * iq2);
    float hxy = g1 * (txy - a1x * a1y * iq1) + g2 * (txy - a2x * a2y * iq2) + (g1 * r1z + g2 * r2z) * zxy;
    bool au = (u <= 0.0f && gx > 0.0f) || (u >= 1.0f && gx < 0.0f);
    bool av = (v <= 0.0f && gy > 0.0f) || (v >= 1.0f && gy < 0.0f);
    if (au && av) return false;
    float igs = 1.0f / (g1 + g2);
    float su, sv;
    if (au) {
        su = 0.0f;
        sv = (hyy > 0.0f) ? -gy / hyy : -gy * igs;
    } else if (av) {
        sv = 0.0f;
        su = (hxx > 0.0f) ? -gx / hxx : -gx * igs;
    } else {
        float det = hxx * hyy - hxy * hxy;
        if (det > 0.0f && hxx > 0.0f) {
            float idet = 1.0f / det;
            su = -(hyy * gx - hxy * gy) * idet;
            sv = -(hxx * gy - hxy * gx) * idet;
        } else {
            su = -gx * igs;
            sv = -gy * igs;
        }
    }
    u = __saturatef(u + su * idx_);
    v = __saturatef(v + sv * idy);
    return true;
}

__device__ __forceinline__ float facet_eval32(const Facet32& F, const float A[3], const float B[3], float na,
                                              float nb, float u, float v)
{
    float x = fmaf(u, F.dx, F.x0), y = fmaf(v, F.dy, F.y0);
    float h = F.z00 + F.b * u + F.c * v + F.e * u * v;
    float r1x = x - A[0], r1y = y - A[1], r1z = h - A[2];
    float r2x = x - B[0], r2y = y - B[1], r2z = h - B[2];
    float q1 = r1x * r1x + r1y * r1y + r1z * r1z;
    float q2 = r2x * r2x + r2y * r2y + r2z * r2z;
    return na * (q1 * rsqrtf(q1)) + nb * (q2 * rsqrtf(q2));
}

// FP64 final Newton step on facet (fi, fj) from (u, v); returns the optical path of the
// result and its two leg lengths (|X-A|, |X-B|).
__device__ __forceinline__ double final_step64(const DemView& d, int fi, int fj, const double A[3], const double B[3],
                                               double na, double nb, double u, double v, double& dA, double& dB)
{
    Facet64 F;
    facet_load(d, fi, fj, F);
    {
        double x = F.x0 + u * F.dx, y = F.y0 + v * F.dy;
        double h = F.z00 + F.b * u + F.c * v + F.e * u * v;
        double idx_ = 1.0 / F.dx, idy = 1.0 / F.dy;
        double zx = (F.b + F.e * v) * idx_;
        double zy = (F.c + F.e * u) * idy;
        double zxy = F.e * idx_ * idy;
        double r1x = x - A[0], r1y = y - A[1], r1z = h - A[2];
        double r2x = x - B[0], r2y = y - B[1], r2z = h - B[2];
        double q1 = r1x * r1x + r1y * r1y + r1z * r1z;
        double q2 = r2x * r2x + r2y * r2y + r2z * r2z;
        double s1 = rsqrt(q1), s2 = rsqrt(q2);
        double g1 = na * s1, g2 = nb * s2;
        double iq1 = s1 * s1, iq2 = s2 * s2;
        double a1x = r1x + r1z * zx, a1y = r1y + r1z * zy;
        double a2x = r2x + r2z * zx, a2y = r2y + r2z * zy;
        double gx = g1 * a1x + g2 * a2x;
        double gy = g1 * a1y + g2 * a2y;
        double txx = 1.0 + zx * zx, tyy = 1.0 + zy * zy, txy = zx * zy;
        double hxx = g1 * (txx - a1x * a1x * iq1) + g2 * (txx - a2x * a2x * iq2);
        double hyy = g1 * (tyy - a1y * a1y * iq1) + g2 * (tyy - a2y * a2y * iq2);
        double hxy = g1 * (txy - a1x * a1y * iq1) + g2 * (txy - a2x * a2y * iq2) + (g1 * r1z + g2 * r2z) * zxy;
        bool au = (u <= 0.0 && gx > 0.0) || (u >= 1.0 && gx < 0.0);
        bool av = (v <= 0.0 && gy > 0.0) || (v >= 1.0 && gy < 0.0);
        if (!(au && av)) {
            double igs = 1.0 / (g1 + g2);
            double su, sv;
            if (au) {
                su = 0.0;
                sv = (hyy > 0.0) ? -gy / hyy : -gy * igs;
            } else if (av) {
                sv = 0.0;
                su = (hxx > 0.0) ? -gx / hxx : -gx * igs;
            } else {
                double det = hxx * hyy - hxy * hxy;
                if (det > 0.0 && hxx > 0.0) {
                    double idet = 1.0 / det;
                    su = -(hyy * gx - hxy * gy) * idet;
                    sv = -(hxx * gy - hxy * gx) * idet;
                } else {
                    su = -gx * igs;
                    sv = -gy * igs;
                }
            }
            u = clamp01(u + su * idx_);
            v = clamp01(v + sv * idy);
        }
    }
    double x = F.x0 + u * F.dx, y = F.y0 + v * F.dy;
    double h = F.z00 + F.b * u + F.c * v + F.e * u * v;
    double r1x = x - A[0], r1y = y - A[1], r1z = h - A[2];
    double r2x = x - B[0], r2y = y - B[1], r2z = h - B[2];
    dA = sqrt(r1x * r1x + r1y * r1y + r1z * r1z);
    dB = sqrt(r2x * r2x + r2y * r2y + r2z * r2z);
    return na * dA + nb * dB;
}

// Mixed-precision crossing solve A (index na) -> B (index nb).  A32/B32: the endpoints in
// the FP32 frame.  Returns the FP64 optical path; dA, dB: FP64 leg lengths.
__device__ __forceinline__ double solve_mixed(const DemView& d, const MixedCtx& m, const double A[3],
                                              const double B[3], const float A32[3], const float B32[3],
                                              float na, float nb, int W, double& dA, double& dB)
{
    // 1. flat-interface start (FP32)
    const bool lower_b = nb >= na;
    const float* Lp = lower_b ? B32 : A32;
    const float* Up = lower_b ? A32 : B32;
    const float nl = lower_b ? nb : na, nu = lower_b ? na : nb;
    float h0 = height32(m, Lp[0], Lp[1]);
    float hx = Lp[0] - Up[0], hy = Lp[1] - Up[1];
    float D = sqrtf(hx * hx + hy * hy);
    float sx = Lp[0], sy = Lp[1];
    if (D >= 1e-6f) {
        float ha = fabsf(Up[2] - h0), hb = fabsf(Lp[2] - h0);
        float s = fminf(fmaxf(D * ha / (ha + hb + 1e-30f), 0.f), D);
#pragma unroll
        for (int it = 0; it < kFlatIters; it++) {
            float q1 = s * s + ha * ha, r = D - s, q2 = r * r + hb * hb;
            float i1 = rsqrtf(q1), i2 = rsqrtf(q2);
            float g = nu * s * i1 - nl * r * i2;
            float gp = nu * ha * ha * i1 * i1 * i1 + nl * hb * hb * i2 * i2 * i2;
            if (gp > 0.f) s = fminf(fmaxf(s - g / gp, 0.f), D);
        }
        sx = Up[0] + hx * (s / D);
        sy = Up[1] + hy * (s / D);
    }
    // 2. node scan (FP32), strict < in i-major, j-minor order
    int is = min(max(__float2int_rn(sx / m.stepx), 0), m.nx - 1);
    int js = min(max(__float2int_rn(sy / m.stepy), 0), m.ny - 1);
    int ia = max(is - W, 0), ib = min(is + W, m.nx - 1);
    int ja = max(js - W, 0), jb = min(js + W, m.ny - 1);
    float bestL = INFINITY;
    int bi = is, bj = js;
    for (int i = ia; i <= ib; i++) {
        float xi = (float)i * m.stepx;
        float dxa = xi - A32[0], dxb = xi - B32[0];
        float sxa = dxa * dxa, sxb = dxb * dxb;
        const float* zrow = m.z32 + i;
        for (int j = ja; j <= jb; j++) {
            float yj = (float)j * m.stepy;
            float zij = __ldg(zrow + (int64_t)j * m.nx);
            float dya = yj - A32[1], dyb = yj - B32[1];
            float dza = zij - A32[2], dzb = zij - B32[2];
            float qa = fmaf(dza, dza, fmaf(dya, dya, sxa));
            float qb = fmaf(dzb, dzb, fmaf(dyb, dyb, sxb));
            float L = na * (qa * rsqrtf(qa)) + nb * (qb * rsqrtf(qb));
            if (L < bestL) {
                bestL = L;
                bi = i;
                bj = j;
            }
        }
    }
    // 3. polish the facets around the best node (FP32)
    int bfi = min(bi, m.nx - 2), bfj = min(bj, m.ny - 2);     // fallback facet
    float bestF = INFINITY, bu = (float)(bi - bfi), bv = (float)(bj - bfj);
#pragma unroll 1
    for (int k = 0; k < 4; k++) {
        int fi = bi - 1 + (k >> 1), fj = bj - 1 + (k & 1);
        if (fi < 0 || fj < 0 || fi > m.nx - 2 || fj > m.ny - 2) continue;
        Facet32 F;
        F.x0 = (float)fi * m.stepx;
        F.y0 = (float)fj * m.stepy;
        F.dx = m.stepx;
        F.dy = m.stepy;
        float z00 = zf(m, fi, fj), z01 = zf(m, fi + 1, fj), z10 = zf(m, fi, fj + 1), z11 = zf(m, fi + 1, fj + 1);
        F.z00 = z00;
        F.b = z01 - z00;
        F.c = z10 - z00;
        F.e = z11 - z01 - z10 + z00;
        float u = (float)(bi - fi), v = (float)(bj - fj);
#pragma unroll 1
        for (int it = 0; it < kPolishIters; it++)
            if (!facet_step32(F, A32, B32, na, nb, u, v)) break;
        float L = facet_eval32(F, A32, B32, na, nb, u, v);
        if (L < bestF) {
            bestF = L;
            bu = u;
            bv = v;
            bfi = fi;
            bfj = fj;
        }
    }
    // 4. FP64 final step
    return final_step64(d, bfi, bfj, A, B, (double)na, (double)nb, (double)bu, (double)bv, dA, dB);
}

}  // namespace

template <int FP16>
__global__ void __launch_bounds__(128) k_bp_mixed(BpArgs a, MixedCtx m)
{
    const int* __restrict__ ref_bin_i = a.ref_bin_i;
    const float* __restrict__ ref_bin_f = a.ref_bin_f;
    const int np = a.np;
    const float k_bin = (float)(a.fs_eff / a.c);
    const float k_phase = (float)(2.0 * 3.14159265358979323846 / a.lambda);
    const float n1f = (float)a.n1, n2f = (float)a.n2;
    const int64_t nr = a.nr;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < a.v_count;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t v = a.v_begin + k;
        const int yi = (int)(v % a.ny);
        const int xi = (int)((v / a.ny) % a.nx);
        const int zi = (int)(v / ((int64_t)a.nx * a.ny));
        const double P[3] = {__ldg(a.gx + xi), __ldg(a.gy + yi), __ldg(a.gz + zi)};
        const float P32[3] = {(float)(P[0] - m.ox), (float)(P[1] - m.oy), (float)P[2]};
        float accr = 0.f, acci = 0.f, cmpr = 0.f, cmpi = 0.f;
        for (int i = 0; i < np; i++) {
            const double T[3] = {__ldg(a.tx + 3 * i), __ldg(a.tx + 3 * i + 1), __ldg(a.tx + 3 * i + 2)};
            const double R[3] = {__ldg(a.rx + 3 * i), __ldg(a.rx + 3 * i + 1), __ldg(a.rx + 3 * i + 2)};
            const float T32[3] = {(float)(T[0] - m.ox), (float)(T[1] - m.oy), (float)T[2]};
            const float R32[3] = {(float)(R[0] - m.ox), (float)(R[1] - m.oy), (float)R[2]};
            double r1t, r2t, r2r, r1r;
            double Lida = solve_mixed(a.dem, m, T, P, T32, P32, n1f, n2f, a.W, r1t, r2t);
            double Lvol = solve_mixed(a.dem, m, P, R, P32, R32, n2f, n1f, a.W, r2r, r1r);
            // per-pulse legs: n1*r1Tx + n2*r2Tx + n2*r2Rx + n1*r1Rx
            const double L = Lida + Lvol;
            const float dL = (float)(L - __ldg(a.ref_L + i));
            // fast-time bin: integer anchor + FP32 offset
            const float t = __ldg(ref_bin_f + i) + dL * k_bin;
            const float fl = floorf(t);
            const int64_t lo = (int64_t)__ldg(ref_bin_i + i) + (int64_t)fl;
            const float q = t - fl;
            const bool exact = (q == 0.0f);
            if (lo >= 0 && (lo < nr - 1 || (lo == nr - 1 && exact))) {
                float s0r, s0i, s1r = 0.f, s1i = 0.f;
                const int64_t base = (int64_t)i * nr + lo;
                if constexpr (FP16) {
                    const float sc = __ldg(a.scale16 + i);
                    float2 f0 = __half22float2(a.rc16[base]);
                    s0r = f0.x * sc;
                    s0i = f0.y * sc;
                    if (!exact) {
                        float2 f1 = __half22float2(a.rc16[base + 1]);
                        s1r = f1.x * sc;
                        s1i = f1.y * sc;
                    }
                } else {
                    float2 f0 = __ldg(a.rc32 + base);
                    s0r = f0.x;
                    s0i = f0.y;
                    if (!exact) {
                        float2 f1 = __ldg(a.rc32 + base + 1);
                        s1r = f1.x;
                        s1i = f1.y;
                    }
                }
                const float w0 = 1.0f - q;
                const float vr = exact ? s0r : fmaf(w0, s0r, q * s1r);
                const float vi = exact ? s0i : fmaf(w0, s0i, q * s1i);
                // carrier phase: FP64-reduced anchor + FP32 offset, reduced again to [-pi, pi]
                float ph = __ldg(a.ref_phase + i) + dL * k_phase;
                const float kk = rintf(ph * 0.15915494309189535f);
                ph = fmaf(-kk, 6.28318548202514648f, ph);
                ph = fmaf(-kk, -1.7484555e-7f, ph);
                float sn, cs;
                __sincosf(ph, &sn, &cs);
                const float cr = vr * cs - vi * sn;
                const float ci = vr * sn + vi * cs;
                // Kahan-compensated sums
                float y = cr - cmpr;
                float tt = accr + y;
                cmpr = (tt - accr) - y;
                accr = tt;
                y = ci - cmpi;
                tt = acci + y;
                cmpi = (tt - acci) - y;
                acci = tt;
            }
        }
        a.out[((int64_t)xi * a.ny + yi) * a.nz + zi] =
            make_double2((double)accr - (double)cmpr, (double)acci - (double)cmpi);
    }
}

cudaError_t launch_bp_mixed(const BpArgs& a, int legs, int fp16, cudaStream_t st)
{
    // the mean-over-pulses legs of the reference (proc_test_script.cpp:518-548) are served
    // by the FP64 form only
    if (legs == 0) return cudaErrorNotSupported;
    MixedCtx m;
    m.z32 = a.dem.z32;
    m.nx = a.dem.nx;
    m.ny = a.dem.ny;
    m.stepx = (float)a.dem.stepx;
    m.stepy = (float)a.dem.stepy;
    m.ox = a.dem.x0;
    m.oy = a.dem.y0;
    int64_t blocks64 = (a.v_count + 127) / 128;
    int blocks = (int)(blocks64 < 1 ? 1 : (blocks64 > (int64_t)1 << 30 ? (int64_t)1 << 30 : blocks64));
    if (fp16)
        k_bp_mixed<1><<<blocks, 128, 0, st>>>(a, m);
    else
        k_bp_mixed<0><<<blocks, 128, 0, st>>>(a, m);
    return cudaGetLastError();
}

}  // namespace bsar
