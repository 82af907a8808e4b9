// dev_common.cuh -- device-side DEM view and the reference's DEM / Fermat arithmetic.
//
// Everything in the FP64 section is written to reproduce the reference's results bit
// for bit: the translation units that include it are compiled with --fmad=false, and
// every expression keeps the reference's operation order (sqrt and division are IEEE
// correctly rounded in CUDA, as on the host).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "dev_view.hpp"

namespace bsar {

// std::min / std::max as libstdc++ defines them (their NaN order is part of the result).
__device__ __forceinline__ double std_min(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double std_max(double a, double b) { return (a < b) ? b : a; }

// First i with v[i] <= x <= v[i+1] (the reference's linear scan,
// src/raw_data_processing.cpp:625-640); -1 when none.  For non-decreasing axes the
// first match is found by a lower bound over v[1..n-1]; otherwise by the scan itself.
__device__ __forceinline__ int axis_interval(const double* __restrict__ v, int n, double x, int asc)
{
    if (n < 2) return -1;
    if (asc) {
        int lo = 1, hi = n;
        while (lo < hi) {
            int mid = (lo + hi) >> 1;
            if (__ldg(v + mid) < x) lo = mid + 1; else hi = mid;
        }
        if (lo >= n) return -1;
        int i = lo - 1;
        return (x >= __ldg(v + i) && x <= __ldg(v + i + 1)) ? i : -1;
    }
    for (int i = 0; i + 1 < n; i++)
        if (x >= __ldg(v + i) && x <= __ldg(v + i + 1)) return i;
    return -1;
}

// One axis of interpolateDEMElevation: indices (i0, i1) and the clamped weight,
// src/raw_data_processing.cpp:621-671.  An unmatched axis keeps (0, 0), its span is
// replaced by 1.0 and the weight is clamp(x - v[0], 0, 1).
struct AxisLookup {
    int i0, i1;
    double w;
};

__device__ __forceinline__ AxisLookup axis_lookup(const double* __restrict__ v, int n, double x, int asc)
{
    AxisLookup r;
    int i = axis_interval(v, n, x, asc);
    r.i0 = i < 0 ? 0 : i;
    r.i1 = i < 0 ? 0 : i + 1;
    double d = __ldg(v + r.i1) - __ldg(v + r.i0);
    if (d == 0) d = 1.0;
    double w = (x - __ldg(v + r.i0)) / d;
    r.w = std_max(0.0, std_min(1.0, w));
    return r;
}

// The height combination of interpolateDEMElevation, :649-677.
__device__ __forceinline__ double dem_combine(const DemView& d, const AxisLookup& ax, const AxisLookup& ay)
{
    const double* __restrict__ Z = d.z;
    double z00 = __ldg(Z + (int64_t)ay.i0 * d.nx + ax.i0);
    if (ax.i0 == ax.i1 && ay.i0 == ay.i1) return z00;
    double z01 = __ldg(Z + (int64_t)ay.i0 * d.nx + ax.i1);
    double z10 = __ldg(Z + (int64_t)ay.i1 * d.nx + ax.i0);
    double z11 = __ldg(Z + (int64_t)ay.i1 * d.nx + ax.i1);
    double wx = ax.w, wy = ay.w;
    return z00 * (1 - wx) * (1 - wy) + z01 * wx * (1 - wy) + z10 * (1 - wx) * wy + z11 * wx * wy;
}

// interpolateDEMElevation, src/raw_data_processing.cpp:615-680.
__device__ __forceinline__ double dem_elevation(const DemView& d, double x, double y)
{
    if (d.empty) return 0.0;
    AxisLookup ax = axis_lookup(d.xv, d.nx, x, d.asc_x);
    AxisLookup ay = axis_lookup(d.yv, d.ny, y, d.asc_y);
    return dem_combine(d, ax, ay);
}

// Optical path n1*|X-P1| + n2*|P2-X| as the grid search writes it (:532-534).
__device__ __forceinline__ double grid_optical(double px, double py, double pz, double x1, double y1,
                                               double z1, double x2, double y2, double z2,
                                               double n1, double n2)
{
    double d1 = sqrt((px - x1) * (px - x1) + (py - y1) * (py - y1) + (pz - z1) * (pz - z1));
    double d2 = sqrt((x2 - px) * (x2 - px) + (y2 - py) * (y2 - py) + (z2 - pz) * (z2 - pz));
    return n1 * d1 + n2 * d2;
}

// One level of the reference's grid search (:509-551) with a G x G grid.  The y-axis
// lookups of the G columns do not depend on the row, so they are made once per level.
// Column tables of one search level in shared memory, [column][thread] (consecutive
// lanes, consecutive words): the G column positions and y-axis lookups stay out of the
// registers.  TPB is the largest block the calling kernel launches with.
template <int TPB> struct GridCols {
    double py[15][TPB];
    double w[15][TPB];
    int2 ii[15][TPB];
};

template <int G, int TPB>
__device__ __forceinline__ void grid_level(const DemView& d, double x1, double y1, double z1,
                                           double x2, double y2, double z2, double n1, double n2,
                                           double R, double& bestX, double& bestY, double& minOP,
                                           GridCols<TPB>* cols)
{
    const double minX = bestX - R, maxX = bestX + R;
    const double minY = bestY - R, maxY = bestY + R;
    const int t = threadIdx.x;
#pragma unroll
    for (int j = 0; j < G; j++) {
        const double py = minY + j * (maxY - minY) / (G - 1);
        cols->py[j][t] = py;
        if (!d.empty) {
            const AxisLookup a = axis_lookup(d.yv, d.ny, py, d.asc_y);
            cols->w[j][t] = a.w;
            cols->ii[j][t] = make_int2(a.i0, a.i1);
        }
    }
    for (int i = 0; i < G; i++) {
        double px = minX + i * (maxX - minX) / (G - 1);
        AxisLookup ax;
        if (!d.empty) ax = axis_lookup(d.xv, d.nx, px, d.asc_x);
#pragma unroll
        for (int j = 0; j < G; j++) {
            const double py = cols->py[j][t];
            double pz = 0.0;
            if (!d.empty) {
                const int2 ii = cols->ii[j][t];
                const AxisLookup ay{ii.x, ii.y, cols->w[j][t]};
                pz = dem_combine(d, ax, ay);
            }
            double op = grid_optical(px, py, pz, x1, y1, z1, x2, y2, z2, n1, n2);
            if (op < minOP) {
                minOP = op;
                bestX = px;
                bestY = py;
            }
        }
    }
}

// calculateRefractionPoint, src/raw_data_processing.cpp:455-572.
template <int TPB>
__device__ __forceinline__ void refraction_grid(const DemView& d, double x1, double y1, double z1,
                                                double x2, double y2, double z2, double n1,
                                                double n2, double out[3])
{
    __shared__ GridCols<TPB> cols;
    double bestX = (x1 + x2) / 2.0;
    double bestY = (y1 + y2) / 2.0;
    double dd = sqrt((x2 - x1) * (x2 - x1) + (y2 - y1) * (y2 - y1));
    double R = std_max(dd, 500.0);
    double minOP = 1e9;
    grid_level<15, TPB>(d, x1, y1, z1, x2, y2, z2, n1, n2, R, bestX, bestY, minOP, &cols);
    R /= 5.0;
#pragma unroll 1
    for (int level = 1; level < 5; level++) {
        grid_level<11, TPB>(d, x1, y1, z1, x2, y2, z2, n1, n2, R, bestX, bestY, minOP, &cols);
        R /= 3.0;
    }
    out[0] = bestX;
    out[1] = bestY;
    out[2] = dem_elevation(d, bestX, bestY);
}

// ---------------------------------------------------------------------------------
// Newton Fermat solver, FP64.  Steps: flat-interface Snell start; node scan of
// +-W DEM nodes around it; active-set projected Newton on the facets sharing the best
// node; one final step on the winning facet.  (No reference counterpart; the oracle's
// bo_refraction_newton restates it.)
// ---------------------------------------------------------------------------------
constexpr int kFlatIters = 4;
constexpr int kPolishIters = 3;

struct Facet64 {
    double x0, y0, dx, dy, z00, b, c, e;
};

__device__ __forceinline__ void facet_load(const DemView& d, int fi, int fj, Facet64& F)
{
    const double* __restrict__ Z = d.z;
    int64_t nx = d.nx;
    F.x0 = __ldg(d.xv + fi);
    F.y0 = __ldg(d.yv + fj);
    F.dx = __ldg(d.xv + fi + 1) - F.x0;
    F.dy = __ldg(d.yv + fj + 1) - F.y0;
    double z00 = __ldg(Z + fj * nx + fi), z01 = __ldg(Z + fj * nx + fi + 1);
    double z10 = __ldg(Z + (fj + 1) * nx + fi), z11 = __ldg(Z + (fj + 1) * nx + fi + 1);
    F.z00 = z00;
    F.b = z01 - z00;
    F.c = z10 - z00;
    F.e = z11 - z01 - z10 + z00;
}

__device__ __forceinline__ double clamp01(double t) { return t < 0.0 ? 0.0 : (t > 1.0 ? 1.0 : t); }

__device__ __forceinline__ bool facet_step(const Facet64& F, const double A[3], const double B[3],
                                           double na, double nb, double& u, double& v)
{
    double x = F.x0 + u * F.dx, y = F.y0 + v * F.dy;
    double h = F.z00 + F.b * u + F.c * v + F.e * u * v;
    double zx = (F.b + F.e * v) / F.dx;
    double zy = (F.c + F.e * u) / F.dy;
    double zxy = F.e / (F.dx * F.dy);
    double r1x = x - A[0], r1y = y - A[1], r1z = h - A[2];
    double r2x = x - B[0], r2y = y - B[1], r2z = h - B[2];
    double q1 = r1x * r1x + r1y * r1y + r1z * r1z;
    double q2 = r2x * r2x + r2y * r2y + r2z * r2z;
    double g1 = na / sqrt(q1), g2 = nb / sqrt(q2);
    double a1x = r1x + r1z * zx, a1y = r1y + r1z * zy;
    double a2x = r2x + r2z * zx, a2y = r2y + r2z * zy;
    double gx = g1 * a1x + g2 * a2x;
    double gy = g1 * a1y + g2 * a2y;
    double txx = 1.0 + zx * zx, tyy = 1.0 + zy * zy, txy = zx * zy;
    double hxx = g1 * (txx - a1x * a1x / q1) + g2 * (txx - a2x * a2x / q2);
    double hyy = g1 * (tyy - a1y * a1y / q1) + g2 * (tyy - a2y * a2y / q2);
    double hxy = g1 * (txy - a1x * a1y / q1) + g2 * (txy - a2x * a2y / q2) + (g1 * r1z + g2 * r2z) * zxy;
    bool au = (u <= 0.0 && gx > 0.0) || (u >= 1.0 && gx < 0.0);
    bool av = (v <= 0.0 && gy > 0.0) || (v >= 1.0 && gy < 0.0);
    double gs = g1 + g2;
    double su, sv;
    if (au && av) return false;
    if (au) {
        su = 0.0;
        sv = (hyy > 0.0) ? -gy / hyy : -gy / gs;
    } else if (av) {
        sv = 0.0;
        su = (hxx > 0.0) ? -gx / hxx : -gx / gs;
    } else {
        double det = hxx * hyy - hxy * hxy;
        if (det > 0.0 && hxx > 0.0) {
            su = -(hyy * gx - hxy * gy) / det;
            sv = -(hxx * gy - hxy * gx) / det;
        } else {
            su = -gx / gs;
            sv = -gy / gs;
        }
    }
    u = clamp01(u + su / F.dx);
    v = clamp01(v + sv / F.dy);
    return true;
}

__device__ __forceinline__ double facet_eval(const Facet64& F, const double A[3], const double B[3],
                                             double na, double nb, double u, double v, double X[3])
{
    X[0] = F.x0 + u * F.dx;
    X[1] = F.y0 + v * F.dy;
    X[2] = F.z00 + F.b * u + F.c * v + F.e * u * v;
    double r1x = X[0] - A[0], r1y = X[1] - A[1], r1z = X[2] - A[2];
    double r2x = X[0] - B[0], r2y = X[1] - B[1], r2z = X[2] - B[2];
    return na * sqrt(r1x * r1x + r1y * r1y + r1z * r1z) + nb * sqrt(r2x * r2x + r2y * r2y + r2z * r2z);
}

__device__ __forceinline__ void flat_start(const double U[3], const double L[3], double nu, double nl,
                                           double h0, int iters, double& sx, double& sy)
{
    double hx = L[0] - U[0], hy = L[1] - U[1];
    double D = sqrt(hx * hx + hy * hy);
    if (!(D >= 1e-9)) {
        sx = L[0];
        sy = L[1];
        return;
    }
    double ha = fabs(U[2] - h0), hb = fabs(L[2] - h0);
    double s = D * ha / (ha + hb + 1e-30);
    if (!(s >= 0.0)) s = 0.0;
    if (s > D) s = D;
    for (int it = 0; it < iters; it++) {
        double q1 = sqrt(s * s + ha * ha);
        double r = D - s;
        double q2 = sqrt(r * r + hb * hb);
        double g = nu * s / q1 - nl * r / q2;
        double gp = nu * ha * ha / (q1 * q1 * q1) + nl * hb * hb / (q2 * q2 * q2);
        if (!(gp > 0.0)) break;
        s = s - g / gp;
        if (s < 0.0) s = 0.0;
        if (s > D) s = D;
    }
    sx = U[0] + hx * (s / D);
    sy = U[1] + hy * (s / D);
}

__device__ __forceinline__ int nearest_node(double v0, double step, int n, double s)
{
    double t = floor((s - v0) / step + 0.5);
    if (!(t >= 0.0)) return 0;
    if (t > (double)(n - 1)) return n - 1;
    return (int)t;
}

// Crossing point of the path A (index na) -> B (index nb), FP64.
__device__ __forceinline__ void refraction_newton(const DemView& d, const double A[3], const double B[3],
                                                  double na, double nb, int W, double out[3])
{
    const bool lower_b = nb >= na;
    const double* Lp = lower_b ? B : A;
    const double* Up = lower_b ? A : B;
    double nl = lower_b ? nb : na, nu = lower_b ? na : nb;
    double h0 = dem_elevation(d, Lp[0], Lp[1]);
    double sx, sy;
    if (d.empty || d.nx < 2 || d.ny < 2) {
        flat_start(Up, Lp, nu, nl, h0, 4 * kFlatIters, sx, sy);
        out[0] = sx;
        out[1] = sy;
        out[2] = dem_elevation(d, sx, sy);
        return;
    }
    flat_start(Up, Lp, nu, nl, h0, kFlatIters, sx, sy);
    int is = nearest_node(d.x0, d.stepx, d.nx, sx), js = nearest_node(d.y0, d.stepy, d.ny, sy);
    int ia = max(is - W, 0), ib = min(is + W, d.nx - 1);
    int ja = max(js - W, 0), jb = min(js + W, d.ny - 1);
    double bestL = INFINITY;
    int bi = is, bj = js;
    const double* __restrict__ Z = d.z;
    for (int i = ia; i <= ib; i++) {
        double xi = __ldg(d.xv + i);
        double r1x = xi - A[0], r2x = xi - B[0];
        for (int j = ja; j <= jb; j++) {
            double yj = __ldg(d.yv + j);
            double zij = __ldg(Z + (int64_t)j * d.nx + i);
            double r1y = yj - A[1], r1z = zij - A[2];
            double r2y = yj - B[1], r2z = zij - B[2];
            double L = na * sqrt(r1x * r1x + r1y * r1y + r1z * r1z) + nb * sqrt(r2x * r2x + r2y * r2y + r2z * r2z);
            if (L < bestL) {
                bestL = L;
                bi = i;
                bj = j;
            }
        }
    }
    // fallback facet (kept only when no facet path compares below +inf, e.g. NaN input)
    int bfi = min(bi, d.nx - 2), bfj = min(bj, d.ny - 2);
    double bestF = INFINITY, bu = (double)(bi - bfi), bv = (double)(bj - bfj);
#pragma unroll 1
    for (int k = 0; k < 4; k++) {
        int fi = bi - 1 + (k >> 1), fj = bj - 1 + (k & 1);
        if (fi < 0 || fj < 0 || fi > d.nx - 2 || fj > d.ny - 2) continue;
        Facet64 F;
        facet_load(d, fi, fj, F);
        double u = (double)(bi - fi), v = (double)(bj - fj);
#pragma unroll 1
        for (int it = 0; it < kPolishIters; it++)
            if (!facet_step(F, A, B, na, nb, u, v)) break;
        double X[3];
        double L = facet_eval(F, A, B, na, nb, u, v, X);
        if (L < bestF) {
            bestF = L;
            bu = u;
            bv = v;
            bfi = fi;
            bfj = fj;
        }
    }
    Facet64 F;
    facet_load(d, bfi, bfj, F);
    facet_step(F, A, B, na, nb, bu, bv);
    facet_eval(F, A, B, na, nb, bu, bv, out);
}

// Dispatch on the solver (0 = grid, 1 = Newton).
// TPB: the largest block size the calling kernel launches with (the grid search keeps
// one column of shared-memory tables per thread).
template <int SOLVER, int TPB>
__device__ __forceinline__ void refraction_point(const DemView& d, const double A[3], const double B[3],
                                                 double na, double nb, int W, double out[3])
{
    if constexpr (SOLVER == 0)
        refraction_grid<TPB>(d, A[0], A[1], A[2], B[0], B[1], B[2], na, nb, out);
    else
        refraction_newton(d, A, B, na, nb, W, out);
}

}  // namespace bsar
