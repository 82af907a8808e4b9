/*
 * bsar_oracle.c -- CPU restatement of the bistatic SAR back-projection hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle: it is linked by the
 * tests, by __graft_entry__.smoke() and by the CPU-baseline leg of bench.py, and
 * by nothing else.  The product path (c-_bistatic_sar_b200/) never calls it.
 *
 * Every function restates one function of the reference project
 * (DavidAtenciaMondragon/c-_bistatic_sar) in plain C, in the same operation
 * order, so that with -ffp-contract=off it reproduces the reference's FP64
 * results bit for bit.  The restatement is pinned against the reference's own
 * compiled sources (oracle/_ref, built by oracle/Makefile) and against the
 * committed fixtures in tests/golden/.
 *
 * The Newton Fermat solver at the end has no reference counterpart: it restates
 * the algorithm of the product's Newton kernels (same steps, FP64) so the mixed
 * GPU form can be gated against an FP64 CPU result.
 *
 * Layouts used throughout:
 *   complex arrays   interleaved (re, im) doubles
 *   point arrays     n x 3 row-major (x, y, z)
 *   DEM              z[j * nx + i] = Z_DEM[j][i]  (row j <-> Y_vec[j], column i <-> X_vec[i]);
 *                    entries the reference would find missing in a ragged Z_DEM are 0.0
 *   pulses           pulse-major: sample s of pulse p at [p * n + s]
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

typedef struct bo_dem {
    int64_t nx, ny;       /* X_vec.size(), Y_vec.size() */
    const double *xv, *yv;
    const double *z;      /* ny * nx */
    int32_t empty;        /* X_vec, Y_vec or Z_DEM empty -> elevation 0 */
    int32_t pad;
} bo_dem;

/* std::min / std::max exactly as libstdc++ defines them (NaN-order matters). */
static inline double std_min(double a, double b) { return (b < a) ? b : a; }
static inline double std_max(double a, double b) { return (a < b) ? b : a; }

/* First interval [v[i], v[i+1]] containing x, linear scan; none -> (0, 0).
 * src/raw_data_processing.cpp:621-640 */
static void axis_interval(const double *v, int64_t n, double x, int64_t *i0, int64_t *i1)
{
    *i0 = 0;
    *i1 = 0;
    for (int64_t i = 0; i + 1 < n; i++) {
        if (x >= v[i] && x <= v[i + 1]) {
            *i0 = i;
            *i1 = i + 1;
            return;
        }
    }
}

/* interpolateDEMElevation, src/raw_data_processing.cpp:615-680 */
double bo_dem_elevation(const bo_dem *d, double x, double y)
{
    if (d->empty) return 0.0;                                   /* :616-618 */
    int64_t i0, i1, j0, j1;
    axis_interval(d->xv, d->nx, x, &i0, &i1);                   /* :625-631 */
    axis_interval(d->yv, d->ny, y, &j0, &j1);                   /* :634-640 */
    /* :643-646 clamps are no-ops for indices produced above */
    const double *Z = d->z;
    const int64_t nx = d->nx;
    double z00 = Z[j0 * nx + i0];                               /* :649-652 */
    double z01 = Z[j0 * nx + i1];
    double z10 = Z[j1 * nx + i0];
    double z11 = Z[j1 * nx + i1];
    if (i0 == i1 && j0 == j1) return z00;                       /* :655-657 */
    double dx = d->xv[i1] - d->xv[i0];                          /* :659-662 */
    double dy = d->yv[j1] - d->yv[j0];
    if (dx == 0) dx = 1.0;                                      /* :664-665 */
    if (dy == 0) dy = 1.0;
    double wx = (x - d->xv[i0]) / dx;                           /* :667-668 */
    double wy = (y - d->yv[j0]) / dy;
    wx = std_max(0.0, std_min(1.0, wx));                        /* :670-671 */
    wy = std_max(0.0, std_min(1.0, wy));
    return z00 * (1 - wx) * (1 - wy) +                          /* :674-677 */
           z01 * wx * (1 - wy) +
           z10 * (1 - wx) * wy +
           z11 * wx * wy;
}

void bo_dem_elevation_batch(const bo_dem *d, const double *xy, int64_t n, double *z)
{
    for (int64_t k = 0; k < n; k++) z[k] = bo_dem_elevation(d, xy[2 * k], xy[2 * k + 1]);
}

/* calculateRefractionPoint, src/raw_data_processing.cpp:455-572:
 * 5-level coarse-to-fine grid search (15x15 then four 11x11) minimising
 * n1*|X-P1| + n2*|P2-X| over X on the DEM surface. */
void bo_refraction_grid(double x1, double y1, double z1, double x2, double y2, double z2,
                        const bo_dem *d, double n1, double n2, double out[3])
{
    double midX = (x1 + x2) / 2.0;                              /* :478-479 */
    double midY = (y1 + y2) / 2.0;
    double directDistance = sqrt((x2 - x1) * (x2 - x1) + (y2 - y1) * (y2 - y1)); /* :483 */
    double searchRadius = std_max(directDistance, 500.0);       /* :484 */
    double bestX = midX, bestY = midY;                          /* :496-497 */
    double minOpticalPath = 1e9;
    double currentRadius = searchRadius;
    for (int level = 0; level < 5; level++) {                   /* :507 */
        int gridSize = (level == 0) ? 15 : 11;                  /* :508 */
        double minX = bestX - currentRadius;
        double maxX = bestX + currentRadius;
        double minY = bestY - currentRadius;
        double maxY = bestY + currentRadius;
        for (int i = 0; i < gridSize; i++) {                    /* :523-543 */
            for (int j = 0; j < gridSize; j++) {
                double px = minX + i * (maxX - minX) / (gridSize - 1);
                double py = minY + j * (maxY - minY) / (gridSize - 1);
                double pz = bo_dem_elevation(d, px, py);
                double d1 = sqrt((px - x1) * (px - x1) + (py - y1) * (py - y1) + (pz - z1) * (pz - z1));
                double d2 = sqrt((x2 - px) * (x2 - px) + (y2 - py) * (y2 - py) + (z2 - pz) * (z2 - pz));
                double opticalPath = n1 * d1 + n2 * d2;
                if (opticalPath < minOpticalPath) {             /* :536 strict < */
                    minOpticalPath = opticalPath;
                    bestX = px;
                    bestY = py;
                }
            }
        }
        currentRadius /= (level == 0) ? 5.0 : 3.0;              /* :551 */
    }
    out[0] = bestX;                                             /* :555-557 */
    out[1] = bestY;
    out[2] = bo_dem_elevation(d, bestX, bestY);
}

/* calculateReflectionPoint, src/raw_data_processing.cpp:575-612 */
void bo_reflection_point(double txX, double txY, double txZ, double rxX, double rxY, double rxZ,
                         const bo_dem *d, double out[3])
{
    (void)txZ;
    (void)rxZ;
    double midX = (txX + rxX) / 2.0;
    double midY = (txY + rxY) / 2.0;
    double minDist = 1e9, bestZ = 0.0;
    if (!d->empty) {
        for (int64_t i = 0; i < d->nx; i++) {
            for (int64_t j = 0; j < d->ny; j++) {
                double dx = d->xv[i] - midX;
                double dy = d->yv[j] - midY;
                double dist = sqrt(dx * dx + dy * dy);
                if (dist < minDist) {
                    minDist = dist;
                    bestZ = d->z[j * d->nx + i];
                }
            }
        }
    }
    out[0] = midX;
    out[1] = midY;
    out[2] = bestZ;
}

/* ---------------------------------------------------------------------------------
 * Newton Fermat solver (FP64).  No reference counterpart: restates, step for step,
 * the algorithm of the product's Newton kernels, so the GPU forms can be gated
 * against it.  Objective f(X) = na*|X-A| + nb*|X-B| for X on the bilinear DEM.
 *   1. start: flat-interface Snell point.  h0 = DEM height under the endpoint with
 *      the larger index; BO_FLAT_ITERS 1-D Newton steps along the horizontal A-B line.
 *   2. node scan: f at every DEM node within +-W nodes of the node nearest the start
 *      (W = search_nodes); strict < in i-major, j-minor order keeps the first minimum.
 *   3. polish: on each of the (up to) 4 facets that share the best node, starting at
 *      that node, BO_POLISH_ITERS active-set projected Newton steps in the facet's
 *      (u, v) box; the facet with the smallest f wins (strict <, fixed facet order).
 *   4. final step: one more projected Newton step on the winning facet.
 * Requires strictly ascending DEM axes; empty or 1-wide DEMs use the flat start.
 * ------------------------------------------------------------------------------- */
#define BO_FLAT_ITERS 4
#define BO_POLISH_ITERS 3

typedef struct bo_facet {
    double x0, y0, dx, dy, z00, b, c, e;
} bo_facet;

static void facet_load(const bo_dem *d, int64_t fi, int64_t fj, bo_facet *F)
{
    const double *Z = d->z;
    int64_t nx = d->nx;
    F->x0 = d->xv[fi];
    F->y0 = d->yv[fj];
    F->dx = d->xv[fi + 1] - F->x0;
    F->dy = d->yv[fj + 1] - F->y0;
    double z00 = Z[fj * nx + fi], z01 = Z[fj * nx + fi + 1];
    double z10 = Z[(fj + 1) * nx + fi], z11 = Z[(fj + 1) * nx + fi + 1];
    F->z00 = z00;
    F->b = z01 - z00;
    F->c = z10 - z00;
    F->e = z11 - z01 - z10 + z00;
}

static double clamp01(double t) { return t < 0.0 ? 0.0 : (t > 1.0 ? 1.0 : t); }

/* One active-set projected Newton step in the facet box; returns 0 when the
 * iterate is a corner minimum (no step possible). */
static int facet_step(const bo_facet *F, const double A[3], const double B[3], double na,
                      double nb, double *u, double *v)
{
    double x = F->x0 + *u * F->dx, y = F->y0 + *v * F->dy;
    double h = F->z00 + F->b * *u + F->c * *v + F->e * *u * *v;
    double zx = (F->b + F->e * *v) / F->dx;
    double zy = (F->c + F->e * *u) / F->dy;
    double zxy = F->e / (F->dx * F->dy);
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
    double hxy = g1 * (txy - a1x * a1y / q1) + g2 * (txy - a2x * a2y / q2) +
                 (g1 * r1z + g2 * r2z) * zxy;
    int au = (*u <= 0.0 && gx > 0.0) || (*u >= 1.0 && gx < 0.0);
    int av = (*v <= 0.0 && gy > 0.0) || (*v >= 1.0 && gy < 0.0);
    double gs = g1 + g2;
    double su, sv;
    if (au && av) return 0;
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
    *u = clamp01(*u + su / F->dx);
    *v = clamp01(*v + sv / F->dy);
    return 1;
}

static double facet_eval(const bo_facet *F, const double A[3], const double B[3], double na,
                         double nb, double u, double v, double X[3])
{
    X[0] = F->x0 + u * F->dx;
    X[1] = F->y0 + v * F->dy;
    X[2] = F->z00 + F->b * u + F->c * v + F->e * u * v;
    double r1x = X[0] - A[0], r1y = X[1] - A[1], r1z = X[2] - A[2];
    double r2x = X[0] - B[0], r2y = X[1] - B[1], r2z = X[2] - B[2];
    return na * sqrt(r1x * r1x + r1y * r1y + r1z * r1z) + nb * sqrt(r2x * r2x + r2y * r2y + r2z * r2z);
}

/* Flat-interface Snell start; (sx, sy) is the horizontal crossing estimate. */
static void flat_start(const double U[3], const double L[3], double nu, double nl, double h0,
                       int iters, double *sx, double *sy)
{
    double hx = L[0] - U[0], hy = L[1] - U[1];
    double D = sqrt(hx * hx + hy * hy);
    if (!(D >= 1e-9)) {
        *sx = L[0];
        *sy = L[1];
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
    *sx = U[0] + hx * (s / D);
    *sy = U[1] + hy * (s / D);
}

/* Node index nearest to s on an ascending axis with mean spacing (v[n-1]-v[0])/(n-1). */
static int64_t nearest_node(const double *v, int64_t n, double s)
{
    double step = (v[n - 1] - v[0]) / (double)(n - 1);
    double t = floor((s - v[0]) / step + 0.5);
    if (!(t >= 0.0)) return 0;
    if (t > (double)(n - 1)) return n - 1;
    return (int64_t)t;
}

void bo_refraction_newton(double x1, double y1, double z1, double x2, double y2, double z2,
                          const bo_dem *d, double n1, double n2, int32_t search_nodes,
                          double out[3])
{
    const double A[3] = {x1, y1, z1}, B[3] = {x2, y2, z2};
    const int lower_b = n2 >= n1;
    const double *Lp = lower_b ? B : A, *Up = lower_b ? A : B;
    double nl = lower_b ? n2 : n1, nu = lower_b ? n1 : n2;
    double h0 = bo_dem_elevation(d, Lp[0], Lp[1]);
    double sx, sy;
    if (d->empty || d->nx < 2 || d->ny < 2) {
        flat_start(Up, Lp, nu, nl, h0, 4 * BO_FLAT_ITERS, &sx, &sy);
        out[0] = sx;
        out[1] = sy;
        out[2] = bo_dem_elevation(d, sx, sy);
        return;
    }
    flat_start(Up, Lp, nu, nl, h0, BO_FLAT_ITERS, &sx, &sy);
    int64_t is = nearest_node(d->xv, d->nx, sx), js = nearest_node(d->yv, d->ny, sy);
    int64_t W = search_nodes;
    int64_t ia = is - W < 0 ? 0 : is - W, ib = is + W > d->nx - 1 ? d->nx - 1 : is + W;
    int64_t ja = js - W < 0 ? 0 : js - W, jb = js + W > d->ny - 1 ? d->ny - 1 : js + W;
    double bestL = INFINITY;
    int64_t bi = is, bj = js;
    for (int64_t i = ia; i <= ib; i++) {
        for (int64_t j = ja; j <= jb; j++) {
            double X[3] = {d->xv[i], d->yv[j], d->z[j * d->nx + i]};
            double r1x = X[0] - A[0], r1y = X[1] - A[1], r1z = X[2] - A[2];
            double r2x = X[0] - B[0], r2y = X[1] - B[1], r2z = X[2] - B[2];
            double L = n1 * sqrt(r1x * r1x + r1y * r1y + r1z * r1z) +
                       n2 * sqrt(r2x * r2x + r2y * r2y + r2z * r2z);
            if (L < bestL) {
                bestL = L;
                bi = i;
                bj = j;
            }
        }
    }
    /* fallback facet (kept only when no facet path compares below +inf, e.g. NaN input) */
    int64_t bfi = bi < d->nx - 2 ? bi : d->nx - 2, bfj = bj < d->ny - 2 ? bj : d->ny - 2;
    double bestF = INFINITY, bu = (double)(bi - bfi), bv = (double)(bj - bfj);
    for (int k = 0; k < 4; k++) {
        int64_t fi = bi - 1 + (k >> 1), fj = bj - 1 + (k & 1);
        if (fi < 0 || fj < 0 || fi > d->nx - 2 || fj > d->ny - 2) continue;
        bo_facet F;
        facet_load(d, fi, fj, &F);
        double u = (double)(bi - fi), v = (double)(bj - fj);
        for (int it = 0; it < BO_POLISH_ITERS; it++)
            if (!facet_step(&F, A, B, n1, n2, &u, &v)) break;
        double X[3];
        double L = facet_eval(&F, A, B, n1, n2, u, v, X);
        if (L < bestF) {
            bestF = L;
            bu = u;
            bv = v;
            bfi = fi;
            bfj = fj;
        }
    }
    bo_facet F;
    facet_load(d, bfi, bfj, &F);
    facet_step(&F, A, B, n1, n2, &bu, &bv);                 /* 4. final step */
    facet_eval(&F, A, B, n1, n2, bu, bv, out);
}

/* calculaSlantRangeFermat, src/raw_data_processing.cpp:112-255, for one target P
 * over n pulses.  solver 0 = reference grid search, 1 = Newton.
 * ranges: 4 x n (r1Tx, r2Tx, r1Rx, r2Rx); ida/volta/refl: n x 3 (refl may be NULL). */
void bo_slant_range_fermat(const bo_dem *d, const double *tx, const double *rx, int64_t n,
                           const double P[3], double n1, double n2, int32_t solver,
                           int32_t search_nodes, double *ranges, double *ida, double *volta,
                           double *refl)
{
    double Px = P[0], Py = P[1], Pz = P[2];
    for (int64_t i = 0; i < n; i++) {
        double TxX = tx[3 * i], TxY = tx[3 * i + 1], TxZ = tx[3 * i + 2];
        double RxX = rx[3 * i], RxY = rx[3 * i + 1], RxZ = rx[3 * i + 2];
        double a[3], b[3];
        if (solver == 0) {
            bo_refraction_grid(TxX, TxY, TxZ, Px, Py, Pz, d, n1, n2, a);   /* :166-172 */
            bo_refraction_grid(Px, Py, Pz, RxX, RxY, RxZ, d, n2, n1, b);   /* :175-181 */
        } else {
            bo_refraction_newton(TxX, TxY, TxZ, Px, Py, Pz, d, n1, n2, search_nodes, a);
            bo_refraction_newton(Px, Py, Pz, RxX, RxY, RxZ, d, n2, n1, search_nodes, b);
        }
        if (ida) memcpy(ida + 3 * i, a, sizeof a);
        if (volta) memcpy(volta + 3 * i, b, sizeof b);
        if (refl) bo_reflection_point(TxX, TxY, TxZ, RxX, RxY, RxZ, d, refl + 3 * i);
        if (ranges) {
            ranges[i] = sqrt((TxX - a[0]) * (TxX - a[0]) + (TxY - a[1]) * (TxY - a[1]) +
                             (TxZ - a[2]) * (TxZ - a[2]));                  /* :197-201 */
            ranges[n + i] = sqrt((Px - a[0]) * (Px - a[0]) + (Py - a[1]) * (Py - a[1]) +
                                 (Pz - a[2]) * (Pz - a[2]));                /* :204-208 */
            ranges[2 * n + i] = sqrt((RxX - b[0]) * (RxX - b[0]) + (RxY - b[1]) * (RxY - b[1]) +
                                     (RxZ - b[2]) * (RxZ - b[2]));          /* :211-215 */
            ranges[3 * n + i] = sqrt((Px - b[0]) * (Px - b[0]) + (Py - b[1]) * (Py - b[1]) +
                                     (Pz - b[2]) * (Pz - b[2]));            /* :218-222 */
        }
    }
}

/* splineInterpolation, src/interpolation.cpp:4-51, one pulse of n complex samples. */
void bo_spline_upsample(const double *in, int64_t n, int32_t factor, double *out)
{
    size_t un = (size_t)n;
    size_t newSize = un * (size_t)factor;
    for (size_t i = 0; i < newSize; i++) {
        double pos = (double)i / factor;                          /* :18 */
        size_t idx = (size_t)pos;
        double frac = pos - idx;
        if (idx >= un - 1) {                                      /* :22-25 */
            idx = un - 2;
            frac = 1.0;
        }
        double t = frac, t2 = t * t, t3 = t2 * t;
        double h1 = 2 * t3 - 3 * t2 + 1;                          /* :33-36 */
        double h2 = -2 * t3 + 3 * t2;
        double h3 = t3 - 2 * t2 + t;
        double h4 = t3 - t2;
        for (int c = 0; c < 2; c++) {
            double p0 = in[2 * idx + c], p1 = in[2 * (idx + 1) + c];
            double dPrev = (idx > 0) ? (p0 - in[2 * (idx - 1) + c]) : 0;            /* :39-42 */
            double dNext = (idx < un - 2) ? (in[2 * (idx + 2) + c] - p1) : 0;
            out[2 * i + c] = h1 * p0 + h2 * p1 + h3 * dPrev + h4 * dNext;           /* :45-46 */
        }
    }
}

void bo_spline_upsample_batch(const double *in, int64_t n, int64_t batch, int32_t factor, double *out)
{
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < batch; p++)
        bo_spline_upsample(in + 2 * n * p, n, factor, out + 2 * n * factor * p);
}

/* ------------------------- FFT, src/fft_utils.cpp ------------------------------ */
static int is_pow2(uint64_t n) { return n > 0 && (n & (n - 1)) == 0; }

static uint64_t next_pow2(uint64_t n)                             /* :187-196 */
{
    if (n <= 1) return 1;
    uint64_t p = 1;
    while (p < n) p *= 2;
    return p;
}

/* FFTProcessor::fft, src/fft_utils.cpp:11-44: bit reversal, then radix-2 DIT stages
 * with twiddles advanced by the recurrence w *= wlen.  Non-power-of-two: unchanged. */
void bo_fft(double *a, int64_t n)
{
    uint64_t N = (uint64_t)n;
    if (N <= 1 || !is_pow2(N)) return;
    uint64_t j = 0;                                               /* :164-181 */
    for (uint64_t i = 1; i < N; i++) {
        uint64_t bit = N >> 1;
        while (j & bit) {
            j ^= bit;
            bit >>= 1;
        }
        j ^= bit;
        if (i < j) {
            double tr = a[2 * i], ti = a[2 * i + 1];
            a[2 * i] = a[2 * j];
            a[2 * i + 1] = a[2 * j + 1];
            a[2 * j] = tr;
            a[2 * j + 1] = ti;
        }
    }
    for (uint64_t len = 2; len <= N; len *= 2) {
        double angle = -2.0 * M_PI / len;
        double wlr = cos(angle), wli = sin(angle);
        for (uint64_t i = 0; i < N; i += len) {
            double wr = 1.0, wi = 0.0;
            for (uint64_t k = 0; k < len / 2; k++) {
                double *u = a + 2 * (i + k), *v = a + 2 * (i + k + len / 2);
                double vr = v[0] * wr - v[1] * wi;
                double vi = v[0] * wi + v[1] * wr;
                double ur = u[0], ui = u[1];
                u[0] = ur + vr;
                u[1] = ui + vi;
                v[0] = ur - vr;
                v[1] = ui - vi;
                double nwr = wr * wlr - wi * wli;
                double nwi = wr * wli + wi * wlr;
                wr = nwr;
                wi = nwi;
            }
        }
    }
}

/* FFTProcessor::ifft, src/fft_utils.cpp:46-61 */
void bo_ifft(double *a, int64_t n)
{
    for (int64_t i = 0; i < n; i++) a[2 * i + 1] = -a[2 * i + 1];
    bo_fft(a, n);
    for (int64_t i = 0; i < n; i++) {
        a[2 * i] = a[2 * i] / (double)n;
        a[2 * i + 1] = -a[2 * i + 1] / (double)n;
    }
}

/* fftCorrelation (conj=1, src/fft_utils.cpp:63-101) and fftConvolution (conj=0,
 * :103-138) of one signal against a reference; out has max(ns, nr) entries. */
static void correlate_one(const double *sig, int64_t ns, const double *ref, int64_t nr,
                          int conj, double *out, double *ws)
{
    int64_t N = ns > nr ? ns : nr;
    int64_t P = (int64_t)next_pow2((uint64_t)N);
    double *fs = ws, *fr = ws + 2 * P;
    memset(fs, 0, sizeof(double) * 2 * P);
    memset(fr, 0, sizeof(double) * 2 * P);
    memcpy(fs, sig, sizeof(double) * 2 * ns);
    memcpy(fr, ref, sizeof(double) * 2 * nr);
    bo_fft(fs, P);
    bo_fft(fr, P);
    for (int64_t k = 0; k < P; k++) {
        double a = fs[2 * k], b = fs[2 * k + 1];
        double c = fr[2 * k], e = conj ? -fr[2 * k + 1] : fr[2 * k + 1];
        fs[2 * k] = a * c - b * e;
        fs[2 * k + 1] = a * e + b * c;
    }
    bo_ifft(fs, P);
    memcpy(out, fs, sizeof(double) * 2 * N);
}

/* Pulse compression loop of processRawData, src/raw_data_processing.cpp:431-446
 * (conj=1) and the echo synthesis loop :406-421 (conj=0), for `batch` pulses. */
void bo_fft_correlate_batch(const double *sig, int64_t ns, int64_t batch, const double *ref,
                            int64_t nr, int32_t conj, double *out)
{
    int64_t N = ns > nr ? ns : nr;
    int64_t P = (int64_t)next_pow2((uint64_t)N);
#pragma omp parallel
    {
        double *ws = (double *)malloc(sizeof(double) * 4 * P);
#pragma omp for schedule(static)
        for (int64_t b = 0; b < batch; b++)
            correlate_one(sig + 2 * ns * b, ns, ref, nr, conj, out + 2 * N * b, ws);
        free(ws);
    }
}

/* createCHIRP, src/raw_data_processing.cpp:257-290; returns the sample count. */
int64_t bo_create_chirp(double f0, double f1, double T, double fs, double *out, int64_t cap)
{
    double k = (f1 - f0) / T;
    int N = (int)(T * fs) + 1;
    for (int n = 0; n < N && n < cap; n++) {
        double t = n / fs;
        double phase = 2.0 * M_PI * (f0 * t + (k / 2.0) * t * t);
        out[2 * n] = cos(phase);
        out[2 * n + 1] = sin(phase);
    }
    return N;
}

/* fftshifted matched-filter reference of length nmax built from the chirp,
 * src/raw_data_processing.cpp:371-394. */
void bo_matched_reference(const double *chirp, int64_t nc, int64_t nmax, double *ref)
{
    memset(ref, 0, sizeof(double) * 2 * nmax);
    int64_t half = nc / 2;
    for (int64_t i = 0; i < nc - half; i++) {
        ref[2 * i] = chirp[2 * (half + i)];
        ref[2 * i + 1] = chirp[2 * (half + i) + 1];
    }
    int64_t start = nmax - half;
    for (int64_t i = 0; i < half; i++) {
        ref[2 * (start + i)] = chirp[2 * i];
        ref[2 * (start + i) + 1] = chirp[2 * i + 1];
    }
}

/* ------------------------- back-projection ------------------------------------
 * The inline voxel loop of proc_test_script.cpp:451-767, one voxel at a time.
 *   rc       upsampled range-compressed pulses, pulse-major, np x nr complex
 *   legs     0: R1t/R1r = mean over all pulses (proc_test_script.cpp:518-548)
 *            1: R1t/R1r = the per-pulse r1Tx/r1Rx of calculaSlantRangeFermat
 *   solver   0: grid search (reference), 1: Newton (search_nodes = node-scan half width)
 *   fs_eff   sampling rate of rc (reference: Rx.fs * 4, proc_test_script.cpp:220-223)
 *   voxels   indices in the reference's flat order z -> x -> y (y fastest),
 *            proc_test_script.cpp:132-151; NULL = all nx*ny*nz in that order
 *   out      complex per listed voxel (NULL voxels: image [x][y][z], z fastest,
 *            the layout of output[x][y][z], proc_test_script.cpp:761-767)
 */
typedef struct bo_bp_args {
    const bo_dem *dem;
    const double *tx, *rx;
    int64_t np;
    const double *rc;
    int64_t nr;
    const double *gx, *gy, *gz;
    int64_t nx, ny, nz;
    double n1, n2, c, fs_eff, lambda;
    int32_t legs, solver;
    int32_t search_nodes, pad;
} bo_bp_args;

static void bp_voxel(const bo_bp_args *A, const double P[3], double *ida, double *volta,
                     double *ranges, double acc[2])
{
    int64_t np = A->np;
    bo_slant_range_fermat(A->dem, A->tx, A->rx, np, P, A->n1, A->n2, A->solver, A->search_nodes,
                          ranges, ida, volta, NULL);
    double pr = 0.0, pi = 0.0;
    for (int64_t i = 0; i < np; i++) {
        const double *a = ida + 3 * i, *b = volta + 3 * i;
        double dx = P[0] - a[0], dy = P[1] - a[1], dz = P[2] - a[2];
        double R2t = sqrt(dx * dx + dy * dy + dz * dz);             /* :497-505 */
        dx = P[0] - b[0];
        dy = P[1] - b[1];
        dz = P[2] - b[2];
        double R2r = sqrt(dx * dx + dy * dy + dz * dz);             /* :507-516 */
        double R1t, R1r;
        if (A->legs == 0) {
            double s = 0.0;                                         /* :518-531 */
            for (int64_t k = 0; k < np; k++) {
                double ex = A->tx[3 * k] - a[0], ey = A->tx[3 * k + 1] - a[1],
                       ez = A->tx[3 * k + 2] - a[2];
                s += sqrt(ex * ex + ey * ey + ez * ez);
            }
            R1t = s / (double)np;
            s = 0.0;                                                /* :533-548 */
            for (int64_t k = 0; k < np; k++) {
                double ex = A->rx[3 * k] - b[0], ey = A->rx[3 * k + 1] - b[1],
                       ez = A->rx[3 * k + 2] - b[2];
                s += sqrt(ex * ex + ey * ey + ez * ez);
            }
            R1r = s / (double)np;
        } else {
            R1t = ranges[i];
            R1r = ranges[2 * np + i];
        }
        double n1 = A->n1, n2 = A->n2;
        double t_val = (1.0 / A->c) * (n1 * R1t + n2 * R2t + n2 * R2r + n1 * R1r);   /* :565 */
        double rngBin = 1.0 + (t_val * A->fs_eff);                                  /* :569 */
        double phi = (2.0 * M_PI / A->lambda) * (n1 * R1t + n2 * R2t + n2 * R2r + n1 * R1r); /* :573 */
        double b0 = rngBin - 1.0;                                                   /* :593 */
        int lo = (int)floor(b0);
        int hi = (int)ceil(b0);
        if (lo >= 0 && hi < (int)A->nr) {                                           /* :599 */
            double q = b0 - lo;
            const double *s0 = A->rc + 2 * ((int64_t)lo + i * A->nr);
            const double *s1 = A->rc + 2 * ((int64_t)hi + i * A->nr);
            double vr, vi;
            if (lo == hi) {
                vr = s0[0];
                vi = s0[1];
            } else {
                vr = (1.0 - q) * s0[0] + q * s1[0];                                /* :635 */
                vi = (1.0 - q) * s0[1] + q * s1[1];
            }
            double cr = cos(phi), ci = sin(phi);                                    /* :638 */
            pr += vr * cr - vi * ci;                                                /* :641 */
            pi += vr * ci + vi * cr;
        }
    }
    acc[0] = pr;
    acc[1] = pi;
}

void bo_backproject(const bo_bp_args *A, const int64_t *voxels, int64_t nvox, double *out)
{
    int64_t total = A->nx * A->ny * A->nz;
    int64_t count = voxels ? nvox : total;
#pragma omp parallel
    {
        double *ida = (double *)malloc(sizeof(double) * 3 * A->np);
        double *volta = (double *)malloc(sizeof(double) * 3 * A->np);
        double *ranges = (double *)malloc(sizeof(double) * 4 * A->np);
#pragma omp for schedule(dynamic, 1)
        for (int64_t k = 0; k < count; k++) {
            int64_t v = voxels ? voxels[k] : k;
            int64_t yi = v % A->ny;                                 /* :761-763 */
            int64_t xi = (v / A->ny) % A->nx;
            int64_t zi = v / (A->nx * A->ny);
            double P[3] = {A->gx[xi], A->gy[yi], A->gz[zi]};
            double acc[2];
            bp_voxel(A, P, ida, volta, ranges, acc);
            int64_t o = voxels ? k : (xi * A->ny + yi) * A->nz + zi;
            out[2 * o] = acc[0];
            out[2 * o + 1] = acc[1];
        }
        free(ida);
        free(volta);
        free(ranges);
    }
}
