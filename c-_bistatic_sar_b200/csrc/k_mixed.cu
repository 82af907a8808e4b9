// k_mixed.cu -- the mixed-precision back-projection kernel.
//
// One thread per voxel, voxels of a CTA consecutive in the reference's flat order
// (y fastest), every thread walking the pulses in order.  Lanes of a warp solve the same
// pulse for neighbouring voxels, so their DEM windows, Tx/Rx loads and sample gathers
// coincide or sit next to each other.
//
// DEM tile: at start every CTA stages a TI x TJ FP32 tile of the DEM around its voxels
// (shifted by the scene's mean crossing offset) into shared memory with one TMA 2-D
// tiled load (cp.async.bulk.tensor, no multicast) completing on an mbarrier; node scans
// whose window lies inside the tile read it from there, others read the FP32 DEM in
// global memory.
//
// Per (voxel, pulse):
//   Fermat, twice (Tx -> voxel, voxel -> Rx):
//     FP32  flat-interface start; node scan of the (2W+1)^2 DEM nodes around it
//           (compile-time W for the common widths) ranking na|N-A| + nb|N-B|; when the
//           runner-up is within kTieM metres of the best, the candidates within kTieM are
//           re-ranked in FP64 with the FP64 solver's arithmetic and scan order, so both
//           forms pick the same node; active-set Newton polish on the 4 facets around it
//     FP64  one final Newton step on the winning facet; its leg lengths give the
//           bistatic optical path L in FP64
//   delay / phase: dL = L - L_ref(pulse) rounded to FP32; the fast-time bin and carrier
//           phase are FP32 offsets from per-pulse FP64 anchors (integer bin + fraction,
//           phase reduced to [-pi, pi) in FP64)
//   gather: two complex64 (or FP16 complex x pulse scale) samples, linear interpolation
//           (proc_test_script.cpp:589-636), times exp(j phi), Kahan-compensated FP32 sum.
#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>

#include "dev_common.cuh"
#include "kernels.hpp"

namespace bsar {

namespace {

constexpr int TI = kMixedTileI;    // tile columns (x); 272 B rows, a multiple of 16 B
constexpr int TJ = kMixedTileJ;    // tile rows (y)
// FP32 node-scan ranking ambiguity threshold, metres of optical path.  The largest FP32
// error of a node's ranking value measured against FP64 over 6e9 medium-scene solves was
// 4.8e-6 m (in units of L / ng), so two nodes are mis-ordered only within ~1e-5 m.
constexpr float kTieM = 5.0e-5f;
// A FP32 flat start closer than this to a node-cell boundary is redone in FP64: metres
// of start-position error (the largest measured FP32 start error was 3.1e-5 node units,
// 7.6e-6 m) plus the FP32 quantisation of the node coordinate (ulps of the largest index).
constexpr float kStartBandM = 2.5e-5f;
constexpr float kStartBandUlps = 8.0f;
constexpr long kWaitSpins = 1L << 24;

struct Facet32 {
    float x0, y0, dx, dy, z00, b, c, e;
    float idx, idy;     // 1 / dx, 1 / dy
};

struct MixedCtx {
    const float* __restrict__ z32;  // pitch-padded FP32 heights, z32[j * pitch + i]
    int pitch;
    int nx, ny;
    float stepx, stepy;             // uniform node spacing
    float istepx, istepy;           // 1 / spacing
    double ox, oy;                  // origin of the FP32 frame (first DEM node)
    double idx64, idy64;            // 1 / spacing, FP64
    float start_band;               // node units: FP32 starts this close to a cell boundary go FP64
    int prune;                      // node scans may skip what the lower bound excludes
    float zmin;                     // lowest FP32 height of the DEM
};

// Start heights under a voxel (the lower endpoint of both of its paths when the ground
// index exceeds the air index): FP32 bilinear for the FP32 start, the FP64 DEM lookup for
// the FP64 start.  Computed once per voxel instead of once per solve.
struct VoxelStart {
    float h32;
    double h64;
};

}  // namespace

// Start band of a DEM (node units), see kStartBandM.
float mixed_start_band(const DemView& d)
{
    const double step = d.stepx < d.stepy ? d.stepx : d.stepy;
    const double nmax = (double)(d.nx > d.ny ? d.nx : d.ny);
    return (float)((double)kStartBandM / step + (double)kStartBandUlps * nmax * 0x1.0p-23);
}

namespace {

// A DEM tile in shared memory: node (i, j) at s[(j - j0) * TI + (i - i0)].
struct Tile {
    const float* s;
    int i0, j0;
    bool ok;
};

__device__ __forceinline__ float zf(const MixedCtx& m, int i, int j) { return __ldg(m.z32 + (int64_t)j * m.pitch + i); }

// FP32 bilinear height (clamped to the DEM) for the flat-interface start.
__device__ __forceinline__ float height32(const MixedCtx& m, float x, float y)
{
    float fx = x * m.istepx, fy = y * m.istepy;
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
    const float idx_ = F.idx, idy = F.idy;
    float zx = (F.b + F.e * v) * idx_;
    float zy = (F.c + F.e * u) * idy;
    float r1x = x - A[0], r1y = y - A[1], r1z = h - A[2];
    float r2x = x - B[0], r2y = y - B[1], r2z = h - B[2];
    float q1 = r1x * r1x + r1y * r1y + r1z * r1z;
    float q2 = r2x * r2x + r2y * r2y + r2z * r2z;
    float s1 = rsqrtf(q1), s2 = rsqrtf(q2);
    float g1 = na * s1, g2 = nb * s2;
    float a1x = r1x + r1z * zx, a1y = r1y + r1z * zy;
    float a2x = r2x + r2z * zx, a2y = r2y + r2z * zy;
    float gx = g1 * a1x + g2 * a2x;
    float gy = g1 * a1y + g2 * a2y;
    // active set first: a corner the gradient pushes outward of on both axes is this
    // facet's minimum, and the Hessian is not needed
    bool au = (u <= 0.0f && gx > 0.0f) || (u >= 1.0f && gx < 0.0f);
    bool av = (v <= 0.0f && gy > 0.0f) || (v >= 1.0f && gy < 0.0f);
    if (au && av) return false;
    float zxy = F.e * idx_ * idy;
    float iq1 = s1 * s1, iq2 = s2 * s2;
    float txx = 1.0f + zx * zx, tyy = 1.0f + zy * zy, txy = zx * zy;
    float hxx = g1 * (txx - a1x * a1x * iq1) + g2 * (txx - a2x * a2x * iq2);
    float hyy = g1 * (tyy - a1y * a1y * iq1) + g2 * (tyy - a2y * a2y * iq2);
    float hxy = g1 * (txy - a1x * a1y * iq1) + g2 * (txy - a2x * a2y * iq2) + (g1 * r1z + g2 * r2z) * zxy;
    // approximate reciprocals (2 ulp): they set a Newton step's length, which the FP64
    // final step corrects, so a correctly rounded one buys nothing
    float igs = __fdividef(1.0f, g1 + g2);
    float su, sv;
    if (au) {
        su = 0.0f;
        sv = (hyy > 0.0f) ? -gy * __fdividef(1.0f, hyy) : -gy * igs;
    } else if (av) {
        sv = 0.0f;
        su = (hxx > 0.0f) ? -gx * __fdividef(1.0f, hxx) : -gx * igs;
    } else {
        float det = hxx * hyy - hxy * hxy;
        if (det > 0.0f && hxx > 0.0f) {
            float idet = __fdividef(1.0f, det);
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
                                               double na, double nb, double u, double v, double& dA, double& dB,
                                               double* X, double idx_, double idy)
{
    Facet64 F;
    facet_load(d, fi, fj, F);
    {
        double x = F.x0 + u * F.dx, y = F.y0 + v * F.dy;
        double h = F.z00 + F.b * u + F.c * v + F.e * u * v;
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
            // one division: the reciprocal of the pivot the taken branch needs
            double det = hxx * hyy - hxy * hxy;
            const bool newton = !au && !av && det > 0.0 && hxx > 0.0;
            const bool axis = (au && hyy > 0.0) || (av && !au && hxx > 0.0);
            const double piv = newton ? det : (axis ? (au ? hyy : hxx) : g1 + g2);
            const double ip = 1.0 / piv;
            double su, sv;
            if (newton) {
                su = -(hyy * gx - hxy * gy) * ip;
                sv = -(hxx * gy - hxy * gx) * ip;
            } else if (au) {
                su = 0.0;
                sv = -gy * ip;
            } else if (av) {
                sv = 0.0;
                su = -gx * ip;
            } else {
                su = -gx * ip;
                sv = -gy * ip;
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
    if (X) {
        X[0] = x;
        X[1] = y;
        X[2] = h;
    }
    return na * dA + nb * dB;
}

// Node optical path in FP64 with the FP64 solver's exact arithmetic (no contraction):
// na*sqrt(|N-A|^2) + nb*sqrt(|N-B|^2), sums and products in the same order.
__device__ __forceinline__ double node_l64(const DemView& d, int i, int j, const double A[3], const double B[3],
                                           double na, double nb)
{
    double xi = __ldg(d.xv + i), yj = __ldg(d.yv + j), zij = __ldg(d.z + (int64_t)j * d.nx + i);
    double r1x = __dsub_rn(xi, A[0]), r1y = __dsub_rn(yj, A[1]), r1z = __dsub_rn(zij, A[2]);
    double r2x = __dsub_rn(xi, B[0]), r2y = __dsub_rn(yj, B[1]), r2z = __dsub_rn(zij, B[2]);
    double q1 = __dadd_rn(__dadd_rn(__dmul_rn(r1x, r1x), __dmul_rn(r1y, r1y)), __dmul_rn(r1z, r1z));
    double q2 = __dadd_rn(__dadd_rn(__dmul_rn(r2x, r2x), __dmul_rn(r2y, r2y)), __dmul_rn(r2z, r2z));
    return __dadd_rn(__dmul_rn(na, __dsqrt_rn(q1)), __dmul_rn(nb, __dsqrt_rn(q2)));
}

// Node ranking values.  G is the voxel-side endpoint of the path (index ng), E the
// other one (index ne); the scans rank L' = re |N-E| + |N-G| = L / ng with re = ne / ng.

// Branch-free ranking update: best value / position and runner-up value.
__device__ __forceinline__ void rank(float L, int i, int j, float& v1, float& v2, int& bi, int& bj)
{
    v2 = fminf(v2, fmaxf(v1, L));
    bool p = L < v1;
    v1 = p ? L : v1;
    bi = p ? i : bi;
    bj = p ? j : bj;
}

struct Rank {
    float v1, v2;
    int bi, bj;
};

// Generic node scan over [ia, ib] x [ja, jb]: both legs per node, z from the tile when
// `in_tile`, else from global memory.
__device__ __noinline__ Rank scan_generic(const MixedCtx m, const float* ts, int ti0, int tj0, bool in_tile, int ia,
                                          int ib, int ja, int jb, float ex, float ey, float ez, float gx, float gy,
                                          float gz, float re, Rank r)
{
    for (int i = ia; i <= ib; i++) {
        float xi = (float)i * m.stepx;
        float dxe = xi - ex, dxg = xi - gx;
        float sxe = dxe * dxe, sxg = dxg * dxg;
        for (int j = ja; j <= jb; j++) {
            float yj = (float)j * m.stepy;
            float dye = yj - ey, dyg = yj - gy;
            float z = in_tile ? ts[(j - tj0) * TI + (i - ti0)] : zf(m, i, j);
            float dze = z - ez, dzg = z - gz;
            float qe = fmaf(dze, dze, fmaf(dye, dye, sxe));
            float qg = fmaf(dzg, dzg, fmaf(dyg, dyg, sxg));
            rank(fmaf(re, qe * rsqrtf(qe), qg * rsqrtf(qg)), i, j, r.v1, r.v2, r.bi, r.bj);
        }
    }
    return r;
}

// Per-warp table over the union of the 32 lanes' windows: (z, re |N-E|) per node, the
// height next to the E-leg term (all lanes solve the same pulse, so this leg does not
// depend on the voxel), so the scan reads both with one 8-byte load.  Lane l fills column
// j0 + l.  Warp-uniform; `ok` is false when the union does not fit.
constexpr int TBJ = 32;
// table rows for a compile-time node-scan half width: the window plus slack for the
// spread of the 32 lanes' window centres
template <int WT> struct TableRows { static constexpr int v = WT > 0 ? 2 * WT + 1 + (WT >= 12 ? 5 : 7) : 1; };

struct AirTable {
    float2* t;
    int i0, j0;
    bool ok;
};

template <int TBI>
__device__ __forceinline__ AirTable build_air_table(const MixedCtx& m, const Tile& T, float2* buf, int is, int js, int W,
                                                    float ex, float ey, float ez, float re)
{
    const unsigned full = 0xffffffffu;
    int i0 = max(__reduce_min_sync(full, is) - W, 0), i1 = min(__reduce_max_sync(full, is) + W, m.nx - 1);
    int j0 = max(__reduce_min_sync(full, js) - W, 0), j1 = min(__reduce_max_sync(full, js) + W, m.ny - 1);
    AirTable A{buf, i0, j0, false};
    __syncwarp();                       // readers of the previous table are done
    if (i1 - i0 + 1 > TBI || j1 - j0 + 1 > TBJ) return A;
    const int lane = threadIdx.x & 31;
    const int j = j0 + lane;
    const bool in_tile = T.ok && i0 >= T.i0 && i1 < T.i0 + TI && j0 >= T.j0 && j1 < T.j0 + TJ;
    if (j <= j1) {
        float dy = (float)j * m.stepy - ey;
        float sy = dy * dy;
        for (int i = i0; i <= i1; i++) {
            float z = in_tile ? T.s[(j - T.j0) * TI + (i - T.i0)] : zf(m, i, j);
            float dx = (float)i * m.stepx - ex, dz = z - ez;
            float q = fmaf(dz, dz, fmaf(dx, dx, sy));
            buf[(i - i0) * TBJ + lane] = make_float2(z, re * (q * rsqrtf(q)));
        }
    }
    __syncwarp();
    A.ok = true;
    return A;
}

// Full (2W+1)^2 window inside the DEM and the warp table: height and E leg from the
// table (one 8-byte load per node), the G leg per node, columns unrolled with
// compile-time offsets.  The best node's row is updated once per row.
template <int W>
__device__ __forceinline__ void scan_table_inl(const MixedCtx& m, const AirTable& AT, int is, int js, float gx,
                                               float gy, float gz, float& v1, float& v2, int& bi, int& bj)
{
    constexpr int NJ = 2 * W + 1;
    float syg[NJ];
#pragma unroll
    for (int c = 0; c < NJ; c++) {
        float dy = (float)(js - W + c) * m.stepy - gy;
        syg[c] = dy * dy;
    }
    const float2* row0 = AT.t + (is - W - AT.i0) * TBJ + (js - W - AT.j0);
    int bc = bj - (js - W);
#pragma unroll 1
    for (int r = 0; r < NJ; r++) {
        const int i = is - W + r;
        const float dx = (float)i * m.stepx - gx;
        const float sxg = dx * dx;
        const float2* row = row0 + r * TBJ;
        const float v1_row = v1;
#pragma unroll
        for (int c = 0; c < NJ; c++) {
            const float2 e = row[c];
            const float dz = e.x - gz;
            const float q = fmaf(dz, dz, sxg + syg[c]);
            const float L = fmaf(q, rsqrtf(q), e.y);
            v2 = fminf(v2, fmaxf(v1, L));
            const bool p = L < v1;
            v1 = p ? L : v1;
            bc = p ? c : bc;
        }
        bi = (v1 < v1_row) ? i : bi;
    }
    bj = js - W + bc;
}

// Out of line for the widths that prune: it runs for the exhaustive flag and for warps
// whose lanes do not all have full windows, so its body stays out of the pulse loop's
// instruction stream.
template <int W>
__device__ __noinline__ Rank scan_table(const MixedCtx m, const float2* tab, int ti0, int tj0, int is, int js, float gx,
                                        float gy, float gz, Rank rk)
{
    const AirTable AT{const_cast<float2*>(tab), ti0, tj0, true};
    scan_table_inl<W>(m, AT, is, js, gx, gy, gz, rk.v1, rk.v2, rk.bi, rk.bj);
    return rk;
}

// Columns of a window row in groups of four for the pruned scan; a trailing single column
// joins the last group (13 columns: 0-3, 4-7, 8-12).
template <int W> struct ColGroups {
    static constexpr int NJ = 2 * W + 1;
    static constexpr int N = (NJ % 4 == 1) ? NJ / 4 : (NJ + 3) / 4;
    __host__ __device__ static constexpr int first(int k) { return 4 * k; }
    __host__ __device__ static constexpr int last(int k) { return k == N - 1 ? NJ - 1 : 4 * k + 3; }
};

// The table scan with exact pruning: rows, and groups of columns inside a row, whose
// ranking values provably all exceed the pruning threshold are skipped.  The result (best
// value, best node, and whether the runner-up lies within the tie band) is that of
// scan_table, bit for bit:
//  * a skipped node's value exceeds v1 + tie at the time of the skip, so it is neither the
//    minimum nor within the tie band of the final minimum, and v2 - v1 >= tie is decided
//    as before;
//  * an exact FP32 tie between two nodes puts v2 == v1 and sends the lane to the FP64
//    re-rank, so the order in which rows are visited (centre outward) does not choose
//    between equal values.
// The bound.  The E leg e(N) = re |N - E| is convex, so it lies above its tangent plane
// at the start node N0: e(N) >= K + a.(N - G), a = re (N0 - E) / |N0 - E|.  On a row
// (x fixed) with every height above zlo, the ranking value is at least
//     K + a_x X + a_z Zl + min_Y [a_y Y + sqrt(X^2 + Zl^2 + Y^2)]
// (X, Y, Zl: offsets from the voxel G; Zl from the row's lowest height), valid while
// a_z Z + |N - G| grows with the height Z over the window (checked once per solve).  With
// t = thr - K - a_x X - a_z Zl, the row holds no node at or below thr when t < 0 or
// t^2 < (1 - a_y^2)(X^2 + Zl^2); a column group, whose Y lies in [Ylo, Yhi] and whose own
// lowest height gives Zl, holds none when t < 0 or the parabola
// (1 - a_y^2) Y^2 + 2 t a_y Y + X^2 + Zl^2 - t^2 is positive on [Ylo, Yhi].  The
// threshold is v1 + tie, or sooner the value of `seed` (the previous pulse's best node,
// when it lies in this window) + tie, widened by a margin far above the FP32 rounding of
// the values and of the bound.  Warp-uniform: a row or group is skipped only when no lane
// of the warp needs it, so all 32 lanes must call together.
template <int W>
__device__ __forceinline__ void scan_pruned(const MixedCtx& m, const AirTable& AT, int is, int js, const float E[3],
                                            float gx, float gy, float gz, float re, float tie, int seed, float& v1,
                                            float& v2, int& bi, int& bj)
{
    using CG = ColGroups<W>;
    constexpr int NJ = 2 * W + 1;
    const unsigned full = 0xffffffffu;
    float syg[NJ];
#pragma unroll
    for (int c = 0; c < NJ; c++) {
        float dy = (float)(js - W + c) * m.stepy - gy;
        syg[c] = dy * dy;
    }
    const float2* row0 = AT.t + (is - W - AT.i0) * TBJ + (js - W - AT.j0);
    // tangent plane of the E leg at the start node N0
    const float2 n0 = row0[W * TBJ + W];
    const float x0 = (float)is * m.stepx, y0 = (float)js * m.stepy;
    // approximate divisions (2 ulp): the tangent plane and the parabola's vertex move by
    // ~1e-7 relative, which changes the bound by far less than the threshold's margin
    // (2e-4 m + 4e-6 |T|), so the skips stay exact
    const float kk = __fdividef(re * re, n0.y);                    // re / |N0 - E|
    const float ax = (x0 - E[0]) * kk, ay = (y0 - E[1]) * kk, az = (n0.x - E[2]) * kk;
    const float K = n0.y + ax * (gx - x0) + ay * (gy - y0) + az * (gz - n0.x);
    const float sy2 = 1.0f - ay * ay;
    const float yv_t = __fdividef(-ay, sy2);                       // vertex of the parabola: Y = t * yv_t
    const float ay2 = 2.0f * ay;
    const float yfirst = (float)(js - W) * m.stepy - gy;
    // height monotonicity over the window, from the DEM's lowest height (else nothing is
    // pruned): d/dZ [a_z Z + |N - G|] = a_z + Z / |N - G| (Z above the voxel) is positive
    // for every node only if the voxel lies below the DEM's lowest height (Z >= Zt > 0),
    // and, for a_z < 0, Z^2 >= a_z^2 |N - G|^2 at the window's farthest corner
    const float Zt = m.zmin - gz;
    const float hx = fabsf(x0 - gx) + (float)W * m.stepx, hy = fabsf(y0 - gy) + (float)W * m.stepy;
    const bool bound_ok = sy2 > 1e-3f &&           // |a| = re: the bound needs the E leg's index below the G leg's
                          Zt > 0.0f && (az >= 0.0f || az * az * (hx * hx + hy * hy + Zt * Zt) <= Zt * Zt);
    // seed: the previous pulse's best node, ranked with the scan's own arithmetic
    float thr_seed = INFINITY;
    {
        const int si = seed >> 16, sj = seed & 0xffff;
        if (seed >= 0 && abs(si - is) <= W && abs(sj - js) <= W) {
            const float2 e = row0[(si - is + W) * TBJ + (sj - js + W)];
            const float dx = (float)si * m.stepx - gx, dy = (float)sj * m.stepy - gy;
            const float dz = e.x - gz;
            const float q = fmaf(dz, dz, dx * dx + dy * dy);
            thr_seed = fmaf(q, rsqrtf(q), e.y);
        }
    }
    const float never = bound_ok ? 0.0f : INFINITY;     // +inf: keep every node
    int bc = bj - (js - W);
#pragma unroll 1
    for (int k = 0; k < NJ; k++) {
        const int d = (k + 1) >> 1;
        const int r = (k & 1) ? W - d : W + d;          // rows from the start node outward
        const int i = is - W + r;
        const float dx = (float)i * m.stepx - gx;
        const float sxg = dx * dx;
        const float2* row = row0 + r * TBJ;
        float T = fminf(thr_seed, v1) + tie + never;
        T = T + fmaf(4e-6f, fabsf(T), 2e-4f);
        const float R = T - K - ax * dx;
        float2 e[NJ];
#pragma unroll
        for (int c = 0; c < NJ; c++) e[c] = row[c];
        float zg[CG::N];
#pragma unroll
        for (int g = 0; g < CG::N; g++) {
            zg[g] = e[CG::first(g)].x;
#pragma unroll
            for (int c = CG::first(g) + 1; c <= CG::last(g); c++) zg[g] = fminf(zg[g], e[c].x);
        }
        // the whole row (Y free) against its lowest height
        {
            float zr = zg[0];
#pragma unroll
            for (int g = 1; g < CG::N; g++) zr = fminf(zr, zg[g]);
            const float zl = zr - gz;
            const float t = R - az * zl;
            const bool skip = t < 0.0f || t * t < sy2 * fmaf(zl, zl, sxg);
            if (!__any_sync(full, !skip)) continue;
        }
        const float v1_row = v1;
#pragma unroll
        for (int g = 0; g < CG::N; g++) {
            const int c0 = CG::first(g), c1 = CG::last(g);
            const float zl = zg[g] - gz;
            const float t = R - az * zl;
            const float ylo = fmaf((float)c0, m.stepy, yfirst), yhi = fmaf((float)c1, m.stepy, yfirst);
            const float yc = fminf(fmaxf(t * yv_t, ylo), yhi);
            const float q = fmaf(fmaf(sy2, yc, ay2 * t), yc, fmaf(-t, t, fmaf(zl, zl, sxg)));
            const bool skip = t < 0.0f || q > 0.0f;
            if (!__any_sync(full, !skip)) continue;
#pragma unroll
            for (int c = c0; c <= c1; c++) {
                const float dz = e[c].x - gz;
                const float qq = fmaf(dz, dz, sxg + syg[c]);
                const float L = fmaf(qq, rsqrtf(qq), e[c].y);
                v2 = fminf(v2, fmaxf(v1, L));
                const bool p = L < v1;
                v1 = p ? L : v1;
                bc = p ? c : bc;
            }
        }
        bi = (v1 < v1_row) ? i : bi;
    }
    bj = js - W + bc;
}

// Narrowest node-scan half width whose table scan is pruned.
constexpr int kPruneMinW = 6;

template <int W, bool TABLE>
__device__ __forceinline__ void node_scan(const MixedCtx& m, const Tile& T, const AirTable& AT, int is, int js, int Wr,
                                          const float E[3], const float G[3], float re, float tie, int seed, float& v1,
                                          float& v2, int& bi, int& bj)
{
    const int ia = max(is - Wr, 0), ib = min(is + Wr, m.nx - 1);
    const int ja = max(js - Wr, 0), jb = min(js + Wr, m.ny - 1);
    const bool in_tile = T.ok && ia >= T.i0 && ib < T.i0 + TI && ja >= T.j0 && jb < T.j0 + TJ;
    if constexpr (W > 0 && W < kPruneMinW && TABLE) {
        // small windows: every node, inline (the bound tests would cost more than they save)
        if (AT.ok && Wr == W && ia == is - W && ib == is + W && ja == js - W && jb == js + W) {
            scan_table_inl<W>(m, AT, is, js, G[0], G[1], G[2], v1, v2, bi, bj);
            return;
        }
    }
    if constexpr (W >= kPruneMinW && TABLE) {
        const bool full_window = AT.ok && Wr == W && ia == is - W && ib == is + W && ja == js - W && jb == js + W;
        // the pruned scan votes across the warp: only when every lane takes it
        const bool all_full = __all_sync(0xffffffffu, full_window);
        if (all_full && m.prune) {
            scan_pruned<W>(m, AT, is, js, E, G[0], G[1], G[2], re, tie, seed, v1, v2, bi, bj);
            return;
        }
        if (full_window) {
            const Rank r = scan_table<W>(m, AT.t, AT.i0, AT.j0, is, js, G[0], G[1], G[2], Rank{v1, v2, bi, bj});
            v1 = r.v1;
            v2 = r.v2;
            bi = r.bi;
            bj = r.bj;
            return;
        }
    }
    Rank r = scan_generic(m, T.s, T.i0, T.j0, in_tile, ia, ib, ja, jb, E[0], E[1], E[2], G[0], G[1], G[2], re,
                          Rank{v1, v2, bi, bj});
    v1 = r.v1;
    v2 = r.v2;
    bi = r.bi;
    bj = r.bj;
}

// FP64 re-ranking of the nodes within the FP32 ambiguity band, with the FP64 solver's
// arithmetic and order (i-major, j-minor, strict <).
__device__ __noinline__ int2 rerank64(const DemView d, const MixedCtx m, const float* ts, int ti0, int tj0, bool tok,
                                      int is, int js, int Wr, float ex, float ey, float ez, float gx, float gy,
                                      float gz, float re, float limit, double Ax, double Ay, double Az, double Bx,
                                      double By, double Bz, double na, double nb, int2 best_ij)
{
    const int ia = max(is - Wr, 0), ib = min(is + Wr, m.nx - 1);
    const int ja = max(js - Wr, 0), jb = min(js + Wr, m.ny - 1);
    const bool in_tile = tok && ia >= ti0 && ib < ti0 + TI && ja >= tj0 && jb < tj0 + TJ;
    const double A[3] = {Ax, Ay, Az}, B[3] = {Bx, By, Bz};
    double best = INFINITY;
    for (int i = ia; i <= ib; i++) {
        float xi = (float)i * m.stepx;
        float dxe = xi - ex, dxg = xi - gx;
        for (int j = ja; j <= jb; j++) {
            float yj = (float)j * m.stepy;
            float dye = yj - ey, dyg = yj - gy;
            float z = in_tile ? ts[(j - tj0) * TI + (i - ti0)] : zf(m, i, j);
            float dze = z - ez, dzg = z - gz;
            float qe = dxe * dxe + dye * dye + dze * dze;
            float qg = dxg * dxg + dyg * dyg + dzg * dzg;
            if (re * sqrtf(qe) + sqrtf(qg) <= limit) {
                double L = node_l64(d, i, j, A, B, na, nb);
                if (L < best) {
                    best = L;
                    best_ij = make_int2(i, j);
                }
            }
        }
    }
    return best_ij;
}

// Warp-cooperative form of rerank64: each lane whose FP32 runner-up lies within the tie
// band (`need`) has its window re-ranked by the whole warp, 32 nodes at a time, with the
// same FP32 filter and FP64 node values; the smallest FP64 value with the lowest i-major
// index wins, which is the node the FP64 scan's strict < keeps.  All 32 lanes call it.
__device__ __noinline__ int2 rerank64_warp(const DemView d, const MixedCtx m, const float* ts, int ti0, int tj0,
                                           bool tok, bool need, int is, int js, int Wr, float ex, float ey, float ez,
                                           float gx, float gy, float gz, float re, float limit, double Ax, double Ay,
                                           double Az, double Bx, double By, double Bz, double na, double nb,
                                           int2 best_ij)
{
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    unsigned pending = __ballot_sync(full, need);
    int2 result = best_ij;
    while (pending) {
        const int l = __ffs(pending) - 1;
        pending &= pending - 1;
        const int lis = __shfl_sync(full, is, l), ljs = __shfl_sync(full, js, l);
        const float lex = __shfl_sync(full, ex, l), ley = __shfl_sync(full, ey, l), lez = __shfl_sync(full, ez, l);
        const float lgx = __shfl_sync(full, gx, l), lgy = __shfl_sync(full, gy, l), lgz = __shfl_sync(full, gz, l);
        const float llim = __shfl_sync(full, limit, l);
        const double A[3] = {__shfl_sync(full, Ax, l), __shfl_sync(full, Ay, l), __shfl_sync(full, Az, l)};
        const double B[3] = {__shfl_sync(full, Bx, l), __shfl_sync(full, By, l), __shfl_sync(full, Bz, l)};
        const int ia = max(lis - Wr, 0), ib = min(lis + Wr, m.nx - 1);
        const int ja = max(ljs - Wr, 0), jb = min(ljs + Wr, m.ny - 1);
        const bool in_tile = tok && ia >= ti0 && ib < ti0 + TI && ja >= tj0 && jb < tj0 + TJ;
        const int nj = jb - ja + 1, n = (ib - ia + 1) * nj;
        double best = INFINITY;
        int bidx = 0x7fffffff;
        for (int k = lane; k < n; k += 32) {
            const int i = ia + k / nj, j = ja + k % nj;
            float xi = (float)i * m.stepx, yj = (float)j * m.stepy;
            float dxe = xi - lex, dxg = xi - lgx;
            float dye = yj - ley, dyg = yj - lgy;
            float z = in_tile ? ts[(j - tj0) * TI + (i - ti0)] : zf(m, i, j);
            float dze = z - lez, dzg = z - lgz;
            float qe = dxe * dxe + dye * dye + dze * dze;
            float qg = dxg * dxg + dyg * dyg + dzg * dzg;
            if (re * sqrtf(qe) + sqrtf(qg) <= llim) {
                double L = node_l64(d, i, j, A, B, na, nb);
                if (L < best) {
                    best = L;
                    bidx = k;
                }
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const double ob = __shfl_xor_sync(full, best, o);
            const int oi = __shfl_xor_sync(full, bidx, o);
            if (ob < best || (ob == best && oi < bidx)) {
                best = ob;
                bidx = oi;
            }
        }
        if (lane == l && bidx != 0x7fffffff) result = make_int2(ia + bidx / nj, ja + bidx % nj);
    }
    return result;
}

// FP64 flat-interface start and its nearest node, exactly as the FP64 solver makes them
// (used when the FP32 start lies within rounding distance of a node-cell boundary).
__device__ __noinline__ int2 start_node64(const DemView d, double Ax, double Ay, double Az, double Bx, double By,
                                          double Bz, double na, double nb, double h0_known)
{
    const double A[3] = {Ax, Ay, Az}, B[3] = {Bx, By, Bz};
    const bool lower_b = nb >= na;
    const double* Lp = lower_b ? B : A;
    const double* Up = lower_b ? A : B;
    double nl = lower_b ? nb : na, nu = lower_b ? na : nb;
    const double h0 = isnan(h0_known) ? dem_elevation(d, Lp[0], Lp[1]) : h0_known;
    double sx, sy;
    flat_start(Up, Lp, nu, nl, h0, kFlatIters, sx, sy);
    return make_int2(nearest_node(d.x0, d.stepx, d.nx, sx), nearest_node(d.y0, d.stepy, d.ny, sy));
}

// Mixed-precision crossing solve A (index na) -> B (index nb); the voxel-side endpoint G
// is B when g_is_b, else A.  A32/B32: the endpoints in the FP32 frame.  With TABLE the
// warp builds and uses the shared E-leg table (all 32 lanes must call together).
// Returns the FP64 optical path; dA, dB: FP64 leg lengths; X (optional): the crossing.
// seed (table form): in, the node this lane chose for the same leg at the previous pulse
// ((i << 16) | j, or -1), which only speeds up the pruned scan; out, the node chosen now.
template <int WT, bool TABLE>
__device__ __forceinline__ double solve_mixed(const DemView& d, const MixedCtx& m, const Tile& T, float2* table_buf,
                                              const double A[3], const double B[3],
                                              const float A32[3], const float B32[3], float na, float nb,
                                              bool g_is_b, int W, const VoxelStart& vs, int& seed, double& dA,
                                              double& dB, double* X = nullptr)
{
    // 1. flat-interface start (FP32); the lower endpoint is normally the voxel itself
    const bool lower_b = nb >= na;
    const bool lp_is_g = lower_b == g_is_b;
    const float* Lp = lower_b ? B32 : A32;
    const float* Up = lower_b ? A32 : B32;
    const float nl = lower_b ? nb : na, nu = lower_b ? na : nb;
    const float h0 = lp_is_g ? vs.h32 : height32(m, Lp[0], Lp[1]);
    float hx = Lp[0] - Up[0], hy = Lp[1] - Up[1];
    const float D2 = hx * hx + hy * hy;
    float D = D2 * rsqrtf(D2);
    float sx = Lp[0], sy = Lp[1];
    if (D >= 1e-6f) {
        float ha = fabsf(Up[2] - h0), hb = fabsf(Lp[2] - h0);
        float s = fminf(fmaxf(__fdividef(D * ha, ha + hb + 1e-30f), 0.f), D);
#pragma unroll
        for (int it = 0; it < kFlatIters; it++) {
            float q1 = s * s + ha * ha, r = D - s, q2 = r * r + hb * hb;
            float i1 = rsqrtf(q1), i2 = rsqrtf(q2);
            float g = nu * s * i1 - nl * r * i2;
            float gp = nu * ha * ha * i1 * i1 * i1 + nl * hb * hb * i2 * i2 * i2;
            if (gp > 0.f) s = fminf(fmaxf(s - __fdividef(g, gp), 0.f), D);
        }
        const float t = __fdividef(s, D);
        sx = Up[0] + hx * t;
        sy = Up[1] + hy * t;
    }
    // 2. node scan (FP32, L / ng), FP64 re-rank of near ties.  The window centre is the
    //    node nearest the start; a start within rounding distance of a cell boundary is
    //    redone in FP64 so both forms scan the same window.
    const float fx = sx * m.istepx, fy = sy * m.istepy;
    int is = min(max(__float2int_rn(fx), 0), m.nx - 1);
    int js = min(max(__float2int_rn(fy), 0), m.ny - 1);
    if (fabsf(fabsf(fx - rintf(fx)) - 0.5f) < m.start_band || fabsf(fabsf(fy - rintf(fy)) - 0.5f) < m.start_band) {
        const int2 s64 = start_node64(d, A[0], A[1], A[2], B[0], B[1], B[2], (double)na, (double)nb,
                                      lp_is_g ? vs.h64 : (double)NAN);
        is = s64.x;
        js = s64.y;
    }
    const float* E = g_is_b ? A32 : B32;
    const float* G = g_is_b ? B32 : A32;
    const float ng = g_is_b ? nb : na;
    const float re = __fdividef(g_is_b ? na : nb, ng);
    AirTable AT{table_buf, 0, 0, false};
    if constexpr (TABLE && WT > 0)
        AT = build_air_table<TableRows<WT>::v>(m, T, table_buf, is, js, W, E[0], E[1], E[2], re);
    float v1 = INFINITY, v2 = INFINITY;
    int bi = is, bj = js;
    const float tie = kTieM / ng;
    node_scan<WT, TABLE>(m, T, AT, is, js, W, E, G, re, tie, seed, v1, v2, bi, bj);
    const bool need = !(v2 - v1 >= tie);
    if constexpr (TABLE) {
        if (__any_sync(0xffffffffu, need)) {
            const int2 b = rerank64_warp(d, m, T.s, T.i0, T.j0, T.ok, need, is, js, W, E[0], E[1], E[2], G[0], G[1],
                                         G[2], re, v1 + tie, A[0], A[1], A[2], B[0], B[1], B[2], (double)na,
                                         (double)nb, make_int2(bi, bj));
            bi = b.x;
            bj = b.y;
        }
    } else if (need) {
        const int2 b = rerank64(d, m, T.s, T.i0, T.j0, T.ok, is, js, W, E[0], E[1], E[2], G[0], G[1], G[2], re,
                                v1 + tie, A[0], A[1], A[2], B[0], B[1], B[2], (double)na, (double)nb,
                                make_int2(bi, bj));
        bi = b.x;
        bj = b.y;
    }
    seed = (bi < 32768 && bj < 65536) ? (bi << 16) | bj : -1;
    // 3. polish the facets around the best node (FP32); heights from the DEM tile when the
    //    node's 3 x 3 neighbourhood lies in it.  The nine heights are loaded once (indices
    //    clamped to the DEM; a facet that would need a clamped one is not polished), and the
    //    path's gradient at the node is formed once: with G = na (N - A)/|N - A| +
    //    nb (N - B)/|N - B|, a facet with the node at its corner (u0, v0) has the gradient
    //    (Gx + Gz zx, Gy + Gz zy), zx and zy the facet's slopes along the edges through the
    //    node (one-sided differences: backward where u0 = 1, forward where u0 = 0).  When it
    //    points out of the facet on both axes, the corner is that facet's minimum and the
    //    facet keeps the node's path; the others take the Newton steps.
    const bool nt = T.ok && bi - 1 >= T.i0 && bi + 1 < T.i0 + TI && bj - 1 >= T.j0 && bj + 1 < T.j0 + TJ;
    auto zt = [&](int i, int j) { return nt ? T.s[(j - T.j0) * TI + (i - T.i0)] : zf(m, i, j); };
    const int im = max(bi - 1, 0), ip = min(bi + 1, m.nx - 1);
    const int jm = max(bj - 1, 0), jp = min(bj + 1, m.ny - 1);
    const float zmm = zt(im, jm), zm0 = zt(im, bj), zmp = zt(im, jp);
    const float z0m = zt(bi, jm), z00n = zt(bi, bj), z0p = zt(bi, jp);
    const float zpm = zt(ip, jm), zp0 = zt(ip, bj), zpp = zt(ip, jp);
    float Lnode, gxb, gxf, gyb, gyf;
    {
        float xn = (float)bi * m.stepx, yn = (float)bj * m.stepy;
        float r1x = xn - A32[0], r1y = yn - A32[1], r1z = z00n - A32[2];
        float r2x = xn - B32[0], r2y = yn - B32[1], r2z = z00n - B32[2];
        float q1 = r1x * r1x + r1y * r1y + r1z * r1z, q2 = r2x * r2x + r2y * r2y + r2z * r2z;
        const float s1 = rsqrtf(q1), s2 = rsqrtf(q2);
        Lnode = na * (q1 * s1) + nb * (q2 * s2);
        const float g1 = na * s1, g2 = nb * s2;
        const float Gx = g1 * r1x + g2 * r2x, Gy = g1 * r1y + g2 * r2y, Gz = g1 * r1z + g2 * r2z;
        gxb = fmaf(Gz, (z00n - zm0) * m.istepx, Gx);
        gxf = fmaf(Gz, (zp0 - z00n) * m.istepx, Gx);
        gyb = fmaf(Gz, (z00n - z0m) * m.istepy, Gy);
        gyf = fmaf(Gz, (z0p - z00n) * m.istepy, Gy);
    }
    int bfi = min(bi, m.nx - 2), bfj = min(bj, m.ny - 2);     // fallback facet
    float bestF = INFINITY, bu = (float)(bi - bfi), bv = (float)(bj - bfj);
#pragma unroll 1
    for (int k = 0; k < 4; k++) {
        const bool kx = k >> 1, ky = k & 1;       // facet on the +x / +y side of the node
        int fi = bi - 1 + kx, fj = bj - 1 + ky;
        if (fi < 0 || fj < 0 || fi > m.nx - 2 || fj > m.ny - 2) continue;
        float u = (float)(bi - fi), v = (float)(bj - fj);
        float L = Lnode;
        const bool corner = (kx ? gxf > 0.0f : gxb < 0.0f) && (ky ? gyf > 0.0f : gyb < 0.0f);
        if (!corner) {
            Facet32 F;
            F.x0 = (float)fi * m.stepx;
            F.y0 = (float)fj * m.stepy;
            F.dx = m.stepx;
            F.dy = m.stepy;
            F.idx = m.istepx;
            F.idy = m.istepy;
            // corners (fi, fj), (fi + 1, fj), (fi, fj + 1), (fi + 1, fj + 1) of the 3 x 3 block
            const float z00 = kx ? (ky ? z00n : z0m) : (ky ? zm0 : zmm);
            const float z01 = kx ? (ky ? zp0 : zpm) : (ky ? z00n : z0m);
            const float z10 = kx ? (ky ? z0p : z00n) : (ky ? zmp : zm0);
            const float z11 = kx ? (ky ? zpp : zp0) : (ky ? z0p : z00n);
            F.z00 = z00;
            F.b = z01 - z00;
            F.c = z10 - z00;
            F.e = z11 - z01 - z10 + z00;
            bool moved = false;
#pragma unroll 1
            for (int it = 0; it < kPolishIters; it++) {
                if (!facet_step32(F, A32, B32, na, nb, u, v)) break;
                moved = true;
            }
            // a facet whose corner is already its minimum keeps the best node's path
            if (moved) L = facet_eval32(F, A32, B32, na, nb, u, v);
        }
        if (L < bestF) {
            bestF = L;
            bu = u;
            bv = v;
            bfi = fi;
            bfj = fj;
        }
    }
    // 4. FP64 final step
    return final_step64(d, bfi, bfj, A, B, (double)na, (double)nb, (double)bu, (double)bv, dA, dB, X, m.idx64,
                        m.idy64);
}

// ------------------------------- TMA tile staging -----------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint32_t mbar_try_wait_parity(uint32_t bar, uint32_t parity)
{
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    return done;
}

// A copy that missed its deadline may still be in flight: wait for it (bounded) before
// the CTA's shared memory is released.
__device__ void drain_tile(uint64_t* mbar, uint32_t parity)
{
    const uint32_t bar = smem_u32(mbar);
    uint32_t done = 0;
    for (long s = 0; s < kWaitSpins && !done; s++) done = mbar_try_wait_parity(bar, parity);
}

// Arms `mbar` and has one elected thread load the tile with a TMA 2-D tiled copy that
// completes on it; every thread then waits for the barrier's phase `parity`, at most
// `polls` polls (the draining wait before exit has its own fixed limit, kWaitSpins).
// Returns false (and raises *status) if the copy did not complete in time.  The caller
// has initialised the barrier and synchronised the CTA after the previous tile's readers.
__device__ bool stage_tile(const void* tmap, float* tile, uint64_t* mbar, int i0, int j0, uint32_t parity, long long polls,
                           int* status)
{
    const uint32_t bar = smem_u32(mbar);
    if (threadIdx.x == 0) {
        const uint32_t bytes = TI * TJ * sizeof(float);
        // the tensor map sits in global memory written by host copies (a request slot is
        // reused by later requests): acquire it for the tensormap proxy before the copy
        asm volatile("fence.proxy.tensormap::generic.acquire.sys [%0], 128;" ::"l"(reinterpret_cast<uint64_t>(tmap))
                     : "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
        asm volatile(
            "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
                "r"(smem_u32(tile)), "l"(reinterpret_cast<uint64_t>(tmap)), "r"(i0), "r"(j0), "r"(bar)
            : "memory");
    }
    uint32_t done = 0;
    for (long long s = 0; s < polls && !done; s++) done = mbar_try_wait_parity(bar, parity);
    if (!done && status) atomicExch(status, 1);
    return done != 0;
}

__device__ __forceinline__ MixedCtx req_ctx(const MixedReq& r)
{
    MixedCtx m;
    m.z32 = r.z32;
    m.pitch = r.pitch;
    m.nx = r.a.dem.nx;
    m.ny = r.a.dem.ny;
    m.stepx = r.stepx;
    m.stepy = r.stepy;
    m.istepx = r.istepx;
    m.istepy = r.istepy;
    m.ox = r.ox;
    m.oy = r.oy;
    m.idx64 = r.idx64;
    m.idy64 = r.idy64;
    m.start_band = r.start_band;
    m.prune = !r.exhaustive;
    m.zmin = r.zmin;
    return m;
}

// One voxel of a request over pulses [p0, p1) (k: index in the request's voxel range;
// k >= v_count repeats the last voxel without storing it, so whole warps stay active).
// The sum goes to dst at the voxel's image index.
template <int WT, bool CH>
__device__ __forceinline__ void voxel_mixed(const BpArgs& a, const MixedCtx& m, const Tile& T, float2* table_buf,
                                            bool fp16, int64_t kk, int p0, int p1,
                                            double2* __restrict__ dst)
{
    const int np = CH ? p1 : a.np;
    const float k_bin = (float)(a.fs_eff / a.c);
    const float k_phase = (float)(2.0 * 3.14159265358979323846 / a.lambda);
    const float n1f = (float)a.n1, n2f = (float)a.n2;
    const int64_t nr = a.nr;
    const int64_t k = kk < a.v_count ? kk : a.v_count - 1;
    const int64_t v = a.v_begin + k;
    const int yi = (int)(v % a.ny);
    const int xi = (int)((v / a.ny) % a.nx);
    const int zi = (int)(v / ((int64_t)a.nx * a.ny));
    const double P[3] = {__ldg(a.gx + xi), __ldg(a.gy + yi), __ldg(a.gz + zi)};
    const float P32[3] = {(float)(P[0] - m.ox), (float)(P[1] - m.oy), (float)P[2]};
    const VoxelStart vs{height32(m, P32[0], P32[1]), dem_elevation(a.dem, P[0], P[1])};
    float accr = 0.f, acci = 0.f, cmpr = 0.f, cmpi = 0.f;
    int seed0 = -1, seed1 = -1;     // each leg's node at the previous pulse (pruning hint)
    for (int i = CH ? p0 : 0; i < np; i++) {
        const double Tx[3] = {__ldg(a.tx + 3 * i), __ldg(a.tx + 3 * i + 1), __ldg(a.tx + 3 * i + 2)};
        const double Rx[3] = {__ldg(a.rx + 3 * i), __ldg(a.rx + 3 * i + 1), __ldg(a.rx + 3 * i + 2)};
        const float T32[3] = {(float)(Tx[0] - m.ox), (float)(Tx[1] - m.oy), (float)Tx[2]};
        const float R32[3] = {(float)(Rx[0] - m.ox), (float)(Rx[1] - m.oy), (float)Rx[2]};
        // per-pulse legs: n1*r1Tx + n2*r2Tx (Tx -> voxel) + n2*r2Rx + n1*r1Rx (voxel -> Rx);
        // one solver body serves both legs
        double L = 0.0;
#pragma unroll 1
        for (int leg = 0; leg < 2; leg++) {
            // endpoints selected element-wise so they stay in registers
            const double A[3] = {leg ? P[0] : Tx[0], leg ? P[1] : Tx[1], leg ? P[2] : Tx[2]};
            const double B[3] = {leg ? Rx[0] : P[0], leg ? Rx[1] : P[1], leg ? Rx[2] : P[2]};
            const float A32[3] = {leg ? P32[0] : T32[0], leg ? P32[1] : T32[1], leg ? P32[2] : T32[2]};
            const float B32[3] = {leg ? R32[0] : P32[0], leg ? R32[1] : P32[1], leg ? R32[2] : P32[2]};
            double dA, dB;
            int seed = leg ? seed1 : seed0;
            L += solve_mixed<WT, true>(a.dem, m, T, table_buf, A, B, A32, B32, leg ? n2f : n1f,
                                       leg ? n1f : n2f, leg == 0, a.W, vs, seed, dA, dB);
            seed1 = leg ? seed : seed1;
            seed0 = leg ? seed0 : seed;
        }
        const float dL = (float)(L - __ldg(a.ref_L + i));
        // fast-time bin: integer anchor + FP32 offset
        const float t = __ldg(a.ref_bin_f + i) + dL * k_bin;
        const float fl = floorf(t);
        const int64_t lo = (int64_t)__ldg(a.ref_bin_i + i) + (int64_t)fl;
        const float q = t - fl;
        const bool exact = (q == 0.0f);
        if (lo >= 0 && (lo < nr - 1 || (lo == nr - 1 && exact))) {
            float s0r, s0i, s1r = 0.f, s1i = 0.f;
            const int64_t base = (int64_t)i * nr + lo;
            if (fp16) {
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
            const float kr = rintf(ph * 0.15915494309189535f);
            ph = fmaf(-kr, 6.28318548202514648f, ph);
            ph = fmaf(-kr, -1.7484555e-7f, ph);
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
    if (kk < a.v_count)
        (CH ? dst : a.out)[((int64_t)xi * a.ny + yi) * a.nz + zi] =
            make_double2((double)accr - (double)cmpr, (double)acci - (double)cmpi);
}

// The last of a tile's pulse chunks to finish adds the chunks' sums, in chunk order, into
// the image (partial sums of the other CTAs are read from L2).
__device__ __forceinline__ void reduce_chunks(const BpArgs& a, const double2* __restrict__ partial, int K,
                                              int64_t kk)
{
    if (kk >= a.v_count) return;
    const int64_t v = a.v_begin + kk;
    const int yi = (int)(v % a.ny);
    const int xi = (int)((v / a.ny) % a.nx);
    const int zi = (int)(v / ((int64_t)a.nx * a.ny));
    const int64_t idx = ((int64_t)xi * a.ny + yi) * a.nz + zi;
    const int64_t nvox = (int64_t)a.nx * a.ny * a.nz;
    double sr = 0.0, si = 0.0;
    for (int c = 0; c < K; c++) {
        const double2 q = __ldcg(partial + c * nvox + idx);
        sr += q.x;
        si += q.y;
    }
    a.out[idx] = make_double2(sr, si);
}

}  // namespace

// Persistent mixed back-projection.  Every CTA takes work items -- one request and 128
// consecutive voxels of it -- from the batch's list through an atomic counter until the
// list is exhausted, so tiles of several requests share one launch.  The 128 voxels of a
// work item are the same 128 a one-request launch gives a CTA, so a voxel's arithmetic
// (warp tables, DEM tile, sums) does not depend on what else is in the batch.
// CH: the instantiation for batches holding small-grid requests whose tiles run in pulse
// chunks (MixedChunks); the last chunk of a tile to finish adds the chunks' sums in chunk
// order.  Batches without chunks run the other instantiation, which never reads them.
// The DEM tile is staged only for wide node scans (WT = 12, and the generic width): a
// 25 x 25 scan builds 30-row warp tables every pulse and reads them from the tile faster
// than through L1.  For 7 x 7 and 13 x 13 scans the tile's bookkeeping costs registers
// (twice the spills) and its 17 KB per CTA shrinks L1, and the kernel runs faster with the
// heights read from global memory -- the same FP32 values, so the same image.
template <int WT> struct StagesTile { static constexpr bool v = WT == 0 || WT >= 12; };

template <int WT, bool CH>
__global__ void __launch_bounds__(128, 4) k_bp_mixed(MixedBatch b)
{
    constexpr bool kTile = StagesTile<WT>::v;
    __shared__ alignas(128) float tile_s[kTile ? TI * TJ : 32];
    __shared__ alignas(16) float2 air_s[4][TableRows<WT>::v * TBJ];   // one (z, E-leg) table per warp
    __shared__ alignas(8) uint64_t mbar;
    __shared__ int2 work;
    __shared__ int last_chunk;
    float2* table_buf = air_s[threadIdx.x >> 5];
    const int ntiles = b.ntiles_dev ? *b.ntiles_dev : b.ntiles;
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    uint32_t parity = 0;
    bool copy_pending = false;     // a tile copy that timed out may still land
    for (;;) {
        __syncthreads();           // previous work item done (tile, table, `work`)
        if (threadIdx.x == 0) {
            const int t = atomicAdd(b.counter, 1);
            work = (t < ntiles) ? (b.tiles ? b.tiles[t] : make_int2(0, t)) : make_int2(-1, -1);
        }
        __syncthreads();
        const int2 w = work;
        if (w.x < 0) break;
        const MixedReq& R = b.reqs[w.x];
        const BpArgs& a = R.a;
        const MixedCtx m = req_ctx(R);
        // work item -> (128-voxel tile, pulse chunk); the unchunked kernel has one chunk
        const int K = CH ? max(b.chunks[w.x].nchunk, 1) : 1;
        const int tile = CH ? w.y / K : w.y;
        const int chunk = CH ? w.y - tile * K : 0;
        Tile T{tile_s, 0, 0, false};
        if (kTile && R.use_tile && !copy_pending) {
            // DEM tile centred on this work item's voxels plus the mean crossing offset
            const int64_t v0 = a.v_begin + (int64_t)tile * 128;
            const int64_t vl = min(v0 + 128, a.v_begin + a.v_count) - 1;
            const int64_t vm = (v0 + vl) / 2;
            const double cx = __ldg(a.gx + (int)((vm / a.ny) % a.nx)) + R.off_x;
            const double cy = __ldg(a.gy + (int)(vm % a.ny)) + R.off_y;
            const int ci = (int)floor((cx - m.ox) / m.stepx), cj = (int)floor((cy - m.oy) / m.stepy);
            T.i0 = ((ci - TI / 2) >> 2) << 2;      // TMA: x offset a multiple of 4 floats (16 B)
            T.j0 = cj - TJ / 2;
            const bool seen = stage_tile(R.tmap, tile_s, &mbar, T.i0, T.j0, parity, b.wait_polls, b.status);
            parity ^= 1u;
            // one view for the whole CTA: the tile is used only if every thread saw it land,
            // and a copy is still in flight only if the thread that issued it did not
            T.ok = __syncthreads_and(seen);
            copy_pending = __syncthreads_or(threadIdx.x == 0 && !seen);
        }
        if constexpr (!CH) {
            voxel_mixed<WT, false>(a, m, T, table_buf, R.fp16 != 0, (int64_t)w.y * 128 + threadIdx.x, 0, 0,
                                   nullptr);
        } else {
            const int p0 = (int)((int64_t)chunk * a.np / K), p1 = (int)((int64_t)(chunk + 1) * a.np / K);
            double2* dst = K == 1 ? a.out : b.chunks[w.x].partial + chunk * ((int64_t)a.nx * a.ny * a.nz);
            voxel_mixed<WT, true>(a, m, T, table_buf, R.fp16 != 0, (int64_t)tile * 128 + threadIdx.x, p0, p1,
                                  dst);
            // the work item again from shared memory, so none of it stays live over the pulses
            const volatile int* wv = reinterpret_cast<volatile int*>(&work);
            const int2 w2 = make_int2(wv[0], wv[1]);
            const MixedChunks C = b.chunks[w2.x];
            if (C.nchunk > 1) {
                const int tile2 = w2.y / C.nchunk;
                __threadfence();   // this chunk's sums before the count that publishes them
                __syncthreads();
                if (threadIdx.x == 0) last_chunk = atomicAdd(C.tile_done + tile2, 1) == C.nchunk - 1;
                __syncthreads();
                if (last_chunk) {
                    __threadfence();
                    reduce_chunks(b.reqs[w2.x].a, C.partial, C.nchunk, (int64_t)tile2 * 128 + threadIdx.x);
                }
            }
        }
    }
    if (copy_pending) drain_tile(&mbar, parity ^ 1u);
}

static MixedCtx mixed_ctx(const DemView& d, int pitch)
{
    MixedCtx m;
    m.z32 = d.z32;
    m.pitch = pitch;
    m.nx = d.nx;
    m.ny = d.ny;
    m.stepx = (float)d.stepx;
    m.stepy = (float)d.stepy;
    m.istepx = (float)(1.0 / d.stepx);
    m.istepy = (float)(1.0 / d.stepy);
    m.ox = d.x0;
    m.oy = d.y0;
    m.idx64 = 1.0 / d.stepx;
    m.idy64 = 1.0 / d.stepy;
    m.start_band = mixed_start_band(d);
    m.prune = 0;
    m.zmin = -INFINITY;
    return m;
}

// Crossing points of the mixed solver (FP32 scan and polish, FP64 final step) for n
// (start, end) pairs: the data behind the mixed form's crossing-point error.
__global__ void k_refraction_mixed(DemView d, MixedCtx m, const double* __restrict__ p1, const double* __restrict__ p2,
                                   int64_t n, float na, float nb, int W, double* __restrict__ out)
{
    const Tile T{nullptr, 0, 0, false};
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const double A[3] = {p1[3 * k], p1[3 * k + 1], p1[3 * k + 2]};
        const double B[3] = {p2[3 * k], p2[3 * k + 1], p2[3 * k + 2]};
        const float A32[3] = {(float)(A[0] - m.ox), (float)(A[1] - m.oy), (float)A[2]};
        const float B32[3] = {(float)(B[0] - m.ox), (float)(B[1] - m.oy), (float)B[2]};
        double dA, dB, X[3];
        const VoxelStart vs{height32(m, B32[0], B32[1]), dem_elevation(d, B[0], B[1])};
        int seed = -1;
        solve_mixed<0, false>(d, m, T, nullptr, A, B, A32, B32, na, nb, true, W, vs, seed, dA, dB, X);
        out[3 * k] = X[0];
        out[3 * k + 1] = X[1];
        out[3 * k + 2] = X[2];
    }
}

cudaError_t launch_refraction_mixed(const DemView& d, int pitch, const double* p1, const double* p2, int64_t n,
                                    double n1, double n2, int W, double* out, cudaStream_t st)
{
    int64_t b = (n + 127) / 128;
    int blocks = (int)(b < 1 ? 1 : (b > 148 * 64 ? 148 * 64 : b));
    k_refraction_mixed<<<blocks, 128, 0, st>>>(d, mixed_ctx(d, pitch), p1, p2, n, (float)n1, (float)n2, W, out);
    return cudaGetLastError();
}

// Shared-memory carve-out for 4 resident CTAs per SM (DEM tile + 4 warp tables each),
// set once per device; the rest of the unified L1 stays cache for the sample gathers.
template <int WT, bool CH> static void set_carveout()
{
    cudaFuncAttributes fa{};
    if (cudaFuncGetAttributes(&fa, k_bp_mixed<WT, CH>) != cudaSuccess) return;
    const double need = 4.0 * (double)(fa.sharedSizeBytes + 1024);
    int pct = (int)(100.0 * need / (228.0 * 1024.0)) + 1;
    pct = pct > 100 ? 100 : pct;
    cudaFuncSetAttribute(k_bp_mixed<WT, CH>, cudaFuncAttributePreferredSharedMemoryCarveout, pct);
}

static void mixed_setup_device()
{
    static std::atomic<uint64_t> done{0};
    int dev = 0;
    cudaGetDevice(&dev);
    const uint64_t bit = 1ull << (dev & 63);
    if (done.load() & bit) return;
    set_carveout<0, false>();
    set_carveout<3, false>();
    set_carveout<6, false>();
    set_carveout<12, false>();
    set_carveout<0, true>();
    set_carveout<3, true>();
    set_carveout<6, true>();
    set_carveout<12, true>();
    done.fetch_or(bit);
}

int mixed_chunks(int64_t voxels, int pulses)
{
    constexpr int kMinChunkPulses = 128;   // below this a chunk's fixed cost (DEM tile, start heights) shows
    const int64_t tiles = (voxels + 127) / 128;
    const int64_t ctas = mixed_grid_ctas();
    if (tiles <= 0 || pulses < 2 * kMinChunkPulses || tiles * 2 > ctas) return 1;
    int64_t k = ctas / tiles;
    if (k > 8) k = 8;
    if (k > pulses / kMinChunkPulses) k = pulses / kMinChunkPulses;
    return (int)k;
}

// Resident CTAs of the current device, looked up once per device: the pulse-chunk count
// (and with it a small grid's summation order) follows the device the call runs on, so
// GPUs of different kinds in one process each get their own.
int mixed_grid_ctas()
{
    mixed_setup_device();
    constexpr int kDevs = 64;
    static std::atomic<int> ctas[kDevs];
    int dev = 0;
    cudaGetDevice(&dev);
    std::atomic<int>* slot = (dev >= 0 && dev < kDevs) ? &ctas[dev] : nullptr;
    int n = slot ? slot->load() : 0;
    if (!n) {
        int sms = 148, per = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_bp_mixed<6, false>, 128, 0);
        n = sms * (per > 0 ? per : 1);
        if (slot) slot->store(n);
    }
    return n;
}

template <bool CH> static void launch_w(const MixedBatch& b, int W, int grid, cudaStream_t st)
{
    switch (W) {
    case 3: k_bp_mixed<3, CH><<<grid, 128, 0, st>>>(b); break;
    case 6: k_bp_mixed<6, CH><<<grid, 128, 0, st>>>(b); break;
    case 12: k_bp_mixed<12, CH><<<grid, 128, 0, st>>>(b); break;
    default: k_bp_mixed<0, CH><<<grid, 128, 0, st>>>(b); break;
    }
}

cudaError_t launch_bp_mixed(const MixedBatch& b, int W, int grid, cudaStream_t st, bool chunked)
{
    mixed_setup_device();
    if (chunked)
        launch_w<true>(b, W, grid, st);
    else
        launch_w<false>(b, W, grid, st);
    return cudaGetLastError();
}

}  // namespace bsar
