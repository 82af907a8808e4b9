// k_plain.cu -- FP64 ("plain") kernels: DEM lookups, Fermat solves and the
// back-projection of the reference's imager, compiled with --fmad=false so that the
// grid-search form reproduces the reference bit for bit.
//
// Back-projection layout: one warp per voxel, its 32 lanes on 32 consecutive pulses.
// Each lane solves its pulse's two crossing points and forms the pulse's contribution;
// the warp then adds the 32 contributions to the voxel sum in pulse order through
// shuffles, so the FP64 sum has exactly the reference's order (pulse 0, 1, 2, ...,
// proc_test_script.cpp:589-641) while 32 pulses are solved in parallel.
#include <cuda_runtime.h>

#include <cstdint>

#include "dev_common.cuh"
#include "kernels.hpp"

namespace bsar {

__global__ void k_dem_elevation(DemView d, const double2* __restrict__ xy, int64_t n, double* __restrict__ z)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        double2 p = xy[k];
        z[k] = dem_elevation(d, p.x, p.y);
    }
}

template <int SOLVER>
__global__ void __launch_bounds__(64) k_refraction_points(DemView d, const double* __restrict__ p1, const double* __restrict__ p2,
                                    int64_t n, double n1, double n2, int W, double* __restrict__ out)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        double A[3] = {p1[3 * k], p1[3 * k + 1], p1[3 * k + 2]};
        double B[3] = {p2[3 * k], p2[3 * k + 1], p2[3 * k + 2]};
        double o[3];
        refraction_point<SOLVER, 64>(d, A, B, n1, n2, W, o);
        out[3 * k] = o[0];
        out[3 * k + 1] = o[1];
        out[3 * k + 2] = o[2];
    }
}

// calculateReflectionPoint, src/raw_data_processing.cpp:575-612: nearest DEM node to
// the Tx/Rx midpoint (strict <, i-major, j-minor).
__device__ void reflection_point(const DemView& d, double txX, double txY, double rxX, double rxY, double out[3])
{
    double midX = (txX + rxX) / 2.0;
    double midY = (txY + rxY) / 2.0;
    double minDist = 1e9, bestZ = 0.0;
    if (!d.empty) {
        // every node in scan order; on equally spaced axes only the 3 x 3 nodes around the
        // nearest one (rounding puts it within one node of the true nearest), scanned in
        // the same order, so the first minimum is the same node
        int ia = 0, ib = d.nx - 1, ja = 0, jb = d.ny - 1;
        if (d.uniform) {
            const int ci = nearest_node(d.x0, d.stepx, d.nx, midX), cj = nearest_node(d.y0, d.stepy, d.ny, midY);
            ia = max(ci - 1, 0);
            ib = min(ci + 1, d.nx - 1);
            ja = max(cj - 1, 0);
            jb = min(cj + 1, d.ny - 1);
        }
        for (int i = ia; i <= ib; i++) {
            double dx = __ldg(d.xv + i) - midX;
            for (int j = ja; j <= jb; j++) {
                double dy = __ldg(d.yv + j) - midY;
                double dist = sqrt(dx * dx + dy * dy);
                if (dist < minDist) {
                    minDist = dist;
                    bestZ = __ldg(d.z + (int64_t)j * d.nx + i);
                }
            }
        }
    }
    out[0] = midX;
    out[1] = midY;
    out[2] = bestZ;
}

// calculaSlantRangeFermat, src/raw_data_processing.cpp:112-255: one thread per pulse.
template <int SOLVER>
__global__ void __launch_bounds__(64) k_slant_range(DemView d, const double* __restrict__ tx, const double* __restrict__ rx, int64_t np,
                              double Px, double Py, double Pz, double n1, double n2, int W,
                              double* __restrict__ ranges, double* __restrict__ ida, double* __restrict__ volta,
                              double* __restrict__ refl)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < np; i += (int64_t)gridDim.x * blockDim.x) {
        double T[3] = {tx[3 * i], tx[3 * i + 1], tx[3 * i + 2]};
        double R[3] = {rx[3 * i], rx[3 * i + 1], rx[3 * i + 2]};
        double P[3] = {Px, Py, Pz};
        double a[3], b[3];
        refraction_point<SOLVER, 64>(d, T, P, n1, n2, W, a);   // :166-172
        refraction_point<SOLVER, 64>(d, P, R, n2, n1, W, b);   // :175-181
        for (int c = 0; c < 3; c++) {
            ida[3 * i + c] = a[c];
            volta[3 * i + c] = b[c];
        }
        if (refl) {
            double r[3];
            reflection_point(d, T[0], T[1], R[0], R[1], r);
            for (int c = 0; c < 3; c++) refl[3 * i + c] = r[c];
        }
        ranges[i] = sqrt((T[0] - a[0]) * (T[0] - a[0]) + (T[1] - a[1]) * (T[1] - a[1]) + (T[2] - a[2]) * (T[2] - a[2]));
        ranges[np + i] = sqrt((P[0] - a[0]) * (P[0] - a[0]) + (P[1] - a[1]) * (P[1] - a[1]) + (P[2] - a[2]) * (P[2] - a[2]));
        ranges[2 * np + i] = sqrt((R[0] - b[0]) * (R[0] - b[0]) + (R[1] - b[1]) * (R[1] - b[1]) + (R[2] - b[2]) * (R[2] - b[2]));
        ranges[3 * np + i] = sqrt((P[0] - b[0]) * (P[0] - b[0]) + (P[1] - b[1]) * (P[1] - b[1]) + (P[2] - b[2]) * (P[2] - b[2]));
    }
}

// ---------------------------------------------------------------------------------
// Back-projection, FP64: proc_test_script.cpp:491-669 for every voxel.
// ---------------------------------------------------------------------------------
template <int SOLVER, int LEGS>
__global__ void __launch_bounds__(128) k_bp_plain(BpArgs a)
{
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int np = a.np;
    const double* __restrict__ tx = a.tx;
    const double* __restrict__ rx = a.rx;
    const double2* __restrict__ rc = a.rc64;
    const double two_pi_over_lambda = 2.0 * 3.14159265358979323846 / a.lambda;
    const double inv_c = 1.0 / a.c;
    for (int64_t k = warp; k < a.v_count; k += nwarps) {
        const int64_t v = a.v_begin + k;
        const int yi = (int)(v % a.ny);
        const int xi = (int)((v / a.ny) % a.nx);
        const int zi = (int)(v / ((int64_t)a.nx * a.ny));
        const double P[3] = {__ldg(a.gx + xi), __ldg(a.gy + yi), __ldg(a.gz + zi)};
        double accr = 0.0, acci = 0.0;
        for (int c0 = 0; c0 < np; c0 += 32) {
            const int i = c0 + lane;
            double cr = 0.0, ci = 0.0;
            int valid = 0;
            if (i < np) {
                const double T[3] = {__ldg(tx + 3 * i), __ldg(tx + 3 * i + 1), __ldg(tx + 3 * i + 2)};
                const double R[3] = {__ldg(rx + 3 * i), __ldg(rx + 3 * i + 1), __ldg(rx + 3 * i + 2)};
                double ia[3], vb[3];
                refraction_point<SOLVER, 128>(a.dem, T, P, a.n1, a.n2, a.W, ia);   // ida
                refraction_point<SOLVER, 128>(a.dem, P, R, a.n2, a.n1, a.W, vb);   // volta
                double dx = P[0] - ia[0], dy = P[1] - ia[1], dz = P[2] - ia[2];
                const double R2t = sqrt(dx * dx + dy * dy + dz * dz);          // :497-505
                dx = P[0] - vb[0];
                dy = P[1] - vb[1];
                dz = P[2] - vb[2];
                const double R2r = sqrt(dx * dx + dy * dy + dz * dz);          // :507-516
                double R1t, R1r;
                if constexpr (LEGS == 0) {                                     // :518-548
                    double s = 0.0;
                    for (int q = 0; q < np; q++) {
                        double ex = __ldg(tx + 3 * q) - ia[0], ey = __ldg(tx + 3 * q + 1) - ia[1],
                               ez = __ldg(tx + 3 * q + 2) - ia[2];
                        s += sqrt(ex * ex + ey * ey + ez * ez);
                    }
                    R1t = s / (double)np;
                    s = 0.0;
                    for (int q = 0; q < np; q++) {
                        double ex = __ldg(rx + 3 * q) - vb[0], ey = __ldg(rx + 3 * q + 1) - vb[1],
                               ez = __ldg(rx + 3 * q + 2) - vb[2];
                        s += sqrt(ex * ex + ey * ey + ez * ez);
                    }
                    R1r = s / (double)np;
                } else {                                                       // r1Tx / r1Rx, :197-215
                    R1t = sqrt((T[0] - ia[0]) * (T[0] - ia[0]) + (T[1] - ia[1]) * (T[1] - ia[1]) +
                               (T[2] - ia[2]) * (T[2] - ia[2]));
                    R1r = sqrt((R[0] - vb[0]) * (R[0] - vb[0]) + (R[1] - vb[1]) * (R[1] - vb[1]) +
                               (R[2] - vb[2]) * (R[2] - vb[2]));
                }
                const double n1 = a.n1, n2 = a.n2;
                const double t_val = inv_c * (n1 * R1t + n2 * R2t + n2 * R2r + n1 * R1r);          // :565
                const double rngBin = 1.0 + (t_val * a.fs_eff);                                   // :569
                const double phi = two_pi_over_lambda * (n1 * R1t + n2 * R2t + n2 * R2r + n1 * R1r); // :573
                const double b = rngBin - 1.0;                                                    // :593
                // (int)floor(b) >= 0 && (int)ceil(b) < nr  <=>  0 <= b <= nr - 1 (NaN fails both)
                if (b >= 0.0 && b <= (double)(a.nr - 1)) {
                    const double lo_d = floor(b);
                    const int64_t lo = (int64_t)lo_d;
                    const int64_t hi = (int64_t)ceil(b);
                    const double q = b - lo_d;
                    const double2* row = rc + (int64_t)i * a.nr;
                    const double2 s0 = __ldg(row + lo);
                    double vr, vi;
                    if (lo == hi) {
                        vr = s0.x;
                        vi = s0.y;
                    } else {
                        const double2 s1 = __ldg(row + hi);
                        vr = (1.0 - q) * s0.x + q * s1.x;                                         // :635
                        vi = (1.0 - q) * s0.y + q * s1.y;
                    }
                    double sn, cs;
                    sincos(phi, &sn, &cs);                                                        // :638
                    cr = vr * cs - vi * sn;
                    ci = vr * sn + vi * cs;
                    valid = 1;
                }
            }
            const int nlanes = min(32, np - c0);
            for (int l = 0; l < nlanes; l++) {                                                     // :641 in pulse order
                const double xr = __shfl_sync(FULL, cr, l);
                const double xim = __shfl_sync(FULL, ci, l);
                const int vv = __shfl_sync(FULL, valid, l);
                if (vv) {
                    accr += xr;
                    acci += xim;
                }
            }
        }
        if (lane == 0) a.out[((int64_t)xi * a.ny + yi) * a.nz + zi] = make_double2(accr, acci);
    }
}

// Per-pulse reference optical path to the grid centre (FP64, Newton, per-pulse legs)
// and its carrier phase reduced to [-pi, pi) in FP64: the mixed form's anchors.
__global__ void k_ref_ranges(DemView d, const double* __restrict__ tx, const double* __restrict__ rx, int np,
                             double cx, double cy, double cz, double n1, double n2, int W, double lambda,
                             double bin_per_m, double* __restrict__ ref_L, float* __restrict__ ref_phase,
                             int* __restrict__ ref_bin_i, float* __restrict__ ref_bin_f, double* __restrict__ offsets)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x) {
        const double T[3] = {tx[3 * i], tx[3 * i + 1], tx[3 * i + 2]};
        const double R[3] = {rx[3 * i], rx[3 * i + 1], rx[3 * i + 2]};
        const double P[3] = {cx, cy, cz};
        double ia[3], vb[3];
        refraction_newton(d, T, P, n1, n2, W, ia);
        refraction_newton(d, P, R, n2, n1, W, vb);
        auto dist = [](const double* u, const double* w) {
            double x = u[0] - w[0], y = u[1] - w[1], z = u[2] - w[2];
            return sqrt(x * x + y * y + z * z);
        };
        double L = n1 * dist(T, ia) + n2 * dist(P, ia) + n2 * dist(P, vb) + n1 * dist(R, vb);
        ref_L[i] = L;
        double cyc = L / lambda;
        double frac = cyc - rint(cyc);               // exact: cyc - rint(cyc) has no rounding
        ref_phase[i] = (float)(frac * 6.283185307179586476925);
        double b = L * bin_per_m;                    // fast-time bin of the anchor
        double bf = floor(b);
        ref_bin_i[i] = (int)bf;
        ref_bin_f[i] = (float)(b - bf);
        // crossing offsets from the centre (x, y) of both solves: DEM tile placement
        offsets[4 * i] = ia[0] - cx;
        offsets[4 * i + 1] = ia[1] - cy;
        offsets[4 * i + 2] = vb[0] - cx;
        offsets[4 * i + 3] = vb[1] - cy;
    }
}

// ------------------------------- launchers ------------------------------------------
static int grid_for(int64_t n, int threads)
{
    int64_t b = (n + threads - 1) / threads;
    if (b > 148 * 32) b = 148 * 32;
    return (int)(b < 1 ? 1 : b);
}

cudaError_t launch_dem_elevation(const DemView& d, const double* xy, int64_t n, double* z, cudaStream_t st)
{
    k_dem_elevation<<<grid_for(n, 128), 128, 0, st>>>(d, (const double2*)xy, n, z);
    return cudaGetLastError();
}

cudaError_t launch_refraction_points(const DemView& d, const double* p1, const double* p2, int64_t n, double n1,
                                     double n2, int solver, int W, double* out, cudaStream_t st)
{
    if (solver == 0)
        k_refraction_points<0><<<grid_for(n, 64), 64, 0, st>>>(d, p1, p2, n, n1, n2, W, out);
    else
        k_refraction_points<1><<<grid_for(n, 64), 64, 0, st>>>(d, p1, p2, n, n1, n2, W, out);
    return cudaGetLastError();
}

cudaError_t launch_slant_range(const DemView& d, const double* tx, const double* rx, int64_t np,
                               const double* target, double n1, double n2, int solver, int W, double* ranges,
                               double* ida, double* volta, double* refl, cudaStream_t st)
{
    if (solver == 0)
        k_slant_range<0><<<grid_for(np, 64), 64, 0, st>>>(d, tx, rx, np, target[0], target[1], target[2], n1, n2, W,
                                                          ranges, ida, volta, refl);
    else
        k_slant_range<1><<<grid_for(np, 64), 64, 0, st>>>(d, tx, rx, np, target[0], target[1], target[2], n1, n2, W,
                                                          ranges, ida, volta, refl);
    return cudaGetLastError();
}

cudaError_t launch_bp_plain(const BpArgs& a, int solver, int legs, cudaStream_t st)
{
    // one warp per voxel; 4 warps per CTA; enough CTAs to cover the voxel range
    int64_t ctas = (a.v_count + 3) / 4;
    int blocks = (int)(ctas > (int64_t)148 * 512 ? (int64_t)148 * 512 : (ctas < 1 ? 1 : ctas));
    if (solver == 0 && legs == 0) k_bp_plain<0, 0><<<blocks, 128, 0, st>>>(a);
    else if (solver == 0) k_bp_plain<0, 1><<<blocks, 128, 0, st>>>(a);
    else if (legs == 0) k_bp_plain<1, 0><<<blocks, 128, 0, st>>>(a);
    else k_bp_plain<1, 1><<<blocks, 128, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_ref_ranges(const DemView& d, const double* tx, const double* rx, int np, const double* center,
                              double n1, double n2, int W, double lambda, double bin_per_m, double* ref_L,
                              float* ref_phase, int* ref_bin_i, float* ref_bin_f, double* offsets, cudaStream_t st)
{
    k_ref_ranges<<<grid_for(np, 64), 64, 0, st>>>(d, tx, rx, np, center[0], center[1], center[2], n1, n2, W, lambda,
                                                  bin_per_m, ref_L, ref_phase, ref_bin_i, ref_bin_f, offsets);
    return cudaGetLastError();
}

}  // namespace bsar
