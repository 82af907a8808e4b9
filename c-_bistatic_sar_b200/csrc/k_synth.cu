// k_synth.cu -- echo synthesis on the GPU (the step before the path: the simulator's
// processRawData builds raw echoes from refracted two-way delays,
// src/raw_data_processing.cpp:292-421).
//
//   k_echo_paths   per (pulse, scatterer): the FP64 Newton crossings Tx -> scatterer and
//                  scatterer -> Rx, the bistatic optical path L and the carrier factor
//                  a * exp(-j 2 pi fc L / c)
//   k_echo_synth   per fast-time sample: the sum over scatterers of the carrier factor
//                  times the chirp centred on the delay (the reference's centred-chirp
//                  convention, at the exact fractional delay), plus complex Gaussian
//                  noise from a counter-based generator (splitmix64 + Box-Muller)
//
// With `ref_bins` the envelope follows the simulator exactly instead: the echo's chirp is
// centred on sample 1 + round(t * fs) (src/raw_data_processing.cpp:329) and wraps around
// the pulse as its circular convolution with the fftshifted chirp does (:371-406); the
// carrier phase stays exact in both modes.
//
// Compiled with --fmad=false like the other FP64 translation units.
#include <cuda_runtime.h>

#include <cstdint>

#include "dev_common.cuh"
#include "kernels.hpp"

namespace bsar {

__global__ void k_echo_paths(DemView d, const double* __restrict__ tx, const double* __restrict__ rx, int np,
                             const double* __restrict__ spos, const double* __restrict__ samp, int ns_, double n1,
                             double n2, int W, double c, double fc, double fs, int ref_bins,
                             double* __restrict__ tau, double2* __restrict__ carrier)
{
    const int64_t total = (int64_t)np * ns_;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x) {
        const int p = (int)(k / ns_), s = (int)(k % ns_);
        const double T[3] = {tx[3 * p], tx[3 * p + 1], tx[3 * p + 2]};
        const double R[3] = {rx[3 * p], rx[3 * p + 1], rx[3 * p + 2]};
        const double P[3] = {spos[3 * s], spos[3 * s + 1], spos[3 * s + 2]};
        double a[3], b[3];
        refraction_newton(d, T, P, n1, n2, W, a);
        refraction_newton(d, P, R, n2, n1, W, b);
        auto dist = [](const double* u, const double* w) {
            double x = u[0] - w[0], y = u[1] - w[1], z = u[2] - w[2];
            return sqrt(x * x + y * y + z * z);
        };
        const double L = n1 * dist(T, a) + n2 * dist(P, a) + n2 * dist(P, b) + n1 * dist(R, b);
        // ref_bins: the simulator's echo bin (an integer sample index) instead of the delay
        tau[k] = ref_bins ? 1.0 + round((L / c) * fs) : L / c;
        // exp(-j 2 pi fc tau) with the phase reduced in cycles first
        double cyc = fc * (L / c);
        cyc -= rint(cyc);
        double sn, cs;
        sincospi(-2.0 * cyc, &sn, &cs);
        carrier[k] = make_double2(samp[s] * cs, samp[s] * sn);
    }
}

__device__ __forceinline__ uint64_t splitmix64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

__device__ __forceinline__ double unit53(uint64_t x) { return (double)(x >> 11) * 0x1.0p-53; }

__global__ void k_echo_synth(const double* __restrict__ tau, const double2* __restrict__ carrier, int np, int ns_,
                             int nsamp, double fs, double f0, double kchirp, int nc, double sigma, uint64_t seed,
                             int ref_bins, double2* __restrict__ raw)
{
    const int64_t total = (int64_t)np * nsamp;
    const int half = nc / 2;
    const double tmax = (double)(nc - 1) / fs;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x) {
        const int p = (int)(k / nsamp), n = (int)(k % nsamp);
        double re = 0.0, im = 0.0;
        for (int s = 0; s < ns_; s++) {
            double t;                                           // time inside the chirp
            if (ref_bins) {
                // the simulator drops echoes whose bin falls outside the pulse (:357-359);
                // otherwise the chirp sample index of this output in the circular convolution
                const double bin = tau[(int64_t)p * ns_ + s];
                if (!(bin >= 0.0 && bin < (double)nsamp)) continue;
                int64_t m = ((int64_t)n - (int64_t)bin + half) % nsamp;
                if (m < 0) m += nsamp;
                t = m < nc ? (double)m / fs : -1.0;
            } else {
                t = (double)n / fs - tau[(int64_t)p * ns_ + s] + (double)half / fs;
            }
            if (t >= 0.0 && t <= tmax) {
                const double cyc = f0 * t + 0.5 * kchirp * t * t;                           // phase in cycles
                double sn, cs;
                sincospi(2.0 * (cyc - rint(cyc)), &sn, &cs);
                const double2 cr = carrier[(int64_t)p * ns_ + s];
                re += cr.x * cs - cr.y * sn;
                im += cr.x * sn + cr.y * cs;
            }
        }
        if (sigma > 0.0) {
            const uint64_t h1 = splitmix64(seed ^ splitmix64((uint64_t)k * 2 + 1));
            const uint64_t h2 = splitmix64(h1 ^ 0xD1B54A32D192ED03ull);
            const double u1 = 1.0 - unit53(h1), u2 = unit53(h2);
            const double r = sqrt(-2.0 * log(u1)) * sigma * 0.70710678118654752440;
            double sn, cs;
            sincospi(2.0 * u2, &sn, &cs);
            re += r * cs;
            im += r * sn;
        }
        raw[k] = make_double2(re, im);
    }
}

cudaError_t launch_echo_synth(const DemView& d, const double* tx, const double* rx, int np, const double* spos,
                              const double* samp, int nscat, double n1, double n2, int W, double c, double fc,
                              double fs, double f0, double f1, double T, int nsamp, double sigma, uint64_t seed,
                              int ref_bins, double* tau, double2* carrier, double2* raw, cudaStream_t st)
{
    const int64_t npairs = (int64_t)np * nscat;
    int b1 = (int)((npairs + 63) / 64);
    if (b1 > 148 * 64) b1 = 148 * 64;
    if (b1 < 1) b1 = 1;
    k_echo_paths<<<b1, 64, 0, st>>>(d, tx, rx, np, spos, samp, nscat, n1, n2, W, c, fc, fs, ref_bins, tau, carrier);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const int nc = (int)(T * fs) + 1;   // createCHIRP's sample count (src/raw_data_processing.cpp:271)
    const int64_t total = (int64_t)np * nsamp;
    int b2 = (int)((total + 255) / 256);
    if (b2 > 148 * 128) b2 = 148 * 128;
    k_echo_synth<<<b2, 256, 0, st>>>(tau, carrier, np, nscat, nsamp, fs, f0, (f1 - f0) / T, nc, sigma, seed, ref_bins,
                                     raw);
    return cudaGetLastError();
}

}  // namespace bsar
