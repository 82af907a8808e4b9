// ref_harness.cpp -- extern "C" entry points over the reference's OWN compiled
// functions (src/raw_data_processing.cpp, src/fft_utils.cpp, src/interpolation.cpp,
// and the file readers / writers src/binary_reader.cpp, src/data_export.cpp,
// src/load_dem_simple.cpp of DavidAtenciaMondragon/c-_bistatic_sar, compiled unmodified
// by oracle/Makefile).
//
// TEST INFRASTRUCTURE ONLY: used to pin the C restatement (bsar_oracle.c), to
// generate the golden fixtures under tests/golden/, and as the timed CPU
// reference arm of bench.py.  The product never links it.
//
// The back-projection loop of the reference lives inline in main()
// (proc_test_script.cpp:451-767) and cannot be called, so ref_backproject below
// restates it around the reference's own calculaSlantRangeFermat.
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <vector>

#include <fcntl.h>
#include <omp.h>
#include <unistd.h>

#include "binary_reader.h"
#include "data_export.h"
#include "fft_utils.h"
#include "interpolation.h"
#include "load_dem.h"
#include "raw_data_processing.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

namespace {

using cvec = std::vector<std::complex<double>>;

ProcessedDEM make_dem(int64_t nx, int64_t ny, const double* xv, const double* yv, const double* z)
{
    ProcessedDEM d;
    d.X_vec.assign(xv, xv + nx);
    d.Y_vec.assign(yv, yv + ny);
    d.Z_DEM.resize(ny);
    for (int64_t j = 0; j < ny; j++) d.Z_DEM[j].assign(z + j * nx, z + (j + 1) * nx);
    return d;
}

std::vector<std::vector<double>> make_points(const double* p, int64_t n)
{
    std::vector<std::vector<double>> v(n, std::vector<double>(3));
    for (int64_t i = 0; i < n; i++)
        for (int k = 0; k < 3; k++) v[i][k] = p[3 * i + k];
    return v;
}

cvec make_cvec(const double* p, int64_t n)
{
    cvec v(n);
    for (int64_t i = 0; i < n; i++) v[i] = {p[2 * i], p[2 * i + 1]};
    return v;
}

void store_cvec(const cvec& v, double* out)
{
    for (size_t i = 0; i < v.size(); i++) {
        out[2 * i] = v[i].real();
        out[2 * i + 1] = v[i].imag();
    }
}

// The reference prints progress lines from inside calculaSlantRangeFermat on every
// call; silence stdout around the calls so timing is not dominated by the terminal.
struct QuietStdout {
    int saved = -1;
    explicit QuietStdout(bool on)
    {
        if (!on) return;
        fflush(stdout);
        std::cout.flush();
        saved = dup(1);
        int devnull = open("/dev/null", O_WRONLY);
        if (devnull >= 0) {
            dup2(devnull, 1);
            close(devnull);
        }
    }
    ~QuietStdout()
    {
        if (saved < 0) return;
        fflush(stdout);
        std::cout.flush();
        dup2(saved, 1);
        close(saved);
    }
};

}  // namespace

extern "C" {

void ref_dem_elevation(int64_t nx, int64_t ny, const double* xv, const double* yv, const double* z,
                       const double* xy, int64_t n, double* out)
{
    ProcessedDEM d = make_dem(nx, ny, xv, yv, z);
    for (int64_t k = 0; k < n; k++) out[k] = interpolateDEMElevation(xy[2 * k], xy[2 * k + 1], d);
}

void ref_refraction_points(int64_t nx, int64_t ny, const double* xv, const double* yv,
                           const double* z, const double* p1, const double* p2, int64_t n,
                           double n1, double n2, double* out)
{
    ProcessedDEM d = make_dem(nx, ny, xv, yv, z);
    for (int64_t k = 0; k < n; k++) {
        std::vector<double> r = calculateRefractionPoint(p1[3 * k], p1[3 * k + 1], p1[3 * k + 2],
                                                         p2[3 * k], p2[3 * k + 1], p2[3 * k + 2],
                                                         d, n1, n2, false);
        for (int c = 0; c < 3; c++) out[3 * k + c] = r[c];
    }
}

void ref_slant_range_fermat(int64_t nx, int64_t ny, const double* xv, const double* yv,
                            const double* z, const double* tx, const double* rx, int64_t np,
                            const double* P, double n1, double n2, double* ranges, double* ida,
                            double* volta, double* refl)
{
    ProcessedDEM d = make_dem(nx, ny, xv, yv, z);
    TrajectoryMatrix t = prepareTrajectoryData(make_points(tx, np), make_points(rx, np),
                                               std::vector<double>{P[0], P[1], P[2]});
    Environment env{n1, n2};
    ReflectionPoints rp;
    RefractionPoints fp;
    RangeData r;
    {
        QuietStdout q(true);
        r = calculaSlantRangeFermat(d, t, env, rp, fp, false);
    }
    for (int64_t i = 0; i < np; i++) {
        ranges[i] = r.r1Tx[i];
        ranges[np + i] = r.r2Tx[i];
        ranges[2 * np + i] = r.r1Rx[i];
        ranges[3 * np + i] = r.r2Rx[i];
        for (int c = 0; c < 3; c++) {
            ida[3 * i + c] = fp.P_refrac_ida[i][c];
            volta[3 * i + c] = fp.P_refrac_volta[i][c];
            if (refl) refl[3 * i + c] = rp.P_reflection[i][c];
        }
    }
}

void ref_spline_upsample(const double* in, int64_t n, int64_t batch, int32_t factor, double* out)
{
    for (int64_t b = 0; b < batch; b++) {
        cvec r = splineInterpolation(make_cvec(in + 2 * n * b, n), factor);
        store_cvec(r, out + 2 * n * factor * b);
    }
}

void ref_fft(double* data, int64_t n, int32_t inverse)
{
    cvec v = make_cvec(data, n);
    if (inverse)
        FFTProcessor::ifft(v);
    else
        FFTProcessor::fft(v);
    store_cvec(v, data);
}

// Pulse compression as driven per pulse in processRawData (src/raw_data_processing.cpp:431-446)
// (conj=1: fftCorrelation) or echo synthesis (:406-421, conj=0: fftConvolution).
void ref_fft_correlate_batch(const double* sig, int64_t ns, int64_t batch, const double* ref,
                             int64_t nr, int32_t conj, int32_t nthreads, double* out)
{
    cvec r = make_cvec(ref, nr);
    int64_t N = ns > nr ? ns : nr;
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
    for (int64_t b = 0; b < batch; b++) {
        cvec s = make_cvec(sig + 2 * ns * b, ns);
        cvec o = conj ? FFTProcessor::fftCorrelation(s, r) : FFTProcessor::fftConvolution(s, r);
        (void)N;
        store_cvec(o, out + 2 * N * b);
    }
}

int64_t ref_create_chirp(double f0, double f1, double T, double fs, double* out, int64_t cap)
{
    RadarTx tx{};
    tx.FreqMenor = f0;
    tx.FreqMaior = f1;
    tx.DuracaoPulso = T;
    tx.fs = fs;
    cvec c;
    {
        QuietStdout q(true);
        c = createCHIRP(tx);
    }
    for (int64_t i = 0; i < (int64_t)c.size() && i < cap; i++) {
        out[2 * i] = c[i].real();
        out[2 * i + 1] = c[i].imag();
    }
    return (int64_t)c.size();
}

// Restatement of the inline voxel loop, proc_test_script.cpp:451-767, calling the
// reference's own calculaSlantRangeFermat for every voxel.
//   rc      upsampled range-compressed data, pulse-major np x nr (rCompData,
//           indexed rg + az*nr, proc_test_script.cpp:341-343, 607-608)
//   legs    0 = mean leg distances (:518-548, as shipped), 1 = per-pulse r1Tx / r1Rx
//   voxels  flat indices in the order z -> x -> y (y fastest) of
//           generateFlatGridCoordinates (:132-151); NULL = every voxel, in which
//           case out is the image [x][y][z] (z fastest) of output[x][y][z] (:761-767)
//   nthreads  <= 0: min(omp_get_max_threads(), 12) as shipped (:428)
void ref_backproject(int64_t dnx, int64_t dny, const double* xv, const double* yv, const double* z,
                     const double* tx, const double* rx, int64_t np, const double* rc, int64_t nr,
                     const double* gx, int64_t nx, const double* gy, int64_t ny, const double* gz,
                     int64_t nz, double n1, double n2, double c, double fs, double lambda,
                     int32_t legs, const int64_t* voxels, int64_t nvox, int32_t nthreads,
                     double* out)
{
    ProcessedDEM dem = make_dem(dnx, dny, xv, yv, z);
    std::vector<std::vector<double>> Tx = make_points(tx, np), Rx = make_points(rx, np);
    Environment env{n1, n2};
    const int64_t total = nx * ny * nz;
    const int64_t count = voxels ? nvox : total;
    int nt = nthreads > 0 ? nthreads : std::min(omp_get_max_threads(), 12);
    QuietStdout q(true);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
    for (int64_t k = 0; k < count; k++) {
        int64_t v = voxels ? voxels[k] : k;
        size_t y_idx = v % ny;
        size_t x_idx = (v / ny) % nx;
        size_t z_idx = v / (nx * ny);
        std::vector<double> target_pos{gx[x_idx], gy[y_idx], gz[z_idx]};
        TrajectoryMatrix trajectories = prepareTrajectoryData(Tx, Rx, target_pos);
        ReflectionPoints reflections;
        RefractionPoints refractions;
        RangeData ranges = calculaSlantRangeFermat(dem, trajectories, env, reflections, refractions, false);
        std::complex<double> allPower(0.0, 0.0);
        const std::vector<double>& P = target_pos;
        const size_t n = refractions.P_refrac_ida.size();
        for (size_t i = 0; i < n; ++i) {
            const auto& a = refractions.P_refrac_ida[i];
            const auto& b = refractions.P_refrac_volta[i];
            double dx = P[0] - a[0], dy = P[1] - a[1], dz = P[2] - a[2];
            double R2t = std::sqrt(dx * dx + dy * dy + dz * dz);
            dx = P[0] - b[0];
            dy = P[1] - b[1];
            dz = P[2] - b[2];
            double R2r = std::sqrt(dx * dx + dy * dy + dz * dz);
            double R1t, R1r;
            if (legs == 0) {
                double s = 0.0;
                for (const auto& t : trajectories.Tx) {
                    double ex = t[0] - a[0], ey = t[1] - a[1], ez = t[2] - a[2];
                    s += std::sqrt(ex * ex + ey * ey + ez * ez);
                }
                R1t = s / trajectories.Tx.size();
                s = 0.0;
                for (const auto& r : trajectories.Rx) {
                    double ex = r[0] - b[0], ey = r[1] - b[1], ez = r[2] - b[2];
                    s += std::sqrt(ex * ex + ey * ey + ez * ez);
                }
                R1r = s / trajectories.Rx.size();
            } else {
                R1t = ranges.r1Tx[i];
                R1r = ranges.r1Rx[i];
            }
            double t_val = (1.0 / c) * (n1 * R1t + n2 * R2t + n2 * R2r + n1 * R1r);
            double rngBin = 1.0 + (t_val * fs);
            double phi = (2.0 * M_PI / lambda) * (n1 * R1t + n2 * R2t + n2 * R2r + n1 * R1r);
            double rb = rngBin - 1.0;
            int idxLast = static_cast<int>(std::floor(rb));
            int idxNext = static_cast<int>(std::ceil(rb));
            if (idxLast >= 0 && idxNext < static_cast<int>(nr)) {
                double qf = rb - idxLast;
                size_t idxAz = std::min(i, (size_t)np - 1);
                size_t l = static_cast<size_t>(idxLast) + idxAz * nr;
                size_t h = static_cast<size_t>(idxNext) + idxAz * nr;
                std::complex<double> vl(rc[2 * l], rc[2 * l + 1]), vh(rc[2 * h], rc[2 * h + 1]);
                std::complex<double> iv = (idxLast == idxNext) ? vl : (1.0 - qf) * vl + qf * vh;
                std::complex<double> ph = std::exp(std::complex<double>(0.0, phi));
                allPower += iv * ph;
            }
        }
        int64_t o = voxels ? k : (int64_t)((x_idx * ny + y_idx) * nz + z_idx);
        out[2 * o] = allPower.real();
        out[2 * o + 1] = allPower.imag();
    }
}

// readBinary<double> (src/binary_reader.cpp:8-95): returns the element count (-1 on an
// exception); dims (up to 8), the complex flag and the values (complex128, up to cap).
int64_t ref_read_binary(const char* path, uint64_t* dims, int32_t* ndims, int32_t* is_complex, double* out,
                        int64_t cap)
{
    try {
        MatrixInfo info;
        std::vector<std::complex<double>> v = readBinary<double>(path, info);
        *ndims = (int32_t)info.dimensions.size();
        for (size_t k = 0; k < info.dimensions.size() && k < 8; k++) dims[k] = info.dimensions[k];
        *is_complex = info.isComplex ? 1 : 0;
        for (int64_t i = 0; i < (int64_t)v.size() && i < cap; i++) {
            out[2 * i] = v[i].real();
            out[2 * i + 1] = v[i].imag();
        }
        return (int64_t)v.size();
    } catch (const std::exception&) {
        return -1;
    }
}

// exportComplexMatrix (src/data_export.cpp:71-138) of a rows x cols complex128 matrix.
void ref_export_complex_matrix(const char* path, int64_t rows, int64_t cols, const double* data)
{
    std::vector<std::vector<std::complex<double>>> m(rows, std::vector<std::complex<double>>(cols));
    for (int64_t i = 0; i < rows; i++)
        for (int64_t j = 0; j < cols; j++) m[i][j] = {data[2 * (i * cols + j)], data[2 * (i * cols + j) + 1]};
    exportComplexMatrix(path, m);
}

// export3DComplexMatrix (src/data_export.cpp:180-309) of an [x][y][z] complex128 image.
void ref_export_3d(const char* path, int64_t nx, int64_t ny, int64_t nz, const double* img, const double* gx,
                   const double* gy, const double* gz)
{
    std::vector<std::vector<std::vector<std::complex<double>>>> o(
        nx, std::vector<std::vector<std::complex<double>>>(ny, std::vector<std::complex<double>>(nz)));
    for (int64_t x = 0; x < nx; x++)
        for (int64_t y = 0; y < ny; y++)
            for (int64_t z = 0; z < nz; z++) {
                const int64_t k = (x * ny + y) * nz + z;
                o[x][y][z] = {img[2 * k], img[2 * k + 1]};
            }
    std::vector<double> ax, ay, az;
    if (gx) ax.assign(gx, gx + nx);
    if (gy) ay.assign(gy, gy + ny);
    if (gz) az.assign(gz, gz + nz);
    export3DComplexMatrix(path, o, nx, ny, nz, ax, ay, az);
}

// The simulator's processRawData (src/raw_data_processing.cpp:292-452) on given per-pulse
// ranges (r1Tx, r2Tx, r1Rx, r2Rx, each np long): one target of cross section rcs, an
// M-sample pulse (System::IndiceMaximo), the chirp f0 -> f1 over T at fs, wavelength lamb.
// Outputs are pulse-major (np x M complex): aux (the placed deltas), raw (after the
// convolution with the fftshifted chirp) and root (after pulse compression); chirp gets
// createCHIRP's samples (returns their count).
int64_t ref_process_raw_data(int64_t np, const double* tx, const double* rx, const double* P, const double* ranges,
                             double f0, double f1, double T, double fs, double lamb, double rcs, double c, int32_t M,
                             double n1, double n2, double* aux, double* raw, double* root, double* chirp,
                             int64_t chirp_cap)
{
    TrajectoryMatrix traj;
    traj.Tx = make_points(tx, np);
    traj.Rx = make_points(rx, np);
    traj.P = {P[0], P[1], P[2]};
    RangeData r;
    r.r1Tx.assign(ranges, ranges + np);
    r.r2Tx.assign(ranges + np, ranges + 2 * np);
    r.r1Rx.assign(ranges + 2 * np, ranges + 3 * np);
    r.r2Rx.assign(ranges + 3 * np, ranges + 4 * np);
    RadarTx rtx{};
    rtx.FreqMenor = f0;
    rtx.FreqMaior = f1;
    rtx.DuracaoPulso = T;
    rtx.fs = fs;
    rtx.lamb = lamb;
    RadarRx rrx{};
    rrx.fs = fs;
    Target tg{};
    tg.pos[0] = P[0];
    tg.pos[1] = P[1];
    tg.pos[2] = P[2];
    tg.rcs = rcs;
    System sys{};
    sys.VelocidadeLuz = c;
    sys.IndiceMaximo = M;
    sys.NumeroPulsos = (int)np;
    Environment env{n1, n2};
    RawDataResult res;
    {
        QuietStdout q(true);
        res = processRawData(traj, r, rtx, rrx, tg, sys, env);
    }
    for (int64_t i = 0; i < np; i++)
        for (int32_t b = 0; b < M; b++) {
            const int64_t o = 2 * (i * M + b);
            aux[o] = res.auxData[b][i].real();
            aux[o + 1] = res.auxData[b][i].imag();
            raw[o] = res.rawData[b][i].real();
            raw[o + 1] = res.rawData[b][i].imag();
            root[o] = res.rootData[b][i].real();
            root[o + 1] = res.rootData[b][i].imag();
        }
    for (int64_t k = 0; k < (int64_t)res.chirp.size() && k < chirp_cap; k++) {
        chirp[2 * k] = res.chirp[k].real();
        chirp[2 * k + 1] = res.chirp[k].imag();
    }
    return (int64_t)res.chirp.size();
}

// loadDEM (src/load_dem_simple.cpp:9-224): sizes first (z == NULL), then the arrays
// (z[j*nx + i] = Z_DEM[j][i]; rows shorter than nx read as 0).
void ref_load_dem(const char* path, int64_t* nx, int64_t* ny, double* xv, double* yv, double* z)
{
    ProcessedDEM d = loadDEM(path);
    *nx = (int64_t)d.X_vec.size();
    *ny = (int64_t)d.Y_vec.size();
    if (!z) return;
    for (size_t i = 0; i < d.X_vec.size(); i++) xv[i] = d.X_vec[i];
    for (size_t j = 0; j < d.Y_vec.size(); j++) yv[j] = d.Y_vec[j];
    for (size_t j = 0; j < d.Y_vec.size(); j++)
        for (size_t i = 0; i < d.X_vec.size(); i++)
            z[j * d.X_vec.size() + i] = (j < d.Z_DEM.size() && i < d.Z_DEM[j].size()) ? d.Z_DEM[j][i] : 0.0;
}

}  // extern "C"
