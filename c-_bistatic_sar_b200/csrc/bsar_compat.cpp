// bsar_compat.cpp -- the reference's C++ call surface (include/bsar_compat.h) over the
// C ABI of libbsar.so.  Each function converts the reference's nested std::vector
// layouts to flat arrays, calls one bsar_* entry point on a process-wide context, and
// converts back.  Errors from the library surface as std::runtime_error (or
// std::invalid_argument for arguments the library rejects).
#include "bsar_compat.h"

#include <cmath>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <type_traits>
#include <memory>
#include <mutex>
#include <sstream>
#include <stdexcept>
#include <string>

#include "bsar.h"

namespace {

constexpr double kPi = 3.14159265358979323846;

struct Ctx {
    bsar_ctx* ctx = nullptr;
    ~Ctx()
    {
        if (ctx) bsar_destroy(ctx);
    }
};

// One context per process, created on first use (device from BSAR_DEVICE, default 0).
bsar_ctx* context()
{
    static std::once_flag once;
    static Ctx c;
    std::call_once(once, [] {
        bsar_opts o{};
        const char* dev = std::getenv("BSAR_DEVICE");
        o.device = dev ? std::atoi(dev) : 0;
        if (bsar_create(&c.ctx, &o) != BSAR_OK)
            throw std::runtime_error("bsar: no usable CUDA device (bsar_create failed)");
    });
    if (!c.ctx) throw std::runtime_error("bsar: no usable CUDA device");
    return c.ctx;
}

void check(bsar_status s)
{
    if (s == BSAR_OK) return;
    std::string msg = std::string("bsar: ") + bsar_status_string(s) + ": " + bsar_last_error(context());
    if (s == BSAR_ERR_INVALID_ARG) throw std::invalid_argument(msg);
    throw std::runtime_error(msg);
}

// Host-only entry points (no context): a failure names the file.
void check_files(bsar_status s, const std::string& path)
{
    if (s != BSAR_OK) throw std::runtime_error(std::string("bsar: ") + bsar_status_string(s) + ": " + path);
}

// ProcessedDEM -> packed heights (entries missing from a ragged Z_DEM read 0.0, as the
// reference's bounds checks do, src/raw_data_processing.cpp:649-652).
struct FlatDem {
    std::vector<double> z;
    bsar_dem d{};
    explicit FlatDem(const ProcessedDEM& dem)
    {
        const size_t nx = dem.X_vec.size(), ny = dem.Y_vec.size();
        const bool empty = nx == 0 || ny == 0 || dem.Z_DEM.empty();
        if (!empty) {
            z.assign(nx * ny, 0.0);
            for (size_t j = 0; j < ny && j < dem.Z_DEM.size(); j++)
                for (size_t i = 0; i < nx && i < dem.Z_DEM[j].size(); i++) z[j * nx + i] = dem.Z_DEM[j][i];
        }
        d.nx = empty ? 0 : (int64_t)nx;
        d.ny = empty ? 0 : (int64_t)ny;
        d.x_vec = dem.X_vec.data();
        d.y_vec = dem.Y_vec.data();
        d.z = z.data();
    }
};

std::vector<double> flatten3(const std::vector<std::vector<double>>& p)
{
    std::vector<double> f(3 * p.size());
    for (size_t i = 0; i < p.size(); i++)
        for (int k = 0; k < 3; k++) f[3 * i + k] = p[i].size() > (size_t)k ? p[i][k] : 0.0;
    return f;
}

std::vector<std::vector<double>> unflatten3(const std::vector<double>& f)
{
    std::vector<std::vector<double>> p(f.size() / 3, std::vector<double>(3));
    for (size_t i = 0; i < p.size(); i++)
        for (int k = 0; k < 3; k++) p[i][k] = f[3 * i + k];
    return p;
}

const bsar_fermat_opts kGrid{BSAR_SOLVER_GRID, BSAR_FP64, 0.0};

std::vector<std::complex<double>> correlate(const std::vector<std::complex<double>>& s,
                                            const std::vector<std::complex<double>>& r, int conj)
{
    size_t N = std::max(s.size(), r.size());
    std::vector<std::complex<double>> out(N);
    if (N == 0) return out;
    check(bsar_fft_correlate(context(), reinterpret_cast<const double*>(s.data()), (int64_t)s.size(), 1,
                             reinterpret_cast<const double*>(r.data()), (int64_t)r.size(), conj,
                             reinterpret_cast<double*>(out.data())));
    return out;
}

}  // namespace

// ------------------------------ raw_data_processing --------------------------------

TrajectoryMatrix prepareTrajectoryData(const TrajectoryPoints& trajTx, const TrajectoryPoints& trajRx,
                                       const Target& target)
{
    TrajectoryMatrix t;
    const size_t n = trajTx.Px.size();
    t.Tx.assign(n, std::vector<double>(3));
    t.Rx.assign(n, std::vector<double>(3));
    for (size_t i = 0; i < n; i++) {
        t.Tx[i] = {trajTx.Px[i], trajTx.Py[i], trajTx.Pz[i]};
        t.Rx[i] = {trajRx.Px[i], trajRx.Py[i], trajRx.Pz[i]};
    }
    t.P = {target.pos[0], target.pos[1], target.pos[2]};
    return t;
}

TrajectoryMatrix prepareTrajectoryData(const std::vector<std::vector<double>>& Tx,
                                       const std::vector<std::vector<double>>& Rx,
                                       const std::vector<double>& target_pos)
{
    return TrajectoryMatrix{Tx, Rx, target_pos};
}

ProcessedDEM prepareDEMData(const ProcessedDEM& demData) { return demData; }

// n1 = 1, n2 = 4 unless build/output/proc/environment.txt (or $BSAR_ENVIRONMENT_FILE)
// sets them with lines "n1=..." / "n2=..." (src/raw_data_processing.cpp:14-46).
Environment initializeEnvironment()
{
    Environment env{1.0, 4.0};
    const char* path = std::getenv("BSAR_ENVIRONMENT_FILE");
    std::ifstream f(path ? path : "build/output/proc/environment.txt");
    std::string line;
    while (f && std::getline(f, line)) {
        std::istringstream iss(line);
        std::string key, value;
        if (std::getline(iss, key, '=') && std::getline(iss, value)) {
            if (key == "n1") env.n1 = std::stod(value);
            else if (key == "n2") env.n2 = std::stod(value);
        }
    }
    return env;
}

RangeData calculaSlantRangeFermat(const ProcessedDEM& demData, const TrajectoryMatrix& trajectories,
                                  const Environment& env, ReflectionPoints& strReflexao,
                                  RefractionPoints& strRefraccoes, bool /*bPlotVerbose*/)
{
    const size_t n = trajectories.Tx.size();
    RangeData r;
    r.r1Tx.resize(n);
    r.r2Tx.resize(n);
    r.r1Rx.resize(n);
    r.r2Rx.resize(n);
    strRefraccoes.P_refrac_ida.assign(n, std::vector<double>(3));
    strRefraccoes.P_refrac_volta.assign(n, std::vector<double>(3));
    strReflexao.P_reflection.assign(n, std::vector<double>(3));
    if (n == 0) return r;
    FlatDem dem(demData);
    std::vector<double> tx = flatten3(trajectories.Tx), rx = flatten3(trajectories.Rx);
    double P[3] = {trajectories.P.at(0), trajectories.P.at(1), trajectories.P.at(2)};
    std::vector<double> ranges(4 * n), ida(3 * n), volta(3 * n), refl(3 * n);
    check(bsar_slant_range_fermat(context(), &dem.d, tx.data(), rx.data(), (int64_t)n, P, env.n1, env.n2, &kGrid,
                                  ranges.data(), ida.data(), volta.data(), refl.data()));
    for (size_t i = 0; i < n; i++) {
        r.r1Tx[i] = ranges[i];
        r.r2Tx[i] = ranges[n + i];
        r.r1Rx[i] = ranges[2 * n + i];
        r.r2Rx[i] = ranges[3 * n + i];
    }
    strRefraccoes.P_refrac_ida = unflatten3(ida);
    strRefraccoes.P_refrac_volta = unflatten3(volta);
    strReflexao.P_reflection = unflatten3(refl);
    return r;
}

// createCHIRP, src/raw_data_processing.cpp:257-290: exp(j 2 pi (f0 t + k/2 t^2)),
// t = n / fs, n < int(T fs) + 1 (scene set-up, computed once on the host).
std::vector<std::complex<double>> createCHIRP(const RadarTx& radarTx)
{
    const double f0 = radarTx.FreqMenor, f1 = radarTx.FreqMaior, T = radarTx.DuracaoPulso, fs = radarTx.fs;
    const double k = (f1 - f0) / T;
    const int N = static_cast<int>(T * fs) + 1;
    std::vector<std::complex<double>> chirp(N);
    for (int i = 0; i < N; i++) {
        double t = i / fs;
        double ph = 2.0 * kPi * (f0 * t + (k / 2.0) * t * t);
        chirp[i] = std::complex<double>(std::cos(ph), std::sin(ph));
    }
    return chirp;
}

// processRawData, src/raw_data_processing.cpp:292-452: target deltas at bin
// 1 + round(t fs), raw = IFFT(FFT(aux) . FFT(ref)) and root = IFFT(FFT(raw) . conj(FFT(ref)))
// per pulse column; both correlations run on the GPU as one batched call each.
RawDataResult processRawData(const TrajectoryMatrix& trajectories, const RangeData& ranges, const RadarTx& radarTx,
                             const RadarRx& radarRx, const Target& target, const System& system,
                             const Environment& env)
{
    RawDataResult res;
    const double c = system.VelocidadeLuz;
    const size_t np = trajectories.Tx.size();
    const int M = system.IndiceMaximo;
    res.chirp = createCHIRP(radarTx);
    res.auxData.assign(M, std::vector<std::complex<double>>(np, 0.0));
    res.rawData.assign(M, std::vector<std::complex<double>>(np, 0.0));
    res.rootData.assign(M, std::vector<std::complex<double>>(np, 0.0));
    for (size_t i = 0; i < np; i++) {
        double L = env.n1 * ranges.r1Tx[i] + env.n2 * ranges.r2Tx[i] + env.n1 * ranges.r1Rx[i] + env.n2 * ranges.r2Rx[i];
        double t = L / c;
        int bin = 1 + static_cast<int>(std::round(t * radarRx.fs));
        double phi = -(2.0 * kPi / radarTx.lamb) * L;
        if (bin >= 0 && bin < M) res.auxData[bin][i] = target.rcs * std::complex<double>(std::cos(phi), std::sin(phi));
    }
    // fftshifted reference [second half, zeros, first half] (:371-394)
    std::vector<std::complex<double>> ref(M, 0.0);
    const int nc = (int)res.chirp.size(), half = nc / 2;
    for (int i = 0; i < nc - half && i < M; i++) ref[i] = res.chirp[half + i];
    for (int i = 0; i < half && M - half + i >= 0; i++) ref[M - half + i] = res.chirp[i];
    if (np == 0 || M == 0) return res;
    // pulse-major columns
    std::vector<std::complex<double>> cols(np * (size_t)M), raw(np * (size_t)M), root(np * (size_t)M);
    for (size_t i = 0; i < np; i++)
        for (int r = 0; r < M; r++) cols[i * M + r] = res.auxData[r][i];
    check(bsar_fft_correlate(context(), reinterpret_cast<const double*>(cols.data()), M, (int64_t)np,
                             reinterpret_cast<const double*>(ref.data()), M, 0, reinterpret_cast<double*>(raw.data())));
    check(bsar_fft_correlate(context(), reinterpret_cast<const double*>(raw.data()), M, (int64_t)np,
                             reinterpret_cast<const double*>(ref.data()), M, 1, reinterpret_cast<double*>(root.data())));
    for (size_t i = 0; i < np; i++)
        for (int r = 0; r < M; r++) {
            res.rawData[r][i] = raw[i * M + r];
            res.rootData[r][i] = root[i * M + r];
        }
    return res;
}

std::vector<double> calculateRefractionPoint(double x1, double y1, double z1, double x2, double y2, double z2,
                                             const ProcessedDEM& demData, double n1, double n2, bool)
{
    FlatDem dem(demData);
    double a[3] = {x1, y1, z1}, b[3] = {x2, y2, z2}, o[3];
    check(bsar_refraction_points(context(), &dem.d, a, b, 1, n1, n2, &kGrid, o));
    return {o[0], o[1], o[2]};
}

std::vector<double> calculateReflectionPoint(double txX, double txY, double txZ, double rxX, double rxY, double rxZ,
                                             const ProcessedDEM& demData)
{
    FlatDem dem(demData);
    double tx[3] = {txX, txY, txZ}, rx[3] = {rxX, rxY, rxZ}, P[3] = {txX, txY, txZ};
    double ranges[4], ida[3], volta[3], refl[3];
    check(bsar_slant_range_fermat(context(), &dem.d, tx, rx, 1, P, 1.0, 1.0, &kGrid, ranges, ida, volta, refl));
    return {refl[0], refl[1], refl[2]};
}

double interpolateDEMElevation(double x, double y, const ProcessedDEM& demData)
{
    FlatDem dem(demData);
    double xy[2] = {x, y}, z = 0.0;
    check(bsar_dem_elevation(context(), &dem.d, xy, 1, &z));
    return z;
}

std::vector<std::complex<double>> correlateWithReference(const std::vector<std::complex<double>>& signal,
                                                         const std::vector<std::complex<double>>& reference)
{
    return correlate(signal, reference, 1);
}

// ------------------------------ interpolation --------------------------------------

std::vector<std::complex<double>> splineInterpolation(const std::vector<std::complex<double>>& data, int factor)
{
    std::vector<std::complex<double>> out(data.size() * (size_t)std::max(factor, 0));
    if (out.empty()) return out;
    check(bsar_spline_upsample(context(), reinterpret_cast<const double*>(data.data()), (int64_t)data.size(), 1, factor,
                               reinterpret_cast<double*>(out.data())));
    return out;
}

// ------------------------------ fft_utils -------------------------------------------

void FFTProcessor::fft(std::vector<std::complex<double>>& input)
{
    if (input.size() <= 1) return;
    if (!isPowerOfTwo(input.size())) {
        // src/fft_utils.cpp:17-20: warn and leave the data unchanged
        std::cerr << "Warning: FFT input size " << input.size() << " is not a power of 2. Consider padding."
                  << std::endl;
        return;
    }
    check(bsar_fft(context(), reinterpret_cast<double*>(input.data()), (int64_t)input.size(), 1, 0));
}

void FFTProcessor::ifft(std::vector<std::complex<double>>& input)
{
    if (input.size() <= 1) {
        for (auto& x : input) x = std::conj(std::conj(x)) / static_cast<double>(input.size() ? input.size() : 1);
        return;
    }
    if (!isPowerOfTwo(input.size())) {
        // the reference conjugates, skips the transform, conjugates back and scales by 1/N
        std::cerr << "Warning: FFT input size " << input.size() << " is not a power of 2. Consider padding."
                  << std::endl;
        for (auto& x : input) x = x / static_cast<double>(input.size());
        return;
    }
    check(bsar_fft(context(), reinterpret_cast<double*>(input.data()), (int64_t)input.size(), 1, 1));
}

std::vector<std::complex<double>> FFTProcessor::fftCorrelation(const std::vector<std::complex<double>>& signal,
                                                               const std::vector<std::complex<double>>& reference)
{
    return correlate(signal, reference, 1);
}

std::vector<std::complex<double>> FFTProcessor::fftConvolution(const std::vector<std::complex<double>>& signal,
                                                               const std::vector<std::complex<double>>& reference)
{
    return correlate(signal, reference, 0);
}

// element-wise product over the shorter length (src/fft_utils.cpp:140-152)
std::vector<std::complex<double>> FFTProcessor::multiply(const std::vector<std::complex<double>>& a,
                                                         const std::vector<std::complex<double>>& b)
{
    const size_t n = std::min(a.size(), b.size());
    std::vector<std::complex<double>> r(n);
    for (size_t i = 0; i < n; i++) r[i] = a[i] * b[i];
    return r;
}

// zero padding to the next power of two (src/fft_utils.cpp:154-162)
std::vector<std::complex<double>> FFTProcessor::padToPowerOfTwo(const std::vector<std::complex<double>>& input)
{
    std::vector<std::complex<double>> p(nextPowerOfTwo(input.size()), 0.0);
    std::copy(input.begin(), input.end(), p.begin());
    return p;
}

bool FFTProcessor::isPowerOfTwo(size_t n) { return n > 0 && (n & (n - 1)) == 0; }

size_t FFTProcessor::nextPowerOfTwo(size_t n)
{
    size_t p = 1;
    while (p < n) p *= 2;
    return p;
}

// ------------------------------ batched imager --------------------------------------

// ---------------------------------------------------------------------------------
// Files: readBinary / export* / loadDEM over the library's file entry points (host code;
// no device needed).
// ---------------------------------------------------------------------------------
template <typename T> std::vector<std::complex<T>> readBinary(const std::string& filename, MatrixInfo& info)
{
    bsar_matrix_header h{};
    bsar_status st = bsar_matrix_read_header(filename.c_str(), &h);
    if (st == BSAR_ERR_NOT_FOUND) throw std::runtime_error("bsar: cannot open file " + filename);
    if (st != BSAR_OK) throw std::runtime_error("bsar: cannot read the header of " + filename);
    std::vector<std::complex<double>> v(h.total);
    if (h.total && bsar_matrix_read(filename.c_str(), reinterpret_cast<double*>(v.data()), h.total) != BSAR_OK)
        throw std::runtime_error("bsar: cannot read all values of " + filename);
    info.dimensions.assign(h.dims, h.dims + h.ndims);
    info.isComplex = h.is_complex != 0;
    info.dataType = std::string(h.dtype, h.dtype_len);
    info.totalElements = (size_t)h.total;
    if constexpr (std::is_same<T, double>::value) {
        return v;
    } else {
        std::vector<std::complex<T>> o(v.size());
        for (size_t k = 0; k < v.size(); k++) o[k] = std::complex<T>((T)v[k].real(), (T)v[k].imag());
        return o;
    }
}
template std::vector<std::complex<double>> readBinary<double>(const std::string&, MatrixInfo&);

template <typename T> std::vector<T> readRealBinary(const std::string& filename, MatrixInfo& info)
{
    auto c = readBinary<T>(filename, info);
    std::vector<T> r(c.size());
    for (size_t k = 0; k < c.size(); k++) r[k] = c[k].real();
    return r;
}
template std::vector<double> readRealBinary<double>(const std::string&, MatrixInfo&);

void exportComplexMatrix(const std::string& filename, const std::vector<std::vector<std::complex<double>>>& data)
{
    if (data.empty() || data[0].empty()) {
        std::cerr << "Error: Empty data matrix" << std::endl;
        return;
    }
    // rows x cols(first row), then every row as given (ragged rows as the reference writes them)
    std::vector<std::complex<double>> flat;
    for (const auto& row : data) flat.insert(flat.end(), row.begin(), row.end());
    const uint64_t dims[2] = {data.size(), data[0].size()};
    if (flat.size() == dims[0] * dims[1]) {
        if (bsar_matrix_write(filename.c_str(), 2, dims, 1, reinterpret_cast<const double*>(flat.data())) != BSAR_OK)
            std::cerr << "Error: Could not open file " << filename << std::endl;
        return;
    }
    std::ofstream f(filename, std::ios::binary);
    if (!f.is_open()) {
        std::cerr << "Error: Could not open file " << filename << std::endl;
        return;
    }
    const uint32_t nd = 2, cplx = 1, tlen = 6;
    char name[16] = {'d', 'o', 'u', 'b', 'l', 'e'};
    f.write(reinterpret_cast<const char*>(&nd), 4);
    f.write(reinterpret_cast<const char*>(&cplx), 4);
    f.write(reinterpret_cast<const char*>(&tlen), 4);
    f.write(name, 16);
    f.write(reinterpret_cast<const char*>(dims), 16);
    f.write(reinterpret_cast<const char*>(flat.data()), 16 * flat.size());
}

void exportRealMatrix(const std::string& filename, const std::vector<std::vector<double>>& data)
{
    std::ofstream f(filename);
    if (!f.is_open()) {
        std::cerr << "Error: Could not open file " << filename << std::endl;
        return;
    }
    f << std::fixed << std::setprecision(6);
    for (const auto& row : data) {
        for (size_t j = 0; j < row.size(); j++) {
            if (j) f << ",";
            f << row[j];
        }
        f << std::endl;
    }
}

void exportVector(const std::string& filename, const std::vector<double>& data)
{
    std::ofstream f(filename);
    if (!f.is_open()) {
        std::cerr << "Error: Could not open file " << filename << std::endl;
        return;
    }
    f << std::fixed << std::setprecision(6);
    for (size_t i = 0; i < data.size(); i++) {
        if (i) f << ",";
        f << data[i];
    }
    f << std::endl;
}

void export3DComplexMatrix(const std::string& filename,
                           const std::vector<std::vector<std::vector<std::complex<double>>>>& output3D, size_t nx,
                           size_t ny, size_t nz, const std::vector<double>& grid_x, const std::vector<double>& grid_y,
                           const std::vector<double>& grid_z)
{
    if (output3D.size() != nx || (nx > 0 && output3D[0].size() != ny) ||
        (nx > 0 && ny > 0 && output3D[0][0].size() != nz)) {
        std::cerr << "Error: 3-D matrix dimensions do not match nx, ny, nz" << std::endl;
        return;
    }
    std::vector<std::complex<double>> img(nx * ny * nz);
    for (size_t x = 0; x < nx; x++)
        for (size_t y = 0; y < ny; y++)
            for (size_t z = 0; z < nz; z++) img[(x * ny + y) * nz + z] = output3D[x][y][z];
    const bool axes = !grid_x.empty() && !grid_y.empty() && !grid_z.empty();
    if (bsar_image_export(filename.c_str(), reinterpret_cast<const double*>(img.data()), (int64_t)nx, (int64_t)ny,
                          (int64_t)nz, axes ? grid_x.data() : nullptr, axes ? grid_y.data() : nullptr,
                          axes ? grid_z.data() : nullptr) != BSAR_OK)
        std::cerr << "Error: could not write " << filename << std::endl;
}

ProcessedDEM loadDEM(const std::string& filename)
{
    int64_t nx = 0, ny = 0;
    int32_t flags = 0;
    if (bsar_dem_load_esri(filename.c_str(), &nx, &ny, nullptr, nullptr, nullptr, &flags) != BSAR_OK)
        throw std::invalid_argument("bsar: cannot parse the DEM file " + filename);
    std::vector<double> xv(nx), yv(ny), z((size_t)nx * ny);
    check_files(bsar_dem_load_esri(filename.c_str(), &nx, &ny, xv.data(), yv.data(), z.data(), &flags), filename);
    ProcessedDEM d;
    d.X_vec = xv;
    d.Y_vec = yv;
    d.Z_DEM.assign(ny, std::vector<double>(nx));
    for (int64_t j = 0; j < ny; j++)
        for (int64_t i = 0; i < nx; i++) d.Z_DEM[j][i] = z[(size_t)j * nx + i];
    return d;
}

namespace bsar_compat {

std::vector<std::vector<std::vector<std::complex<double>>>> backprojectImage(
    const ProcessedDEM& demData, const std::vector<std::vector<double>>& Tx, const std::vector<std::vector<double>>& Rx,
    const std::vector<std::complex<double>>& rCompData, size_t interpRangeSamples, const std::vector<double>& grid_x,
    const std::vector<double>& grid_y, const std::vector<double>& grid_z, const Environment& env, double c, double fs,
    double lambda, const ImageOptions& o)
{
    const size_t nx = grid_x.size(), ny = grid_y.size(), nz = grid_z.size();
    std::vector<std::vector<std::vector<std::complex<double>>>> out(
        nx, std::vector<std::vector<std::complex<double>>>(ny, std::vector<std::complex<double>>(nz)));
    if (nx * ny * nz == 0) return out;
    if (Tx.size() != Rx.size() || interpRangeSamples == 0 || rCompData.size() < Tx.size() * interpRangeSamples)
        throw std::invalid_argument("bsar: trajectories and rCompData do not match");
    FlatDem dem(demData);
    std::vector<double> tx = flatten3(Tx), rx = flatten3(Rx);
    bsar_scene_desc s{};
    s.dem = dem.d;
    s.n_pulses = (int64_t)Tx.size();
    s.tx = tx.data();
    s.rx = rx.data();
    s.n_samples = (int64_t)interpRangeSamples;
    s.samples = reinterpret_cast<const double*>(rCompData.data());
    s.samples_kind = BSAR_SAMPLES_COMPRESSED;
    s.upsample = 1;   // the data are already upsampled
    s.n1 = env.n1;
    s.n2 = env.n2;
    s.c = c;
    s.fc = c / lambda;
    s.fs = fs;
    bsar_ctx* ctx = context();
    bsar_scene_id sid = 0;
    check(bsar_scene_upload(ctx, &s, &sid));
    bsar_grid g{(int64_t)nx, (int64_t)ny, (int64_t)nz, grid_x.data(), grid_y.data(), grid_z.data()};
    bsar_bp_opts bo{o.solver, o.legs, o.precision, 0, o.search_radius_m};
    std::vector<std::complex<double>> img(nx * ny * nz);
    bsar_status st = bsar_backproject(ctx, sid, &g, &bo, reinterpret_cast<double*>(img.data()));
    bsar_scene_release(ctx, sid);
    check(st);
    for (size_t x = 0; x < nx; x++)
        for (size_t y = 0; y < ny; y++)
            for (size_t z = 0; z < nz; z++) out[x][y][z] = img[(x * ny + y) * nz + z];
    return out;
}

}  // namespace bsar_compat
