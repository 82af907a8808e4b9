// Driver for the C++ drop-in layer (libbsar_compat.so): calls the reference's call
// surface exactly as proc_test_script.cpp / gs_test_script.cpp do and prints the results
// for the test to compare with the oracle.  Builds against either include/bsar_compat.h
// (-DUSE_BSAR_HEADER) or the reference's own headers.
#include <complex>
#include <cstdio>
#include <vector>

#ifdef USE_BSAR_HEADER
#include "bsar_compat.h"
#else
#include "fft_utils.h"
#include "interpolation.h"
#include "raw_data_processing.h"
#endif

int main()
{
    // 12 x 10 DEM at 0.5 m around (20, 0): a tilted plane with a ripple
    ProcessedDEM dem;
    for (int i = 0; i < 12; i++) dem.X_vec.push_back(17.0 + 0.5 * i);
    for (int j = 0; j < 10; j++) dem.Y_vec.push_back(-2.25 + 0.5 * j);
    dem.Z_DEM.assign(10, std::vector<double>(12));
    for (int j = 0; j < 10; j++)
        for (int i = 0; i < 12; i++) dem.Z_DEM[j][i] = 0.02 * i - 0.01 * j + 0.03 * ((i * 7 + j * 3) % 5 - 2);
    std::vector<std::vector<double>> Tx, Rx;
    for (int k = 0; k < 6; k++) {
        Tx.push_back({-4.0 + 1.5 * k, 2.0 - 0.7 * k, 30.0});
        Rx.push_back({1.0 + 1.5 * k, 2.0 - 0.7 * k, 30.0});
    }
    std::vector<double> P = {20.1, -0.2, -5.0};
    TrajectoryMatrix traj = prepareTrajectoryData(Tx, Rx, P);
    Environment env{1.0, 2.0};
    ReflectionPoints refl;
    RefractionPoints refr;
    RangeData r = calculaSlantRangeFermat(prepareDEMData(dem), traj, env, refl, refr, false);
    for (size_t i = 0; i < Tx.size(); i++)
        std::printf("range %zu %.17g %.17g %.17g %.17g\n", i, r.r1Tx[i], r.r2Tx[i], r.r1Rx[i], r.r2Rx[i]);
    for (size_t i = 0; i < Tx.size(); i++)
        std::printf("ida %zu %.17g %.17g %.17g\n", i, refr.P_refrac_ida[i][0], refr.P_refrac_ida[i][1],
                    refr.P_refrac_ida[i][2]);
    std::printf("elev %.17g\n", interpolateDEMElevation(19.3, 0.4, dem));
    std::vector<double> cp = calculateRefractionPoint(Tx[0][0], Tx[0][1], Tx[0][2], P[0], P[1], P[2], dem, 1.0, 2.0);
    std::printf("refr %.17g %.17g %.17g\n", cp[0], cp[1], cp[2]);
    std::vector<std::complex<double>> sig(64);
    for (int n = 0; n < 64; n++) sig[n] = std::complex<double>(std::cos(0.3 * n), std::sin(0.11 * n * n));
    std::vector<std::complex<double>> up = splineInterpolation(sig, 4);
    for (size_t n = 0; n < up.size(); n += 37) std::printf("spline %zu %.17g %.17g\n", n, up[n].real(), up[n].imag());
    std::vector<std::complex<double>> ref(sig.begin(), sig.begin() + 16);
    std::vector<std::complex<double>> corr = FFTProcessor::fftCorrelation(sig, ref);
    for (size_t n = 0; n < corr.size(); n += 9) std::printf("corr %zu %.17g %.17g\n", n, corr[n].real(), corr[n].imag());
    std::vector<std::complex<double>> f = sig;
    FFTProcessor::fft(f);
    std::printf("fft0 %.17g %.17g\n", f[5].real(), f[5].imag());
    std::vector<std::complex<double>> odd(12, 1.0);
    FFTProcessor::fft(odd);   // not a power of two: unchanged, with the reference's warning
    std::printf("fftodd %.17g\n", odd[3].real());
#ifdef USE_BSAR_HEADER
    // the imager's voxel loop in one call: 6 pulses, 256 upsampled samples each
    std::vector<std::complex<double>> rc(6 * 256);
    for (size_t n = 0; n < rc.size(); n++) rc[n] = std::complex<double>(std::sin(0.05 * n), std::cos(0.031 * n));
    std::vector<double> gx = {20.0, 20.1}, gy = {-0.1, 0.0, 0.1}, gz = {-5.0};
    auto img = bsar_compat::backprojectImage(dem, Tx, Rx, rc, 256, gx, gy, gz, env, 3e8, 2.0e9, 0.3);
    for (size_t x = 0; x < gx.size(); x++)
        for (size_t y = 0; y < gy.size(); y++)
            std::printf("img %zu %zu %.17g %.17g\n", x, y, img[x][y][0].real(), img[x][y][0].imag());
#endif
    return 0;
}
