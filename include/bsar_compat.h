/*
 * bsar_compat.h -- the reference's C++ call surface for the back-projection path,
 * implemented by libbsar_compat.so on top of the C ABI of bsar.h.
 *
 * A program written against DavidAtenciaMondragon/c-_bistatic_sar (proc_test_script.cpp,
 * gs_test_script.cpp) links libbsar_compat.so in place of the reference's
 * src/raw_data_processing.cpp, src/interpolation.cpp and src/fft_utils.cpp.  The types
 * below have the member names, types and order of the reference's structs (include/
 * radar_params.h, funcao_espiral.h, raw_data_processing.h) so objects compiled against
 * either header share one layout and one set of mangled names; a translation unit
 * includes either this header or the reference's, not both.
 *
 * Every function computes on the GPU through bsar.h; there is no CPU fallback (a missing
 * device raises std::runtime_error from the first call).  The Fermat functions run the
 * reference's grid search in FP64 and return its results bit for bit.
 *
 * The batched bsar_compat::backprojectImage replaces the imager's OpenMP voxel loop
 * (proc_test_script.cpp:436-767) with one call.
 */
#ifndef BSAR_COMPAT_H
#define BSAR_COMPAT_H

#include <complex>
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

/* ---------------- types (layout of the reference's structs) ---------------------- */

/* transmitter parameters, include/radar_params.h:7-28 */
struct RadarTx {
    double FreqPortadora, NumVoltasEsp, RaioMenorEsp, RaioMaiorEsp, AltMaiorEsp, AltMenorEsp, Vt, PRF, lamb, fs,
        PotenciaTx, GananciaAnt, FreqMenor, FreqMaior, DuracaoPulso, AperturaAzimut, AperturaElev, Yaw, InclElev,
        Temperatura;
};

/* receiver parameters, include/radar_params.h:31-47 */
struct RadarRx {
    double NumVoltasEsp, RaioMenorEsp, RaioMaiorEsp, AltMaiorEsp, AltMenorEsp, Vt, PRF, fs, GananciaAnt,
        AperturaAzimut, AperturaElev, Yaw, InclElev, Temperatura, B;
};

/* point target, include/radar_params.h:50-53 */
struct Target {
    double pos[3];
    double rcs;
};

/* system constants, include/radar_params.h:56-66 */
struct System {
    double VelocidadeLuz;
    int IndiceMaximo;
    int NumeroPulsos;
    bool PlotarGrafico;
    double RefGeografico[3];
    double xMin, xMax;
    double yMin, yMax;
    double discGrid;
    double ratioUp;
};

/* refractive indices above / below the surface, include/radar_params.h:69-72 */
struct Environment {
    double n1;
    double n2;
};

/* DEM: axes and heights Z_DEM[row of Y_vec][column of X_vec], include/radar_params.h:75-79 */
struct ProcessedDEM {
    std::vector<double> X_vec;
    std::vector<double> Y_vec;
    std::vector<std::vector<double>> Z_DEM;
};

/* trajectory as coordinate vectors, include/funcao_espiral.h:7-11 */
struct TrajectoryPoints {
    std::vector<double> Px;
    std::vector<double> Py;
    std::vector<double> Pz;
};

/* Tx / Rx positions (N x 3) and the target, include/raw_data_processing.h:11-15 */
struct TrajectoryMatrix {
    std::vector<std::vector<double>> Tx;
    std::vector<std::vector<double>> Rx;
    std::vector<double> P;
};

/* per-pulse leg lengths, include/raw_data_processing.h:18-23 */
struct RangeData {
    std::vector<double> r1Tx;
    std::vector<double> r2Tx;
    std::vector<double> r1Rx;
    std::vector<double> r2Rx;
};

/* crossing points of the outbound (ida) and return (volta) paths, N x 3,
 * include/raw_data_processing.h:26-29 */
struct RefractionPoints {
    std::vector<std::vector<double>> P_refrac_ida;
    std::vector<std::vector<double>> P_refrac_volta;
};

/* include/raw_data_processing.h:32-35 */
struct ReflectionPoints {
    std::vector<std::vector<double>> P_reflection;
};

/* simulator matrices [range row][pulse column], include/raw_data_processing.h:38-43 */
struct RawDataResult {
    std::vector<std::vector<std::complex<double>>> auxData;
    std::vector<std::vector<std::complex<double>>> rawData;
    std::vector<std::vector<std::complex<double>>> rootData;
    std::vector<std::complex<double>> chirp;
};

/* ---------------- functions of include/raw_data_processing.h --------------------- */

TrajectoryMatrix prepareTrajectoryData(const TrajectoryPoints& trajTx, const TrajectoryPoints& trajRx,
                                       const Target& target);                                    /* :54 */
TrajectoryMatrix prepareTrajectoryData(const std::vector<std::vector<double>>& Tx,
                                       const std::vector<std::vector<double>>& Rx,
                                       const std::vector<double>& target_pos);                   /* :59 */
ProcessedDEM prepareDEMData(const ProcessedDEM& demData);                                        /* :72 */
Environment initializeEnvironment();                                                             /* :82 */
RangeData calculaSlantRangeFermat(const ProcessedDEM& demData, const TrajectoryMatrix& trajectories,
                                  const Environment& env, ReflectionPoints& strReflexao,
                                  RefractionPoints& strRefraccoes, bool bPlotVerbose = false);   /* :102 */
std::vector<std::complex<double>> createCHIRP(const RadarTx& radarTx);                           /* :115 */
RawDataResult processRawData(const TrajectoryMatrix& trajectories, const RangeData& ranges, const RadarTx& radarTx,
                             const RadarRx& radarRx, const Target& target, const System& system,
                             const Environment& env);                                            /* :126 */
std::vector<double> calculateRefractionPoint(double x1, double y1, double z1, double x2, double y2, double z2,
                                             const ProcessedDEM& demData, double n1, double n2,
                                             bool bPlotVerbose = false);                        /* :135 */
std::vector<double> calculateReflectionPoint(double txX, double txY, double txZ, double rxX, double rxY,
                                             double rxZ, const ProcessedDEM& demData);           /* :141 */
double interpolateDEMElevation(double x, double y, const ProcessedDEM& demData);                 /* :146 */
std::vector<std::complex<double>> correlateWithReference(const std::vector<std::complex<double>>& signal,
                                                         const std::vector<std::complex<double>>& reference); /* :149 */

/* ---------------- include/interpolation.h:8 -------------------------------------- */
std::vector<std::complex<double>> splineInterpolation(const std::vector<std::complex<double>>& data, int factor);

/* ---------------- include/fft_utils.h:13-85 --------------------------------------- */
class FFTProcessor {
public:
    static void fft(std::vector<std::complex<double>>& input);
    static void ifft(std::vector<std::complex<double>>& input);
    static std::vector<std::complex<double>> fftCorrelation(const std::vector<std::complex<double>>& signal,
                                                            const std::vector<std::complex<double>>& reference);
    static std::vector<std::complex<double>> fftConvolution(const std::vector<std::complex<double>>& signal,
                                                            const std::vector<std::complex<double>>& reference);
    static std::vector<std::complex<double>> multiply(const std::vector<std::complex<double>>& a,
                                                      const std::vector<std::complex<double>>& b);
    static std::vector<std::complex<double>> padToPowerOfTwo(const std::vector<std::complex<double>>& input);

private:
    static void bitReverse(std::vector<std::complex<double>>& input);
    static bool isPowerOfTwo(size_t n);
    static size_t nextPowerOfTwo(size_t n);
};

/* ---------------- include/binary_reader.h:10-31 ---------------------------------- */
struct MatrixInfo {
    std::vector<uint64_t> dimensions;
    bool isComplex;
    std::string dataType;
    size_t totalElements;
};
template <typename T> std::vector<std::complex<T>> readBinary(const std::string& filename, MatrixInfo& info);
template <typename T> std::vector<T> readRealBinary(const std::string& filename, MatrixInfo& info);

/* ---------------- include/data_export.h:31-70 ------------------------------------- */
void exportComplexMatrix(const std::string& filename, const std::vector<std::vector<std::complex<double>>>& data);
void exportRealMatrix(const std::string& filename, const std::vector<std::vector<double>>& data);
void exportVector(const std::string& filename, const std::vector<double>& data);
void export3DComplexMatrix(const std::string& filename,
                           const std::vector<std::vector<std::vector<std::complex<double>>>>& output3D, size_t nx,
                           size_t ny, size_t nz, const std::vector<double>& grid_x = {},
                           const std::vector<double>& grid_y = {}, const std::vector<double>& grid_z = {});

/* ---------------- include/load_dem.h:17 ------------------------------------------- */
ProcessedDEM loadDEM(const std::string& filename);

/* ---------------- batched imager (no reference counterpart) ----------------------- */
namespace bsar_compat {

struct ImageOptions {
    int solver = 0;              /* 0: the reference's grid search, 1: Newton           */
    int legs = 0;                /* 0: mean over pulses (as shipped), 1: per pulse       */
    int precision = 0;           /* 0: FP64, 1: mixed, 2: mixed with FP16 samples       */
    double search_radius_m = 0;  /* Newton node-scan radius; 0 selects 1.5 m            */
};

/* The voxel loop of proc_test_script.cpp:436-767 in one call.
 *   rCompData       upsampled range-compressed data, rg + az * interpRangeSamples
 *                   (proc_test_script.cpp:341-343)
 *   c, fs, lambda   strSystem.VelocidadeLuz, strRadarRx.fs (already x factorInterp),
 *                   strRadarTx.lamb (:213, :220-223, :559-563)
 * Returns output[x][y][z] (:408-414, :761-767). */
std::vector<std::vector<std::vector<std::complex<double>>>> backprojectImage(
    const ProcessedDEM& dem, const std::vector<std::vector<double>>& Tx, const std::vector<std::vector<double>>& Rx,
    const std::vector<std::complex<double>>& rCompData, size_t interpRangeSamples, const std::vector<double>& grid_x,
    const std::vector<double>& grid_y, const std::vector<double>& grid_z, const Environment& env, double c,
    double fs, double lambda, const ImageOptions& options = ImageOptions());

}  // namespace bsar_compat

#endif /* BSAR_COMPAT_H */
