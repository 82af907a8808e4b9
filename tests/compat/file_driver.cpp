// File-level driver for the C++ drop-in layer: the reference's readers and writers
// (readBinary, exportComplexMatrix, exportRealMatrix, exportVector,
// export3DComplexMatrix, loadDEM) called as the imager and simulator call them.
// Builds against include/bsar_compat.h (-DUSE_BSAR_HEADER) or the reference's headers.
//   file_driver <dem.asc> <in.bin> <out_dir>
#include <complex>
#include <cstdio>
#include <string>
#include <vector>

#ifdef USE_BSAR_HEADER
#include "bsar_compat.h"
#else
#include "binary_reader.h"
#include "data_export.h"
#include "load_dem.h"
#endif

int main(int argc, char** argv)
{
    if (argc < 4) return 2;
    const std::string out = argv[3];
    ProcessedDEM dem = loadDEM(argv[1]);
    std::printf("dem %zu %zu\n", dem.X_vec.size(), dem.Y_vec.size());
    for (size_t j = 0; j < dem.Z_DEM.size(); j++)
        for (size_t i = 0; i < dem.Z_DEM[j].size(); i++) std::printf("z %zu %zu %.17g\n", j, i, dem.Z_DEM[j][i]);
    MatrixInfo info;
    std::vector<std::complex<double>> v = readBinary<double>(argv[2], info);
    std::printf("info %zu %d %zu %zu\n", info.dimensions.size(), info.isComplex ? 1 : 0, info.dataType.size(),
                info.totalElements);
    for (size_t k = 0; k < v.size(); k++) std::printf("v %.17g %.17g\n", v[k].real(), v[k].imag());
    std::vector<double> re = readRealBinary<double>(argv[2], info);
    std::printf("real %zu\n", re.size());
    std::vector<std::vector<std::complex<double>>> m(3, std::vector<std::complex<double>>(4));
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 4; j++) m[i][j] = {0.25 * i - j, 1.0 / (1 + i + j)};
    exportComplexMatrix(out + "/m.bin", m);
    std::vector<std::vector<double>> r = {{1.5, -2.25, 3.125}, {4.0, 5.0, 6.0}};
    exportRealMatrix(out + "/r.csv", r);
    exportVector(out + "/v.csv", {0.1, 0.2, 0.30000000000000004});
    const size_t nx = 3, ny = 2, nz = 4;
    std::vector<std::vector<std::vector<std::complex<double>>>> o(
        nx, std::vector<std::vector<std::complex<double>>>(ny, std::vector<std::complex<double>>(nz)));
    for (size_t x = 0; x < nx; x++)
        for (size_t y = 0; y < ny; y++)
            for (size_t z = 0; z < nz; z++) o[x][y][z] = {(double)(x + 10 * y + 100 * z), -(double)x};
    export3DComplexMatrix(out + "/img.bin", o, nx, ny, nz, {19.2, 19.24, 19.28}, {-0.8, -0.76}, {-5.8, -5.72, -5.64, -5.56});
    return 0;
}
