// Concurrency driver for the C++ drop-in layer: the imager calls calculaSlantRangeFermat
// for every voxel from up to 12 OpenMP threads at once (proc_test_script.cpp:428,451,484),
// so the layer must be reentrant.  This driver solves a set of voxels serially, then again
// from 12 threads with the imager's dynamic schedule, and prints how many results differ
// (bit for bit) and how many calls failed.
#include <omp.h>

#include <cstdio>
#include <stdexcept>
#include <vector>

#include "bsar_compat.h"

struct Solve {
    RangeData r;
    RefractionPoints refr;
};

static Solve solve(const ProcessedDEM& dem, const std::vector<std::vector<double>>& Tx,
                   const std::vector<std::vector<double>>& Rx, const std::vector<double>& P, const Environment& env)
{
    Solve s;
    ReflectionPoints refl;
    TrajectoryMatrix traj = prepareTrajectoryData(Tx, Rx, P);
    s.r = calculaSlantRangeFermat(dem, traj, env, refl, s.refr, false);
    return s;
}

static bool same(const Solve& a, const Solve& b)
{
    return a.r.r1Tx == b.r.r1Tx && a.r.r2Tx == b.r.r2Tx && a.r.r1Rx == b.r.r1Rx && a.r.r2Rx == b.r.r2Rx &&
           a.refr.P_refrac_ida == b.refr.P_refrac_ida && a.refr.P_refrac_volta == b.refr.P_refrac_volta;
}

int main()
{
    ProcessedDEM dem;
    for (int i = 0; i < 24; i++) dem.X_vec.push_back(14.0 + 0.5 * i);
    for (int j = 0; j < 20; j++) dem.Y_vec.push_back(-4.75 + 0.5 * j);
    dem.Z_DEM.assign(20, std::vector<double>(24));
    for (int j = 0; j < 20; j++)
        for (int i = 0; i < 24; i++) dem.Z_DEM[j][i] = 0.015 * i - 0.01 * j + 0.04 * ((i * 5 + j * 3) % 7 - 3);
    std::vector<std::vector<double>> Tx, Rx;
    for (int k = 0; k < 16; k++) {
        Tx.push_back({-6.0 + 0.8 * k, 3.0 - 0.4 * k, 30.0});
        Rx.push_back({-1.0 + 0.8 * k, 3.0 - 0.4 * k, 30.0});
    }
    Environment env{1.0, 2.0};
    std::vector<std::vector<double>> voxels;
    for (int x = 0; x < 8; x++)
        for (int y = 0; y < 6; y++)
            for (int z = 0; z < 2; z++) voxels.push_back({19.0 + 0.3 * x, -1.0 + 0.35 * y, -5.0 - 0.4 * z});
    const int n = (int)voxels.size();

    std::vector<Solve> serial(n), threaded(n);
    for (int v = 0; v < n; v++) serial[v] = solve(dem, Tx, Rx, voxels[v], env);

    int failed = 0;
    omp_set_num_threads(12);
    // every voxel twice, in the imager's schedule: the first result is kept, the second
    // compared on the spot while other threads' calls are in flight
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : failed)
    for (int v = 0; v < 2 * n; v++) {
        const int k = v / 2;
        try {
            Solve s = solve(dem, Tx, Rx, voxels[k], env);
            if (v % 2 == 0) threaded[k] = s;
            else if (!same(s, serial[k])) failed++;
        } catch (const std::exception&) {
            failed++;
        }
    }
    int differ = 0;
    for (int v = 0; v < n; v++) differ += !same(serial[v], threaded[v]);
    std::printf("voxels %d threads %d differ %d failed %d\n", n, omp_get_max_threads(), differ, failed);
    return 0;
}
