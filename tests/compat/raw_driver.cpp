// Driver for processRawData (the simulator's echo model, src/raw_data_processing.cpp:292-452):
// reads one target's trajectories, per-pulse ranges and radar parameters from a binary
// file, calls processRawData through the reference's call surface and writes auxData,
// rawData and rootData pulse-major (np x M complex doubles).  Builds against
// include/bsar_compat.h (-DUSE_BSAR_HEADER, the GPU shims) or the reference's own headers.
//
// Input file: int64 np, int64 M, then doubles tx[np*3], rx[np*3], P[3], ranges[4*np]
// (r1Tx, r2Tx, r1Rx, r2Rx), f0, f1, T, fs, lamb, rcs, c, n1, n2.
#include <complex>
#include <cstdint>
#include <cstdio>
#include <vector>

#ifdef USE_BSAR_HEADER
#include "bsar_compat.h"
#else
#include "raw_data_processing.h"
#endif

int main(int argc, char** argv)
{
    if (argc != 3) return 2;
    FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 3;
    int64_t np = 0, M = 0;
    if (std::fread(&np, 8, 1, f) != 1 || std::fread(&M, 8, 1, f) != 1) return 4;
    std::vector<double> tx(3 * np), rx(3 * np), P(3), rg(4 * np), sc(9);
    if (std::fread(tx.data(), 8, tx.size(), f) != tx.size() || std::fread(rx.data(), 8, rx.size(), f) != rx.size() ||
        std::fread(P.data(), 8, 3, f) != 3 || std::fread(rg.data(), 8, rg.size(), f) != rg.size() ||
        std::fread(sc.data(), 8, sc.size(), f) != sc.size())
        return 5;
    std::fclose(f);
    TrajectoryMatrix traj;
    for (int64_t i = 0; i < np; i++) {
        traj.Tx.push_back({tx[3 * i], tx[3 * i + 1], tx[3 * i + 2]});
        traj.Rx.push_back({rx[3 * i], rx[3 * i + 1], rx[3 * i + 2]});
    }
    traj.P = P;
    RangeData r;
    r.r1Tx.assign(rg.begin(), rg.begin() + np);
    r.r2Tx.assign(rg.begin() + np, rg.begin() + 2 * np);
    r.r1Rx.assign(rg.begin() + 2 * np, rg.begin() + 3 * np);
    r.r2Rx.assign(rg.begin() + 3 * np, rg.end());
    RadarTx rtx{};
    rtx.FreqMenor = sc[0];
    rtx.FreqMaior = sc[1];
    rtx.DuracaoPulso = sc[2];
    rtx.fs = sc[3];
    rtx.lamb = sc[4];
    RadarRx rrx{};
    rrx.fs = sc[3];
    Target tg{};
    tg.pos[0] = P[0];
    tg.pos[1] = P[1];
    tg.pos[2] = P[2];
    tg.rcs = sc[5];
    System sys{};
    sys.VelocidadeLuz = sc[6];
    sys.IndiceMaximo = (int)M;
    sys.NumeroPulsos = (int)np;
    Environment env{sc[7], sc[8]};
    RawDataResult res = processRawData(traj, r, rtx, rrx, tg, sys, env);
    FILE* o = std::fopen(argv[2], "wb");
    if (!o) return 6;
    for (const auto* m : {&res.auxData, &res.rawData, &res.rootData})
        for (int64_t i = 0; i < np; i++)
            for (int64_t b = 0; b < M; b++) {
                const double v[2] = {(*m)[b][i].real(), (*m)[b][i].imag()};
                std::fwrite(v, 8, 2, o);
            }
    std::fclose(o);
    return 0;
}
