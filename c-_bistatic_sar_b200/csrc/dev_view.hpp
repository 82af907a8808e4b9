// dev_view.hpp -- the DEM as kernels see it (plain struct shared by host and device code).
#pragma once

namespace bsar {

// Axes, heights z[j * nx + i] = Z_DEM[j][i] and a few host-precomputed facts.
struct DemView {
    const double* xv;
    const double* yv;
    const double* z;
    const float* z32;   // FP32 copy of z (mixed kernels), may be null
    int nx, ny;
    int empty;          // X_vec / Y_vec / Z_DEM empty -> height 0
    int asc_x, asc_y;   // axis non-decreasing: binary search finds the reference's first match
    int uniform;        // both axes strictly ascending and equally spaced (required by the Newton solver)
    double x0, y0;      // xv[0], yv[0]
    double stepx, stepy;// (v[n-1] - v[0]) / (n - 1)
};

}  // namespace bsar
