// Prints the register FFT's host-built table layouts (kernels.hpp) for 4096, 8192 and
// 16384 points: per length, the second-pass twiddle table's source indices, then the
// stored order of the matched-filter spectrum.  tests/test_rf_tables.py checks them.
#include "kernels.hpp"

#include <cstdio>

int main()
{
    for (int L = 12; L <= 14; L++) {
        const long long n = bsar::rf_twiddle_count(L);
        std::printf("%d %lld", L, n);
        for (long long e = 0; e < n; e++) std::printf(" %lld", (long long)bsar::rf_twiddle_source(L, e));
        std::printf("\n");
        for (int o = 0; o < (1 << L); o++) std::printf("%d ", bsar::rf_spectrum_index(L, o));
        std::printf("\n");
    }
    return 0;
}
