// ref_chunking_shim.cpp -- exposes the REFERENCE's build_pulse_segments
// (include/classical_spin/lattice/pulse_chunking.h, compiled in place from the
// reference tree by oracle/Makefile target `ref`) to the oracle tests.
#include "classical_spin/lattice/pulse_chunking.h"

#include <vector>

extern "C" int refchunk_segments(double T_start, double T_end, const double* centers, int n_centers,
                                 double window, double T_step, double free_dt_factor, double* segs,
                                 int max_segs) {
    const std::vector<double> c(centers, centers + n_centers);
    const auto s = classical_spin_pulse_chunking::build_pulse_segments(T_start, T_end, c, window, T_step,
                                                                       free_dt_factor);
    for (size_t i = 0; i < s.size() && (int)i < max_segs; ++i) {
        segs[3 * i] = s[i].t0;
        segs[3 * i + 1] = s[i].t1;
        segs[3 * i + 2] = s[i].dt_init;
    }
    return (int)s.size();
}
