// ref_mixed_shim.cu -- C entry points around the REFERENCE's own mixed SU(2)/SU(3)
// GPU integrator.
//
// Test infrastructure only.  Compiled (by oracle/Makefile, target `ref`) together
// with the reference sources src/gpu/mixed_lattice_gpu.cu and
// src/gpu/gpu_common_helpers.cu, read in place from the reference tree, into
// oracle/_ref/libref_mixed.so.  It calls the reference's `namespace mixed_gpu` API
// (include/classical_spin/gpu/mixed_lattice_gpu_api.h) as MixedLattice's host glue
// does, so tests can pin the B200 mixed path and the numpy restatement in
// mixed_oracle.py to the reference's own arithmetic on a B200.  Entry points return
// a negative value on a C++ exception.
#include "classical_spin/gpu/mixed_lattice_gpu_api.h"

#include <cstdint>
#include <cstring>
#include <vector>

namespace {
template <class T>
std::vector<T> vec(const T* p, int64_t n) { return n > 0 ? std::vector<T>(p, p + n) : std::vector<T>(); }
std::vector<size_t> idx(const int64_t* p, int64_t n) {
    std::vector<size_t> v(n > 0 ? n : 0);
    for (int64_t i = 0; i < n; ++i) v[i] = (size_t)p[i];
    return v;
}
}  // namespace

extern "C" {

// dims = {N2, NA2, N3, NA3, z2, z3, zm2, zm3}
void* refmix_create(const int64_t* dims, const double* f2, const double* o2, const double* j2, const int64_t* p2,
                    const int64_t* c2, const double* f3, const double* o3, const double* j3, const int64_t* p3,
                    const int64_t* c3, const double* m2, const int64_t* mp2, const int64_t* mc2, const double* m3,
                    const int64_t* mp3, const int64_t* mc3) {
    try {
        const int64_t N2 = dims[0], NA2 = dims[1], N3 = dims[2], NA3 = dims[3];
        const int64_t z2 = dims[4], z3 = dims[5], zm2 = dims[6], zm3 = dims[7];
        return mixed_gpu::create_gpu_mixed_lattice_data(
            (size_t)N2, 3, (size_t)NA2, (size_t)N3, 8, (size_t)NA3, (size_t)z2, (size_t)z3, (size_t)zm2, (size_t)zm3,
            vec(f2, N2 * 3), vec(o2, N2 * 9), vec(j2, N2 * z2 * 9), idx(p2, N2 * z2), idx(c2, N2),
            vec(f3, N3 * 8), vec(o3, N3 * 64), vec(j3, N3 * z3 * 64), idx(p3, N3 * z3), idx(c3, N3),
            vec(m2, N2 * zm2 * 24), std::vector<size_t>(), idx(mp2, N2 * zm2), idx(mc2, N2),
            vec(m3, N3 * zm3 * 24), idx(mp3, N3 * zm3), idx(mc3, N3));
    } catch (...) {
        return nullptr;
    }
}

void refmix_destroy(void* h) {
    mixed_gpu::destroy_gpu_mixed_lattice_data((mixed_gpu::GPUMixedLatticeDataHandle*)h);
}

int refmix_set_pulse(void* h, int sub, const double* fd, int64_t n, double amp, double width, double freq, double t1,
                     double t2) {
    try {
        auto* x = (mixed_gpu::GPUMixedLatticeDataHandle*)h;
        if (sub == 2) mixed_gpu::set_gpu_pulse_SU2(x, vec(fd, n), amp, width, freq, t1, t2);
        else mixed_gpu::set_gpu_pulse_SU3(x, vec(fd, n), amp, width, freq, t1, t2);
        return 0;
    } catch (...) {
        return -1;
    }
}

int refmix_set_spins(void* h, const double* s, int64_t n) {
    try {
        mixed_gpu::set_gpu_mixed_spins((mixed_gpu::GPUMixedLatticeDataHandle*)h, vec(s, n));
        return 0;
    } catch (...) {
        return -1;
    }
}

int refmix_get_spins(void* h, double* s, int64_t n) {
    try {
        std::vector<double> v;
        mixed_gpu::get_gpu_mixed_spins((mixed_gpu::GPUMixedLatticeDataHandle*)h, v);
        if ((int64_t)v.size() != n) return -2;
        std::memcpy(s, v.data(), n * sizeof(double));
        return 0;
    } catch (...) {
        return -1;
    }
}

int refmix_step(void* h, double t, double dt, const char* method) {
    try {
        mixed_gpu::step_mixed_gpu((mixed_gpu::GPUMixedLatticeDataHandle*)h, t, dt, method);
        return 0;
    } catch (...) {
        return -1;
    }
}

// Saved rows into times[max_rows], states[max_rows][n]; returns the row count (or < 0).
int64_t refmix_integrate(void* h, double T0, double T1, double dt, int64_t save, const char* method, double* times,
                         double* states, int64_t n, int64_t max_rows) {
    try {
        std::vector<std::pair<double, std::vector<double>>> traj;
        mixed_gpu::integrate_mixed_gpu((mixed_gpu::GPUMixedLatticeDataHandle*)h, T0, T1, dt, (size_t)save, traj,
                                       method);
        const int64_t rows = (int64_t)traj.size();
        for (int64_t r = 0; r < rows && r < max_rows; ++r) {
            times[r] = traj[r].first;
            if ((int64_t)traj[r].second.size() != n) return -2;
            std::memcpy(states + r * n, traj[r].second.data(), n * sizeof(double));
        }
        return rows;
    } catch (...) {
        return -1;
    }
}

int refmix_magnetization(void* h, double* m2, double* ms2, double* m3, double* ms3) {
    try {
        std::vector<double> a, b, c, d;
        mixed_gpu::compute_magnetization_mixed_gpu((mixed_gpu::GPUMixedLatticeDataHandle*)h, a, b, c, d);
        std::memcpy(m2, a.data(), 3 * sizeof(double));
        std::memcpy(ms2, b.data(), 3 * sizeof(double));
        std::memcpy(m3, c.data(), 8 * sizeof(double));
        std::memcpy(ms3, d.data(), 8 * sizeof(double));
        return 0;
    } catch (...) {
        return -1;
    }
}

int refmix_normalize(void* h, double l2, double l3) {
    try {
        mixed_gpu::normalize_spins_mixed_gpu((mixed_gpu::GPUMixedLatticeDataHandle*)h, l2, l3);
        return 0;
    } catch (...) {
        return -1;
    }
}

}  // extern "C"
