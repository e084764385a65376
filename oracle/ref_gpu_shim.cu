// ref_gpu_shim.cu -- C entry points around the REFERENCE's own GPU integrator.
//
// Test infrastructure only.  Compiled (by oracle/Makefile, target `ref`)
// together with the reference sources src/gpu/lattice_gpu.cu and
// src/gpu/gpu_common_helpers.cu, read in place from the reference tree, into
// oracle/_ref/libref_gpu.so.  It calls the reference's `namespace gpu` API
// (include/classical_spin/gpu/lattice_gpu_api.h) exactly as the reference's
// Lattice host glue does (lattice.h:5429-5602, 5617-5855), so tests can pin
// the CPU restatement in ll_oracle.cpp to the reference's own arithmetic on
// a B200.  Every entry point returns a negative value on a C++ exception.
#include "classical_spin/gpu/lattice_gpu_api.h"

#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

extern "C" {

void* refgpu_create(int64_t N, int64_t n_atoms, int64_t zmax, const double* field,
                    const double* onsite, const double* bilinear, const int64_t* partners,
                    const int64_t* counts) {
    try {
        std::vector<double> f(field, field + 3 * N), o(onsite, onsite + 9 * N),
            b(bilinear, bilinear + 9 * N * zmax);
        std::vector<size_t> p(partners, partners + N * zmax), c(counts, counts + N);
        return gpu::create_gpu_lattice_data((size_t)N, 3, (size_t)n_atoms, (size_t)zmax, f, o, b, p, c);
    } catch (...) {
        return nullptr;
    }
}

void refgpu_destroy(void* h) { gpu::destroy_gpu_lattice_data((gpu::GPULatticeDataHandle*)h); }

int refgpu_set_pulse(void* h, const double* fd, int64_t n, double amp, double width, double freq,
                     double t1, double t2) {
    try {
        gpu::set_gpu_pulse((gpu::GPULatticeDataHandle*)h, std::vector<double>(fd, fd + n), amp, width,
                           freq, t1, t2);
        return 0;
    } catch (...) {
        return -1;
    }
}

int refgpu_set_spins(void* h, const double* s, int64_t n) {
    try {
        gpu::set_gpu_spins((gpu::GPULatticeDataHandle*)h, std::vector<double>(s, s + n));
        return 0;
    } catch (...) {
        return -1;
    }
}

int refgpu_get_spins(void* h, double* s, int64_t n) {
    try {
        std::vector<double> v;
        gpu::get_gpu_spins((gpu::GPULatticeDataHandle*)h, v);
        if ((int64_t)v.size() != n) return -2;
        std::memcpy(s, v.data(), n * sizeof(double));
        return 0;
    } catch (...) {
        return -1;
    }
}

// integrate_gpu: copies up to max_rows saved (t, state) pairs; returns the row count.
int64_t refgpu_integrate(void* h, double T0, double T1, double dt, int64_t save_interval,
                         const char* method, double* times, double* states, int64_t N3,
                         int64_t max_rows) {
    try {
        std::vector<std::pair<double, std::vector<double>>> traj;
        gpu::integrate_gpu((gpu::GPULatticeDataHandle*)h, T0, T1, dt, (size_t)save_interval, traj,
                           std::string(method));
        const int64_t n = (int64_t)traj.size();
        for (int64_t r = 0; r < n && r < max_rows; ++r) {
            if (times) times[r] = traj[r].first;
            if (states && (int64_t)traj[r].second.size() == N3)
                std::memcpy(states + r * N3, traj[r].second.data(), N3 * sizeof(double));
        }
        return n;
    } catch (...) {
        return -1;
    }
}

int refgpu_step(void* h, double t, double dt, const char* method) {
    try {
        gpu::step_gpu((gpu::GPULatticeDataHandle*)h, t, dt, std::string(method));
        return 0;
    } catch (...) {
        return -1;
    }
}

// integrate_gpu_batched: mags [rows][B][3][3]; returns the row count.
int64_t refgpu_batched(void* h, const double* init, int64_t N3, const double* tau2, int64_t B,
                       const double* afm, const double* frames, int64_t n_atoms, double T0,
                       double T1, double dt, int64_t save_interval, double* times, double* mags,
                       int64_t max_rows) {
    try {
        gpu::BatchedMagResult r = gpu::integrate_gpu_batched(
            (gpu::GPULatticeDataHandle*)h, std::vector<double>(init, init + N3),
            std::vector<double>(tau2, tau2 + B), std::vector<double>(afm, afm + n_atoms),
            std::vector<double>(frames, frames + 9 * n_atoms), T0, T1, dt, (size_t)save_interval,
            "rk4");
        const int64_t n = (int64_t)r.n_time_points;
        for (int64_t i = 0; i < n && i < max_rows; ++i) {
            if (times) times[i] = r.times[i];
            if (mags) std::memcpy(mags + i * B * 9, r.mag_data.data() + i * B * 9, B * 9 * sizeof(double));
        }
        return n;
    } catch (...) {
        return -1;
    }
}

}  // extern "C"
