/*
 * Header-only drop-in for the reference's host GPU API (namespace gpu,
 * include/classical_spin/gpu/lattice_gpu_api.h:24-216 of ze-bang/Classical_MCMC_Spin),
 * implemented over the C ABI in cmd.h (libcmd_b200.so).
 *
 * Put this repository's include/ ahead of the reference's on the include path
 * and link -lcmd_b200: Lattice (lattice.h:5422-5966) compiles unchanged.  The
 * include guard is the reference header's own, so whichever copy is found
 * first is the only one seen.
 *
 * Behaviour kept from the reference (lattice_gpu.cu:627-796):
 *   - a NULL handle, or a handle without spins, makes every call a no-op
 *     (compute_energy_gpu returns 0.0);
 *   - integrate_gpu appends (t, state) pairs to `trajectory`, every
 *     save_interval steps and once more at the end (integrator.cuh:470-488);
 *   - an unknown method warns on std::cerr and runs "ssprk53"
 *     (integrator.cuh:454-458); integrate_gpu_batched warns and runs "rk4"
 *     for any other method (lattice_gpu.cu:781-784);
 *   - compute_magnetization_gpu adds the new means to whatever the output
 *     vectors hold (they are resized, not cleared, lattice_gpu.cu:736-757).
 * Differences: compute_energy_gpu returns the energy (the reference throws,
 * lattice_gpu.cu:298-303); spin_dim must be 3 and vector sizes must match the
 * lattice (std::invalid_argument otherwise); device errors throw
 * std::runtime_error carrying cmd_last_error().
 */
#ifndef LATTICE_GPU_API_H
#define LATTICE_GPU_API_H

#include <cstddef>
#include <cstdint>
#include <iostream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "cmd.h"

namespace gpu {

struct GPULatticeDataHandle {
    cmd_handle* h = nullptr;
    size_t lattice_size = 0;
    size_t n_atoms = 0;
    bool has_state = false;
};

namespace shim {

inline void check(int rc, const char* what) {
    if (rc == CMD_OK) return;
    const std::string msg = std::string(what) + ": " + cmd_last_error();
    if (rc == CMD_ERR_INVALID_ARG) throw std::invalid_argument(msg);
    throw std::runtime_error(msg);
}

// Method names of the reference GPU integrator (integrator.cuh:91-458); -1 if unknown.
inline int method_code(const std::string& m) {
    if (m == "ssprk53") return CMD_SSPRK53;
    if (m == "rk4") return CMD_RK4;
    if (m == "dopri5" || m == "rk54" || m == "rkf54") return CMD_DOPRI5_FIXED;
    if (m == "rk5" || m == "rkck54") return CMD_CASH_KARP_FIXED;
    if (m == "euler") return CMD_EULER;
    if (m == "rk2" || m == "midpoint") return CMD_MIDPOINT;
    if (m == "rk78" || m == "rkf78") return CMD_RK78;
    if (m == "bulirsch_stoer" || m == "bs") return CMD_BULIRSCH_STOER;
    return -1;
}

inline int method_or_default(const std::string& m) {
    const int c = method_code(m);
    if (c >= 0) return c;
    std::cerr << "Warning: Unknown GPU integration method '" << m << "', using ssprk53" << std::endl;
    return CMD_SSPRK53;
}

inline bool ready(const GPULatticeDataHandle* x) { return x && x->h && x->has_state; }

}  // namespace shim

inline GPULatticeDataHandle* create_gpu_lattice_data(size_t lattice_size, size_t spin_dim, size_t N_atoms,
                                                     size_t max_bilinear, const std::vector<double>& flat_field,
                                                     const std::vector<double>& flat_onsite,
                                                     const std::vector<double>& flat_bilinear,
                                                     const std::vector<size_t>& flat_partners,
                                                     const std::vector<size_t>& num_bilinear_per_site) {
    if (spin_dim != 3) throw std::invalid_argument("create_gpu_lattice_data: spin_dim must be 3");
    const size_t N = lattice_size;
    if (flat_field.size() != 3 * N || flat_onsite.size() != 9 * N || flat_bilinear.size() != 9 * N * max_bilinear ||
        flat_partners.size() != N * max_bilinear || num_bilinear_per_site.size() != N)
        throw std::invalid_argument("create_gpu_lattice_data: array sizes do not match the lattice");
    const std::vector<int64_t> partners(flat_partners.begin(), flat_partners.end());
    const std::vector<int64_t> counts(num_bilinear_per_site.begin(), num_bilinear_per_site.end());
    cmd_lattice_desc d{};
    d.lattice_size = (int64_t)N;
    d.spin_dim = 3;
    d.n_atoms = (int32_t)N_atoms;
    d.max_bilinear = (int32_t)max_bilinear;
    d.field = flat_field.data();
    d.onsite = flat_onsite.data();
    d.bilinear = flat_bilinear.data();
    d.partners = partners.data();
    d.counts = counts.data();
    cmd_handle* h = nullptr;
    shim::check(cmd_create(&d, &h), "create_gpu_lattice_data");
    GPULatticeDataHandle* x = new GPULatticeDataHandle;
    x->h = h;
    x->lattice_size = N;
    x->n_atoms = N_atoms;
    return x;
}

inline void destroy_gpu_lattice_data(GPULatticeDataHandle* handle) {
    if (!handle) return;
    cmd_destroy(handle->h);
    delete handle;
}

inline void set_gpu_pulse(GPULatticeDataHandle* handle, const std::vector<double>& flat_field_drive,
                          double pulse_amp, double pulse_width, double pulse_freq, double t_pulse_1,
                          double t_pulse_2) {
    if (!handle || !handle->h) return;
    if (flat_field_drive.size() != 2 * 3 * handle->n_atoms)
        throw std::invalid_argument("set_gpu_pulse: flat_field_drive must hold 2 * N_atoms * 3 values");
    shim::check(cmd_set_pulse(handle->h, flat_field_drive.data(), pulse_amp, pulse_width, pulse_freq, t_pulse_1,
                              t_pulse_2),
                "set_gpu_pulse");
}

inline void set_gpu_spins(GPULatticeDataHandle* handle, const std::vector<double>& flat_spins) {
    if (!handle || !handle->h) return;
    shim::check(cmd_set_spins(handle->h, flat_spins.data(), (int64_t)flat_spins.size()), "set_gpu_spins");
    handle->has_state = true;
}

inline void get_gpu_spins(GPULatticeDataHandle* handle, std::vector<double>& flat_spins) {
    if (!shim::ready(handle)) return;
    flat_spins.resize(3 * handle->lattice_size);
    shim::check(cmd_get_spins(handle->h, flat_spins.data(), (int64_t)flat_spins.size()), "get_gpu_spins");
}

inline void integrate_gpu(GPULatticeDataHandle* handle, double T_start, double T_end, double dt,
                          size_t save_interval, std::vector<std::pair<double, std::vector<double>>>& trajectory,
                          const std::string& method = "ssprk53") {
    if (!shim::ready(handle)) return;
    const int m = shim::method_or_default(method);
    const size_t n3 = 3 * handle->lattice_size;
    int64_t rows = 0;
    const int rc = cmd_integrate(handle->h, T_start, T_end, dt, (int64_t)save_interval, m, nullptr, nullptr,
                                 nullptr, 0, &rows);
    if (rows <= 0) shim::check(rc == CMD_OK ? CMD_ERR_INVALID_ARG : rc, "integrate_gpu");
    std::vector<double> times((size_t)rows), states((size_t)rows * n3);
    shim::check(cmd_integrate(handle->h, T_start, T_end, dt, (int64_t)save_interval, m, times.data(), nullptr,
                              states.data(), rows, &rows),
                "integrate_gpu");
    trajectory.reserve(trajectory.size() + (size_t)rows);
    for (int64_t r = 0; r < rows; ++r)
        trajectory.emplace_back(times[(size_t)r], std::vector<double>(states.begin() + r * n3,
                                                                      states.begin() + (r + 1) * n3));
}

inline void step_gpu(GPULatticeDataHandle* handle, double t, double dt, const std::string& method = "ssprk53") {
    if (!shim::ready(handle)) return;
    shim::check(cmd_step(handle->h, t, dt, shim::method_or_default(method)), "step_gpu");
}

inline double compute_energy_gpu(GPULatticeDataHandle* handle) {
    if (!shim::ready(handle)) return 0.0;
    double e = 0.0;
    shim::check(cmd_energy(handle->h, &e), "compute_energy_gpu");
    return e;
}

inline void normalize_spins_gpu(GPULatticeDataHandle* handle, double spin_length) {
    if (!shim::ready(handle)) return;
    shim::check(cmd_normalize(handle->h, spin_length), "normalize_spins_gpu");
}

inline void compute_magnetization_gpu(GPULatticeDataHandle* handle, std::vector<double>& mag_local,
                                      std::vector<double>& mag_staggered) {
    if (!shim::ready(handle)) return;
    double ml[3], ms[3];
    shim::check(cmd_magnetization(handle->h, ml, ms), "compute_magnetization_gpu");
    mag_local.resize(3, 0.0);
    mag_staggered.resize(3, 0.0);
    const double N = (double)handle->lattice_size;
    for (int d = 0; d < 3; ++d) {
        mag_local[d] = mag_local[d] / N + ml[d];
        mag_staggered[d] = mag_staggered[d] / N + ms[d];
    }
}

struct BatchedMagResult {
    size_t B;
    size_t spin_dim;
    size_t n_time_points;
    std::vector<double> times;     // [n_time_points]
    std::vector<double> mag_data;  // [n_time_points][B][3][spin_dim]: M_antiferro, M_local, M_global
};

inline BatchedMagResult integrate_gpu_batched(GPULatticeDataHandle* handle,
                                              const std::vector<double>& flat_initial_state,
                                              const std::vector<double>& tau2_values,
                                              const std::vector<double>& afm_signs,
                                              const std::vector<double>& sublattice_frames, double T_start,
                                              double T_end, double dt, size_t save_interval = 1,
                                              const std::string& method = "rk4") {
    if (!handle || !handle->h || tau2_values.empty()) return BatchedMagResult{};
    if (method != "rk4")
        std::cerr << "[integrate_gpu_batched] method='" << method
                  << "' is not supported in batched mode; using rk4." << std::endl;
    const int64_t B = (int64_t)tau2_values.size();
    const double* afm = afm_signs.empty() ? nullptr : afm_signs.data();
    const double* frames = sublattice_frames.empty() ? nullptr : sublattice_frames.data();
    if (flat_initial_state.size() != 3 * handle->lattice_size)
        throw std::invalid_argument("integrate_gpu_batched: flat_initial_state must hold lattice_size * 3 values");
    if (afm && afm_signs.size() != handle->n_atoms)
        throw std::invalid_argument("integrate_gpu_batched: afm_signs must hold N_atoms values");
    if (frames && sublattice_frames.size() != 9 * handle->n_atoms)
        throw std::invalid_argument("integrate_gpu_batched: sublattice_frames must hold N_atoms * 9 values");
    int64_t rows = 0;
    const int rc = cmd_integrate_batched(handle->h, flat_initial_state.data(), tau2_values.data(), B, afm, frames,
                                         T_start, T_end, dt, (int64_t)save_interval, CMD_RK4, nullptr, nullptr, 0,
                                         &rows);
    if (rows <= 0) shim::check(rc == CMD_OK ? CMD_ERR_INVALID_ARG : rc, "integrate_gpu_batched");
    BatchedMagResult r;
    r.B = (size_t)B;
    r.spin_dim = 3;
    r.times.resize((size_t)rows);
    r.mag_data.resize((size_t)rows * B * 9);
    shim::check(cmd_integrate_batched(handle->h, flat_initial_state.data(), tau2_values.data(), B, afm, frames,
                                      T_start, T_end, dt, (int64_t)save_interval, CMD_RK4, r.times.data(),
                                      r.mag_data.data(), rows, &rows),
                "integrate_gpu_batched");
    r.n_time_points = (size_t)rows;
    return r;
}

}  // namespace gpu

#endif  // LATTICE_GPU_API_H
