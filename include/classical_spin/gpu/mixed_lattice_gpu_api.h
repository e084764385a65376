/*
 * Header-only drop-in for the reference's host GPU API for mixed SU(2)/SU(3)
 * lattices (namespace mixed_gpu, include/classical_spin/gpu/mixed_lattice_gpu_api.h:25-214
 * of ze-bang/Classical_MCMC_Spin), implemented over the C ABI in cmd_mixed.h
 * (libcmd_b200.so).
 *
 * Put this repository's include/ ahead of the reference's on the include path and
 * link -lcmd_b200: MixedLattice compiles unchanged.  The include guard is the
 * reference header's own.
 *
 * Behaviour kept from the reference (mixed_lattice_gpu.cu:567-761): a NULL handle,
 * or a handle without spins, makes every call a no-op; integrate_mixed_gpu appends
 * (t, state) pairs every save_interval steps and once more at the end; an unknown
 * method warns on std::cerr and runs "ssprk53"; get_mixed_lattice_dims of a NULL
 * handle gives zeros.  Differences: spin dimensions must be 3 and 8, mismatched
 * vector sizes throw std::invalid_argument, device errors throw std::runtime_error
 * carrying cmd_last_error(), and "rk45" (a CPU-path method) is not a mixed method.
 */
#ifndef MIXED_LATTICE_GPU_API_H
#define MIXED_LATTICE_GPU_API_H

#include <array>
#include <cstddef>
#include <cstdint>
#include <iostream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "cmd.h"
#include "cmd_mixed.h"

namespace mixed_gpu {

struct GPUMixedLatticeDataHandle {
    cmd_mixed* h = nullptr;
    size_t n2 = 0, n3 = 0, na2 = 0, na3 = 0;
    bool has_state = false;
};

namespace shim {

inline void check(int rc, const char* what) {
    if (rc == CMD_OK) return;
    const std::string msg = std::string(what) + ": " + cmd_last_error();
    if (rc == CMD_ERR_INVALID_ARG) throw std::invalid_argument(msg);
    throw std::runtime_error(msg);
}

// Method names of the reference GPU integrator (integrator.cuh:91-458), ssprk53 for the rest.
inline int method_or_default(const std::string& m) {
    if (m == "ssprk53") return CMD_SSPRK53;
    if (m == "rk4") return CMD_RK4;
    if (m == "dopri5" || m == "rk54" || m == "rkf54") return CMD_DOPRI5_FIXED;
    if (m == "rk5" || m == "rkck54") return CMD_CASH_KARP_FIXED;
    if (m == "euler") return CMD_EULER;
    if (m == "rk2" || m == "midpoint") return CMD_MIDPOINT;
    if (m == "rk78" || m == "rkf78") return CMD_RK78;
    if (m == "bulirsch_stoer" || m == "bs") return CMD_BULIRSCH_STOER;
    std::cerr << "Warning: Unknown GPU integration method '" << m << "', using ssprk53" << std::endl;
    return CMD_SSPRK53;
}

inline bool ready(const GPUMixedLatticeDataHandle* x) { return x && x->h && x->has_state; }

inline std::vector<int64_t> idx(const std::vector<size_t>& v) { return std::vector<int64_t>(v.begin(), v.end()); }

}  // namespace shim

inline GPUMixedLatticeDataHandle* create_gpu_mixed_lattice_data(
    size_t lattice_size_SU2, size_t spin_dim_SU2, size_t N_atoms_SU2, size_t lattice_size_SU3, size_t spin_dim_SU3,
    size_t N_atoms_SU3, size_t max_bilinear_SU2, size_t max_bilinear_SU3, size_t max_mixed_bilinear,
    size_t max_mixed_bilinear_SU3, const std::vector<double>& flat_field_SU2, const std::vector<double>& flat_onsite_SU2,
    const std::vector<double>& flat_bilinear_SU2, const std::vector<size_t>& flat_partners_SU2,
    const std::vector<size_t>& num_bilinear_per_site_SU2, const std::vector<double>& flat_field_SU3,
    const std::vector<double>& flat_onsite_SU3, const std::vector<double>& flat_bilinear_SU3,
    const std::vector<size_t>& flat_partners_SU3, const std::vector<size_t>& num_bilinear_per_site_SU3,
    const std::vector<double>& flat_mixed_bilinear, const std::vector<size_t>& /*flat_mixed_partners_SU2, unused*/,
    const std::vector<size_t>& flat_mixed_partners_SU3, const std::vector<size_t>& num_mixed_per_site_SU2,
    const std::vector<double>& flat_mixed_bilinear_SU3, const std::vector<size_t>& flat_mixed_partners_SU2_from_SU3,
    const std::vector<size_t>& num_mixed_per_site_SU3) {
    if (spin_dim_SU2 != 3 || spin_dim_SU3 != 8)
        throw std::invalid_argument("create_gpu_mixed_lattice_data: spin dimensions must be 3 and 8");
    const size_t N2 = lattice_size_SU2, N3 = lattice_size_SU3;
    const size_t z2 = max_bilinear_SU2, z3 = max_bilinear_SU3, zm2 = max_mixed_bilinear, zm3 = max_mixed_bilinear_SU3;
    if (flat_field_SU2.size() != 3 * N2 || flat_onsite_SU2.size() != 9 * N2 || flat_bilinear_SU2.size() != 9 * N2 * z2 ||
        flat_partners_SU2.size() != N2 * z2 || num_bilinear_per_site_SU2.size() != N2 ||
        flat_field_SU3.size() != 8 * N3 || flat_onsite_SU3.size() != 64 * N3 ||
        flat_bilinear_SU3.size() != 64 * N3 * z3 || flat_partners_SU3.size() != N3 * z3 ||
        num_bilinear_per_site_SU3.size() != N3 || flat_mixed_bilinear.size() != 24 * N2 * zm2 ||
        flat_mixed_partners_SU3.size() != N2 * zm2 || (zm2 > 0 && num_mixed_per_site_SU2.size() != N2) ||
        flat_mixed_bilinear_SU3.size() != 24 * N3 * zm3 || flat_mixed_partners_SU2_from_SU3.size() != N3 * zm3 ||
        (zm3 > 0 && num_mixed_per_site_SU3.size() != N3))
        throw std::invalid_argument("create_gpu_mixed_lattice_data: array sizes do not match the lattice");
    const std::vector<int64_t> p2 = shim::idx(flat_partners_SU2), c2 = shim::idx(num_bilinear_per_site_SU2);
    const std::vector<int64_t> p3 = shim::idx(flat_partners_SU3), c3 = shim::idx(num_bilinear_per_site_SU3);
    const std::vector<int64_t> mp2 = shim::idx(flat_mixed_partners_SU3), mc2 = shim::idx(num_mixed_per_site_SU2);
    const std::vector<int64_t> mp3 = shim::idx(flat_mixed_partners_SU2_from_SU3), mc3 = shim::idx(num_mixed_per_site_SU3);
    cmd_mixed_desc d{};
    d.n_su2 = (int64_t)N2;
    d.n_su3 = (int64_t)N3;
    d.spin_dim_su2 = 3;
    d.spin_dim_su3 = 8;
    d.n_atoms_su2 = (int32_t)N_atoms_SU2;
    d.n_atoms_su3 = (int32_t)N_atoms_SU3;
    d.max_bilinear_su2 = (int32_t)z2;
    d.max_bilinear_su3 = (int32_t)z3;
    d.max_mixed_su2 = (int32_t)zm2;
    d.max_mixed_su3 = (int32_t)zm3;
    d.field_su2 = flat_field_SU2.data();
    d.onsite_su2 = flat_onsite_SU2.data();
    d.bilinear_su2 = flat_bilinear_SU2.data();
    d.partners_su2 = p2.data();
    d.counts_su2 = c2.data();
    d.field_su3 = flat_field_SU3.data();
    d.onsite_su3 = flat_onsite_SU3.data();
    d.bilinear_su3 = flat_bilinear_SU3.data();
    d.partners_su3 = p3.data();
    d.counts_su3 = c3.data();
    d.mixed_su2 = flat_mixed_bilinear.data();
    d.mixed_partners_su3 = mp2.data();
    d.mixed_counts_su2 = mc2.data();
    d.mixed_su3 = flat_mixed_bilinear_SU3.data();
    d.mixed_partners_su2 = mp3.data();
    d.mixed_counts_su3 = mc3.data();
    cmd_mixed* h = nullptr;
    shim::check(cmd_mixed_create(&d, &h), "create_gpu_mixed_lattice_data");
    GPUMixedLatticeDataHandle* x = new GPUMixedLatticeDataHandle;
    x->h = h;
    x->n2 = N2;
    x->n3 = N3;
    x->na2 = N_atoms_SU2;
    x->na3 = N_atoms_SU3;
    return x;
}

inline void destroy_gpu_mixed_lattice_data(GPUMixedLatticeDataHandle* handle) {
    if (!handle) return;
    cmd_mixed_destroy(handle->h);
    delete handle;
}

inline void set_gpu_pulse_SU2(GPUMixedLatticeDataHandle* handle, const std::vector<double>& flat_field_drive,
                              double pulse_amp, double pulse_width, double pulse_freq, double t_pulse_1,
                              double t_pulse_2) {
    if (!handle || !handle->h) return;
    if (flat_field_drive.size() != 2 * 3 * handle->na2)
        throw std::invalid_argument("set_gpu_pulse_SU2: flat_field_drive must hold 2 * N_atoms_SU2 * 3 values");
    shim::check(cmd_mixed_set_pulse(handle->h, 2, flat_field_drive.data(), pulse_amp, pulse_width, pulse_freq,
                                    t_pulse_1, t_pulse_2),
                "set_gpu_pulse_SU2");
}

inline void set_gpu_pulse_SU3(GPUMixedLatticeDataHandle* handle, const std::vector<double>& flat_field_drive,
                              double pulse_amp, double pulse_width, double pulse_freq, double t_pulse_1,
                              double t_pulse_2) {
    if (!handle || !handle->h) return;
    if (flat_field_drive.size() != 2 * 8 * handle->na3)
        throw std::invalid_argument("set_gpu_pulse_SU3: flat_field_drive must hold 2 * N_atoms_SU3 * 8 values");
    shim::check(cmd_mixed_set_pulse(handle->h, 3, flat_field_drive.data(), pulse_amp, pulse_width, pulse_freq,
                                    t_pulse_1, t_pulse_2),
                "set_gpu_pulse_SU3");
}

inline void set_gpu_mixed_spins(GPUMixedLatticeDataHandle* handle, const std::vector<double>& flat_spins) {
    if (!handle || !handle->h) return;
    shim::check(cmd_mixed_set_spins(handle->h, flat_spins.data(), (int64_t)flat_spins.size()), "set_gpu_mixed_spins");
    handle->has_state = true;
}

inline void get_gpu_mixed_spins(GPUMixedLatticeDataHandle* handle, std::vector<double>& flat_spins) {
    if (!shim::ready(handle)) return;
    flat_spins.resize(3 * handle->n2 + 8 * handle->n3);
    shim::check(cmd_mixed_get_spins(handle->h, flat_spins.data(), (int64_t)flat_spins.size()), "get_gpu_mixed_spins");
}

inline void integrate_mixed_gpu(GPUMixedLatticeDataHandle* handle, double T_start, double T_end, double dt,
                                size_t save_interval, std::vector<std::pair<double, std::vector<double>>>& trajectory,
                                const std::string& method = "ssprk53") {
    if (!shim::ready(handle)) return;
    const int m = shim::method_or_default(method);
    const size_t V = 3 * handle->n2 + 8 * handle->n3;
    int64_t rows = 0;
    const int rc = cmd_mixed_integrate(handle->h, T_start, T_end, dt, (int64_t)save_interval, m, nullptr, nullptr, 0,
                                       &rows);
    if (rows <= 0) shim::check(rc == CMD_OK ? CMD_ERR_INVALID_ARG : rc, "integrate_mixed_gpu");
    std::vector<double> times((size_t)rows), states((size_t)rows * V);
    shim::check(cmd_mixed_integrate(handle->h, T_start, T_end, dt, (int64_t)save_interval, m, times.data(),
                                    states.data(), rows, &rows),
                "integrate_mixed_gpu");
    trajectory.reserve(trajectory.size() + (size_t)rows);
    for (int64_t r = 0; r < rows; ++r)
        trajectory.emplace_back(times[(size_t)r],
                                std::vector<double>(states.begin() + r * V, states.begin() + (r + 1) * V));
}

inline void step_mixed_gpu(GPUMixedLatticeDataHandle* handle, double t, double dt,
                           const std::string& method = "ssprk53") {
    if (!shim::ready(handle)) return;
    shim::check(cmd_mixed_step(handle->h, t, dt, shim::method_or_default(method)), "step_mixed_gpu");
}

inline void compute_magnetization_mixed_gpu(GPUMixedLatticeDataHandle* handle, std::vector<double>& mag_SU2,
                                            std::vector<double>& mag_staggered_SU2, std::vector<double>& mag_SU3,
                                            std::vector<double>& mag_staggered_SU3) {
    if (!shim::ready(handle)) return;
    mag_SU2.resize(3);
    mag_staggered_SU2.resize(3);
    mag_SU3.resize(8);
    mag_staggered_SU3.resize(8);
    shim::check(cmd_mixed_magnetization(handle->h, mag_SU2.data(), mag_staggered_SU2.data(), mag_SU3.data(),
                                        mag_staggered_SU3.data()),
                "compute_magnetization_mixed_gpu");
}

inline void normalize_spins_mixed_gpu(GPUMixedLatticeDataHandle* handle, double spin_length_SU2,
                                      double spin_length_SU3) {
    if (!shim::ready(handle)) return;
    shim::check(cmd_mixed_normalize(handle->h, spin_length_SU2, spin_length_SU3), "normalize_spins_mixed_gpu");
}

inline void get_mixed_lattice_dims(GPUMixedLatticeDataHandle* handle, size_t& lattice_size_SU2, size_t& spin_dim_SU2,
                                   size_t& N_atoms_SU2, size_t& lattice_size_SU3, size_t& spin_dim_SU3,
                                   size_t& N_atoms_SU3) {
    if (!handle || !handle->h) {
        lattice_size_SU2 = spin_dim_SU2 = N_atoms_SU2 = 0;
        lattice_size_SU3 = spin_dim_SU3 = N_atoms_SU3 = 0;
        return;
    }
    int64_t dims[6];
    shim::check(cmd_mixed_dims(handle->h, dims), "get_mixed_lattice_dims");
    lattice_size_SU2 = (size_t)dims[0];
    spin_dim_SU2 = (size_t)dims[1];
    N_atoms_SU2 = (size_t)dims[2];
    lattice_size_SU3 = (size_t)dims[3];
    spin_dim_SU3 = (size_t)dims[4];
    N_atoms_SU3 = (size_t)dims[5];
}

}  // namespace mixed_gpu

#endif  // MIXED_LATTICE_GPU_API_H
