// The reference's call sequence on its host GPU API (as Lattice makes it, lattice.h:5429-5966),
// compiled against the header-only drop-in include/classical_spin/gpu/lattice_gpu_api.h.
//
// usage: shim_calls <dir>.  Reads <dir>/meta.txt ("N n_atoms max_bilinear") and the raw arrays
// field, onsite, bilinear (double), partners, counts (uint64), spins, drive, afm, frames, tau2
// (double) as <name>.bin; writes its results to <dir>/out_<name>.bin.
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <string>
#include <vector>

#include "classical_spin/gpu/lattice_gpu_api.h"

template <class T>
static std::vector<T> load(const std::string& path) {
    std::ifstream f(path, std::ios::binary | std::ios::ate);
    if (!f) throw std::runtime_error("cannot read " + path);
    const std::streamsize n = f.tellg();
    f.seekg(0);
    std::vector<T> v((size_t)n / sizeof(T));
    f.read(reinterpret_cast<char*>(v.data()), n);
    return v;
}

static void save(const std::string& path, const std::vector<double>& v) {
    std::ofstream f(path, std::ios::binary);
    f.write(reinterpret_cast<const char*>(v.data()), (std::streamsize)(v.size() * sizeof(double)));
}

int main(int argc, char** argv) {
    if (argc != 2) {
        std::fprintf(stderr, "usage: shim_calls <dir>\n");
        return 2;
    }
    const std::string d = std::string(argv[1]) + "/";
    size_t N = 0, n_atoms = 0, zmax = 0;
    {
        std::ifstream m(d + "meta.txt");
        m >> N >> n_atoms >> zmax;
    }
    const auto spins = load<double>(d + "spins.bin");
    try {
        gpu::GPULatticeDataHandle* h = gpu::create_gpu_lattice_data(
            N, 3, n_atoms, zmax, load<double>(d + "field.bin"), load<double>(d + "onsite.bin"),
            load<double>(d + "bilinear.bin"), load<size_t>(d + "partners.bin"), load<size_t>(d + "counts.bin"));

        // No spins yet: the reference's calls are no-ops.
        std::vector<double> untouched = {7.0};
        std::vector<std::pair<double, std::vector<double>>> traj;
        gpu::get_gpu_spins(h, untouched);
        gpu::integrate_gpu(h, 0.0, 1.0, 0.1, 1, traj);
        gpu::step_gpu(h, 0.0, 0.1);
        const double e_none = gpu::compute_energy_gpu(h);
        const double e_null = gpu::compute_energy_gpu(nullptr);
        gpu::set_gpu_spins(nullptr, spins);
        gpu::destroy_gpu_lattice_data(nullptr);
        save(d + "out_noop.bin", {untouched.size() == 1 && untouched[0] == 7.0 ? 1.0 : 0.0, (double)traj.size(),
                                  e_none, e_null});

        gpu::set_gpu_pulse(h, load<double>(d + "drive.bin"), 0.5, 0.4, 0.9, 0.2, 0.6);
        gpu::set_gpu_spins(h, spins);
        gpu::integrate_gpu(h, 0.0, 1.0, 0.02, 5, traj);               // default method: ssprk53
        std::vector<double> times, states;
        for (const auto& p : traj) {
            times.push_back(p.first);
            states.insert(states.end(), p.second.begin(), p.second.end());
        }
        save(d + "out_traj_times.bin", times);
        save(d + "out_traj_states.bin", states);

        std::vector<double> s;
        gpu::step_gpu(h, 1.0, 0.02, "rk4");
        gpu::get_gpu_spins(h, s);
        save(d + "out_step_rk4.bin", s);
        gpu::step_gpu(h, 1.02, 0.02, "no_such_method");              // warns, runs ssprk53
        gpu::get_gpu_spins(h, s);
        save(d + "out_step_fallback.bin", s);

        std::vector<double> ml, ms;
        gpu::compute_magnetization_gpu(h, ml, ms);
        const double e = gpu::compute_energy_gpu(h);
        std::vector<double> scal = {e, ml[0], ml[1], ml[2], ms[0], ms[1], ms[2]};
        std::vector<double> ml2 = {1.0, 2.0, 3.0}, ms2 = {0.0, 0.0, 0.0};
        gpu::compute_magnetization_gpu(h, ml2, ms2);                   // adds to what the vectors hold
        scal.insert(scal.end(), ml2.begin(), ml2.end());
        save(d + "out_scalars.bin", scal);
        gpu::normalize_spins_gpu(h, 2.0);
        gpu::get_gpu_spins(h, s);
        save(d + "out_normalized.bin", s);

        const auto tau2 = load<double>(d + "tau2.bin");
        gpu::BatchedMagResult r = gpu::integrate_gpu_batched(h, spins, tau2, load<double>(d + "afm.bin"),
                                                             load<double>(d + "frames.bin"), -0.5, 1.0, 0.01, 2,
                                                             "dopri5");       // warns, runs rk4
        save(d + "out_batched_times.bin", r.times);
        save(d + "out_batched_mags.bin", r.mag_data);
        save(d + "out_batched_shape.bin", {(double)r.B, (double)r.spin_dim, (double)r.n_time_points});
        gpu::BatchedMagResult empty = gpu::integrate_gpu_batched(h, spins, {}, {}, {}, 0.0, 1.0, 0.1);
        save(d + "out_batched_empty.bin", {(double)empty.B, (double)empty.times.size()});
        gpu::destroy_gpu_lattice_data(h);
    } catch (const std::exception& ex) {
        std::fprintf(stderr, "error: %s\n", ex.what());
        return 1;
    }
    return 0;
}
