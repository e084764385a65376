// The reference's call sequence on its mixed SU(2)/SU(3) host GPU API (as MixedLattice makes
// it), compiled against the header-only drop-in include/classical_spin/gpu/mixed_lattice_gpu_api.h.
//
// usage: mixed_shim_calls <dir>.  Reads <dir>/meta.txt ("n2 na2 n3 na3 z2 z3 zm2 zm3") and the raw
// arrays field2, onsite2, bil2, field3, onsite3, bil3, mix2, mix3, spins, drive2, drive3 (double) and
// part2, cnt2, part3, cnt3, mpart2, mcnt2, mpart3, mcnt3 (uint64) as <name>.bin; writes
// <dir>/out_<name>.bin.
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <string>
#include <vector>

#include "classical_spin/gpu/mixed_lattice_gpu_api.h"

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
        std::fprintf(stderr, "usage: mixed_shim_calls <dir>\n");
        return 2;
    }
    const std::string d = std::string(argv[1]) + "/";
    size_t n2 = 0, na2 = 0, n3 = 0, na3 = 0, z2 = 0, z3 = 0, zm2 = 0, zm3 = 0;
    {
        std::ifstream m(d + "meta.txt");
        m >> n2 >> na2 >> n3 >> na3 >> z2 >> z3 >> zm2 >> zm3;
    }
    auto D = [&](const char* n) { return load<double>(d + n + ".bin"); };
    auto I = [&](const char* n) { return load<size_t>(d + n + ".bin"); };
    try {
        mixed_gpu::GPUMixedLatticeDataHandle* h = mixed_gpu::create_gpu_mixed_lattice_data(
            n2, 3, na2, n3, 8, na3, z2, z3, zm2, zm3, D("field2"), D("onsite2"), D("bil2"), I("part2"), I("cnt2"),
            D("field3"), D("onsite3"), D("bil3"), I("part3"), I("cnt3"), D("mix2"), std::vector<size_t>(),
            I("mpart2"), I("mcnt2"), D("mix3"), I("mpart3"), I("mcnt3"));
        // No spins yet, and NULL handles: the reference's calls are no-ops.
        std::vector<double> untouched = {7.0};
        std::vector<std::pair<double, std::vector<double>>> traj;
        mixed_gpu::get_gpu_mixed_spins(h, untouched);
        mixed_gpu::integrate_mixed_gpu(h, 0.0, 1.0, 0.1, 1, traj);
        size_t a = 1, b = 1, c = 1, e = 1, f = 1, g = 1;
        mixed_gpu::get_mixed_lattice_dims(nullptr, a, b, c, e, f, g);
        std::vector<double> noop = {untouched.size() == 1 && untouched[0] == 7.0 ? 1.0 : 0.0, (double)traj.size(),
                                    (double)(a + b + c + e + f + g)};
        mixed_gpu::get_mixed_lattice_dims(h, a, b, c, e, f, g);
        noop.insert(noop.end(), {(double)a, (double)b, (double)c, (double)e, (double)f, (double)g});
        save(d + "out_noop.bin", noop);

        mixed_gpu::set_gpu_pulse_SU2(h, D("drive2"), 0.6, 0.3, 1.2, 0.05, 0.25);
        mixed_gpu::set_gpu_pulse_SU3(h, D("drive3"), 0.4, 0.2, 0.8, 0.1, 0.3);
        mixed_gpu::set_gpu_mixed_spins(h, D("spins"));
        mixed_gpu::integrate_mixed_gpu(h, 0.0, 0.4, 0.02, 5, traj);          // default method: ssprk53
        std::vector<double> times, states;
        for (const auto& p : traj) {
            times.push_back(p.first);
            states.insert(states.end(), p.second.begin(), p.second.end());
        }
        save(d + "out_traj_times.bin", times);
        save(d + "out_traj_states.bin", states);
        std::vector<double> s;
        mixed_gpu::step_mixed_gpu(h, 0.4, 0.02, "rk4");
        mixed_gpu::get_gpu_mixed_spins(h, s);
        save(d + "out_step_rk4.bin", s);
        mixed_gpu::step_mixed_gpu(h, 0.42, 0.02, "no_such_method");         // warns, runs ssprk53
        mixed_gpu::get_gpu_mixed_spins(h, s);
        save(d + "out_step_fallback.bin", s);
        std::vector<double> m2, ms2, m3, ms3;
        mixed_gpu::compute_magnetization_mixed_gpu(h, m2, ms2, m3, ms3);
        std::vector<double> mags = m2;
        mags.insert(mags.end(), ms2.begin(), ms2.end());
        mags.insert(mags.end(), m3.begin(), m3.end());
        mags.insert(mags.end(), ms3.begin(), ms3.end());
        save(d + "out_mags.bin", mags);
        mixed_gpu::normalize_spins_mixed_gpu(h, 1.5, 0.7);
        mixed_gpu::get_gpu_mixed_spins(h, s);
        save(d + "out_normalized.bin", s);
        mixed_gpu::destroy_gpu_mixed_lattice_data(h);
        mixed_gpu::destroy_gpu_mixed_lattice_data(nullptr);
    } catch (const std::exception& ex) {
        std::fprintf(stderr, "error: %s\n", ex.what());
        return 1;
    }
    return 0;
}
