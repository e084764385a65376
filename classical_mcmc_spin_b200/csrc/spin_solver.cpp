// spin_solver.cpp -- command-line driver for the molecular-dynamics modes of the
// reference's `spin_solver` (src/apps/spin_solver.cpp main :36-374), running on
// the C ABI (include/cmd.h, include/cmd_lattice.h):
//
//   molecular_dynamics  run_molecular_dynamics   runners_lattice.cpp:260-371
//   pump_probe          run_pump_probe           runners_lattice.cpp:376-572
//   2dcs                run_2dcs_spectroscopy    runners_lattice.cpp:578-898
//                       -> pump_probe_spectroscopy_gpu_batched (lattice.h:5617-5855)
//
// Usage:  cmd_spin_solver <file.param> [--parse-only]
//
// The param file is the reference's format (SpinConfig::from_file,
// src/core/spin_config.cpp): `key = value` lines, `#` comments, vectors as
// comma lists.  Systems: honeycomb_kitaev (build_kitaev_honeycomb) and
// pyrochlore_non_kramer (build_pyrochlore_non_kramer).  Keys of modes outside
// this path (annealing, tempering, MC moves) are accepted and ignored: the
// initial state is `initial_spin_config` (the reference's text format) or, when
// that is empty, a seeded random state (`seed`, default 0) -- simulated
// annealing is not part of this build, so an equilibrated state must come from
// a file.
//
// Outputs (per trial directory output_dir/sample_<trial>): initial_spins.txt in
// the reference's format; HDF5 is not available here, so the datasets of the
// reference's trajectory.h5 / pump_probe_spectroscopy.h5 are written as .npy
// files named after their HDF5 paths plus metadata.json for the attributes.
// pump_probe writes pump_probe_trajectory.txt as the reference does.  2dcs also
// writes the analysis step (M_NL and its 2-D spectrum, cmd_nonlinear_spectrum).
//
// Keys this driver adds: seed, cubic_cell (pyrochlore on the 16-site cubic cell),
// md_adaptive (dopri5 with step control instead of the GPU path's fixed step),
// md_save_spins (default true), pump_direction_2 (probe direction in 2dcs).
#include "cmd.h"
#include "cmd_lattice.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <set>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace fs = std::filesystem;

namespace {

struct ConfigError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

std::string trim(const std::string& s) {
    const size_t a = s.find_first_not_of(" \t\r\n");
    if (a == std::string::npos) return "";
    const size_t b = s.find_last_not_of(" \t\r\n");
    return s.substr(a, b - a + 1);
}

std::vector<double> parse_vector(const std::string& v) {     // "1,0,0", "[1, 0, 0]", "(1,0,0)"
    std::string s;
    for (char c : v)
        if (c != '(' && c != ')' && c != '[' && c != ']') s += c;
    std::vector<double> out;
    std::stringstream ss(s);
    std::string item;
    while (std::getline(ss, item, ',')) {
        item = trim(item);
        if (!item.empty()) out.push_back(std::stod(item));
    }
    return out;
}

std::vector<std::vector<double>> parse_vec3_list(const std::string& v, const char* key) {
    const std::vector<double> x = parse_vector(v);
    if (x.empty() || x.size() % 3 != 0)
        throw ConfigError(std::string(key) + " must have a multiple of 3 values (got " + std::to_string(x.size()) +
                          ")");
    std::vector<std::vector<double>> out;
    for (size_t i = 0; i < x.size(); i += 3) out.push_back({x[i], x[i + 1], x[i + 2]});
    return out;
}

bool parse_bool(const std::string& v) {
    std::string s = trim(v);
    std::transform(s.begin(), s.end(), s.begin(), ::tolower);
    if (s == "true" || s == "1" || s == "yes" || s == "on") return true;
    if (s == "false" || s == "0" || s == "no" || s == "off") return false;
    throw ConfigError("bad boolean '" + v + "'");
}

struct Config {
    std::string system = "honeycomb_kitaev";
    std::string mode;
    int64_t L[3] = {24, 24, 1};
    std::map<std::string, double> params;        // SpinConfig::get_param storage
    double field_strength = 0.0;
    std::vector<double> field_direction = {0.0, 1.0, 0.0};
    std::vector<double> g_factor = {1.0, 1.0, 1.0};
    int num_trials = 1;
    std::string output_dir = "output";
    std::string initial_spin_config;
    double spin_length = 1.0;
    double md_time_start = 0.0, md_time_end = 100.0, md_timestep = 0.01;
    int64_t md_save_interval = 1;
    std::string md_integrator = "dopri5";
    double md_abs_tol = 1e-6, md_rel_tol = 1e-6;
    bool md_adaptive = false, md_save_spins = true;
    double pump_amplitude = 1.0, pump_width = 10.0, pump_frequency = 0.0, pump_time = 0.0;
    std::vector<std::vector<double>> pump_directions = {{0.0, 1.0, 0.0}};
    std::vector<std::vector<double>> pump_directions_2;
    double tau_start = -200.0, tau_end = 200.0, tau_step = 1.0;
    bool reuse_m0_for_m1 = true;                 // W1: M1(tau) as a time shift of M0 when stationary
    double stationarity_tol = 1e-6;
    uint64_t seed = 0;
    bool cubic_cell = false;
    std::vector<std::string> ignored;

    double param(const std::string& k, double def) const {
        auto it = params.find(k);
        return it == params.end() ? def : it->second;
    }
};

std::string normalise_system(const std::string& v) {
    const std::string s = trim(v);
    if (s == "honeycomb_kitaev" || s == "HONEYCOMB_KITAEV" || s == "KITAEV") return "honeycomb_kitaev";
    if (s == "pyrochlore_non_kramer" || s == "PYROCHLORE_NON_KRAMER" || s == "non_kramer")
        return "pyrochlore_non_kramer";
    throw ConfigError("system '" + s + "' is not on this path (honeycomb_kitaev, pyrochlore_non_kramer)");
}

std::string normalise_mode(const std::string& v) {
    const std::string s = trim(v);
    if (s == "molecular_dynamics" || s == "MD" || s == "dynamics") return "molecular_dynamics";
    if (s == "pump_probe" || s == "PUMP_PROBE" || s == "pump-probe") return "pump_probe";
    if (s == "2dcs" || s == "2DCS" || s == "spectroscopy" || s == "pump_probe_spectroscopy") return "2dcs";
    throw ConfigError("simulation_mode '" + s + "' is not on this path (molecular_dynamics, pump_probe, 2dcs)");
}

// md_integrator names of the reference GPU integrator (integrator.cuh:91-452); "dopri5" is
// controlled (the CPU path's step control) under md_adaptive = true.  -1: not a method.
const char* const kMethodNames =
    "the GPU path (ssprk53, rk4, dopri5 / rk54 / rkf54, rk5 / rkck54, euler, rk2 / midpoint, rk78 / rkf78, "
    "bs / bulirsch_stoer; md_adaptive = true makes dopri5 step-controlled)";

int method_code(const std::string& m, bool adaptive) {
    if (m == "rk4") return CMD_RK4;
    if (m == "dopri5") return adaptive ? CMD_RK45 : CMD_DOPRI5_FIXED;
    if (m == "rk54" || m == "rkf54") return CMD_DOPRI5_FIXED;
    if (m == "rk5" || m == "rkck54") return CMD_CASH_KARP_FIXED;
    if (m == "ssprk53") return CMD_SSPRK53;
    if (m == "euler") return CMD_EULER;
    if (m == "rk2" || m == "midpoint") return CMD_MIDPOINT;
    if (m == "rk78" || m == "rkf78") return CMD_RK78;
    if (m == "bs" || m == "bulirsch_stoer") return CMD_BULIRSCH_STOER;
    return -1;
}

Config parse_file(const std::string& path) {
    std::ifstream f(path);
    if (!f) throw ConfigError("cannot open " + path);
    Config c;
    std::string line;
    int lineno = 0;
    while (std::getline(f, line)) {
        ++lineno;
        const size_t hash = line.find('#');
        if (hash != std::string::npos) line = line.substr(0, hash);
        line = trim(line);
        if (line.empty()) continue;
        const size_t eq = line.find('=');
        if (eq == std::string::npos) throw ConfigError(path + ":" + std::to_string(lineno) + ": expected key = value");
        const std::string k = trim(line.substr(0, eq)), v = trim(line.substr(eq + 1));
        try {
            if (k == "system") c.system = normalise_system(v);
            else if (k == "simulation_mode" || k == "simulation") c.mode = normalise_mode(v);
            else if (k == "lattice_size") {
                const std::vector<double> x = parse_vector(v);
                if (x.size() != 3) throw ConfigError("lattice_size needs 3 values");
                for (int i = 0; i < 3; ++i) c.L[i] = (int64_t)x[i];
            } else if (k == "field_strength" || k == "h") c.field_strength = std::stod(v);
            else if (k == "field_direction") c.field_direction = parse_vector(v);
            else if (k == "g_factor") c.g_factor = parse_vector(v);
            else if (k == "num_trials") c.num_trials = std::stoi(v);
            else if (k == "output_dir") c.output_dir = v;
            else if (k == "initial_spin_config") c.initial_spin_config = v;
            else if (k == "spin_length") c.spin_length = std::stod(v);
            else if (k == "md_time_start") c.md_time_start = std::stod(v);
            else if (k == "md_time_end") c.md_time_end = std::stod(v);
            else if (k == "md_timestep") c.md_timestep = std::stod(v);
            else if (k == "md_save_interval") c.md_save_interval = std::stoll(v);
            else if (k == "md_integrator") c.md_integrator = v;
            else if (k == "md_abs_tol") c.md_abs_tol = std::stod(v);
            else if (k == "md_rel_tol") c.md_rel_tol = std::stod(v);
            else if (k == "md_adaptive") c.md_adaptive = parse_bool(v);
            else if (k == "md_save_spins") c.md_save_spins = parse_bool(v);
            else if (k == "pump_amplitude") c.pump_amplitude = std::stod(v);
            else if (k == "pump_width") c.pump_width = std::stod(v);
            else if (k == "pump_frequency") c.pump_frequency = std::stod(v);
            else if (k == "pump_time") c.pump_time = std::stod(v);
            else if (k == "pump_direction" || k == "pump_directions") c.pump_directions = parse_vec3_list(v, "pump_direction");
            else if (k == "pump_direction_2" || k == "pump_directions_2") c.pump_directions_2 = parse_vec3_list(v, "pump_direction_2");
            else if (k == "tau_start") c.tau_start = std::stod(v);
            else if (k == "tau_end") c.tau_end = std::stod(v);
            else if (k == "tau_step") c.tau_step = std::stod(v);
            else if (k == "reuse_m0_for_m1") c.reuse_m0_for_m1 = parse_bool(v);
            else if (k == "stationarity_tol") c.stationarity_tol = std::stod(v);
            else if (k == "seed") c.seed = std::stoull(v);
            else if (k == "cubic_cell") c.cubic_cell = parse_bool(v);
            else {
                // Hamiltonian parameters (K, Gamma, Jzz, ...) and keys of other
                // modes: numbers go to the generic parameter map, like get_param.
                try {
                    size_t used = 0;
                    const double x = std::stod(v, &used);
                    if (trim(v.substr(used)).empty()) c.params[k] = x;
                    else c.ignored.push_back(k);
                } catch (const std::exception&) {
                    c.ignored.push_back(k);
                }
            }
        } catch (const ConfigError&) {
            throw;
        } catch (const std::exception& e) {
            throw ConfigError(path + ":" + std::to_string(lineno) + ": bad value for " + k + " (" + e.what() + ")");
        }
    }
    if (c.mode.empty()) throw ConfigError("simulation_mode is missing");
    if (c.field_direction.size() != 3 || c.g_factor.size() != 3)
        throw ConfigError("field_direction and g_factor need 3 values");
    if (!(c.md_timestep > 0.0)) throw ConfigError("md_timestep must be positive");
    if (c.md_save_interval < 1) throw ConfigError("md_save_interval must be >= 1");
    if (c.num_trials < 1) throw ConfigError("num_trials must be >= 1");
    if (c.mode != "2dcs" && method_code(c.md_integrator, c.md_adaptive) < 0)
        throw ConfigError("md_integrator '" + c.md_integrator + "' is not a method of " + kMethodNames);
    for (int i = 0; i < 3; ++i)
        if (c.L[i] < 1) throw ConfigError("lattice_size entries must be >= 1");
    return c;
}

// ---------------------------------------------------------------------------
// Output helpers.

void write_npy(const fs::path& p, const std::vector<double>& data, const std::vector<int64_t>& shape) {
    std::string hdr = "{'descr': '<f8', 'fortran_order': False, 'shape': (";
    for (size_t i = 0; i < shape.size(); ++i) hdr += std::to_string(shape[i]) + (shape.size() == 1 ? "," : (i + 1 < shape.size() ? ", " : ""));
    hdr += "), }";
    const size_t total = 10 + hdr.size() + 1;
    hdr += std::string((64 - total % 64) % 64, ' ') + "\n";
    std::ofstream f(p, std::ios::binary);
    if (!f) throw std::runtime_error("cannot write " + p.string());
    const unsigned char magic[8] = {0x93, 'N', 'U', 'M', 'P', 'Y', 1, 0};
    f.write((const char*)magic, 8);
    const uint16_t hl = (uint16_t)hdr.size();
    f.write((const char*)&hl, 2);
    f.write(hdr.data(), (std::streamsize)hdr.size());
    f.write((const char*)data.data(), (std::streamsize)(data.size() * sizeof(double)));
}

void save_spin_config(const fs::path& p, const std::vector<double>& s) {   // lattice.h:4687-4703
    std::ofstream f(p);
    f << std::scientific << std::setprecision(16);
    for (size_t i = 0; i < s.size() / 3; ++i) f << s[3 * i] << " " << s[3 * i + 1] << " " << s[3 * i + 2] << "\n";
}

std::vector<double> load_spin_config(const std::string& p, int64_t N) {      // lattice.h:4708-4739
    std::ifstream f(p);
    if (!f) throw ConfigError("cannot open initial_spin_config " + p);
    std::vector<double> s((size_t)N * 3);
    std::string line;
    int64_t i = 0;
    while (i < N && std::getline(f, line)) {
        std::istringstream is(line);
        if (!(is >> s[3 * i] >> s[3 * i + 1] >> s[3 * i + 2]))
            throw ConfigError("incomplete spin data at line " + std::to_string(i) + " of " + p);
        ++i;
    }
    if (i != N) throw ConfigError(p + " holds " + std::to_string(i) + " spins, expected " + std::to_string(N));
    return s;
}

struct Json {
    std::ostringstream o;
    bool first = true;
    Json() { o << "{"; }
    Json& num(const std::string& k, double v) {
        o << (first ? "" : ", ") << "\"" << k << "\": " << std::setprecision(17) << v;
        first = false;
        return *this;
    }
    Json& str(const std::string& k, const std::string& v) {
        o << (first ? "" : ", ") << "\"" << k << "\": \"" << v << "\"";
        first = false;
        return *this;
    }
    std::string done() { return o.str() + "}"; }
};

void check(int rc, const char* where) {
    if (rc != CMD_OK) throw std::runtime_error(std::string(where) + ": " + cmd_last_error());
}

// ---------------------------------------------------------------------------
// Lattice and state.

struct Model {
    cmd_lattice* L = nullptr;
    cmd_handle* h = nullptr;
    int64_t N = 0;
    int32_t na = 0;
    ~Model() {
        if (h) cmd_destroy(h);
        if (L) cmd_lattice_free(L);
    }
};

void build_model(const Config& c, Model& m) {
    if (c.system == "honeycomb_kitaev") {
        // build_kitaev_honeycomb (unitcell_builders.cpp:178-283) with its defaults
        const char* keys[11] = {"K", "Gamma", "Gammap", "J", "J2_A", "J2_B", "J3", "J_perp", "Ka", "Kb", "Kc"};
        const double defs[11] = {-1.0, 0.25, -0.02, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        double kp[11];
        for (int i = 0; i < 11; ++i) kp[i] = c.param(keys[i], defs[i]);
        check(cmd_lattice_kitaev(kp, c.field_strength, c.field_direction.data(), c.g_factor.data(), (int32_t)c.L[0],
                                 (int32_t)c.L[1], (int32_t)c.L[2], &m.L),
              "cmd_lattice_kitaev");
    } else {
        // build_pyrochlore_non_kramer (unitcell_builders.cpp:370-471) with its defaults
        const double pp[6] = {c.param("Jpm", 0.0), c.param("Jzz", 1.0), c.param("Jpmpm", 0.0),
                              c.param("J2", 0.0), c.param("delta1", 0.0), c.param("delta2", 0.0)};
        check(cmd_lattice_pyrochlore_nk(pp, c.field_strength, c.field_direction.data(), (int32_t)c.L[0],
                                        (int32_t)c.L[1], (int32_t)c.L[2], c.cubic_cell ? 1 : 0, &m.L),
              "cmd_lattice_pyrochlore_nk");
    }
    int32_t zb = 0, dims[3];
    check(cmd_lattice_sizes(m.L, &m.N, &m.na, &zb, dims), "cmd_lattice_sizes");
    cmd_lattice_desc d;
    check(cmd_lattice_desc_of(m.L, &d), "cmd_lattice_desc_of");
    check(cmd_create(&d, &m.h), "cmd_create");
}

std::vector<double> initial_state(const Config& c, const Model& m, int trial) {
    if (!c.initial_spin_config.empty()) return load_spin_config(c.initial_spin_config, m.N);
    std::vector<double> s((size_t)m.N * 3);
    check(cmd_lattice_random_spins(m.N, c.seed + (uint64_t)trial, c.spin_length, s.data()), "random spins");
    return s;
}

// Per-atom pulse directions, normalised (runners_lattice.cpp:419-431), one
// direction broadcast or one per sublattice (:433-443), then R * d per atom
// (Lattice::set_pulse, lattice_md.cpp:210-224).
std::vector<double> atom_dirs(const std::vector<std::vector<double>>& dirs, int32_t na) {
    if (dirs.size() != 1 && dirs.size() != (size_t)na)
        throw ConfigError("pump_direction must have 1 direction or exactly " + std::to_string(na) +
                          " (one per sublattice); got " + std::to_string(dirs.size()));
    std::vector<double> out((size_t)na * 3);
    for (int32_t a = 0; a < na; ++a) {
        const std::vector<double>& d = dirs[dirs.size() == 1 ? 0 : a];
        const double n = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        for (int k = 0; k < 3; ++k) out[3 * a + k] = n > 1e-10 ? d[k] / n : d[k];
    }
    return out;
}

int method_of(const Config& c) {
    const int m = method_code(c.md_integrator, c.md_adaptive);
    if (m < 0) throw ConfigError("md_integrator '" + c.md_integrator + "' is not a method of " + kMethodNames);
    return m;
}

struct Rows {
    std::vector<double> times, obs, states;
    int64_t n = 0;
};

Rows integrate(const Config& c, const Model& m, double T0, double T1, double dt, int64_t save, int method,
               bool states) {
    Rows r;
    int64_t need = 0;
    if (method == CMD_RK45) {
        check(cmd_set_tolerances(m.h, c.md_abs_tol, c.md_rel_tol, 0), "cmd_set_tolerances");
        cmd_integrate(m.h, T0, T1, dt, save, method, nullptr, nullptr, nullptr, 0, &need);   // size query
        // the query runs nothing but reports the bound; run against it
        std::vector<double> st0((size_t)m.N * 3);
        check(cmd_get_spins(m.h, st0.data(), m.N * 3), "cmd_get_spins");
        for (int attempt = 0; attempt < 2; ++attempt) {
            r.times.assign((size_t)need, 0.0);
            r.obs.assign((size_t)need * 10, 0.0);
            if (states) r.states.assign((size_t)need * m.N * 3, 0.0);
            int64_t got = 0;
            const int rc = cmd_integrate(m.h, T0, T1, dt, save, method, r.times.data(), r.obs.data(),
                                         states ? r.states.data() : nullptr, need, &got);
            if (rc == CMD_OK) {
                r.n = got;
                break;
            }
            if (got <= need) check(rc, "cmd_integrate");
            need = got;
            check(cmd_set_spins(m.h, st0.data(), m.N * 3), "cmd_set_spins");
        }
    } else {
        cmd_integrate(m.h, T0, T1, dt, save, method, nullptr, nullptr, nullptr, 0, &need);
        r.times.assign((size_t)need, 0.0);
        r.obs.assign((size_t)need * 10, 0.0);
        if (states) r.states.assign((size_t)need * m.N * 3, 0.0);
        check(cmd_integrate(m.h, T0, T1, dt, save, method, r.times.data(), r.obs.data(),
                            states ? r.states.data() : nullptr, need, &r.n),
              "cmd_integrate");
    }
    r.times.resize((size_t)r.n);
    r.obs.resize((size_t)r.n * 10);
    if (states) r.states.resize((size_t)r.n * m.N * 3);
    return r;
}

std::vector<double> column3(const std::vector<double>& obs, int64_t n, int off) {
    std::vector<double> out((size_t)n * 3);
    for (int64_t i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) out[3 * i + k] = obs[10 * i + off + k];
    return out;
}

// ---------------------------------------------------------------------------
// Runners.

void run_md(const Config& c, Model& m) {
    const int method = method_of(c);
    for (int trial = 0; trial < c.num_trials; ++trial) {
        const fs::path dir = fs::path(c.output_dir) / ("sample_" + std::to_string(trial));
        fs::create_directories(dir);
        const std::vector<double> s0 = initial_state(c, m, trial);
        save_spin_config(dir / "initial_spins.txt", s0);
        check(cmd_set_spins(m.h, s0.data(), m.N * 3), "cmd_set_spins");
        const Rows r = integrate(c, m, c.md_time_start, c.md_time_end, c.md_timestep, c.md_save_interval, method,
                                 c.md_save_spins);
        write_npy(dir / "trajectory_times.npy", r.times, {r.n});
        write_npy(dir / "trajectory_magnetization_antiferro.npy", column3(r.obs, r.n, 0), {r.n, 3});
        write_npy(dir / "trajectory_magnetization_local.npy", column3(r.obs, r.n, 3), {r.n, 3});
        write_npy(dir / "trajectory_magnetization_global.npy", column3(r.obs, r.n, 6), {r.n, 3});
        std::vector<double> e((size_t)r.n);
        for (int64_t i = 0; i < r.n; ++i) e[i] = r.obs[10 * i + 9];
        write_npy(dir / "trajectory_energy_per_site.npy", e, {r.n});
        if (c.md_save_spins) write_npy(dir / "trajectory_spins.npy", r.states, {r.n, m.N, 3});
        std::ofstream(dir / "metadata.json")
            << Json().str("simulation_mode", c.mode).str("system", c.system).num("lattice_size", (double)m.N)
                   .num("spin_dim", 3).num("N_atoms", m.na).num("dim1", c.L[0]).num("dim2", c.L[1])
                   .num("dim3", c.L[2]).num("T_start", c.md_time_start).num("T_end", c.md_time_end)
                   .num("T_step", c.md_timestep).num("save_interval", (double)c.md_save_interval)
                   .str("integration_method", c.md_integrator).num("rows", (double)r.n).done()
            << "\n";
        std::cout << "[trial " << trial << "] " << r.n << " rows -> " << dir.string() << "\n";
    }
}

void run_pump_probe(const Config& c, Model& m) {
    const int method = method_of(c);
    const std::vector<double> d = atom_dirs(c.pump_directions, m.na);
    const std::vector<double> zero(d.size(), 0.0);
    std::vector<double> fd(2 * d.size());
    check(cmd_lattice_rotate_pulse(m.L, d.data(), zero.data(), fd.data()), "cmd_lattice_rotate_pulse");
    for (int trial = 0; trial < c.num_trials; ++trial) {
        const fs::path dir = fs::path(c.output_dir) / ("sample_" + std::to_string(trial));
        fs::create_directories(dir);
        const std::vector<double> s0 = initial_state(c, m, trial);
        save_spin_config(dir / "initial_spins.txt", s0);
        check(cmd_set_spins(m.h, s0.data(), m.N * 3), "cmd_set_spins");
        // single_pulse_drive_gpu (lattice.h:5860-5903): one pulse at pump_time, second field zero
        check(cmd_set_pulse(m.h, fd.data(), c.pump_amplitude, c.pump_width, c.pump_frequency, c.pump_time, 0.0),
              "cmd_set_pulse");
        const Rows r = integrate(c, m, c.md_time_start, c.md_time_end, c.md_timestep, 1, method, false);
        std::ofstream f(dir / "pump_probe_trajectory.txt");               // runners_lattice.cpp:553-560
        f << std::setprecision(17);
        for (int64_t i = 0; i < r.n; ++i) {
            f << r.times[i];
            for (int k = 0; k < 9; ++k) f << " " << r.obs[10 * i + k];
            f << "\n";
        }
        std::cout << "[trial " << trial << "] " << r.n << " rows -> " << (dir / "pump_probe_trajectory.txt").string()
                  << "\n";
    }
}

void run_2dcs(const Config& c, Model& m) {
    if (c.md_integrator != "rk4")
        std::cout << "note: the batched 2DCS path integrates with rk4 (as integrate_gpu_batched does, "
                     "lattice_gpu.cu:781-784)\n";
    // tau grid (lattice.h:5642-5646)
    const int64_t n_tau = (int64_t)std::abs((c.tau_end - c.tau_start) / c.tau_step) + 1;
    std::vector<double> tau((size_t)n_tau);
    for (int64_t i = 0; i < n_tau; ++i) tau[i] = c.tau_start + (double)i * c.tau_step;
    // time grid of the batched loop: t = T0; while (t < T1 - 1e-12) t += dt (lattice_gpu.cu:557)
    std::vector<double> grid{c.md_time_start};
    double t = c.md_time_start;
    while (t < c.md_time_end - 1e-12) {
        t += c.md_timestep;
        grid.push_back(t);
    }
    const int64_t n_steps = (int64_t)grid.size() - 1, n_t = n_steps + 1;
    const std::vector<double> d1 = atom_dirs(c.pump_directions, m.na);
    const std::vector<double> d2 = c.pump_directions_2.empty() ? d1 : atom_dirs(c.pump_directions_2, m.na);
    std::vector<double> fd(2 * d1.size());
    check(cmd_lattice_rotate_pulse(m.L, d1.data(), d2.data(), fd.data()), "cmd_lattice_rotate_pulse");
    const fs::path dir = fs::path(c.output_dir) / "sample_0";
    fs::create_directories(dir);
    const std::vector<double> s0 = initial_state(c, m, 0);
    save_spin_config(dir / "initial_spins.txt", s0);
    check(cmd_set_spins(m.h, s0.data(), m.N * 3), "cmd_set_spins");
    double e_ground = 0.0;
    check(cmd_energy(m.h, &e_ground), "cmd_energy");
    // W1 guard (lattice.h:5654-5676): a stationary ground state lets M1(tau)
    // be M0 shifted in time; otherwise M1 is integrated (probe-only runs).
    double max_ds = 0.0;
    check(cmd_max_dsdt_no_drive(m.h, &max_ds), "cmd_max_dsdt_no_drive");
    const bool synth = c.reuse_m0_for_m1 && max_ds <= c.stationarity_tol;
    std::cout << "2dcs: max |dS/dt| without drive = " << max_ds << (synth ? " (stationary: M1 = shifted M0)\n"
                                                                           : " (M1 integrated)\n");
    const int64_t B = synth ? 1 + n_tau : 1 + 2 * n_tau;
    // trajectories: 0 = M0 (pump at 0); synthesised: 1 + k = M01(tau_k); else
    // 1 + 2k = M1(tau_k) (probe at tau_k), 2 + 2k = M01(tau_k)
    std::vector<double> t1((size_t)B, 0.0), t2((size_t)B, 0.0), a1((size_t)B, 0.0), a2((size_t)B, 0.0);
    a1[0] = c.pump_amplitude;
    for (int64_t k = 0; k < n_tau; ++k) {
        const int64_t i01 = synth ? 1 + k : 2 + 2 * k;
        if (!synth) {
            t2[1 + 2 * k] = tau[k];
            a2[1 + 2 * k] = c.pump_amplitude;
        }
        t2[i01] = tau[k];
        a1[i01] = c.pump_amplitude;
        a2[i01] = c.pump_amplitude;
    }
    std::vector<double> obs((size_t)B * n_t * 10);
    cmd_batch_desc bd;
    std::memset(&bd, 0, sizeof(bd));
    bd.B = B;
    bd.states = s0.data();
    bd.shared_initial = 1;
    bd.method = CMD_RK4;
    bd.t1 = t1.data();
    bd.t2 = t2.data();
    bd.a1 = a1.data();
    bd.a2 = a2.data();
    bd.d1 = fd.data();
    bd.d2 = fd.data() + 3 * m.na;
    bd.width = c.pump_width;
    bd.freq = c.pump_frequency;
    bd.T0 = c.md_time_start;
    bd.dt = c.md_timestep;
    bd.n_steps = n_steps;
    bd.save_interval = 1;
    bd.obs = obs.data();
    check(cmd_run_batch(m.h, &bd), "cmd_run_batch");
    // ground-state magnetisations (lattice.h:5649-5652): M_antiferro in the
    // (-1)^i convention of magnetization_local_antiferro, M_local, M_global
    double m_ground[9], row[10], ml[3], ms[3];
    check(cmd_observables(m.h, row), "cmd_observables");
    check(cmd_magnetization(m.h, ml, ms), "cmd_magnetization");
    for (int d = 0; d < 3; ++d) {
        m_ground[d] = ms[d];
        m_ground[3 + d] = row[3 + d];
        m_ground[6 + d] = row[6 + d];
    }
    // datasets of pump_probe_spectroscopy.h5 (lattice.h:5749-5851)
    auto traj = [&](int64_t b, int off, double* out) {
        for (int64_t i = 0; i < n_t; ++i)
            for (int k = 0; k < 3; ++k) out[3 * i + k] = obs[((size_t)b * n_t + i) * 10 + off + k];
    };
    const char* names[3] = {"antiferro", "local", "global"};
    write_npy(dir / "reference_times.npy", grid, {n_t});
    std::vector<double> M0[3], M1[3], M01[3];
    for (int q = 0; q < 3; ++q) {
        M0[q].assign((size_t)n_t * 3, 0.0);
        traj(0, 3 * q, M0[q].data());
        M1[q].assign((size_t)n_tau * n_t * 3, 0.0);
        M01[q].assign((size_t)n_tau * n_t * 3, 0.0);
        for (int64_t k = 0; k < n_tau; ++k) {
            traj(synth ? 1 + k : 2 + 2 * k, 3 * q, &M01[q][(size_t)k * n_t * 3]);
            if (!synth) {
                traj(1 + 2 * k, 3 * q, &M1[q][(size_t)k * n_t * 3]);
                continue;
            }
            // synthesize_M1_from_M0 (lattice_md.cpp:283-317): the ground state's
            // magnetisation before tau, M0(t - tau) (nearest grid index) after
            for (int64_t i = 0; i < n_t; ++i) {
                double* dst = &M1[q][((size_t)k * n_t + i) * 3];
                if (grid[i] < tau[k] + grid[0]) {
                    for (int d = 0; d < 3; ++d) dst[d] = m_ground[3 * q + d];
                } else {
                    int64_t idx = (int64_t)std::llround((grid[i] - tau[k] - grid[0]) / c.md_timestep);
                    idx = std::max<int64_t>(0, std::min<int64_t>(n_t - 1, idx));
                    for (int d = 0; d < 3; ++d) dst[d] = M0[q][3 * idx + d];
                }
            }
        }
        write_npy(dir / (std::string("reference_M_") + names[q] + ".npy"), M0[q], {n_t, 3});
        write_npy(dir / (std::string("tau_scan_M1_") + names[q] + ".npy"), M1[q], {n_tau, n_t, 3});
        write_npy(dir / (std::string("tau_scan_M01_") + names[q] + ".npy"), M01[q], {n_tau, n_t, 3});
    }
    write_npy(dir / "tau_scan_tau_values.npy", tau, {n_tau});
    // analysis step on M_local (reader_honeycomb.py:459-553)
    std::vector<double> nl((size_t)3 * n_tau * n_t), sp((size_t)3 * n_tau * n_t);
    for (int comp = 0; comp < 3; ++comp)
        check(cmd_nonlinear_spectrum(M0[1].data(), M1[1].data(), M01[1].data(), n_tau, n_t, comp,
                                     &nl[(size_t)comp * n_tau * n_t], &sp[(size_t)comp * n_tau * n_t]),
              "cmd_nonlinear_spectrum");
    write_npy(dir / "M_NL_local.npy", nl, {3, n_tau, n_t});
    write_npy(dir / "spectrum_local.npy", sp, {3, n_tau, n_t});
    std::ofstream(dir / "metadata.json")
        << Json().str("simulation_mode", c.mode).str("system", c.system).num("lattice_size", (double)m.N)
               .num("spin_dim", 3).num("N_atoms", m.na).num("dim1", c.L[0]).num("dim2", c.L[1]).num("dim3", c.L[2])
               .num("pulse_amp", c.pump_amplitude)
               .num("pulse_width", c.pump_width).num("pulse_freq", c.pump_frequency).num("T_start", c.md_time_start)
               .num("T_end", c.md_time_end).num("T_step", c.md_timestep).num("tau_start", c.tau_start)
               .num("tau_end", c.tau_end).num("tau_step", c.tau_step).num("tau_steps", (double)n_tau)
               .num("ground_state_energy", e_ground / (double)m.N).str("integration_method", "rk4")
               .num("max_dsdt_no_drive", max_ds).num("stationarity_tol", c.stationarity_tol)
               .num("m1_synthesized", synth ? 1 : 0)
               .done()
        << "\n";
    std::cout << "2dcs: " << n_tau << " delays x " << n_t << " times (" << B << " trajectories) -> " << dir.string()
              << "\n";
}

void print_config(const Config& c) {
    Json j;
    j.str("system", c.system).str("simulation_mode", c.mode);
    j.num("L0", (double)c.L[0]).num("L1", (double)c.L[1]).num("L2", (double)c.L[2]);
    j.num("field_strength", c.field_strength).num("num_trials", c.num_trials).str("output_dir", c.output_dir);
    j.str("initial_spin_config", c.initial_spin_config).num("md_time_start", c.md_time_start);
    j.num("md_time_end", c.md_time_end).num("md_timestep", c.md_timestep);
    j.num("md_save_interval", (double)c.md_save_interval).str("md_integrator", c.md_integrator);
    j.num("pump_amplitude", c.pump_amplitude).num("pump_width", c.pump_width);
    j.num("pump_frequency", c.pump_frequency).num("pump_time", c.pump_time);
    j.num("n_pump_directions", (double)c.pump_directions.size());
    j.num("tau_start", c.tau_start).num("tau_end", c.tau_end).num("tau_step", c.tau_step);
    j.num("seed", (double)c.seed).num("cubic_cell", c.cubic_cell ? 1 : 0);
    for (const auto& kv : c.params) j.num("param:" + kv.first, kv.second);
    std::string ign;
    for (const auto& k : c.ignored) ign += (ign.empty() ? "" : ",") + k;
    j.str("ignored", ign);
    std::cout << j.done() << "\n";
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2) {
        std::cerr << "usage: " << argv[0] << " <file.param> [--parse-only]\n";
        return 1;
    }
    Config c;
    try {
        c = parse_file(argv[1]);
    } catch (const std::exception& e) {
        std::cerr << "config error: " << e.what() << "\n";
        return 1;
    }
    if (argc > 2 && std::string(argv[2]) == "--parse-only") {
        print_config(c);
        return 0;
    }
    try {
        Model m;
        build_model(c, m);
        std::cout << c.system << " " << c.L[0] << "x" << c.L[1] << "x" << c.L[2] << ": " << m.N << " spins, mode "
                  << c.mode << "\n";
        if (c.mode == "molecular_dynamics") run_md(c, m);
        else if (c.mode == "pump_probe") run_pump_probe(c, m);
        else run_2dcs(c, m);
    } catch (const ConfigError& e) {
        std::cerr << "config error: " << e.what() << "\n";
        return 1;
    } catch (const std::exception& e) {
        std::cerr << "error: " << e.what() << "\n";
        return 2;
    }
    return 0;
}
