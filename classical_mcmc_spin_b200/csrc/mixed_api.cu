// mixed_api.cu -- C ABI of the mixed SU(2) / SU(3) path (cmd_mixed.h): the
// handle owns the device copies of the lattice tables, the state and the
// integrator workspace; every call runs on the handle's stream.
#include "cmd.h"
#include "cmd_mixed.h"
#include "cmd_internal.h"
#include "mixed.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

using cmd::fail;

namespace {

#define MIX_TRY(x)                                                                               \
    do {                                                                                         \
        cudaError_t e_ = (x);                                                                    \
        if (e_ != cudaSuccess) return fail(CMD_ERR_CUDA, std::string(#x ": ") + cudaGetErrorString(e_)); \
    } while (0)

struct Buf {
    void* p = nullptr;
    size_t bytes = 0;
    int ensure(size_t n) {
        if (n <= bytes) return CMD_OK;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        if (cudaMalloc(&p, std::max<size_t>(n, 8)) != cudaSuccess) {
            p = nullptr;
            return fail(CMD_ERR_OOM, "cudaMalloc failed for the mixed lattice");
        }
        bytes = n;
        return CMD_OK;
    }
    template <class T>
    T* as() const { return static_cast<T*>(p); }
    ~Buf() { if (p) cudaFree(p); }
};

}  // namespace

struct cmd_mixed {
    cmd::MixedDev m{};
    int64_t V = 0;
    Buf tables;                // all coupling tables, one allocation
    Buf drive2, drive3;
    Buf state, work, rows, mag;
    bool has_state = false;
    cudaStream_t stream = nullptr;
};

namespace {

int upload(cmd_mixed* h, const void* src, size_t bytes, char*& cursor) {
    if (bytes) MIX_TRY(cudaMemcpyAsync(cursor, src, bytes, cudaMemcpyHostToDevice, h->stream));
    cursor += (bytes + 255) / 256 * 256;
    return CMD_OK;
}

size_t pad(size_t bytes) { return (bytes + 255) / 256 * 256; }

// Partner tables as int32, -1 where the partner lies outside [0, limit).
std::vector<int> partners(const int64_t* p, size_t n, int64_t limit) {
    std::vector<int> out(n, -1);
    for (size_t i = 0; i < n; ++i)
        if (p && p[i] >= 0 && p[i] < limit) out[i] = (int)p[i];
    return out;
}
std::vector<int> counts(const int64_t* c, size_t n) {
    std::vector<int> out(n, 0);
    for (size_t i = 0; i < n; ++i) out[i] = c ? (int)std::max<int64_t>(0, std::min<int64_t>(c[i], 1 << 30)) : 0;
    return out;
}

int method_mode(int method) {
    switch (method) {
        case CMD_RK4: return cmd::kModeRK4;
        case CMD_DOPRI5_FIXED: return cmd::kModeDopri5Fixed;
        case CMD_CASH_KARP_FIXED: return cmd::kModeCashKarpFixed;
        case CMD_EULER: return cmd::kModeEuler;
        case CMD_MIDPOINT: return cmd::kModeMidpoint;
        case CMD_SSPRK53: return cmd::kModeSSPRK53;
        case CMD_RK78: return cmd::kModeRK78;
        case CMD_BULIRSCH_STOER: return cmd::kModeBulirschStoer;
        default: return -1;
    }
}

// Reference loop (integrator.cuh:470-488): steps taken and the times of the saved rows.
int64_t loop_steps(double T0, double T1, double dt, std::vector<double>* grid) {
    int64_t n = 0;
    double t = T0;
    if (grid) grid->clear();
    while (t < T1) {
        if (grid) grid->push_back(t);
        t += dt;
        ++n;
    }
    if (grid) grid->push_back(t);
    return n;
}

template <int CS>
int launch_cs(cmd_mixed* h, const cmd::MixedRun& r, int threads) {
    auto kern = cmd::mixed_integrate_kernel<CS>;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(CS);
    cfg.blockDim = dim3((unsigned)threads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = h->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = CS;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    MIX_TRY(cudaLaunchKernelEx(&cfg, kern, h->m, r));
    return CMD_OK;
}

// One persistent launch over a cluster sized to the lattice: one site per thread up
// to 8 CTAs of kMixedThreads, the threads loop beyond that.
int run(cmd_mixed* h, int method, double T0, double dt, int64_t n_steps, int64_t save_every, int64_t max_rows) {
    const int mode = method_mode(method);
    if (mode < 0) return fail(CMD_ERR_INVALID_ARG, "the mixed path takes a fixed-step method (any CMD_* but CMD_RK45)");
    if (int rc = h->work.ensure((size_t)11 * h->V * sizeof(double))) return rc;
    if (max_rows > 0)
        if (int rc = h->rows.ensure((size_t)max_rows * h->V * sizeof(double))) return rc;
    cmd::MixedRun r{};
    r.work = h->work.as<double>();
    r.y0 = h->state.as<double>();
    r.y_out = h->state.as<double>();
    r.rows = max_rows > 0 ? h->rows.as<double>() : nullptr;
    r.max_rows = max_rows;
    r.T0 = T0;
    r.dt = dt;
    r.n_steps = n_steps;
    r.save_every = save_every;
    r.mode = mode;
    const int64_t sites = (int64_t)h->m.N2 + h->m.N3;
    const int64_t per = (sites + cmd::kMixedThreads - 1) / cmd::kMixedThreads;
    const int cs = per <= 1 ? 1 : per <= 2 ? 2 : per <= 4 ? 4 : 8;
    const int threads = (int)std::min<int64_t>(cmd::kMixedThreads, std::max<int64_t>(32, ((sites + cs - 1) / cs + 31) / 32 * 32));
    int rc = cs == 1 ? launch_cs<1>(h, r, threads)
           : cs == 2 ? launch_cs<2>(h, r, threads)
           : cs == 4 ? launch_cs<4>(h, r, threads)
                     : launch_cs<8>(h, r, threads);
    if (rc) return rc;
    MIX_TRY(cudaGetLastError());
    return CMD_OK;
}

int check(cmd_mixed* h, bool need_state) {
    if (!h) return fail(CMD_ERR_INVALID_ARG, "NULL handle");
    if (need_state && !h->has_state) return fail(CMD_ERR_STATE, "spins not set (call cmd_mixed_set_spins first)");
    return CMD_OK;
}

}  // namespace

extern "C" {

int cmd_mixed_create(const cmd_mixed_desc* d, cmd_mixed** out) {
    cmd::clear_error();
    if (!d || !out) return fail(CMD_ERR_INVALID_ARG, "NULL argument");
    *out = nullptr;
    if (d->spin_dim_su2 != 3 || d->spin_dim_su3 != 8)
        return fail(CMD_ERR_INVALID_ARG, "spin dimensions must be 3 (SU(2)) and 8 (SU(3))");
    if (d->n_su2 < 0 || d->n_su3 < 0 || d->n_su2 + d->n_su3 <= 0 || d->n_su2 + d->n_su3 >= (1LL << 30))
        return fail(CMD_ERR_INVALID_ARG, "bad site counts");
    if ((d->n_su2 > 0 && d->n_atoms_su2 <= 0) || (d->n_su3 > 0 && d->n_atoms_su3 <= 0))
        return fail(CMD_ERR_INVALID_ARG, "n_atoms must be positive for a non-empty sublattice");
    if (d->max_bilinear_su2 < 0 || d->max_bilinear_su3 < 0 || d->max_mixed_su2 < 0 || d->max_mixed_su3 < 0)
        return fail(CMD_ERR_INVALID_ARG, "negative ELL width");
    const int64_t N2 = d->n_su2, N3 = d->n_su3;
    const int z2 = d->max_bilinear_su2, z3 = d->max_bilinear_su3, zm2 = d->max_mixed_su2, zm3 = d->max_mixed_su3;
    auto need = [](const void* p, int64_t n) { return n == 0 || p != nullptr; };
    if (!need(d->field_su2, N2) || !need(d->onsite_su2, N2) || !need(d->counts_su2, N2) ||
        !need(d->field_su3, N3) || !need(d->onsite_su3, N3) || !need(d->counts_su3, N3) ||
        !need(d->bilinear_su2, N2 * z2) || !need(d->partners_su2, N2 * z2) || !need(d->bilinear_su3, N3 * z3) ||
        !need(d->partners_su3, N3 * z3) || !need(d->mixed_su2, N2 * zm2) || !need(d->mixed_partners_su3, N2 * zm2) ||
        !need(d->mixed_counts_su2, N2 * (zm2 > 0)) || !need(d->mixed_su3, N3 * zm3) ||
        !need(d->mixed_partners_su2, N3 * zm3) || !need(d->mixed_counts_su3, N3 * (zm3 > 0)))
        return fail(CMD_ERR_INVALID_ARG, "missing table");
    cmd_mixed* h = new cmd_mixed;
    auto bail = [&](int rc) {
        if (h->stream) cudaStreamDestroy(h->stream);
        delete h;
        return rc;
    };
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(fail(CMD_ERR_CUDA, "no CUDA device (cudaStreamCreate failed)"));
    const std::vector<int> p2 = partners(d->partners_su2, (size_t)(N2 * z2), N2), c2 = counts(d->counts_su2, N2);
    const std::vector<int> p3 = partners(d->partners_su3, (size_t)(N3 * z3), N3), c3 = counts(d->counts_su3, N3);
    const std::vector<int> mp2 = partners(d->mixed_partners_su3, (size_t)(N2 * zm2), N3);
    const std::vector<int> mc2 = counts(zm2 > 0 ? d->mixed_counts_su2 : nullptr, N2);
    const std::vector<int> mp3 = partners(d->mixed_partners_su2, (size_t)(N3 * zm3), N2);
    const std::vector<int> mc3 = counts(zm3 > 0 ? d->mixed_counts_su3 : nullptr, N3);
    const size_t b_f2 = N2 * 3 * 8, b_o2 = N2 * 9 * 8, b_j2 = N2 * z2 * 9 * 8, b_m2 = N2 * zm2 * 24 * 8;
    const size_t b_f3 = N3 * 8 * 8, b_o3 = N3 * 64 * 8, b_j3 = N3 * z3 * 64 * 8, b_m3 = N3 * zm3 * 24 * 8;
    const size_t total = pad(b_f2) + pad(b_o2) + pad(b_j2) + pad(b_m2) + pad(b_f3) + pad(b_o3) + pad(b_j3) +
                         pad(b_m3) + pad(p2.size() * 4) + pad(c2.size() * 4) + pad(mp2.size() * 4) +
                         pad(mc2.size() * 4) + pad(p3.size() * 4) + pad(c3.size() * 4) + pad(mp3.size() * 4) +
                         pad(mc3.size() * 4);
    if (int rc = h->tables.ensure(total)) return bail(rc);
    char* cur = h->tables.as<char>();
    cmd::MixedDev& m = h->m;
    m.N2 = (int)N2; m.N3 = (int)N3;
    m.NA2 = std::max(1, d->n_atoms_su2); m.NA3 = std::max(1, d->n_atoms_su3);
    m.z2 = z2; m.z3 = z3; m.zm2 = zm2; m.zm3 = zm3;
    int rc = CMD_OK;
    auto put = [&](const void* src, size_t bytes) {
        char* at = cur;
        if (rc == CMD_OK) rc = upload(h, src, bytes, cur);
        return at;
    };
    m.field2 = (const double*)put(d->field_su2, b_f2);
    m.onsite2 = (const double*)put(d->onsite_su2, b_o2);
    m.bil2 = (const double*)put(d->bilinear_su2, b_j2);
    m.mix2 = (const double*)put(d->mixed_su2, b_m2);
    m.field3 = (const double*)put(d->field_su3, b_f3);
    m.onsite3 = (const double*)put(d->onsite_su3, b_o3);
    m.bil3 = (const double*)put(d->bilinear_su3, b_j3);
    m.mix3 = (const double*)put(d->mixed_su3, b_m3);
    m.part2 = (const int*)put(p2.data(), p2.size() * 4);
    m.cnt2 = (const int*)put(c2.data(), c2.size() * 4);
    m.mpart2 = (const int*)put(mp2.data(), mp2.size() * 4);
    m.mcnt2 = (const int*)put(mc2.data(), mc2.size() * 4);
    m.part3 = (const int*)put(p3.data(), p3.size() * 4);
    m.cnt3 = (const int*)put(c3.data(), c3.size() * 4);
    m.mpart3 = (const int*)put(mp3.data(), mp3.size() * 4);
    m.mcnt3 = (const int*)put(mc3.data(), mc3.size() * 4);
    if (rc) return bail(rc);
    // drives start at zero, width 1 (the reference's defaults)
    const size_t bd2 = 2 * (size_t)m.NA2 * 3 * 8, bd3 = 2 * (size_t)m.NA3 * 8 * 8;
    if ((rc = h->drive2.ensure(bd2)) || (rc = h->drive3.ensure(bd3))) return bail(rc);
    if (cudaMemsetAsync(h->drive2.p, 0, bd2, h->stream) != cudaSuccess ||
        cudaMemsetAsync(h->drive3.p, 0, bd3, h->stream) != cudaSuccess)
        return bail(fail(CMD_ERR_CUDA, "cudaMemsetAsync failed"));
    m.drive2 = h->drive2.as<double>();
    m.drive3 = h->drive3.as<double>();
    m.width2 = m.width3 = 1.0;
    h->V = 3 * N2 + 8 * N3;
    if ((rc = h->state.ensure((size_t)h->V * sizeof(double)))) return bail(rc);
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) return bail(fail(CMD_ERR_CUDA, "upload failed"));
    *out = h;
    return CMD_OK;
}

int cmd_mixed_destroy(cmd_mixed* h) {
    cmd::clear_error();
    if (!h) return CMD_OK;
    cudaStreamSynchronize(h->stream);
    cudaStreamDestroy(h->stream);
    delete h;
    return CMD_OK;
}

int cmd_mixed_set_pulse(cmd_mixed* h, int32_t sub, const double* fd, double amp, double width, double freq,
                        double t1, double t2) {
    cmd::clear_error();
    if (int rc = check(h, false)) return rc;
    if (sub != 2 && sub != 3) return fail(CMD_ERR_INVALID_ARG, "sublattice must be 2 (SU(2)) or 3 (SU(3))");
    if (!fd) return fail(CMD_ERR_INVALID_ARG, "NULL field_drive");
    if (!std::isfinite(amp) || !std::isfinite(width) || !std::isfinite(freq) || !std::isfinite(t1) || !std::isfinite(t2))
        return fail(CMD_ERR_INVALID_ARG, "non-finite pulse parameter");
    cmd::MixedDev& m = h->m;
    const size_t n = sub == 2 ? 2 * (size_t)m.NA2 * 3 : 2 * (size_t)m.NA3 * 8;
    MIX_TRY(cudaMemcpyAsync(sub == 2 ? h->drive2.p : h->drive3.p, fd, n * sizeof(double), cudaMemcpyHostToDevice,
                            h->stream));
    MIX_TRY(cudaStreamSynchronize(h->stream));
    if (sub == 2) { m.amp2 = amp; m.width2 = width; m.freq2 = freq; m.t1_2 = t1; m.t2_2 = t2; }
    else { m.amp3 = amp; m.width3 = width; m.freq3 = freq; m.t1_3 = t1; m.t2_3 = t2; }
    return CMD_OK;
}

int cmd_mixed_set_spins(cmd_mixed* h, const double* s, int64_t n) {
    cmd::clear_error();
    if (int rc = check(h, false)) return rc;
    if (!s || n != h->V) return fail(CMD_ERR_INVALID_ARG, "spins must hold n_su2*3 + n_su3*8 values");
    for (int64_t i = 0; i < n; ++i)
        if (!std::isfinite(s[i])) return fail(CMD_ERR_NONFINITE, "non-finite spin component");
    MIX_TRY(cudaMemcpyAsync(h->state.p, s, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    MIX_TRY(cudaStreamSynchronize(h->stream));
    h->has_state = true;
    return CMD_OK;
}

int cmd_mixed_get_spins(cmd_mixed* h, double* s, int64_t n) {
    cmd::clear_error();
    if (int rc = check(h, true)) return rc;
    if (!s || n != h->V) return fail(CMD_ERR_INVALID_ARG, "spins must hold n_su2*3 + n_su3*8 values");
    MIX_TRY(cudaMemcpyAsync(s, h->state.p, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    MIX_TRY(cudaStreamSynchronize(h->stream));
    return CMD_OK;
}

int cmd_mixed_step(cmd_mixed* h, double t, double dt, int method) {
    cmd::clear_error();
    if (int rc = check(h, true)) return rc;
    if (!std::isfinite(t) || !std::isfinite(dt)) return fail(CMD_ERR_INVALID_ARG, "non-finite t or dt");
    if (int rc = run(h, method, t, dt, 1, 1, 0)) return rc;
    MIX_TRY(cudaStreamSynchronize(h->stream));
    return CMD_OK;
}

int cmd_mixed_integrate(cmd_mixed* h, double T0, double T1, double dt, int64_t save_interval, int method,
                        double* times, double* states, int64_t max_rows, int64_t* rows_out) {
    cmd::clear_error();
    if (int rc = check(h, true)) return rc;
    if (save_interval <= 0 || !(dt > 0.0) || !std::isfinite(T0) || !std::isfinite(T1))
        return fail(CMD_ERR_INVALID_ARG, "bad integration window");
    if (method_mode(method) < 0)
        return fail(CMD_ERR_INVALID_ARG, "the mixed path takes a fixed-step method (any CMD_* but CMD_RK45)");
    std::vector<double> grid;
    const int64_t n = loop_steps(T0, T1, dt, &grid);
    const int64_t rows = (n + save_interval - 1) / save_interval + 1;
    if (rows_out) *rows_out = rows;
    if (max_rows < rows) return fail(CMD_ERR_INVALID_ARG, "max_rows too small");
    if (int rc = run(h, method, T0, dt, n, save_interval, states ? rows : 0)) return rc;
    if (states)
        MIX_TRY(cudaMemcpyAsync(states, h->rows.p, (size_t)rows * h->V * sizeof(double), cudaMemcpyDeviceToHost,
                                h->stream));
    MIX_TRY(cudaStreamSynchronize(h->stream));
    if (times) {
        int64_t r = 0;
        for (int64_t k = 0; k < n; k += save_interval) times[r++] = grid[k];
        times[r] = grid[n];
    }
    return CMD_OK;
}

int cmd_mixed_magnetization(cmd_mixed* h, double* m2, double* ms2, double* m3, double* ms3) {
    cmd::clear_error();
    if (int rc = check(h, true)) return rc;
    if (!m2 || !ms2 || !m3 || !ms3) return fail(CMD_ERR_INVALID_ARG, "NULL output");
    if (int rc = h->mag.ensure(22 * sizeof(double))) return rc;
    cmd::mixed_magnetization_kernel<<<11, 256, 0, h->stream>>>(h->state.as<double>(), h->m.N2, h->m.N3, h->m.NA2,
                                                              h->m.NA3, h->mag.as<double>());
    MIX_TRY(cudaGetLastError());
    double out[22];
    MIX_TRY(cudaMemcpyAsync(out, h->mag.p, sizeof(out), cudaMemcpyDeviceToHost, h->stream));
    MIX_TRY(cudaStreamSynchronize(h->stream));
    for (int i = 0; i < 3; ++i) { m2[i] = out[i]; ms2[i] = out[3 + i]; }
    for (int i = 0; i < 8; ++i) { m3[i] = out[6 + i]; ms3[i] = out[14 + i]; }
    return CMD_OK;
}

int cmd_mixed_normalize(cmd_mixed* h, double l2, double l3) {
    cmd::clear_error();
    if (int rc = check(h, true)) return rc;
    const int sites = h->m.N2 + h->m.N3;
    cmd::mixed_normalize_kernel<<<(sites + 255) / 256, 256, 0, h->stream>>>(h->state.as<double>(), h->m.N2, h->m.N3,
                                                                           l2, l3);
    MIX_TRY(cudaGetLastError());
    MIX_TRY(cudaStreamSynchronize(h->stream));
    return CMD_OK;
}

int cmd_mixed_dims(cmd_mixed* h, int64_t* dims) {
    cmd::clear_error();
    if (int rc = check(h, false)) return rc;
    if (!dims) return fail(CMD_ERR_INVALID_ARG, "NULL output");
    dims[0] = h->m.N2; dims[1] = 3; dims[2] = h->m.NA2;
    dims[3] = h->m.N3; dims[4] = 8; dims[5] = h->m.NA3;
    return CMD_OK;
}

}  // extern "C"
