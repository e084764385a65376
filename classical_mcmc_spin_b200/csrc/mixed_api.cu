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
#include <map>
#include <string>
#include <vector>

using cmd::fail;

#define MIX_TRY(x)                                                                               \
    do {                                                                                         \
        cudaError_t e_ = (x);                                                                    \
        if (e_ != cudaSuccess) return fail(CMD_ERR_CUDA, std::string(#x ": ") + cudaGetErrorString(e_)); \
    } while (0)

struct cmd_mixed {
    cmd::MixedDev m{};
    int64_t V = 0;
    cmd::DevBuf tables;        // distinct couplings and index arrays, one allocation
    cmd::DevBuf drive2, drive3;
    cmd::DevBuf state, work, rows, mag;
    bool has_state = false;
    cudaStream_t stream = nullptr;
    ~cmd_mixed() {
        for (cmd::DevBuf* b : {&tables, &drive2, &drive3, &state, &work, &rows, &mag}) b->release();
    }
};

namespace {

size_t pad(size_t bytes) { return (bytes + 255) / 256 * 256; }

constexpr size_t kMixedSmemMax = 200 * 1024;   // distinct couplings copied to shared memory up to this size

// Distinct blocks of w doubles in first-seen order, and the index of each block added.
struct Distinct {
    int w;
    std::vector<double> vals;
    std::map<std::vector<double>, int> seen;
    explicit Distinct(int w_) : w(w_) {}
    int add(const double* p) {
        std::vector<double> k(p, p + w);
        auto it = seen.find(k);
        if (it != seen.end()) return it->second;
        const int id = (int)(vals.size() / w);
        vals.insert(vals.end(), k.begin(), k.end());
        seen.emplace(std::move(k), id);
        return id;
    }
};

// One kind of site: distinct field / on-site / bond / mixed-bond blocks, and the
// per-site and per-(slot, site) indices (slot-major: index n * N + s).
struct KindTables {
    std::vector<int> fi, oi, bi, part, cnt, mi, mpart, mcnt;
};

void build_kind(int64_t N, int z, int zm, int dim, const double* field, const double* onsite,
                const double* bil, const int64_t* partners, const int64_t* counts, int64_t limit_same,
                const double* mix, const int64_t* mpartners, const int64_t* mcounts, int64_t limit_other,
                Distinct& F, Distinct& O, Distinct& B, Distinct& M, KindTables& t) {
    t.fi.assign(N, 0); t.oi.assign(N, 0); t.cnt.assign(N, 0); t.mcnt.assign(N, 0);
    t.bi.assign((size_t)N * z, 0); t.part.assign((size_t)N * z, -1);
    t.mi.assign((size_t)N * zm, 0); t.mpart.assign((size_t)N * zm, -1);
    for (int64_t s = 0; s < N; ++s) {
        t.fi[s] = F.add(field + (size_t)s * dim);
        t.oi[s] = O.add(onsite + (size_t)s * dim * dim);
        t.cnt[s] = (int)std::max<int64_t>(0, std::min<int64_t>(counts[s], z));
        for (int n = 0; n < t.cnt[s]; ++n) {
            const int64_t p = partners[(size_t)s * z + n];
            if (p < 0 || p >= limit_same) continue;
            t.part[(size_t)n * N + s] = (int)p;
            t.bi[(size_t)n * N + s] = B.add(bil + ((size_t)s * z + n) * dim * dim);
        }
        t.mcnt[s] = zm > 0 ? (int)std::max<int64_t>(0, std::min<int64_t>(mcounts[s], zm)) : 0;
        for (int n = 0; n < t.mcnt[s]; ++n) {
            const int64_t p = mpartners[(size_t)s * zm + n];
            if (p < 0 || p >= limit_other) continue;
            t.mpart[(size_t)n * N + s] = (int)p;
            t.mi[(size_t)n * N + s] = M.add(mix + ((size_t)s * zm + n) * 24);
        }
    }
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
cudaLaunchConfig_t config(cmd_mixed* h, int threads, cudaLaunchAttribute* attr) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(CS);
    cfg.blockDim = dim3((unsigned)threads);
    cfg.dynamicSmemBytes = h->m.tab_in_smem ? (size_t)h->m.tab_doubles * sizeof(double) : 0;
    cfg.stream = h->stream;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = CS;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cfg;
}

// Function attributes belong to the current device's context, so they are set
// before every launch (a host-side call of about a microsecond): handles on
// several devices, several host threads and a re-created context all see them.
template <int CS>
int set_attributes() {
    auto kern = cmd::mixed_integrate_kernel<CS>;
    MIX_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMixedSmemMax));
    if (CS > 8) MIX_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    return CMD_OK;
}

template <int CS>
int launch_cs(cmd_mixed* h, const cmd::MixedRun& r, int threads) {
    if (int rc = set_attributes<CS>()) return rc;
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = config<CS>(h, threads, attr);
    MIX_TRY(cudaLaunchKernelEx(&cfg, cmd::mixed_integrate_kernel<CS>, h->m, r));
    return CMD_OK;
}

// Whether a 16-CTA cluster (a non-portable size) of this shape can be resident.
bool cluster16_fits(cmd_mixed* h, int threads) {
    if (set_attributes<16>() != CMD_OK) return false;
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = config<16>(h, threads, attr);
    int n = 0;
    return cudaOccupancyMaxActiveClusters(&n, cmd::mixed_integrate_kernel<16>, &cfg) == cudaSuccess && n >= 1;
}

// One persistent launch over a cluster sized to the lattice: one site per thread up
// to 16 CTAs, the threads loop beyond that (at most kMixedThreads per CTA).
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
    // Up to 128 sites per CTA before the cluster grows (more SMs per trajectory beat
    // more warps per SM here: the stages are latency-bound), up to 16 CTAs.
    const int64_t sites = (int64_t)h->m.N2 + h->m.N3;
    const int64_t per = (sites + 127) / 128;
    int cs = per <= 1 ? 1 : per <= 2 ? 2 : per <= 4 ? 4 : per <= 8 ? 8 : 16;
    auto threads_for = [&](int c) {
        return (int)std::min<int64_t>(cmd::kMixedThreads, std::max<int64_t>(32, ((sites + c - 1) / c + 31) / 32 * 32));
    };
    if (cs == 16 && !cluster16_fits(h, threads_for(16))) cs = 8;
    const int threads = threads_for(cs);
    int rc = cs == 1 ? launch_cs<1>(h, r, threads)
           : cs == 2 ? launch_cs<2>(h, r, threads)
           : cs == 4 ? launch_cs<4>(h, r, threads)
           : cs == 8 ? launch_cs<8>(h, r, threads)
                     : launch_cs<16>(h, r, threads);
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
    Distinct F2(3), O2(9), B2(9), M2(24), F3(8), O3(64), B3(64), M3(24);
    KindTables k2, k3;
    build_kind(N2, z2, zm2, 3, d->field_su2, d->onsite_su2, d->bilinear_su2, d->partners_su2, d->counts_su2, N2,
               d->mixed_su2, d->mixed_partners_su3, d->mixed_counts_su2, N3, F2, O2, B2, M2, k2);
    build_kind(N3, z3, zm3, 8, d->field_su3, d->onsite_su3, d->bilinear_su3, d->partners_su3, d->counts_su3, N3,
               d->mixed_su3, d->mixed_partners_su2, d->mixed_counts_su3, N2, F3, O3, B3, M3, k3);
    std::vector<double> tab;
    cmd::MixedDev& m = h->m;
    // each distinct block at the kernel's odd stride (mixed.cuh kStride*)
    auto append = [&](const Distinct& D, int stride, int& off) {
        off = (int)tab.size();
        const size_t nb = D.vals.size() / D.w;
        tab.resize(tab.size() + nb * stride, 0.0);
        for (size_t b = 0; b < nb; ++b)
            std::copy(D.vals.begin() + b * D.w, D.vals.begin() + (b + 1) * D.w, tab.begin() + off + b * stride);
    };
    append(F2, cmd::kStrideF2, m.off_f2); append(O2, cmd::kStrideO2, m.off_o2);
    append(B2, cmd::kStrideB2, m.off_b2); append(M2, cmd::kStrideM, m.off_m2);
    append(F3, cmd::kStrideF3, m.off_f3); append(O3, cmd::kStrideO3, m.off_o3);
    append(B3, cmd::kStrideB3, m.off_b3); append(M3, cmd::kStrideM, m.off_m3);
    // work slots: warp-sized runs of SU(2) and SU(3) sites in turn, so every CTA gets both kinds
    std::vector<int> order;
    order.reserve(N2 + N3);
    for (int64_t a = 0, b = 0; a < N2 || b < N3;) {
        for (int k = 0; k < 32 && a < N2; ++k) order.push_back((int)a++);
        for (int k = 0; k < 32 && b < N3; ++k) order.push_back((int)(N2 + b++));
    }
    const std::vector<int>* ints[17] = {&k2.fi, &k2.oi, &k2.bi, &k2.part, &k2.cnt, &k2.mi, &k2.mpart, &k2.mcnt,
                                        &k3.fi, &k3.oi, &k3.bi, &k3.part, &k3.cnt, &k3.mi, &k3.mpart, &k3.mcnt,
                                        &order};
    size_t total = pad(tab.size() * sizeof(double));
    for (const auto* v : ints) total += pad(v->size() * sizeof(int));
    if (int rc = h->tables.ensure(total)) return bail(rc);
    char* cur = h->tables.as<char>();
    int rc = CMD_OK;
    auto put = [&](const void* src, size_t bytes) {
        char* at = cur;
        if (rc == CMD_OK && bytes) {
            if (cudaMemcpyAsync(cur, src, bytes, cudaMemcpyHostToDevice, h->stream) != cudaSuccess)
                rc = fail(CMD_ERR_CUDA, "upload of the mixed lattice tables failed");
        }
        cur += pad(bytes);
        return at;
    };
    m.N2 = (int)N2; m.N3 = (int)N3;
    m.NA2 = std::max(1, d->n_atoms_su2); m.NA3 = std::max(1, d->n_atoms_su3);
    m.z2 = z2; m.z3 = z3; m.zm2 = zm2; m.zm3 = zm3;
    m.tab = (const double*)put(tab.data(), tab.size() * sizeof(double));
    m.tab_doubles = (int)tab.size();
    m.tab_in_smem = tab.size() * sizeof(double) <= kMixedSmemMax;
    const int* dev[17];
    for (int i = 0; i < 17; ++i) dev[i] = (const int*)put(ints[i]->data(), ints[i]->size() * sizeof(int));
    m.order = dev[16];
    m.f2i = dev[0]; m.o2i = dev[1]; m.b2i = dev[2]; m.part2 = dev[3]; m.cnt2 = dev[4]; m.m2i = dev[5];
    m.mpart2 = dev[6]; m.mcnt2 = dev[7];
    m.f3i = dev[8]; m.o3i = dev[9]; m.b3i = dev[10]; m.part3 = dev[11]; m.cnt3 = dev[12]; m.m3i = dev[13];
    m.mpart3 = dev[14]; m.mcnt3 = dev[15];
    if (rc) return bail(rc);
    // the host vectors above must outlive the copies
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) return bail(fail(CMD_ERR_CUDA, "upload failed"));
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
