// stream.cu -- streamed RK4 and the streamed discrete adjoint (rk_stream.cuh):
// lattices no resident or cluster variant holds, one launch per RK stage over
// (cell tile, trajectory).
#include "cmd_core.h"
#include "rk_stream.cuh"

namespace cmd {
namespace {

// Steps of the streamed RK4 loop: enqueue(k) launches the four stages of step
// base + k, base read by the kernels from h->snbase.  With graphs on and at
// least two chunks of work, one chunk of kChunk steps (4 kChunk stage launches
// and a base advance) is captured once per distinct set of launch parameters
// (`key`), kept in the handle and replayed; the remaining steps are launched
// directly.  The kernels see the same step numbers either way.
constexpr int64_t kChunk = 128;

template <class F>
int run_steps(cmd_handle* h, cudaStream_t st, int64_t S, const std::vector<unsigned char>& key, F&& enqueue,
              int32_t* nl) {
    CUDA_TRY(cudaMemsetAsync(h->snbase.p, 0, sizeof(long long), st));
    int64_t done = 0;
    if (h->graphs && S >= 2 * kChunk) {
        if (!h->stream_graph || h->stream_graph_key != key) {
            release_stream_graph(h);
            cudaGraph_t g = nullptr;
            CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            for (int64_t k = 0; k < kChunk; ++k) enqueue(k);
            stream_advance_kernel<<<1, 32, 0, st>>>(h->snbase.as<long long>(), kChunk);
            const cudaError_t e = cudaStreamEndCapture(st, &g);
            if (e != cudaSuccess || !g) return fail(CMD_ERR_CUDA, std::string("stream capture: ") + cudaGetErrorString(e));
            const cudaError_t e2 = cudaGraphInstantiate(&h->stream_graph, g, 0);
            cudaGraphDestroy(g);
            if (e2 != cudaSuccess) {
                h->stream_graph = nullptr;
                return fail(CMD_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e2));
            }
            h->stream_graph_key = key;
        }
        for (; done + kChunk <= S; done += kChunk) {
            CUDA_TRY(cudaGraphLaunch(h->stream_graph, st));
            *nl += 4 * (int32_t)kChunk + 1;
        }
    }
    for (int64_t k = 0; done + k < S; ++k) {
        enqueue(k);
        *nl += 4;
        if ((k & 1023) == 0) CUDA_TRY(cudaGetLastError());
    }
    CUDA_TRY(cudaGetLastError());
    return CMD_OK;
}

template <class T>
void key_add(std::vector<unsigned char>& k, const T& v) {
    const unsigned char* p = reinterpret_cast<const unsigned char*>(&v);
    k.insert(k.end(), p, p + sizeof(T));
}

// ---------------------------------------------------------------------------
// Streamed RK4 (rk_stream.cuh): lattices no resident variant holds.  One launch
// per stage over (cell tile, trajectory); same RunSpec contract and outputs as
// run_resident.

template <int NAT, int Z, int LZ>
int stream_forward(cmd_handle* h, const RunSpec& r, cudaStream_t st, int32_t* launches) {
    constexpr int NR = 3 * NAT + 1;
    int32_t nl = 0;
    const int G = (int)h->lay.G;
    const int tiles = (G + cmd::stream_cells<NAT>() - 1) / cmd::stream_cells<NAT>();
    const int64_t V = (int64_t)NAT * 3 * G;
    const int64_t B = r.B;
    if (B > 65535) return fail(CMD_ERR_UNSUPPORTED, "streamed batches are limited to 65535 trajectories");
    if (r.traj && B != 1) return fail(CMD_ERR_UNSUPPORTED, "streamed state saving is for single trajectories");
    const int64_t rows = rows_for(r.n_steps, r.save);
    if (int rc = h->sbuf.ensure((size_t)4 * B * V * sizeof(double))) return rc;
    if (int rc = h->spart.ensure((size_t)B * tiles * cmd::kPart * sizeof(double))) return rc;
    double* base = h->sbuf.as<double>();
    const cmd::SVec y{base, V}, acc{base + B * V, V}, Ya{base + 2 * B * V, V}, Yb{base + 3 * B * V, V};
    cmd::StreamArgs a{};
    a.G = G;
    a.tiles = tiles;
    a.B = (int)B;
    a.nbr = h->nbr.as<int>();
    a.dt = r.dt;
    a.n_steps = r.n_steps;
    a.part = h->spart.as<double>();
    a.n_sites = r.n_sites;
    a.save_every = r.save;
    a.rows = rows;
    a.V = V;
    if (r.obs) {
        if (NR <= 10) {
            a.raw = r.obs;
            a.raw_stride = 10;
        } else {
            if (int rc = h->raw.ensure((size_t)B * rows * NR * sizeof(double))) return rc;
            a.raw = h->raw.as<double>();
            a.raw_stride = NR;
        }
    }
    if (r.pulses && r.n_steps > 0) {
        std::vector<double> grid;
        grid.reserve(r.n_steps);
        double t = r.T0;
        for (int64_t k = 0; k < r.n_steps; ++k) {     // t_k of the reference loop (t += dt)
            grid.push_back(t);
            t += r.dt;
        }
        if (int rc = h->times.ensure(grid.size() * sizeof(double))) return rc;
        if (int rc = h->drive.ensure((size_t)B * r.n_steps * 6 * sizeof(double))) return rc;
        CUDA_TRY(cudaMemcpyAsync(h->times.p, grid.data(), grid.size() * sizeof(double), cudaMemcpyHostToDevice, st));
        const int64_t total = B * r.n_steps * 6;
        const int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 32);
        cmd::drive_table_kernel<<<blocks, 256, 0, st>>>(r.pulses, h->times.as<double>(), r.n_steps, r.dt, r.width,
                                                       r.freq, B, h->drive.as<double>());
        CUDA_TRY(cudaGetLastError());
        ++nl;
        a.times = h->times.as<double>();
        a.drive = h->drive.as<double>();
    }
    static const std::vector<double> zeros(3 * 64, 0.0);
    cmd::Couplings<NAT, Z> cp;
    fill_couplings<NAT, Z>(h, r.d1 ? r.d1 : zeros.data(), r.d2 ? r.d2 : zeros.data(), cp);
    const dim3 grid(tiles, (unsigned)B), gridc((G + 255) / 256, (unsigned)B);
    const int64_t N3 = (int64_t)G * NAT * 3;
    auto save_traj = [&](int64_t row) {
        const cmd::SVec src = y;
        cmd::stream_store_kernel<NAT><<<gridc, 256, 0, st>>>(src, G, r.traj + row * N3);
        ++nl;
    };
    cmd::stream_load_kernel<NAT><<<gridc, 256, 0, st>>>(r.y0, r.y0_stride, G, y);
    CUDA_TRY(cudaGetLastError());
    ++nl;
    const int with_obs = r.obs ? 1 : 0;
    if (r.traj) {                                    // states saved between steps: direct launches
        for (int64_t n = 0; n < r.n_steps; ++n) {
            if (n % r.save == 0) save_traj(n / r.save);
            cmd::stream_stage_kernel<NAT, Z, LZ><<<grid, cmd::kStreamTile, 0, st>>>(cp, a, 0, n, y, y, acc, Ya, with_obs);
            cmd::stream_stage_kernel<NAT, Z, LZ><<<grid, cmd::kStreamTile, 0, st>>>(cp, a, 1, n, Ya, y, acc, Yb, with_obs);
            cmd::stream_stage_kernel<NAT, Z, LZ><<<grid, cmd::kStreamTile, 0, st>>>(cp, a, 2, n, Yb, y, acc, Ya, with_obs);
            cmd::stream_stage_kernel<NAT, Z, LZ><<<grid, cmd::kStreamTile, 0, st>>>(cp, a, 3, n, Ya, y, acc, y, with_obs);
            nl += 4;
            if ((n & 1023) == 0) CUDA_TRY(cudaGetLastError());
        }
        CUDA_TRY(cudaGetLastError());
    } else {
        if (int rc = h->snbase.ensure(sizeof(long long))) return rc;
        a.nbase = h->snbase.as<long long>();
        std::vector<unsigned char> key;
        key_add(key, 1);                             // forward stages of this NAT/Z/LZ
        key_add(key, NAT * 100 + Z * 10 + LZ);
        key_add(key, cp);
        key_add(key, a);
        key_add(key, y);
        key_add(key, acc);
        key_add(key, Ya);
        key_add(key, Yb);
        key_add(key, with_obs);
        key_add(key, grid);
        auto enqueue = [&](int64_t k) {
            cmd::stream_stage_kernel<NAT, Z, LZ><<<grid, cmd::kStreamTile, 0, st>>>(cp, a, 0, k, y, y, acc, Ya, with_obs);
            cmd::stream_stage_kernel<NAT, Z, LZ><<<grid, cmd::kStreamTile, 0, st>>>(cp, a, 1, k, Ya, y, acc, Yb, with_obs);
            cmd::stream_stage_kernel<NAT, Z, LZ><<<grid, cmd::kStreamTile, 0, st>>>(cp, a, 2, k, Yb, y, acc, Ya, with_obs);
            cmd::stream_stage_kernel<NAT, Z, LZ><<<grid, cmd::kStreamTile, 0, st>>>(cp, a, 3, k, Ya, y, acc, y, with_obs);
        };
        if (int rc = run_steps(h, st, r.n_steps, key, enqueue, &nl)) return rc;
        a.nbase = nullptr;                           // the final observation below uses absolute steps
    }
    if (r.traj) save_traj(rows - 1);
    if (r.obs) {
        cmd::stream_obs_kernel<NAT, Z, LZ><<<grid, cmd::kStreamTile, 0, st>>>(cp, a, y);
        cmd::stream_reduce_kernel<NAT><<<(unsigned)B, cmd::kStreamTile, 0, st>>>(a, r.n_steps);
        CUDA_TRY(cudaGetLastError());
        nl += 2;
    }
    if (r.y_out) {
        cmd::stream_store_kernel<NAT><<<gridc, 256, 0, st>>>(y, G, r.y_out);
        CUDA_TRY(cudaGetLastError());
        ++nl;
    }
    if (r.obs) {
        const double* fr = r.frames ? r.frames : h->dframes.as<double>();
        const double* af = r.afm ? r.afm : h->dafm.as<double>();
        launch_finish<NAT>(a.raw, a.raw_stride, B * rows, fr, af, r.n_sites, r.obs, st);
        CUDA_TRY(cudaGetLastError());
        ++nl;
    }
    if (launches) *launches = nl;
    return CMD_OK;
}

template <int NAT, int Z, int LZ, int NQ>
int stream_adjoint(cmd_handle* h, const StreamAdjJob& j, const std::vector<double>& DJ, const std::vector<double>& DB,
                   const std::vector<double>& DA, bool has_DA) {
    cudaStream_t st = h->stream;
    const int G = (int)h->lay.G;
    const int tiles = (G + cmd::stream_cells<NAT>() - 1) / cmd::stream_cells<NAT>();
    const int64_t V = (int64_t)NAT * 3 * G, B = j.B, S = j.S, C = j.C, K = j.K;
    if (int rc = h->sbuf.ensure((size_t)5 * B * V * sizeof(double))) return rc;
    if (int rc = h->spart.ensure(((size_t)B * tiles * cmd::kPart + B) * sizeof(double))) return rc;
    const int vtiles = (G + cmd::kStreamTile - 1) / cmd::kStreamTile;     // VJP: one cell per thread
    if (int rc = h->sgpart.ensure((size_t)B * vtiles * cmd::kPart * sizeof(double))) return rc;
    double* base = h->sbuf.as<double>();
    double* d_loss = h->spart.as<double>() + (size_t)B * tiles * cmd::kPart;
    const bool driven = h->amp != 0.0;
    if (driven) {
        std::vector<cmd::Pulse> pl((size_t)B, cmd::Pulse{h->t1, h->t2, h->amp, h->amp});
        if (int rc = h->pulses.ensure((size_t)B * sizeof(cmd::Pulse))) return rc;
        if (int rc = h->drive.ensure((size_t)B * S * 6 * sizeof(double))) return rc;
        CUDA_TRY(cudaMemcpyAsync(h->pulses.p, pl.data(), pl.size() * sizeof(cmd::Pulse), cudaMemcpyHostToDevice, st));
        const int64_t total = B * S * 6;
        const int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 32);
        cmd::drive_table_kernel<<<blocks, 256, 0, st>>>(h->pulses.as<cmd::Pulse>(), j.times, S, j.dt, h->width,
                                                       h->freq, B, h->drive.as<double>());
        CUDA_TRY(cudaGetLastError());
    }
    cmd::Couplings<NAT, Z> cp;
    fill_couplings<NAT, Z>(h, h->fd.data(), h->fd.data() + 3 * h->NA, cp);
    cmd::StreamArgs a{};
    a.G = G;
    a.tiles = tiles;
    a.B = (int)B;
    a.nbr = h->nbr.as<int>();
    a.dt = j.dt;
    a.n_steps = S;
    a.times = j.times;
    a.drive = driven ? h->drive.as<double>() : nullptr;
    a.part = h->spart.as<double>();
    a.save_every = 1;
    a.rows = S + 1;
    a.target = j.target;
    a.mloc = j.mloc;
    a.loss = d_loss;
    a.n_sites = (double)h->N;
    a.ckpt = j.fwd_only ? nullptr : h->ackpt.as<double>();
    a.ckpt_every = C;
    a.n_ckpt = K;
    a.V = V;
    const dim3 grid(tiles, (unsigned)B), gridc((G + 255) / 256, (unsigned)B);
    const cmd::SVec none{nullptr, 0};
    // forward: loss terms every step, checkpoints every C steps
    {
        const cmd::SVec y{base, V}, acc{base + B * V, V}, Ya{base + 2 * B * V, V}, Yb{base + 3 * B * V, V};
        cmd::stream_load_kernel<NAT><<<gridc, 256, 0, st>>>(j.y0, (long long)G * NAT * 3, G, y);
        if (int rc = h->snbase.ensure(sizeof(long long))) return rc;
        cmd::StreamArgs af = a;                      // steps relative to the device step base
        af.nbase = h->snbase.as<long long>();
        std::vector<unsigned char> key;
        key_add(key, 2);                             // adjoint forward stages of this NAT/Z/LZ
        key_add(key, NAT * 100 + Z * 10 + LZ);
        key_add(key, cp);
        key_add(key, af);
        key_add(key, y);
        key_add(key, acc);
        key_add(key, Ya);
        key_add(key, Yb);
        key_add(key, grid);
        auto enqueue = [&](int64_t k) {
            cmd::stream_stage_kernel<NAT, Z, LZ><<<grid, cmd::kStreamTile, 0, st>>>(cp, af, 0, k, y, y, acc, Ya, 1);
            cmd::stream_stage_kernel<NAT, Z, LZ><<<grid, cmd::kStreamTile, 0, st>>>(cp, af, 1, k, Ya, y, acc, Yb, 1);
            cmd::stream_stage_kernel<NAT, Z, LZ><<<grid, cmd::kStreamTile, 0, st>>>(cp, af, 2, k, Yb, y, acc, Ya, 1);
            cmd::stream_stage_kernel<NAT, Z, LZ><<<grid, cmd::kStreamTile, 0, st>>>(cp, af, 3, k, Ya, y, acc, y, 1);
        };
        int32_t nl = 0;
        if (int rc = run_steps(h, st, S, key, enqueue, &nl)) return rc;
        cmd::stream_obs_kernel<NAT, Z, LZ><<<grid, cmd::kStreamTile, 0, st>>>(cp, a, y);
        cmd::stream_reduce_kernel<NAT><<<(unsigned)B, cmd::kStreamTile, 0, st>>>(a, S);
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaMemcpy2DAsync(j.out, (1 + kAdjParams) * sizeof(double), d_loss, sizeof(double), sizeof(double),
                                   (size_t)B, cudaMemcpyDeviceToDevice, st));
    }
    if (j.fwd_only) return CMD_OK;
    cmd::ParamDerivs<NAT, Z, NQ> pd;
    std::memset(&pd, 0, sizeof(pd));
    for (int q = 0; q < NQ; ++q)
        for (int at = 0; at < NAT; ++at) {
            for (int sl = 0; sl < Z; ++sl)
                std::memcpy(pd.DJ[q][at][sl], &DJ[(((size_t)q * NAT + at) * Z + sl) * 9], 9 * sizeof(double));
            std::memcpy(pd.DB[q][at], &DB[((size_t)q * NAT + at) * 3], 3 * sizeof(double));
            std::memcpy(pd.DA[q][at], &DA[((size_t)q * NAT + at) * 9], 9 * sizeof(double));
        }
    pd.has_DA = has_DA;
    cmd::StreamVjpArgs v{};
    v.G = G;
    v.tiles = vtiles;
    v.nbr = a.nbr;
    v.dt = j.dt;
    v.n_steps = S;
    v.drive = a.drive;
    v.target = j.target;
    v.mloc = j.mloc;
    v.n_sites = a.n_sites;
    v.gpart = h->sgpart.as<double>();
    cmd::StreamArgs ar = a;              // recompute: no observables, no checkpoints
    ar.ckpt = nullptr;
    CUDA_TRY(cudaMemsetAsync(v.gpart, 0, (size_t)B * vtiles * cmd::kPart * sizeof(double), st));
    const dim3 vgrid(vtiles, (unsigned)B);
    cmd::SVec lam{base, V}, lam2{base + B * V, V};
    const cmd::SVec acc{base + 2 * B * V, V}, Sa{base + 3 * B * V, V}, Sb{base + 4 * B * V, V};
    cmd::stream_lam_init_kernel<NAT><<<gridc, 256, 0, st>>>(v, lam);
    double* seg = h->aseg.as<double>();
    auto slot = [&](int64_t jj, int q) { return cmd::SVec{seg + (jj * 4 + q) * V, C * 4 * V}; };
    const double dt = j.dt;
    // One checkpoint segment of len steps: the recompute that stores every
    // stage input, then the reverse sweep; kernel step arguments are nb + jj.
    // The cotangent buffers l / l2 swap once per step.
    auto segment = [&](int64_t len, int64_t nb, const cmd::StreamArgs& sa, const cmd::StreamVjpArgs& sv,
                       cmd::SVec& l, cmd::SVec& l2) {
        for (int64_t jj = 0; jj < len; ++jj) {
            const int64_t n = nb + jj;
            const cmd::SVec y = slot(jj, 0);
            const cmd::SVec last = jj + 1 < len ? slot(jj + 1, 0) : none;
            cmd::stream_stage_kernel<NAT, Z, LZ><<<grid, cmd::kStreamTile, 0, st>>>(cp, sa, 0, n, y, y, acc,
                                                                                   slot(jj, 1), 0);
            cmd::stream_stage_kernel<NAT, Z, LZ><<<grid, cmd::kStreamTile, 0, st>>>(cp, sa, 1, n, slot(jj, 1), y, acc,
                                                                                   slot(jj, 2), 0);
            cmd::stream_stage_kernel<NAT, Z, LZ><<<grid, cmd::kStreamTile, 0, st>>>(cp, sa, 2, n, slot(jj, 2), y, acc,
                                                                                   slot(jj, 3), 0);
            cmd::stream_stage_kernel<NAT, Z, LZ><<<grid, cmd::kStreamTile, 0, st>>>(cp, sa, 3, n, slot(jj, 3), y, acc,
                                                                                   last, 0);
        }
        for (int64_t jj = len - 1; jj >= 0; --jj) {
            const int64_t n = nb + jj;
            auto vjp = cmd::stream_vjp_kernel<NAT, Z, LZ, NQ>;
            vjp<<<vgrid, cmd::kStreamTile, 0, st>>>(cp, pd, sv, 3, n, slot(jj, 3), l, none, dt / 6.0, 0.0, Sa, acc,
                                                   none, 0);
            vjp<<<vgrid, cmd::kStreamTile, 0, st>>>(cp, pd, sv, 2, n, slot(jj, 2), l, Sa, dt / 3.0, dt, Sb, acc,
                                                   none, 1);
            vjp<<<vgrid, cmd::kStreamTile, 0, st>>>(cp, pd, sv, 1, n, slot(jj, 1), l, Sb, dt / 3.0, 0.5 * dt, Sa,
                                                   acc, none, 1);
            vjp<<<vgrid, cmd::kStreamTile, 0, st>>>(cp, pd, sv, 0, n, slot(jj, 0), l, Sa, dt / 6.0, 0.5 * dt, none,
                                                   acc, l2, 2);
            std::swap(l, l2);
        }
    };
    // Full-length segments replay a captured graph of the segment with the
    // kernels' steps relative to the device step base (set to the segment's
    // first step before each replay); one graph per order of the cotangent
    // buffers at the segment's start.  The partial segment (processed first)
    // and, with graphs off, every segment launch directly.
    if (int rc = h->snbase.ensure(sizeof(long long))) return rc;
    cmd::StreamArgs ar_rel = ar;
    ar_rel.nbase = h->snbase.as<long long>();
    cmd::StreamVjpArgs v_rel = v;
    v_rel.nbase = h->snbase.as<long long>();
    const double* lam_start = lam.p;
    for (int64_t sg = K - 1; sg >= 0; --sg) {
        const int64_t n0 = sg * C, n1 = std::min(n0 + C, S);
        CUDA_TRY(cudaMemcpy2DAsync(seg, (size_t)C * 4 * V * sizeof(double), h->ackpt.as<double>() + sg * V,
                                   (size_t)K * V * sizeof(double), (size_t)V * sizeof(double), (size_t)B,
                                   cudaMemcpyDeviceToDevice, st));
        const int64_t len = n1 - n0;
        if (!h->graphs || len != C || K < 3) {
            segment(len, n0, ar, v, lam, lam2);
            CUDA_TRY(cudaGetLastError());
            continue;
        }
        const int par = lam.p == lam_start ? 0 : 1;
        std::vector<unsigned char> key;
        key_add(key, 3);                             // adjoint segment of this NAT/Z/LZ/NQ
        key_add(key, NAT * 1000 + Z * 100 + LZ * 10 + NQ);
        key_add(key, cp);
        key_add(key, pd);
        key_add(key, ar_rel);
        key_add(key, v_rel);
        key_add(key, lam);
        key_add(key, lam2);
        key_add(key, acc);
        key_add(key, Sa);
        key_add(key, Sb);
        key_add(key, seg);
        key_add(key, C);
        key_add(key, grid);
        key_add(key, vgrid);
        key_add(key, dt);
        cmd::stream_set_base_kernel<<<1, 32, 0, st>>>(h->snbase.as<long long>(), n0);
        CUDA_TRY(cudaGetLastError());
        cudaGraphExec_t& ex = h->adj_graph[par];
        if (!ex || h->adj_graph_key[par] != key) {
            if (ex) {
                cudaStreamSynchronize(st);
                cudaGraphExecDestroy(ex);
                ex = nullptr;
            }
            h->adj_graph_key[par].clear();
            cmd::SVec l = lam, l2 = lam2;
            cudaGraph_t g = nullptr;
            CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            segment(len, 0, ar_rel, v_rel, l, l2);
            const cudaError_t e = cudaStreamEndCapture(st, &g);
            if (e != cudaSuccess || !g) {
                if (g) cudaGraphDestroy(g);
                return fail(CMD_ERR_CUDA, std::string("stream capture: ") + cudaGetErrorString(e));
            }
            const cudaError_t e2 = cudaGraphInstantiate(&ex, g, 0);
            cudaGraphDestroy(g);
            if (e2 != cudaSuccess) {
                ex = nullptr;
                return fail(CMD_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e2));
            }
            h->adj_graph_key[par] = key;
        }
        CUDA_TRY(cudaGraphLaunch(ex, st));
        if (len & 1) std::swap(lam, lam2);
    }
    cmd::stream_grad_kernel<<<(unsigned)B, 32, 0, st>>>(v.gpart, vtiles, NQ, j.out + 1, 1 + kAdjParams);
    CUDA_TRY(cudaGetLastError());
    return CMD_OK;
}

// Threads per CTA and shared memory per CTA of variant V on layout L.
}  // namespace

void release_stream_graph(cmd_handle* h) {
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->stream_graph) cudaGraphExecDestroy(h->stream_graph);
    h->stream_graph = nullptr;
    h->stream_graph_key.clear();
    for (int i = 0; i < 2; ++i) {
        if (h->call_graph[i]) cudaGraphExecDestroy(h->call_graph[i]);
        h->call_graph[i] = nullptr;
        h->call_sig[i].clear();
        if (h->adj_graph[i]) cudaGraphExecDestroy(h->adj_graph[i]);
        h->adj_graph[i] = nullptr;
        h->adj_graph_key[i].clear();
    }
}

namespace {

// The node types in order and, per kernel node, its function, grid, block,
// dynamic shared memory and cluster shape: what an in-place update of an
// executable graph may not change.  False when a query fails.
bool graph_signature(cudaGraph_t g, std::vector<unsigned char>& sig) {
    size_t n = 0;
    if (cudaGraphGetNodes(g, nullptr, &n) != cudaSuccess) return false;
    std::vector<cudaGraphNode_t> nodes(n);
    if (n && cudaGraphGetNodes(g, nodes.data(), &n) != cudaSuccess) return false;
    sig.clear();
    key_add(sig, n);
    for (cudaGraphNode_t nd : nodes) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(nd, &t) != cudaSuccess) return false;
        key_add(sig, (int)t);
        if (t != cudaGraphNodeTypeKernel) continue;
        cudaKernelNodeParams p{};
        if (cudaGraphKernelNodeGetParams(nd, &p) != cudaSuccess) return false;
        key_add(sig, p.func);
        key_add(sig, p.gridDim);
        key_add(sig, p.blockDim);
        key_add(sig, p.sharedMemBytes);
        cudaLaunchAttributeValue v{};                  // zeros where the node has no cluster shape
        if (cudaGraphKernelNodeGetAttribute(nd, cudaLaunchAttributeClusterDimension, &v) != cudaSuccess) {
            (void)cudaGetLastError();
            v = cudaLaunchAttributeValue{};
        }
        key_add(sig, v.clusterDim.x);
        key_add(sig, v.clusterDim.y);
        key_add(sig, v.clusterDim.z);
    }
    return true;
}

}  // namespace

int graph_call(cmd_handle* h, int slot, cudaStream_t st, const std::function<int()>& enqueue) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    const bool capture = h->graphs && st != nullptr && st != cudaStreamLegacy && st != cudaStreamPerThread &&
                         cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusNone;
    if (!capture) return enqueue();
    // relaxed: the launch helpers set kernel attributes, which is not stream work
    CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
    const int rc = enqueue();
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(st, &g);
    if (rc != CMD_OK || e != cudaSuccess || !g) {
        if (g) cudaGraphDestroy(g);
        (void)cudaGetLastError();
        if (rc != CMD_OK) return rc;
        return fail(CMD_ERR_CUDA, std::string("stream capture: ") + cudaGetErrorString(e));
    }
    // Same kernels and launch shapes as the kept graph: update its arguments in
    // place; otherwise (or when the update is refused) build a new one.
    std::vector<unsigned char> sig;
    const bool have_sig = graph_signature(g, sig);
    (void)cudaGetLastError();
    cudaGraphExec_t& ex = h->call_graph[slot];
    bool updated = false;
    if (ex && have_sig && sig == h->call_sig[slot]) {
        cudaGraphExecUpdateResultInfo info{};
        updated = cudaGraphExecUpdate(ex, g, &info) == cudaSuccess;
        (void)cudaGetLastError();
    }
    if (ex && !updated) {
        cudaStreamSynchronize(st);                    // the old graph's last launch is done
        cudaGraphExecDestroy(ex);
        ex = nullptr;
    }
    h->call_sig[slot] = have_sig ? sig : std::vector<unsigned char>();
    if (!ex) {
        const cudaError_t e2 = cudaGraphInstantiate(&ex, g, 0);
        if (e2 != cudaSuccess) {
            ex = nullptr;
            cudaGraphDestroy(g);
            return fail(CMD_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e2));
        }
    }
    cudaGraphDestroy(g);
    CUDA_TRY(cudaGraphLaunch(ex, st));
    return CMD_OK;
}

int run_streamed(cmd_handle* h, const RunSpec& r, cudaStream_t st, int32_t* launches) {
    switch (global_type(h->lay)) {
        case 0: return stream_forward<2, 3, 1>(h, r, st, launches);
        case 1: return stream_forward<4, 6, 3>(h, r, st, launches);
        default: return no_instance(h->lay);
    }
}

int run_stream_adjoint(cmd_handle* h, const StreamAdjJob& j, int n_params, const std::vector<double>& DJ,
                       const std::vector<double>& DB, const std::vector<double>& DA, bool has_DA) {
    const int ty = global_type(h->lay);
    if (ty < 0) return no_instance(h->lay);
    // the VJP carries as many parameter cotangents as requested (4 or 5)
    if (n_params <= 4)
        return ty == 0 ? stream_adjoint<2, 3, 1, 4>(h, j, DJ, DB, DA, has_DA)
                       : stream_adjoint<4, 6, 3, 4>(h, j, DJ, DB, DA, has_DA);
    return ty == 0 ? stream_adjoint<2, 3, 1, 5>(h, j, DJ, DB, DA, has_DA)
                   : stream_adjoint<4, 6, 3, 5>(h, j, DJ, DB, DA, has_DA);
}

}  // namespace cmd
