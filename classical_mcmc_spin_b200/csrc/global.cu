// global.cu -- the global-state integrator (rk_global.cuh: fixed-step methods,
// controlled Dormand-Prince for lattices no on-chip tiling holds) and the
// on-chip controlled Dormand-Prince kernels (rk45_onchip.cuh).
#include "cmd_core.h"
#include "rk_global.cuh"

namespace cmd {
namespace {

bool same_couplings(const cmd_handle* a, const cmd_handle* b) {
    return a->lay.J == b->lay.J && a->lay.zc == b->lay.zc && a->field == b->field && a->onsite == b->onsite &&
           a->fd == b->fd && a->width == b->width && a->freq == b->freq && a->frames == b->frames &&
           a->afm == b->afm;
}

}  // namespace

int run_global(cmd_handle* owner, std::vector<GJob>& jobs, int mode, double abs_tol, double rel_tol,
               int64_t max_steps, std::vector<long long>& stats) {
    const int64_t B = (int64_t)jobs.size();
    if (B <= 0) return fail(CMD_ERR_INVALID_ARG, "empty batch");
    const cmd_handle* src[2] = {nullptr, nullptr};
    for (const GJob& j : jobs) {
        const int ty = global_type(j.h->lay);
        if (ty < 0) return no_instance(j.h->lay);
        if (!src[ty]) src[ty] = j.h;
        else if (!same_couplings(src[ty], j.h))
            return fail(CMD_ERR_UNSUPPORTED, "lattices of one unit-cell type must share couplings and pulse settings");
    }
    if (src[0] && src[1] && (src[0]->width != src[1]->width || src[0]->freq != src[1]->freq))
        return fail(CMD_ERR_UNSUPPORTED, "pulse width / frequency must agree across the batch");
    // longest first (cells x expected steps)
    std::vector<int64_t> order(B);
    for (int64_t i = 0; i < B; ++i) order[i] = i;
    auto cost = [&](int64_t i) {
        const GJob& j = jobs[i];
        const double steps = j.n_steps > 0 ? (double)j.n_steps : (j.T1 - j.T0) / std::max(j.dt0, 1e-300);
        return (double)j.h->N * steps;
    };
    std::stable_sort(order.begin(), order.end(), [&](int64_t x, int64_t y) { return cost(x) > cost(y); });
    // Controlled RK45 trajectories on lattices an on-chip tiling holds run on
    // the on-chip kernels (rk45_onchip.cuh), one launch per handle, the launches
    // concurrent on the owner's auxiliary streams; everything else runs on the
    // persistent global-state kernel on the owner's stream.
    std::vector<int> tiling(B, -1);
    if (mode == kModeRK45)
        for (int64_t i = 0; i < B; ++i) tiling[i] = rk45_pick(jobs[i].h);
    std::vector<int64_t> gl;                                   // global-state jobs, longest first
    std::vector<cmd_handle*> gh;                               // on-chip groups (one per handle) ...
    std::vector<std::vector<int64_t>> gj;                      // ... and their jobs, longest first
    for (int64_t q = 0; q < B; ++q) {
        const int64_t i = order[q];
        if (tiling[i] < 0) {
            gl.push_back(i);
            continue;
        }
        size_t k = 0;
        while (k < gh.size() && gh[k] != jobs[i].h) ++k;
        if (k == gh.size()) {
            gh.push_back(jobs[i].h);
            gj.emplace_back();
        }
        gj[k].push_back(i);
    }
    size_t work_total = 0;
    std::vector<size_t> woff(B, 0);
    for (int64_t i : gl) {
        woff[i] = work_total;
        work_total += (size_t)cmd::kGVectors * 3 * jobs[i].h->N;
    }
    if (work_total)
        if (int rc = owner->gwork.ensure(work_total * sizeof(double))) return rc;
    if (int rc = owner->gmeta.ensure((size_t)B * sizeof(cmd::GTraj))) return rc;
    if (int rc = owner->gstat.ensure((size_t)B * 4 * sizeof(long long))) return rc;
    if (int rc = owner->gqueue.ensure(sizeof(int))) return rc;
    std::vector<cmd::GTraj> tr;
    tr.reserve(B);
    long long* dstat = owner->gstat.as<long long>();
    auto push = [&](int64_t i) {
        const GJob& j = jobs[i];
        cmd::GTraj T{};
        T.type = global_type(j.h->lay);
        T.G = (int)j.h->lay.G;
        T.nbr = j.h->nbr.as<int>();
        T.y0 = j.y0;
        T.yout = j.yout;
        T.work = tiling[i] < 0 ? owner->gwork.as<double>() + woff[i] : nullptr;
        T.rows = j.rows;
        T.traj = j.traj;
        T.max_rows = j.max_rows;
        T.T0 = j.T0; T.T1 = j.T1; T.dt0 = j.dt0;
        T.n_steps = j.n_steps;
        T.save_every = j.save_every;
        T.pulse = j.pulse;
        T.stat = dstat + 4 * i;
        tr.push_back(T);
    };
    for (int64_t i : gl) push(i);
    for (const auto& v : gj)
        for (int64_t i : v) push(i);
    cudaStream_t st = owner->stream;
    CUDA_TRY(cudaMemcpyAsync(owner->gmeta.p, tr.data(), B * sizeof(cmd::GTraj), cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemsetAsync(owner->gqueue.p, 0, sizeof(int), st));
    CUDA_TRY(cudaMemsetAsync(owner->gstat.p, 0, B * 4 * sizeof(long long), st));
    const cmd::GTraj* dtr = owner->gmeta.as<cmd::GTraj>();
    while (owner->aux_streams.size() < gh.size() + 1) {
        cudaStream_t s2 = nullptr;
        cudaEvent_t e2 = nullptr;
        CUDA_TRY(cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking));
        owner->aux_streams.push_back(s2);
        CUDA_TRY(cudaEventCreateWithFlags(&e2, cudaEventDisableTiming));
        owner->aux_events.push_back(e2);
    }
    for (size_t k = 0; k < gh.size(); ++k)
        if (int rc = rk45_prepare(gh[k], tiling[gj[k][0]])) return rc;
    // fork: every on-chip group on an auxiliary stream after the uploads above,
    // the global-state kernel on the owner's stream, join; one graph
    const int rc = graph_call(owner, kGraphUneven, st, [&]() -> int {
        if (!gh.empty()) CUDA_TRY(cudaEventRecord(owner->aux_events.back(), st));
        int64_t off = (int64_t)gl.size();
        for (size_t k = 0; k < gh.size(); ++k) {
            cudaStream_t sk = owner->aux_streams[k];
            CUDA_TRY(cudaStreamWaitEvent(sk, owner->aux_events.back(), 0));
            const int64_t n = (int64_t)gj[k].size();
            int rc2 = rk45_launch(gh[k], tiling[gj[k][0]], dtr + off, n, abs_tol, rel_tol, max_steps, sk);
            CUDA_TRY(cudaEventRecord(owner->aux_events[k], sk));      // joined below even after a failed launch
            if (rc2) {
                for (size_t q = 0; q <= k; ++q) cudaStreamWaitEvent(st, owner->aux_events[q], 0);
                return rc2;
            }
            off += n;
        }
        if (!gl.empty()) {
            cmd::GArgs a{};
            a.traj = dtr;
            a.B = (int)gl.size();
            a.queue = owner->gqueue.as<int>();
            a.mode = mode;
            a.abs_tol = abs_tol;
            a.rel_tol = rel_tol;
            a.max_steps = max_steps;
            const cmd_handle* any = src[0] ? src[0] : src[1];
            a.width = any->width;
            a.freq = any->freq;
            cmd::Couplings<2, 3> c0;
            cmd::Couplings<4, 6> c1;
            std::memset(&c0, 0, sizeof(c0));
            std::memset(&c1, 0, sizeof(c1));
            if (src[0]) {
                fill_couplings<2, 3>(src[0], src[0]->fd.data(), src[0]->fd.data() + 3 * src[0]->NA, c0);
                a.frames0 = src[0]->dframes.as<double>();
                a.afm0 = src[0]->dafm.as<double>();
            }
            if (src[1]) {
                fill_couplings<4, 6>(src[1], src[1]->fd.data(), src[1]->fd.data() + 3 * src[1]->NA, c1);
                a.frames1 = src[1]->dframes.as<double>();
                a.afm1 = src[1]->dafm.as<double>();
            }
            auto kern = mode >= cmd::kModeEuler ? cmd::rk_global_kernel<2, 3, 1, 4, 6, 3, true>
                                                : cmd::rk_global_kernel<2, 3, 1, 4, 6, 3, false>;
            int dev = 0, nsm = 148, per_sm = 1;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, 0);
            const int grid = (int)std::min<int64_t>((int64_t)gl.size(), (int64_t)nsm * std::max(per_sm, 1));
            kern<<<grid, 256, 0, st>>>(c0, c1, a);
            const cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) {
                for (size_t k = 0; k < gh.size(); ++k) cudaStreamWaitEvent(st, owner->aux_events[k], 0);
                return fail(CMD_ERR_CUDA, std::string("rk_global_kernel: ") + cudaGetErrorString(e));
            }
        }
        for (size_t k = 0; k < gh.size(); ++k) CUDA_TRY(cudaStreamWaitEvent(st, owner->aux_events[k], 0));   // join
        return CMD_OK;
    });
    if (rc != CMD_OK) return rc;
    stats.assign((size_t)B * 4, 0);
    CUDA_TRY(cudaMemcpyAsync(stats.data(), owner->gstat.p, B * 4 * sizeof(long long), cudaMemcpyDeviceToHost, st));
    return sync(owner);
}

}  // namespace cmd
