// adjoint.cu -- discrete adjoint of the RK4 trajectory (cmd_adjoint_rk4): the
// resident kernel (one CTA or cluster per trajectory, rk_adjoint_cluster.cuh),
// the per-trajectory global-memory pair (rk_adjoint.cuh) and, through
// stream.cu, the streamed stages.
#include "cmd_core.h"
#include "rk4_cluster.cuh"
#include "rk_adjoint.cuh"
#include "rk_adjoint_cluster.cuh"
#include "rk_stream.cuh"

#include <cmath>

namespace cmd {
namespace {

// Derivative tables [q][atom][slot][9], [q][atom][3], [q][atom][9] into the kernel parameter block.
template <int NAT, int Z, int NQ>
void fill_param_derivs(const std::vector<double>& DJ, const std::vector<double>& DB, const std::vector<double>& DA,
                       bool has_DA, cmd::ParamDerivs<NAT, Z, NQ>& pd) {
    std::memset(&pd, 0, sizeof(pd));
    for (int q = 0; q < NQ; ++q)
        for (int at = 0; at < NAT; ++at) {
            for (int s = 0; s < Z; ++s)
                std::memcpy(pd.DJ[q][at][s], &DJ[(((size_t)q * NAT + at) * Z + s) * 9], 9 * sizeof(double));
            std::memcpy(pd.DB[q][at], &DB[((size_t)q * NAT + at) * 3], 3 * sizeof(double));
            std::memcpy(pd.DA[q][at], &DA[((size_t)q * NAT + at) * 9], 9 * sizeof(double));
        }
    pd.has_DA = has_DA;
    for (int q = 0; q < NQ; ++q) {
        pd.dj_any[q] = 0;
        for (int at = 0; at < NAT; ++at)
            for (int s = 0; s < Z; ++s)
                for (int e = 0; e < 9; ++e) pd.dj_any[q] |= pd.DJ[q][at][s][e] != 0.0;
    }
}

template <int NAT, int Z, int LZ>
int launch_adjoint(cmd_handle* h, const cmd::AdjArgs& a, const std::vector<double>& DJ, const std::vector<double>& DB,
                   const std::vector<double>& DA, bool has_DA, int64_t B) {
    cmd::Couplings<NAT, Z> cp;
    fill_couplings<NAT, Z>(h, h->fd.data(), h->fd.data() + 3 * h->NA, cp);
    cmd::adjoint_forward_kernel<NAT, Z, LZ><<<(unsigned)B, cmd::kAdjThreads, 0, h->stream>>>(cp, a);
    CUDA_TRY(cudaGetLastError());
    if (a.forward_only) return CMD_OK;
    cmd::ParamDerivs<NAT, Z, kAdjParams> pd;
    fill_param_derivs<NAT, Z, kAdjParams>(DJ, DB, DA, has_DA, pd);
    cmd::adjoint_backward_kernel<NAT, Z, LZ, kAdjParams><<<(unsigned)B, cmd::kAdjThreads, 0, h->stream>>>(cp, pd, a);
    CUDA_TRY(cudaGetLastError());
    return CMD_OK;
}

// Resident adjoint (rk_adjoint_cluster.cuh): one CTA or one cluster of CS CTAs per
// trajectory, one thread per unit cell.
using AdjClusterFn = int (*)(cmd_handle*, cmd::AdjClusterArgs, const std::vector<double>&, const std::vector<double>&,
                             const std::vector<double>&, bool, int64_t);

template <int NAT, int Z, int LZ, int CS, int MAXT>
int launch_adjoint_cluster(cmd_handle* h, cmd::AdjClusterArgs a, const std::vector<double>& DJ,
                           const std::vector<double>& DB, const std::vector<double>& DA, bool has_DA, int64_t B) {
    auto kern = cmd::adjoint_cluster_kernel<NAT, Z, LZ, CS, MAXT, kAdjParams>;
    const int64_t G = h->lay.G, Gc = cluster_cells(G, CS);
    const int threads = (int)((Gc + 31) / 32 * 32);
    const size_t smem = (size_t)cmd::adj_cluster_smem_doubles(NAT, Gc) * sizeof(double);
    if (threads > MAXT || smem > kMaxSmem) return fail(CMD_ERR_UNSUPPORTED, "lattice too large for this adjoint variant");
    a.nbr = cluster_table(h, CS);
    if (!a.nbr && !h->lay.nbr.empty()) return fail(CMD_ERR_UNSUPPORTED, "no cluster neighbour table for this lattice");
    // Function attributes belong to the current device's context: set on every
    // launch (a host-side call of about a microsecond), so handles on several
    // devices, several host threads and a re-created context all see it.
    CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMaxSmem));
    cmd::Couplings<NAT, Z> cp;
    fill_couplings<NAT, Z>(h, h->fd.data(), h->fd.data() + 3 * h->NA, cp);
    cmd::ParamDerivs<NAT, Z, kAdjParams> pd;
    fill_param_derivs<NAT, Z, kAdjParams>(DJ, DB, DA, has_DA, pd);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(B * CS));
    cfg.blockDim = dim3((unsigned)threads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = h->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = CS;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    CUDA_TRY(cudaLaunchKernelEx(&cfg, kern, cp, pd, a, (int)Gc));
    return CMD_OK;
}

struct AdjClusterVariant {
    int NAT, Z, LZ, CS, MAXT;
    AdjClusterFn fn;
};

const AdjClusterVariant kAdjClusterVariants[] = {
    {2, 3, 1, 1, 576, &launch_adjoint_cluster<2, 3, 1, 1, 576>},
    {2, 3, 1, 2, 576, &launch_adjoint_cluster<2, 3, 1, 2, 576>},
    {2, 3, 1, 4, 576, &launch_adjoint_cluster<2, 3, 1, 4, 576>},
    {4, 6, 3, 1, 256, &launch_adjoint_cluster<4, 6, 3, 1, 256>},
    {4, 6, 3, 2, 256, &launch_adjoint_cluster<4, 6, 3, 2, 256>},
    {4, 6, 3, 4, 256, &launch_adjoint_cluster<4, 6, 3, 4, 256>},
};

// The resident adjoint variant for h's lattice: the smallest cluster whose CTAs hold
// the cells; -1 if none does.
int pick_adjoint_cluster(const cmd_handle* h) {
    const Layout& L = h->lay;
    const int ty = global_type(L);
    if (ty < 0) return -1;
    for (int i = 0; i < (int)(sizeof(kAdjClusterVariants) / sizeof(kAdjClusterVariants[0])); ++i) {
        const AdjClusterVariant& v = kAdjClusterVariants[i];
        if ((ty == 0) != (v.NAT == 2)) continue;
        const int64_t Gc = cluster_cells(L.G, v.CS);
        if ((Gc + 31) / 32 * 32 > v.MAXT) continue;
        if ((size_t)cmd::adj_cluster_smem_doubles(v.NAT, Gc) * sizeof(double) > kMaxSmem) continue;
        if ((int64_t)v.NAT * 3 * Gc >= (1 << cmd::kClusterRankShift)) continue;
        if (v.CS > 1 && !cluster_table(h, v.CS)) continue;
        return i;
    }
    return -1;
}


}  // namespace
}  // namespace cmd

using namespace cmd;

extern "C" {

int cmd_adjoint_rk4(cmd_handle* h, const cmd_adjoint_desc* d) {
    cmd::clear_error();
    if (int rc = check_handle(h, false)) return rc;
    if (!d || d->B <= 0 || !d->states || !d->target || !d->loss || d->n_steps <= 0 || !(d->dt > 0.0))
        return fail(CMD_ERR_INVALID_ARG, "bad adjoint description");
    if (d->n_params < 0 || d->n_params > kAdjParams || (d->n_params > 0 && (!d->dparams || !d->grad)))
        return fail(CMD_ERR_INVALID_ARG, "n_params must be 0..5 with derivative lattices and a grad buffer");
    if (d->path < CMD_ADJ_AUTO || d->path > CMD_ADJ_GLOBAL) return fail(CMD_ERR_INVALID_ARG, "unknown adjoint path");
    const int ty = global_type(h->lay);
    if (ty < 0) return no_instance(h->lay);
    const int NA = h->NA, Z = h->lay.Z;
    // derivative tables per (parameter, atom class, slot) from the theta = e_q lattices
    std::vector<double> DJ((size_t)kAdjParams * NA * Z * 9, 0.0), DB((size_t)kAdjParams * NA * 3, 0.0),
        DA((size_t)kAdjParams * NA * 9, 0.0);
    bool has_DA = false;
    for (int q = 0; q < d->n_params; ++q) {
        const cmd_lattice_desc& p = d->dparams[q];
        if (p.lattice_size != h->N || !p.counts || !p.partners || !p.bilinear || !p.field || !p.onsite)
            return fail(CMD_ERR_INVALID_ARG, "derivative lattice does not match the handle's lattice");
        for (int a = 0; a < NA; ++a) {
            for (int s = 0; s < h->lay.zc[a]; ++s) {
                const int e = h->lay.slot_entry[(size_t)a * Z + s];
                if (e < 0 || e >= p.counts[a]) return fail(CMD_ERR_INVALID_ARG, "derivative lattice bond tables differ");
                std::memcpy(&DJ[(((size_t)q * NA + a) * Z + s) * 9], &p.bilinear[((int64_t)a * p.max_bilinear + e) * 9],
                            9 * sizeof(double));
            }
            std::memcpy(&DB[((size_t)q * NA + a) * 3], &p.field[3 * a], 3 * sizeof(double));
            std::memcpy(&DA[((size_t)q * NA + a) * 9], &p.onsite[9 * a], 9 * sizeof(double));
            for (int k = 0; k < 9; ++k) has_DA |= p.onsite[9 * a + k] != 0.0;
        }
    }
    const int64_t B = d->B, S = d->n_steps, N3 = h->N * 3, V = N3;
    int64_t C = d->checkpoint_every > 0 ? d->checkpoint_every : (int64_t)std::ceil(std::sqrt((double)S));
    C = std::max<int64_t>(1, std::min(C, S));
    const int64_t K = (S + C - 1) / C;
    const bool fwd_only = d->forward_only != 0;
    if (int rc = h->awork.ensure((size_t)B * 5 * V * sizeof(double))) return rc;
    if (!fwd_only) {
        if (int rc = h->ackpt.ensure((size_t)B * K * V * sizeof(double))) return rc;
        if (int rc = h->aseg.ensure((size_t)B * C * 4 * V * sizeof(double))) return rc;
    }
    if (int rc = h->amloc.ensure((size_t)B * (S + 1) * 3 * sizeof(double))) return rc;
    if (int rc = h->aout.ensure((size_t)B * (1 + kAdjParams) * sizeof(double))) return rc;
    if (int rc = h->ain.ensure(((size_t)B * N3 + (size_t)B * (S + 1) * 3 + (S + 1)) * sizeof(double))) return rc;
    if (int rc = h->ameta.ensure((size_t)B * sizeof(cmd::AdjTraj))) return rc;
    for (int64_t i = 0; i < B * N3; ++i)
        if (!std::isfinite(d->states[i])) return fail(CMD_ERR_NONFINITE, "non-finite initial spin");
    double* din = h->ain.as<double>();
    double* dtgt = din + B * N3;
    double* dtimes = dtgt + B * (S + 1) * 3;
    std::vector<double> times((size_t)S + 1);
    double t = d->T0;
    for (int64_t n = 0; n <= S; ++n) { times[n] = t; t += d->dt; }
    CUDA_TRY(cudaMemcpyAsync(din, d->states, B * N3 * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(cudaMemcpyAsync(dtgt, d->target, B * (S + 1) * 3 * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(cudaMemcpyAsync(dtimes, times.data(), times.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    std::vector<cmd::AdjTraj> tr(B);
    double* dout = h->aout.as<double>();
    for (int64_t b = 0; b < B; ++b) {
        cmd::AdjTraj& T = tr[b];
        T.y0 = din + b * N3;
        T.target = dtgt + b * (S + 1) * 3;
        T.ckpt = fwd_only ? nullptr : h->ackpt.as<double>() + b * K * V;
        T.seg = fwd_only ? nullptr : h->aseg.as<double>() + b * C * 4 * V;
        T.work = h->awork.as<double>() + b * 5 * V;
        T.mloc = h->amloc.as<double>() + b * (S + 1) * 3;
        T.loss = dout + b * (1 + kAdjParams);
        T.grad = dout + b * (1 + kAdjParams) + 1;
    }
    CUDA_TRY(cudaMemcpyAsync(h->ameta.p, tr.data(), B * sizeof(cmd::AdjTraj), cudaMemcpyHostToDevice, h->stream));
    cmd::AdjArgs a{};
    a.traj = h->ameta.as<cmd::AdjTraj>();
    a.B = (int)B;
    a.G = (int)h->lay.G;
    a.nbr = h->nbr.as<int>();
    a.times = dtimes;
    a.n_steps = S;
    a.ckpt_every = C;
    a.dt = d->dt;
    if (h->amp != 0.0) a.pulse = cmd::Pulse{h->t1, h->t2, h->amp, h->amp};
    a.width = h->width;
    a.freq = h->freq;
    a.forward_only = fwd_only;
    // resident (one CTA or cluster per trajectory) when a variant holds the lattice; else one
    // CTA per trajectory in global memory when the batch fills the GPU, else streamed stages
    const int cpt = cmd::kStreamTile / std::max(1, h->NA);
    const int tiles = (int)((h->lay.G + cpt - 1) / cpt);
    const int resident = (d->path == CMD_ADJ_AUTO || d->path == CMD_ADJ_RESIDENT) ? pick_adjoint_cluster(h) : -1;
    if (d->path == CMD_ADJ_RESIDENT && resident < 0)
        return fail(CMD_ERR_UNSUPPORTED, "no resident adjoint variant holds this lattice");
    const bool streamed = resident < 0 && B <= 65535 &&
                          (d->path == CMD_ADJ_STREAMED || (d->path == CMD_ADJ_AUTO && B < 148 && tiles >= 2));
    int rc = CMD_OK;
    if (resident >= 0) {
        cmd::AdjClusterArgs ca{};
        ca.traj = a.traj;
        ca.G = a.G;
        ca.n_steps = S;
        ca.ckpt_every = C;
        ca.dt = d->dt;
        ca.forward_only = fwd_only;
        if (h->amp != 0.0) {
            const cmd::Pulse pl{h->t1, h->t2, h->amp, h->amp};
            if (int rc2 = h->pulses.ensure(sizeof(cmd::Pulse))) return rc2;
            if (int rc2 = h->drive.ensure((size_t)S * 6 * sizeof(double))) return rc2;
            CUDA_TRY(cudaMemcpyAsync(h->pulses.p, &pl, sizeof(pl), cudaMemcpyHostToDevice, h->stream));
            const int blocks = (int)std::min<int64_t>((S * 6 + 255) / 256, 148 * 32);
            cmd::drive_table_kernel<<<blocks, 256, 0, h->stream>>>(h->pulses.as<cmd::Pulse>(), dtimes, S, d->dt,
                                                                 h->width, h->freq, 1, h->drive.as<double>());
            CUDA_TRY(cudaGetLastError());
            ca.drive = h->drive.as<double>();
        }
        rc = kAdjClusterVariants[resident].fn(h, ca, DJ, DB, DA, has_DA, B);
    } else if (streamed) {
        StreamAdjJob j{B, S, C, K, fwd_only, din, dtgt, dtimes, h->amloc.as<double>(), dout, d->dt};
        rc = run_stream_adjoint(h, j, d->n_params, DJ, DB, DA, has_DA);
    } else {
        rc = ty == 0 ? launch_adjoint<2, 3, 1>(h, a, DJ, DB, DA, has_DA, B)
                     : launch_adjoint<4, 6, 3>(h, a, DJ, DB, DA, has_DA, B);
    }
    if (rc != CMD_OK) return rc;
    std::vector<double> out((size_t)B * (1 + kAdjParams));
    CUDA_TRY(cudaMemcpyAsync(out.data(), dout, out.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    if (d->m_local)
        CUDA_TRY(cudaMemcpyAsync(d->m_local, h->amloc.p, B * (S + 1) * 3 * sizeof(double), cudaMemcpyDeviceToHost,
                                 h->stream));
    if (int rc2 = sync(h)) return rc2;
    for (int64_t b = 0; b < B; ++b) {
        d->loss[b] = out[b * (1 + kAdjParams)];
        if (!fwd_only)
            for (int q = 0; q < d->n_params; ++q) d->grad[b * d->n_params + q] = out[b * (1 + kAdjParams) + 1 + q];
    }
    return CMD_OK;
}

}  // extern "C"
