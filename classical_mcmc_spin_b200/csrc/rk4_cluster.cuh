// rk4_cluster.cuh -- resident RK4 with one trajectory split over a thread-block
// cluster of CS CTAs (CS SMs), for lattices one CTA cannot hold (48x48
// honeycomb: 2304 cells) and for batches too small to fill the GPU one CTA per
// trajectory (the single plain trajectory, the tail of a scan).
//
// CTA `rank` of the cluster owns cells [rank*Gc, rank*Gc + Gc) and keeps their
// y_n and RK4 sum in registers and their stage inputs in its shared memory
// (double-buffered, [NAT*3][Gc]).  A partner in another CTA's slice is read
// through distributed shared memory (the address of that CTA's buffer from
// cluster.map_shared_rank); the partner table holds (rank << 24) | offset.  One
// cluster barrier per stage (barrier.cluster arrive/wait: release/acquire at
// cluster scope, so every CTA's stage input is visible before it is read).
//
// Observables: each CTA sums its cells (stage 0), warp-reduces (stage 1) and
// finishes its totals in ctot[] (stage 2); in stage 3 rank 0 adds the CTAs'
// totals in rank order and writes the raw row -- the same fixed order on every
// run.  No CTA leaves before the last cross-CTA read (final cluster barrier).
#pragma once

#include "rk4_resident.cuh"

#include <cooperative_groups.h>

namespace cmd {

namespace cg = cooperative_groups;

constexpr int kClusterRankShift = 24;          // partner word: (rank << 24) | offset in that CTA's buffer
constexpr int kClusterOffsetMask = (1 << kClusterRankShift) - 1;

template <int CS>
__device__ __forceinline__ const double* pick_rank(const double* const (&base)[CS], int r) {
    const double* p = base[0];
#pragma unroll
    for (int i = 1; i < CS; ++i)
        if (r == i) p = base[i];
    return p;
}

template <int NAT, int Z, int LZ, int CS, int MAXT>
__global__ void __launch_bounds__(MAXT, 1)
rk4_cluster_kernel(const __grid_constant__ Couplings<NAT, Z> cp, const __grid_constant__ ResidentArgs a, int Gc) {
    constexpr int NL = Z - LZ;
    constexpr int NR = NVals<NAT>::used;
    constexpr int NV = NR <= 4 ? 4 : (NR <= 8 ? 8 : 16);
    extern __shared__ double smem[];
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = (int)cluster.block_rank();
    const long long b = blockIdx.x / CS;
    const int SBc = NAT * 3 * Gc;                  // one stage buffer of this CTA
    double* red = smem + 2 * SBc;                  // [32][kRedStride]
    double* drv = red + 32 * kRedStride;           // [2][6] envelopes of the current / next step
    double* ctot = drv + 12;                       // [NR] this CTA's totals of the row being finished
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
    const int g = rank * Gc + tid;                 // global cell of this thread
    const bool own = tid < Gc && g < a.G;

    const double* base[CS];
#pragma unroll
    for (int r = 0; r < CS; ++r) base[r] = r == rank ? smem : cluster.map_shared_rank(smem, r);

    double y[NAT][3], acc[NAT][3], yc[NAT][3];
    int nb[NAT][NL > 0 ? NL : 1];
    const double* y0 = a.y0 + b * a.y0_stride;
#pragma unroll
    for (int at = 0; at < NAT; ++at) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double v = own ? y0[((long long)g * NAT + at) * 3 + c] : 0.0;
            y[at][c] = v;
            yc[at][c] = v;
            acc[at][c] = 0.0;
            if (own) smem[(at * 3 + c) * Gc + tid] = v;
        }
#pragma unroll
        for (int m = 0; m < NL; ++m) nb[at][m] = own ? a.nbr[((long long)g * NAT + at) * NL + m] : 0;
    }

    const bool drive_on = a.drive != nullptr;
    const double* dtab = drive_on ? a.drive + b * a.n_steps * 6 : nullptr;
    const double dt = a.dt;
    const bool stager = drive_on && warp == 0 && lane < 6;
    if (stager && a.n_steps > 0) drv[lane] = dtab[lane];
    cluster.sync();

    auto field_at = [&](int in, int at, const double (&S)[NAT][3], double (&H)[3]) {
        if (cp.has_field) {
            H[0] = -cp.field[at][0]; H[1] = -cp.field[at][1]; H[2] = -cp.field[at][2];
        } else {
            H[0] = 0.0; H[1] = 0.0; H[2] = 0.0;
        }
        if (cp.has_onsite) {
#pragma unroll
            for (int d = 0; d < 3; ++d)
                bond_acc(H[d], 2.0 * cp.onsite[at][3 * d], 2.0 * cp.onsite[at][3 * d + 1],
                         2.0 * cp.onsite[at][3 * d + 2], S[at][0], S[at][1], S[at][2]);
        }
#pragma unroll
        for (int n = 0; n < LZ; ++n) {
            const int pb = (at + 1 + n) % NAT;
#pragma unroll
            for (int d = 0; d < 3; ++d)
                bond_acc(H[d], cp.J[at][n][3 * d], cp.J[at][n][3 * d + 1], cp.J[at][n][3 * d + 2], S[pb][0],
                         S[pb][1], S[pb][2]);
        }
#pragma unroll
        for (int m = 0; m < NL; ++m) {
            const int n = LZ + m;
            if (n < cp.zc[at]) {
                const int w = nb[at][m];
                const double* src = pick_rank<CS>(base, w >> kClusterRankShift);
                const int p = in + (w & kClusterOffsetMask);
                const double P0 = src[p], P1 = src[p + Gc], P2 = src[p + 2 * Gc];
#pragma unroll
                for (int d = 0; d < 3; ++d)
                    bond_acc(H[d], cp.J[at][n][3 * d], cp.J[at][n][3 * d + 1], cp.J[at][n][3 * d + 2], P0, P1, P2);
            }
        }
    };
    auto reduce_partials = [&](double (&part)[NV]) {
        const double r = warp_reduce_many<NV>(part);
        constexpr int span = 32 / NV;
        if ((lane % span) == 0) red[warp * kRedStride + lane / span] = r;
    };
    // warp q: this CTA's total of value q over its warps -> ctot[q]
    auto finish_cta = [&]() {
        for (int q = warp; q < NR; q += nwarps) {
            double s = lane < nwarps ? red[lane * kRedStride + q] : 0.0;
#pragma unroll
            for (int o = 16; o >= 1; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (lane == 0) ctot[q] = s;
        }
    };
    // rank 0: row = sum over the CTAs (rank order) of their totals
    auto write_row = [&](long long row) {
        if (rank != 0 || a.raw == nullptr) return;
        if (tid < NR) {
            double s = 0.0;
#pragma unroll
            for (int r = 0; r < CS; ++r) s += pick_rank<CS>(base, r)[2 * SBc + 32 * kRedStride + 12 + tid];
            a.raw[(b * a.rows + row) * a.raw_stride + tid] = s;
        }
    };
    auto write_traj = [&](long long row) {
        if (!a.traj || !own) return;
        double* dst = a.traj + (b * a.rows + row) * (long long)a.G * NAT * 3;
#pragma unroll
        for (int at = 0; at < NAT; ++at)
#pragma unroll
            for (int c = 0; c < 3; ++c) dst[((long long)g * NAT + at) * 3 + c] = y[at][c];
    };
    auto cell_obs = [&](int in, double (&part)[NV]) {
        if (!own) return;
#pragma unroll
        for (int at = 0; at < NAT; ++at) {
            double H[3];
            field_at(in, at, yc, H);
            part[3 * at] += yc[at][0];
            part[3 * at + 1] += yc[at][1];
            part[3 * at + 2] += yc[at][2];
            part[3 * NAT] += yc[at][0] * (H[0] - cp.field[at][0]) + yc[at][1] * (H[1] - cp.field[at][1]) +
                             yc[at][2] * (H[2] - cp.field[at][2]);
        }
    };

    long long row = 0;
    long long save_left = 0;
    int in = 0, out = SBc;
    double part[NV];
    for (long long step = 0; step < a.n_steps; ++step) {
        const bool observe = save_left == 0;
        save_left = observe ? a.save_every - 1 : save_left - 1;
        const double* dv = drv + 6 * (step & 1);
        double next_f = 0.0;
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            if (s == 0 && stager && step + 1 < a.n_steps) next_f = dtab[(step + 1) * 6 + lane];
            if (s == 2 && stager && step + 1 < a.n_steps) drv[6 * ((step + 1) & 1) + lane] = next_f;
            const int ti = s == 0 ? 0 : (s == 3 ? 2 : 1);
            const double f1 = drive_on ? dv[2 * ti] : 0.0;
            const double f2 = drive_on ? dv[2 * ti + 1] : 0.0;
            const bool drive_now = drive_on && (f1 != 0.0 || f2 != 0.0);
            if (s == 0) {
#pragma unroll
                for (int q = 0; q < NV; ++q) part[q] = 0.0;
            }
            if (s == 1 && observe) reduce_partials(part);
            if (s == 2 && observe) finish_cta();
            if (s == 3 && observe) {
                write_row(row);
                ++row;
            }
            if (own) {
                const double(&S)[NAT][3] = yc;
                double nx[NAT][3];
#pragma unroll
                for (int at = 0; at < NAT; ++at) {
                    double H[3];
                    field_at(in, at, S, H);
                    if (s == 0 && observe) {
                        part[3 * at] += S[at][0];
                        part[3 * at + 1] += S[at][1];
                        part[3 * at + 2] += S[at][2];
                        part[3 * NAT] += S[at][0] * (H[0] - cp.field[at][0]) + S[at][1] * (H[1] - cp.field[at][1]) +
                                         S[at][2] * (H[2] - cp.field[at][2]);
                    }
                    if (drive_now) {
#pragma unroll
                        for (int d = 0; d < 3; ++d) drive_acc(H[d], cp.d1[at][d], cp.d2[at][d], f1, f2);
                    }
                    const double kk[3] = {H[1] * S[at][2] - H[2] * S[at][1], H[2] * S[at][0] - H[0] * S[at][2],
                                          H[0] * S[at][1] - H[1] * S[at][0]};
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        double v;
                        if (s == 0) {
                            acc[at][c] = kk[c];
                            v = 1.0 * y[at][c] + (0.5 * dt) * kk[c];
                        } else if (s == 1) {
                            acc[at][c] = acc[at][c] + 2.0 * kk[c];
                            v = 1.0 * y[at][c] + (0.5 * dt) * kk[c];
                        } else if (s == 2) {
                            acc[at][c] = acc[at][c] + 2.0 * kk[c];
                            v = 1.0 * y[at][c] + dt * kk[c];
                        } else {
                            y[at][c] += (dt / 6.0) * (acc[at][c] + kk[c]);
                            v = y[at][c];
                        }
                        nx[at][c] = v;
                    }
                }
#pragma unroll
                for (int at = 0; at < NAT; ++at)
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        yc[at][c] = nx[at][c];
                        smem[out + (at * 3 + c) * Gc + tid] = nx[at][c];
                    }
            }
            if (s == 0 && observe) write_traj(row);
            cluster.sync();
            const int tmp = in; in = out; out = tmp;
        }
    }
    // Final observation of y(t_end).
#pragma unroll
    for (int q = 0; q < NV; ++q) part[q] = 0.0;
    cell_obs(in, part);
    write_traj(row);
    reduce_partials(part);
    __syncthreads();
    finish_cta();
    cluster.sync();
    write_row(row);
    if (a.y_out && own) {
        double* dst = a.y_out + b * (long long)a.G * NAT * 3;
#pragma unroll
        for (int at = 0; at < NAT; ++at)
#pragma unroll
            for (int c = 0; c < 3; ++c) dst[((long long)g * NAT + at) * 3 + c] = y[at][c];
    }
    cluster.sync();                                // the last cross-CTA reads are done
}

}  // namespace cmd
