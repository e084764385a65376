// rk4_lean.cuh -- the resident RK4 kernel (rk4_resident.cuh: one CTA per
// trajectory, one unit cell per thread, y_n / the RK4 sum / the own stage input
// in registers, the stage input neighbours read double-buffered in shared
// memory, observables reduced every saved step) with the per-stage integer and
// control work taken out of the step loop:
//   * the shared-memory component stride is the compile-time bound MAXT
//     (buf[(atom*3 + comp)*MAXT + cell]), so a partner's three components and
//     the own atoms' stores use immediate offsets;
//   * four stages per step alternate the two buffers, so the buffer a stage
//     reads is known at compile time: each partner's address is resolved once,
//     before the loop, and the other buffer is a compile-time offset from it;
//   * every atom carries Z bonds (checked on the host).  A per-atom test of
//     the bond count stays in the loop all the same: it is a uniform branch,
//     and without it the compiler moves the coupling loads out of the step
//     loop into registers and spills.
// Same arithmetic, in the same order, as rk4_resident_kernel: the results are
// identical.
#pragma once

#include "rk4_resident.cuh"

namespace cmd {

// Shared memory of the lean kernel in doubles: two stage buffers of stride
// MAXT, the reduction rows and the staged envelopes.
__host__ __device__ constexpr long long lean_smem_doubles(int nat, int maxt) {
    return 2LL * nat * 3 * maxt + 32 * kRedStride + 12;
}

template <int NAT, int Z, int LZ, int MAXT, int MINB>
__global__ void __launch_bounds__(MAXT, MINB)
rk4_lean_kernel(const __grid_constant__ Couplings<NAT, Z> cp, const __grid_constant__ ResidentArgs a) {
    constexpr int NL = Z - LZ;                       // non-local slots per atom
    constexpr int NR = NVals<NAT>::used;
    constexpr int NV = NVals<NAT>::value;
    constexpr int GS = MAXT;                         // component stride in shared memory
    constexpr int SB = NAT * 3 * GS;                 // one stage buffer
    extern __shared__ double smem[];
    double* red = smem + 2 * SB;                     // [32][kRedStride]
    double* drv = red + 32 * kRedStride;             // [2][6] envelopes of the current / next step

    const int G = a.G;
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
    const long long b = blockIdx.x;
    const bool own = tid < G;
    const int g = tid;

    double y[NAT][3], acc[NAT][3], yc[NAT][3];
    // partner n of atom at: word offset of its component-0 slot in buffer 0 (buffer 1 is SB further)
    int pb[NAT][NL > 0 ? NL : 1];
    const double* y0 = a.y0 + b * a.y0_stride;
#pragma unroll
    for (int at = 0; at < NAT; ++at)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double v = own ? y0[((long long)g * NAT + at) * 3 + c] : 0.0;
            y[at][c] = v;
            yc[at][c] = v;
            acc[at][c] = 0.0;
            smem[(at * 3 + c) * GS + g] = v;
        }
#pragma unroll
    for (int at = 0; at < NAT; ++at)
#pragma unroll
        for (int m = 0; m < NL; ++m) {
            // resident-layout offset (atom*3)*G + cell -> (atom*3)*GS + cell
            const int off = own ? a.nbr[((long long)g * NAT + at) * NL + m] : 0;
            const int pat3 = off / G, cell = off - pat3 * G;
            const int w = pat3 * GS + cell;
            pb[at][m] = w;
        }

    const bool drive_on = a.drive != nullptr;
    const double dt = a.dt;
    const int st_e = lane;
    const bool stager = drive_on && warp == 0 && lane < 6;
    const double* dtab = stager ? a.drive + b * a.n_steps * 6 : nullptr;
    if (stager && a.n_steps > 0) drv[st_e] = dtab[st_e];
    __syncthreads();

    auto field_at = [&](int buf, int at, const double (&S)[NAT][3], double (&H)[3]) {
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
            const int pa = (at + 1 + n) % NAT;
#pragma unroll
            for (int d = 0; d < 3; ++d)
                bond_acc(H[d], cp.J[at][n][3 * d], cp.J[at][n][3 * d + 1], cp.J[at][n][3 * d + 2], S[pa][0],
                         S[pa][1], S[pa][2]);
        }
        if (LZ >= cp.zc[at]) return;                  // always false here; keeps the couplings operands
#pragma unroll
        for (int m = 0; m < NL; ++m) {
            const double* p = smem + (pb[at][m] + buf * SB);
            const double P0 = p[0], P1 = p[GS], P2 = p[2 * GS];
#pragma unroll
            for (int d = 0; d < 3; ++d)
                bond_acc(H[d], cp.J[at][LZ + m][3 * d], cp.J[at][LZ + m][3 * d + 1], cp.J[at][LZ + m][3 * d + 2], P0,
                         P1, P2);
        }
    };
    auto reduce_partials = [&](double (&part)[NV]) {
        const double r = warp_reduce_many<NV>(part);
        constexpr int span = 32 / NV;
        if ((lane % span) == 0) red[warp * kRedStride + lane / span] = r;
    };
    auto finish_raw = [&](long long row) {
        if (a.raw == nullptr) return;
        for (int q = warp; q < NR; q += nwarps) {
            double s = lane < nwarps ? red[lane * kRedStride + q] : 0.0;
#pragma unroll
            for (int o = 16; o >= 1; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (lane == 0) a.raw[(b * a.rows + row) * a.raw_stride + q] = s;
        }
    };
    auto write_traj = [&](long long row) {
        if (!a.traj || !own) return;
        double* dst = a.traj + (b * a.rows + row) * (long long)G * NAT * 3;
#pragma unroll
        for (int at = 0; at < NAT; ++at)
#pragma unroll
            for (int c = 0; c < 3; ++c) dst[((long long)g * NAT + at) * 3 + c] = y[at][c];
    };

    long long row = 0;
    long long save_left = 0;
    double part[NV];
    const long long n_steps = a.n_steps;
    for (long long step = 0; step < n_steps; ++step) {
        const bool observe = save_left == 0;
        save_left = observe ? a.save_every - 1 : save_left - 1;
        double next_f = 0.0;
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const int rb = s & 1;                    // buffer read in this stage; the other one is written
            if (s == 0 && stager && step + 1 < n_steps) next_f = dtab[(step + 1) * 6 + st_e];
            if (s == 2 && stager && step + 1 < n_steps) drv[6 * ((step + 1) & 1) + st_e] = next_f;
            const int ti = s == 0 ? 0 : (s == 3 ? 2 : 1);
            if (s == 0) {
#pragma unroll
                for (int q = 0; q < NV; ++q) part[q] = 0.0;
            }
            if (s == 1 && observe) reduce_partials(part);
            if (s == 2 && observe) {
                finish_raw(row);
                ++row;
            }
            const double* dv = drv + 6 * (step & 1);
            const double f1 = drive_on ? dv[2 * ti] : 0.0;
            const double f2 = drive_on ? dv[2 * ti + 1] : 0.0;
            const bool drive_now = drive_on && (f1 != 0.0 || f2 != 0.0);   // 0*d adds exactly 0
            double* wbuf = smem + (rb ^ 1) * SB;
            double nx[NAT][3];
#pragma unroll
            for (int at = 0; at < NAT; ++at) {
                double H[3];
                field_at(rb, at, yc, H);
                if (s == 0 && observe) {
                    part[3 * at] += yc[at][0];
                    part[3 * at + 1] += yc[at][1];
                    part[3 * at + 2] += yc[at][2];
                    part[3 * NAT] += yc[at][0] * (H[0] - cp.field[at][0]) + yc[at][1] * (H[1] - cp.field[at][1]) +
                                     yc[at][2] * (H[2] - cp.field[at][2]);
                }
                if (drive_now) {
#pragma unroll
                    for (int d = 0; d < 3; ++d) drive_acc(H[d], cp.d1[at][d], cp.d2[at][d], f1, f2);
                }
                const double kk[3] = {H[1] * yc[at][2] - H[2] * yc[at][1], H[2] * yc[at][0] - H[0] * yc[at][2],
                                      H[0] * yc[at][1] - H[1] * yc[at][0]};
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
                    nx[at][c] = v;                   // own registers change after the cell
                }
            }
#pragma unroll
            for (int at = 0; at < NAT; ++at)
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    yc[at][c] = nx[at][c];
                    wbuf[(at * 3 + c) * GS + g] = nx[at][c];
                }
            if (s == 0 && observe) write_traj(row);
            __syncthreads();
        }
    }
    // Final observation of y(t_end): one more static-field evaluation for E.
    {
#pragma unroll
        for (int q = 0; q < NV; ++q) part[q] = 0.0;
#pragma unroll
        for (int at = 0; at < NAT; ++at) {
            double H[3];
            field_at(0, at, yc, H);
            if (own) {
                part[3 * at] += yc[at][0];
                part[3 * at + 1] += yc[at][1];
                part[3 * at + 2] += yc[at][2];
                part[3 * NAT] += yc[at][0] * (H[0] - cp.field[at][0]) + yc[at][1] * (H[1] - cp.field[at][1]) +
                                 yc[at][2] * (H[2] - cp.field[at][2]);
            }
        }
        write_traj(row);
        reduce_partials(part);
        __syncthreads();
        finish_raw(row);
    }
    if (a.y_out && own) {
        double* dst = a.y_out + b * (long long)G * NAT * 3;
#pragma unroll
        for (int at = 0; at < NAT; ++at)
#pragma unroll
            for (int c = 0; c < 3; ++c) dst[((long long)g * NAT + at) * 3 + c] = y[at][c];
    }
}

}  // namespace cmd
