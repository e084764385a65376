// rk4_resident.cuh -- one CTA per trajectory, whole RK4 trajectory in one launch.
//
// The Landau-Lifshitz right-hand side of the reference (lattice_md.cpp:39-103,
// LLG_flat_kernel in lattice_gpu.cu:73-117):
//     H_i  = -B_i + 2 A_i S_i + sum_n J_n S_p(n) - drive(t)
//     dS_i/dt = H_i x S_i
// advanced by classic RK4 with the reference GPU stepper's arithmetic
// (integrator.cuh:115-139): stage inputs y + (c dt) k, final
// y += dt/6 (k1 + 2 k2 + 2 k3 + k4).
//
// Layout on chip (B200: 227 KB shared memory and 64K registers per CTA):
//   * one thread owns CPT groups (unit cells) of NAT sites; y_n, the RK
//     accumulator and its own current stage input stay in registers;
//   * the stage input every neighbour needs is published in shared memory,
//     double buffered, class-major SoA: buf[(atom*3 + comp)*G + group], so a
//     warp's 32 consecutive groups hit 32 consecutive doubles;
//   * bonds whose partner lives in the thread's own cell ("local" slots,
//     partner atom (a+1+n) % NAT) are read from registers, all others from
//     shared memory through per-thread int32 offsets loaded once;
//   * the coupling matrices are identical for every cell (checked on the host),
//     so they are kernel parameters: compile-time-indexed constant-bank
//     operands of the DFMAs, no loads at all.
// One __syncthreads per stage.  The observables of step n (M_af, M_local,
// M_global and E) come out of stage 0 of step n (E = 1/2 sum_i S_i.(H_i - B_i)
// from the static field of that stage), are warp-reduced with a butterfly that
// moves NV values in ~NV+log2(32/NV) shuffles, and are finished by one warp
// after the next barrier.  No atomics: every sum has a fixed order.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace cmd {

template <int NAT, int Z>
struct Couplings {
    double J[NAT][Z][9];      // slot-ordered, local slots first
    double field[NAT][3];
    double onsite[NAT][9];
    double frame[NAT][9];
    double afm[NAT];
    double d1[NAT][3];        // pulse directions (frame-rotated)
    double d2[NAT][3];
    int zc[NAT];              // slots in use per class (<= Z)
    int has_field;
    int has_onsite;
};

struct Pulse {
    double t1, t2, a1, a2;
};

struct ResidentArgs {
    int G;                    // groups (cells) per trajectory
    int nonlocal;             // offsets per (group, atom) in nbr
    long long n_steps;
    long long save_every;
    double T0, dt;
    double inv_n;             // unused (kept for ABI of the launch struct)
    double n_sites;           // N as a double (observables are divided by N)
    const int* nbr;           // [G][NAT][nonlocal]
    const double* y0;         // [B or 1][N*3]
    long long y0_stride;      // doubles between trajectories (0: shared)
    double* y_out;            // [B][N*3] or nullptr
    double* obs;              // [B][rows][10] or nullptr
    long long rows;           // rows per trajectory
    double* traj;             // [B][rows][N*3] or nullptr
    const Pulse* pulses;      // [B] or nullptr
    double width, freq;
};

constexpr int kRedStride = 16;  // doubles per warp in the reduction scratch

// Reduce NV (power of two, <= 32) per-lane values over the warp.  Afterwards
// lane l holds the total of value index l / (32 / NV).
template <int NV>
__device__ __forceinline__ double warp_reduce_many(double (&v)[NV]) {
    const int lane = threadIdx.x & 31;
    int o = 16;
#pragma unroll
    for (int half = NV / 2; half >= 1; half >>= 1) {
        const bool upper = (lane & o) != 0;
#pragma unroll
        for (int j = 0; j < half; ++j) {
            const double keep = upper ? v[j + half] : v[j];
            const double send = upper ? v[j] : v[j + half];
            v[j] = keep + __shfl_xor_sync(0xffffffffu, send, o);
        }
        o >>= 1;
    }
    double r = v[0];
#pragma unroll
    for (int q = 16 / NV; q >= 1; q >>= 1) r += __shfl_xor_sync(0xffffffffu, r, q);
    return r;
}

template <int NAT>
struct NVals {
    static constexpr int used = 3 * NAT + 1;
    static constexpr int value = used <= 4 ? 4 : (used <= 8 ? 8 : (used <= 16 ? 16 : 32));
};

// Drive envelope of lattice_md.cpp:45-56: a * exp(-(x/(2w))^2) * cos(freq x).
__device__ __forceinline__ double drive_factor(double amp, double x, double width, double freq) {
    const double u = x / (2.0 * width);
    return amp * exp(-(u * u)) * cos(freq * x);
}

template <int NAT, int Z, int LZ, int CPT, int MAXT>
__global__ void __launch_bounds__(MAXT, 1)
rk4_resident_kernel(const __grid_constant__ Couplings<NAT, Z> cp,
                    const __grid_constant__ ResidentArgs a) {
    constexpr int NL = Z - LZ;                       // non-local slots per atom
    constexpr int NV = NVals<NAT>::value;
    extern __shared__ double smem[];
    const int G = a.G;
    const int SB = NAT * 3 * G;                      // one stage buffer
    double* bufA = smem;
    double* bufB = smem + SB;
    double* red = bufB + SB;                         // [32][kRedStride]
    double* fin = red + 32 * kRedStride;             // [16] final-combine scratch
    double* drv = fin + 16;                          // [2][6] drive factors

    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
    const long long b = blockIdx.x;

    double y[CPT][NAT][3], acc[CPT][NAT][3], yc[CPT][NAT][3];
    int nb[CPT][NAT][NL > 0 ? NL : 1];
    bool own[CPT];

    const double* y0 = a.y0 + b * a.y0_stride;
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
        const int g = tid + k * blockDim.x;
        own[k] = g < G;
#pragma unroll
        for (int at = 0; at < NAT; ++at) {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const double v = own[k] ? y0[((long long)g * NAT + at) * 3 + c] : 0.0;
                y[k][at][c] = v;
                yc[k][at][c] = v;
                acc[k][at][c] = 0.0;
                if (own[k]) bufA[(at * 3 + c) * G + g] = v;
            }
#pragma unroll
            for (int m = 0; m < NL; ++m)
                nb[k][at][m] = own[k] ? a.nbr[((long long)g * NAT + at) * NL + m] : 0;
        }
    }

    Pulse pl{0.0, 0.0, 0.0, 0.0};
    if (a.pulses) pl = a.pulses[b];
    const bool drive_on = a.pulses != nullptr && (pl.a1 != 0.0 || pl.a2 != 0.0);
    const double dt = a.dt;
    double t = a.T0;

    // drive factors for step 0: lanes 0..5 of the last warp
    if (drive_on && warp == nwarps - 1 && lane < 6) {
        const double tt = t + (lane < 2 ? 0.0 : (lane < 4 ? 0.5 * dt : dt));
        drv[lane] = (lane & 1) ? drive_factor(pl.a2, tt - pl.t2, a.width, a.freq)
                               : drive_factor(pl.a1, tt - pl.t1, a.width, a.freq);
    }
    __syncthreads();

    // Field at the current stage input for (k, at); returns static field in Hs.
    auto field_at = [&](const double* in, int k, int at, double (&H)[3]) {
        const double S0 = yc[k][at][0], S1 = yc[k][at][1], S2 = yc[k][at][2];
        if (cp.has_field) {
            H[0] = -cp.field[at][0]; H[1] = -cp.field[at][1]; H[2] = -cp.field[at][2];
        } else {
            H[0] = 0.0; H[1] = 0.0; H[2] = 0.0;
        }
        if (cp.has_onsite) {
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                H[d] += 2.0 * cp.onsite[at][3 * d + 0] * S0;
                H[d] += 2.0 * cp.onsite[at][3 * d + 1] * S1;
                H[d] += 2.0 * cp.onsite[at][3 * d + 2] * S2;
            }
        }
#pragma unroll
        for (int n = 0; n < LZ; ++n) {
            const int pb = (at + 1 + n) % NAT;
            const double P0 = yc[k][pb][0], P1 = yc[k][pb][1], P2 = yc[k][pb][2];
#pragma unroll
            for (int d = 0; d < 3; ++d)
                H[d] += cp.J[at][n][3 * d] * P0 + cp.J[at][n][3 * d + 1] * P1 + cp.J[at][n][3 * d + 2] * P2;
        }
#pragma unroll
        for (int m = 0; m < NL; ++m) {
            const int n = LZ + m;
            if (n < cp.zc[at]) {
                const double* p = in + nb[k][at][m];
                const double P0 = p[0], P1 = p[G], P2 = p[2 * G];
#pragma unroll
                for (int d = 0; d < 3; ++d)
                    H[d] += cp.J[at][n][3 * d] * P0 + cp.J[at][n][3 * d + 1] * P1 + cp.J[at][n][3 * d + 2] * P2;
            }
        }
    };

    // Per-thread observable partials -> per-warp totals in red[warp][*].
    auto reduce_partials = [&](double (&part)[NV]) {
        const double r = warp_reduce_many<NV>(part);
        constexpr int span = 32 / NV;
        if ((lane % span) == 0) red[warp * kRedStride + lane / span] = r;
    };
    // One warp sums the per-warp totals and writes the 10-double row.
    auto finish_row = [&](long long row) {
        if (warp != 0) return;
        constexpr int used = NVals<NAT>::used;
        double s = 0.0;
        if (lane < used)
            for (int w = 0; w < nwarps; ++w) s += red[w * kRedStride + lane];
        if (lane < used) fin[lane] = s;
        __syncwarp();
        if (lane == 0 && a.obs) {
            double ml[3] = {0, 0, 0}, mg[3] = {0, 0, 0}, ma[3] = {0, 0, 0};
#pragma unroll
            for (int at = 0; at < NAT; ++at) {
                const double m0 = fin[3 * at], m1 = fin[3 * at + 1], m2 = fin[3 * at + 2];
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    ml[d] += fin[3 * at + d];
                    const double r = cp.frame[at][3 * d] * m0 + cp.frame[at][3 * d + 1] * m1 +
                                     cp.frame[at][3 * d + 2] * m2;
                    mg[d] += r;
                    ma[d] += cp.afm[at] * r;
                }
            }
            double* o = a.obs + (b * a.rows + row) * 10;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                o[d] = ma[d] / a.n_sites;
                o[3 + d] = ml[d] / a.n_sites;
                o[6 + d] = mg[d] / a.n_sites;
            }
            o[9] = 0.5 * fin[3 * NAT] / a.n_sites;
        }
    };
    auto write_traj = [&](long long row) {
        if (!a.traj) return;
        double* dst = a.traj + (b * a.rows + row) * (long long)G * NAT * 3;
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            if (!own[k]) continue;
            const int g = tid + k * blockDim.x;
#pragma unroll
            for (int at = 0; at < NAT; ++at)
#pragma unroll
                for (int c = 0; c < 3; ++c) dst[((long long)g * NAT + at) * 3 + c] = y[k][at][c];
        }
    };

    long long row = 0;
    bool pending = false;       // a row's per-warp totals wait in red[]
    double* in = bufA;
    double* out = bufB;
    for (long long step = 0; step < a.n_steps; ++step) {
        const bool observe = (step % a.save_every) == 0;
        const double* dv = drv + 6 * (step & 1);
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            double f1 = 0.0, f2 = 0.0;
            if (drive_on) {
                const int ti = s == 0 ? 0 : (s == 3 ? 2 : 1);
                f1 = dv[2 * ti];
                f2 = dv[2 * ti + 1];
            }
            double part[NV];
#pragma unroll
            for (int q = 0; q < NV; ++q) part[q] = 0.0;
#pragma unroll
            for (int k = 0; k < CPT; ++k) {
                if (!own[k]) continue;
                const int g = tid + k * blockDim.x;
                double nx[NAT][3];
#pragma unroll
                for (int at = 0; at < NAT; ++at) {
                    double H[3];
                    field_at(in, k, at, H);
                    const double S0 = yc[k][at][0], S1 = yc[k][at][1], S2 = yc[k][at][2];
                    if (s == 0 && observe) {
                        part[3 * at] += S0; part[3 * at + 1] += S1; part[3 * at + 2] += S2;
                        part[3 * NAT] += S0 * (H[0] - cp.field[at][0]) + S1 * (H[1] - cp.field[at][1]) +
                                         S2 * (H[2] - cp.field[at][2]);
                    }
                    if (drive_on) {
#pragma unroll
                        for (int d = 0; d < 3; ++d) H[d] -= cp.d1[at][d] * f1 + cp.d2[at][d] * f2;
                    }
                    const double k0 = H[1] * S2 - H[2] * S1;
                    const double k1 = H[2] * S0 - H[0] * S2;
                    const double k2 = H[0] * S1 - H[1] * S0;
                    const double kk[3] = {k0, k1, k2};
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        if (s == 0) {
                            acc[k][at][c] = kk[c];
                            nx[at][c] = 1.0 * y[k][at][c] + (0.5 * dt) * kk[c];
                        } else if (s == 1) {
                            acc[k][at][c] = acc[k][at][c] + 2.0 * kk[c];
                            nx[at][c] = 1.0 * y[k][at][c] + (0.5 * dt) * kk[c];
                        } else if (s == 2) {
                            acc[k][at][c] = acc[k][at][c] + 2.0 * kk[c];
                            nx[at][c] = 1.0 * y[k][at][c] + dt * kk[c];
                        } else {
                            y[k][at][c] += (dt / 6.0) * (acc[k][at][c] + kk[c]);
                            nx[at][c] = y[k][at][c];
                        }
                    }
                }
#pragma unroll
                for (int at = 0; at < NAT; ++at)
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        yc[k][at][c] = nx[at][c];
                        out[(at * 3 + c) * G + g] = nx[at][c];
                    }
            }
            if (s == 0 && observe) {
                write_traj(row);
                reduce_partials(part);
            }
            if (s == 1 && pending) {
                finish_row(row);
                ++row;
                pending = false;
            }
            if (s == 3 && drive_on && warp == nwarps - 1 && lane < 6) {
                const double tn = t + dt;
                const double tt = tn + (lane < 2 ? 0.0 : (lane < 4 ? 0.5 * dt : dt));
                drv[6 * ((step + 1) & 1) + lane] =
                    (lane & 1) ? drive_factor(pl.a2, tt - pl.t2, a.width, a.freq)
                               : drive_factor(pl.a1, tt - pl.t1, a.width, a.freq);
            }
            __syncthreads();
            if (s == 0 && observe) pending = true;
            double* tmp = in; in = out; out = tmp;
        }
        t += dt;
    }
    if (pending) {          // defensive: stage 1 always follows stage 0 inside a step
        finish_row(row);
        ++row;
        pending = false;
        __syncthreads();
    }
    // Final observation of y(t_end): one more static-field evaluation for E.
    {
        double part[NV];
#pragma unroll
        for (int q = 0; q < NV; ++q) part[q] = 0.0;
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            if (!own[k]) continue;
#pragma unroll
            for (int at = 0; at < NAT; ++at) {
                double H[3];
                field_at(in, k, at, H);
                const double S0 = yc[k][at][0], S1 = yc[k][at][1], S2 = yc[k][at][2];
                part[3 * at] += S0; part[3 * at + 1] += S1; part[3 * at + 2] += S2;
                part[3 * NAT] += S0 * (H[0] - cp.field[at][0]) + S1 * (H[1] - cp.field[at][1]) +
                                 S2 * (H[2] - cp.field[at][2]);
            }
        }
        write_traj(row);
        reduce_partials(part);
        __syncthreads();
        finish_row(row);
    }
    if (a.y_out) {
        double* dst = a.y_out + b * (long long)G * NAT * 3;
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            if (!own[k]) continue;
            const int g = tid + k * blockDim.x;
#pragma unroll
            for (int at = 0; at < NAT; ++at)
#pragma unroll
                for (int c = 0; c < 3; ++c) dst[((long long)g * NAT + at) * 3 + c] = y[k][at][c];
        }
    }
}

}  // namespace cmd
