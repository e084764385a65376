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
//   * one thread owns CPT groups (unit cells) of NAT sites; y_n and the RK
//     accumulator stay in registers for the whole trajectory (and, with YREG,
//     the thread's own current stage input too);
//   * the stage input every neighbour needs is published in shared memory,
//     double buffered, class-major SoA: buf[(atom*3 + comp)*G + group], so a
//     warp's 32 consecutive groups hit 32 consecutive doubles;
//   * bonds whose partner lives in the thread's own cell ("local" slots,
//     partner atom (a+1+n) % NAT) never touch shared memory; all others are
//     read through per-thread int32 offsets loaded once;
//   * the coupling matrices are identical for every cell (checked on the host),
//     so they are kernel parameters: compile-time-indexed constant-bank
//     operands of the DFMAs, no loads at all.
// One __syncthreads per stage, and nothing serial sits in front of it:
//   * the pulse envelopes of every stage time come from a table filled by a
//     parallel pre-pass (drive_table_kernel), loaded one step ahead;
//   * the per-step observables leave as raw sums (sum of S per atom class and
//     sum_i S_i.(H_i - B_i) over the static field of stage 0), warp-reduced
//     with a butterfly that moves NV values in ~NV+log2(32/NV) shuffles and
//     finished in parallel (warp q sums value q over the warps); a post-pass
//     (finish_rows_kernel) applies the frames and the 1/N.
// No atomics: every sum has a fixed order.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "drive.cuh"

namespace cmd {

template <int NAT, int Z>
struct Couplings {
    double J[NAT][Z][9];      // slot-ordered, local slots first
    double field[NAT][3];
    double onsite[NAT][9];
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
    long long B;              // trajectories
    long long n_steps;
    long long save_every;
    double T0, dt;
    const int* nbr;           // [G][NAT][Z-LZ]
    const double* y0;         // [B or 1][N*3]
    long long y0_stride;      // doubles between trajectories (0: shared)
    double* y_out;            // [B][N*3] or nullptr
    double* raw;              // [B][rows][raw_stride] raw observable sums, or nullptr
    long long raw_stride;     // doubles per raw row (>= 3*NAT+1)
    long long rows;           // rows per trajectory
    double* traj;             // [B][rows][N*3] or nullptr
    const double* drive;      // [B][n_steps][6] envelope table, or nullptr (no drive)
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
    static constexpr int used = 3 * NAT + 1;      // sum S per atom class, then sum S.(H-B)
    static constexpr int value = used <= 4 ? 4 : (used <= 8 ? 8 : (used <= 16 ? 16 : 32));
};

// h += j0*p0 + j1*p1 + j2*p2 as a chain of three fused multiply-adds (one
// rounding per term; the plain expression costs a DMUL, two DFMAs and a DADD).
__device__ __forceinline__ void bond_acc(double& h, double j0, double j1, double j2, double p0, double p1,
                                         double p2) {
    h = fma(j0, p0, h);
    h = fma(j1, p1, h);
    h = fma(j2, p2, h);
}

template <int V>
struct AtomTag {
    static constexpr int value = V;
};

// f(AtomTag<at>) with `at` (0 <= at < NAT) as a compile-time constant, so the
// couplings of the atom stay constant-bank operands.
template <int NAT, int AT = 0, class F>
__device__ __forceinline__ void with_atom(int at, F&& f) {
    if constexpr (AT < NAT) {
        if (at == AT)
            f(AtomTag<AT>{});
        else
            with_atom<NAT, AT + 1>(at, f);
    }
}

// h -= d1*f1 + d2*f2 as two fused multiply-adds.
__device__ __forceinline__ void drive_acc(double& h, double d1, double d2, double f1, double f2) {
    h = fma(-d1, f1, h);
    h = fma(-d2, f2, h);
}


// Envelope table [B][n_steps][6]: for each step n the factors (pulse 1, pulse 2)
// at t_n, t_n + dt/2 and t_n + dt, t_n the accumulated time of the reference loop.
static __global__ void drive_table_kernel(const Pulse* __restrict__ pulses, const double* __restrict__ times,
                                   long long n_steps, double dt, double width, double freq, long long B,
                                   double* __restrict__ out) {
    const long long total = B * n_steps * 6;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const long long b = e / (n_steps * 6);
        const long long r = e - b * n_steps * 6;
        const long long n = r / 6;
        const int q = (int)(r - n * 6);
        const double t = times[n];
        const double tt = q < 2 ? t : (q < 4 ? t + 0.5 * dt : t + dt);
        const Pulse p = pulses[b];
        out[e] = (q & 1) ? drive_factor(p.a2, tt - p.t2, width, freq)
                         : drive_factor(p.a1, tt - p.t1, width, freq);
    }
}

// Raw sums -> {M_af[3], M_local[3], M_global[3], E/N} rows.  `raw` may alias
// `obs` (raw_stride 10): each row is read completely before it is written.
template <int NAT>
__global__ void finish_rows_kernel(const double* raw, long long raw_stride, long long n_rows_total,
                                   const double* __restrict__ frames, const double* __restrict__ afm,
                                   double n_sites, double* obs) {
    constexpr int NR = 3 * NAT + 1;
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < n_rows_total;
         r += (long long)gridDim.x * blockDim.x) {
        double m[NR];
#pragma unroll
        for (int q = 0; q < NR; ++q) m[q] = raw[r * raw_stride + q];
        double ml[3] = {0, 0, 0}, mg[3] = {0, 0, 0}, ma[3] = {0, 0, 0};
#pragma unroll
        for (int at = 0; at < NAT; ++at) {
            const double* R = frames + 9 * at;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                ml[d] += m[3 * at + d];
                const double v = R[3 * d] * m[3 * at] + R[3 * d + 1] * m[3 * at + 1] + R[3 * d + 2] * m[3 * at + 2];
                mg[d] += v;
                ma[d] += afm[at] * v;
            }
        }
        double* o = obs + r * 10;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            o[d] = ma[d] / n_sites;
            o[3 + d] = ml[d] / n_sites;
            o[6 + d] = mg[d] / n_sites;
        }
        o[9] = 0.5 * m[3 * NAT] / n_sites;
    }
}

template <int NAT, int Z, int LZ, int CPT, int MAXT, int MINB, bool YREG, int TPC>
__global__ void __launch_bounds__(MAXT, MINB)
rk4_resident_kernel(const __grid_constant__ Couplings<NAT, Z> cp,
                    const __grid_constant__ ResidentArgs a) {
    constexpr int NL = Z - LZ;                       // non-local slots per atom
    constexpr int NR = NVals<NAT>::used;             // observables per trajectory
    constexpr int NRT = NR * TPC;                    // observables of the CTA's trajectories
    constexpr int NV = NRT <= 4 ? 4 : (NRT <= 8 ? 8 : 16);
    static_assert(NRT <= kRedStride, "observables of a CTA must fit one reduction row");
    extern __shared__ double smem[];
    const int G = a.G;
    const int SB = NAT * 3 * G;                      // one stage buffer
    // Trajectory t of this CTA keeps its two stage buffers at t*2*SB (+ 0 / SB).
    // Shared memory is addressed through 32-bit offsets, which keeps the
    // addressing in the shared window and in 32-bit registers.
    double* red = smem + TPC * 2 * SB;               // [32][kRedStride]
    double* drv = red + 32 * kRedStride;             // [TPC][2][6] envelopes of the current / next step

    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
    const long long b0 = (long long)blockIdx.x * TPC;
    const int ntr = (int)(a.B - b0 < TPC ? a.B - b0 : TPC);   // trajectories of this CTA (uniform)

    double y[TPC][CPT][NAT][3], acc[TPC][CPT][NAT][3];
    double yc[YREG ? TPC : 1][YREG ? CPT : 1][NAT][3];
    int nb[CPT][NAT][NL > 0 ? NL : 1];

#pragma unroll
    for (int t = 0; t < TPC; ++t) {
        const double* y0 = a.y0 + (b0 + t) * a.y0_stride;
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            const int g = tid + k * blockDim.x;
            const bool own = g < G && t < ntr;
#pragma unroll
            for (int at = 0; at < NAT; ++at)
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const double v = own ? y0[((long long)g * NAT + at) * 3 + c] : 0.0;
                    y[t][k][at][c] = v;
                    if (YREG) yc[YREG ? t : 0][YREG ? k : 0][at][c] = v;
                    acc[t][k][at][c] = 0.0;
                    if (own) smem[t * 2 * SB + (at * 3 + c) * G + g] = v;
                }
        }
    }
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
        const int g = tid + k * blockDim.x;
#pragma unroll
        for (int at = 0; at < NAT; ++at)
#pragma unroll
            for (int m = 0; m < NL; ++m) nb[k][at][m] = g < G ? a.nbr[((long long)g * NAT + at) * NL + m] : 0;
    }

    const bool drive_on = a.drive != nullptr;
    const double dt = a.dt;
    // Lanes 0..6*TPC-1 of warp 0 stage the envelopes (lane l: trajectory l/6,
    // value l%6): loaded during stage 0 of step n for step n+1, stored to drv[]
    // during stage 2, read by everyone after the stage-3 barrier.  Nothing
    // waits on the global load.
    const int st_t = lane / 6, st_e = lane - 6 * (lane / 6);
    const bool stager = drive_on && warp == 0 && lane < 6 * TPC && st_t < ntr;
    const double* dtab = stager ? a.drive + (b0 + st_t) * a.n_steps * 6 : nullptr;
    if (stager && a.n_steps > 0) drv[st_t * 12 + st_e] = dtab[st_e];
    __syncthreads();

    // Static field at the current stage input (buffer offset `in`) of cell k,
    // atom at.  S[][] holds the cell's NAT stage-input spins.
    auto field_at = [&](int in, int k, int at, const double (&S)[NAT][3], double (&H)[3]) {
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
                const int p = in + nb[k][at][m];
                const double P0 = smem[p], P1 = smem[p + G], P2 = smem[p + 2 * G];
#pragma unroll
                for (int d = 0; d < 3; ++d)
                    bond_acc(H[d], cp.J[at][n][3 * d], cp.J[at][n][3 * d + 1], cp.J[at][n][3 * d + 2], P0, P1, P2);
            }
        }
    };
    auto load_cell = [&](int in, int t, int k, double (&S)[NAT][3]) {
        const int g = tid + k * blockDim.x;
#pragma unroll
        for (int at = 0; at < NAT; ++at)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                if (YREG) S[at][c] = yc[YREG ? t : 0][YREG ? k : 0][at][c];
                else S[at][c] = smem[in + (at * 3 + c) * G + g];
            }
    };
    // Per-thread partials -> per-warp totals in red[warp][*].
    auto reduce_partials = [&](double (&part)[NV]) {
        const double r = warp_reduce_many<NV>(part);
        constexpr int span = 32 / NV;
        if ((lane % span) == 0) red[warp * kRedStride + lane / span] = r;
    };
    // Warp q sums value q (q = warp, warp + nwarps, ...) over the warps and
    // writes it to its trajectory's row (runs after a barrier).
    auto finish_raw = [&](long long row) {
        if (a.raw == nullptr) return;
        for (int q = warp; q < NRT; q += nwarps) {
            double s = lane < nwarps ? red[lane * kRedStride + q] : 0.0;
#pragma unroll
            for (int o = 16; o >= 1; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            const int t = q / NR;
            if (lane == 0 && t < ntr) a.raw[((b0 + t) * a.rows + row) * a.raw_stride + (q - t * NR)] = s;
        }
    };
    auto write_traj = [&](long long row) {
        if (!a.traj) return;
#pragma unroll
        for (int t = 0; t < TPC; ++t) {
            if (t >= ntr) continue;
            double* dst = a.traj + ((b0 + t) * a.rows + row) * (long long)G * NAT * 3;
#pragma unroll
            for (int k = 0; k < CPT; ++k) {
                const int g = tid + k * blockDim.x;
                if (g >= G) continue;
#pragma unroll
                for (int at = 0; at < NAT; ++at)
#pragma unroll
                    for (int c = 0; c < 3; ++c) dst[((long long)g * NAT + at) * 3 + c] = y[t][k][at][c];
            }
        }
    };

    long long row = 0;
    long long save_left = 0;            // steps until the next saved row
    int in = 0;          // offset (within a trajectory's pair) of the buffer holding the current stage input
    int out = SB;
    // Observables of step n: summed per thread during stage 0, warp-reduced at
    // the start of stage 1 (off the stage-0 barrier's critical path, next to
    // stage 1's own work), finished across warps and written in stage 2.
    double part[NV];
    for (long long step = 0; step < a.n_steps; ++step) {
        const bool observe = save_left == 0;
        save_left = observe ? a.save_every - 1 : save_left - 1;
        double next_f = 0.0;
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            if (s == 0 && stager && step + 1 < a.n_steps) next_f = dtab[(step + 1) * 6 + st_e];
            if (s == 2 && stager && step + 1 < a.n_steps) drv[st_t * 12 + 6 * ((step + 1) & 1) + st_e] = next_f;
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
#pragma unroll
            for (int t = 0; t < TPC; ++t) {
                if (t >= ntr) continue;
                const int tin = t * 2 * SB + in, tout = t * 2 * SB + out;
                const double* dv = drv + t * 12 + 6 * (step & 1);
                const double f1 = drive_on ? dv[2 * ti] : 0.0;
                const double f2 = drive_on ? dv[2 * ti + 1] : 0.0;
                const bool drive_now = drive_on && (f1 != 0.0 || f2 != 0.0);   // 0*d adds exactly 0
#pragma unroll
                for (int k = 0; k < CPT; ++k) {
                    const int g = tid + k * blockDim.x;
                    if (g >= G) continue;
                    double S[NAT][3];
                    load_cell(tin, t, k, S);
                    double nx[YREG ? NAT : 1][3];
#pragma unroll
                    for (int at = 0; at < NAT; ++at) {
                        double H[3];
                        field_at(tin, k, at, S, H);
                        if (s == 0 && observe) {
                            part[t * NR + 3 * at] += S[at][0];
                            part[t * NR + 3 * at + 1] += S[at][1];
                            part[t * NR + 3 * at + 2] += S[at][2];
                            part[t * NR + 3 * NAT] += S[at][0] * (H[0] - cp.field[at][0]) +
                                                      S[at][1] * (H[1] - cp.field[at][1]) +
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
                                acc[t][k][at][c] = kk[c];
                                v = 1.0 * y[t][k][at][c] + (0.5 * dt) * kk[c];
                            } else if (s == 1) {
                                acc[t][k][at][c] = acc[t][k][at][c] + 2.0 * kk[c];
                                v = 1.0 * y[t][k][at][c] + (0.5 * dt) * kk[c];
                            } else if (s == 2) {
                                acc[t][k][at][c] = acc[t][k][at][c] + 2.0 * kk[c];
                                v = 1.0 * y[t][k][at][c] + dt * kk[c];
                            } else {
                                y[t][k][at][c] += (dt / 6.0) * (acc[t][k][at][c] + kk[c]);
                                v = y[t][k][at][c];
                            }
                            if (YREG) nx[YREG ? at : 0][c] = v;     // own registers change after the cell
                            else smem[tout + (at * 3 + c) * G + g] = v;
                        }
                    }
                    if (YREG) {
#pragma unroll
                        for (int at = 0; at < NAT; ++at)
#pragma unroll
                            for (int c = 0; c < 3; ++c) {
                                yc[YREG ? t : 0][YREG ? k : 0][at][c] = nx[YREG ? at : 0][c];
                                smem[tout + (at * 3 + c) * G + g] = nx[YREG ? at : 0][c];
                            }
                    }
                }
            }
            if (s == 0 && observe) write_traj(row);
            __syncthreads();
            const int tmp = in; in = out; out = tmp;
        }
    }
    // Final observation of y(t_end): one more static-field evaluation for E.
    {
#pragma unroll
        for (int q = 0; q < NV; ++q) part[q] = 0.0;
#pragma unroll
        for (int t = 0; t < TPC; ++t) {
            if (t >= ntr) continue;
            const int tin = t * 2 * SB + in;
#pragma unroll
            for (int k = 0; k < CPT; ++k) {
                const int g = tid + k * blockDim.x;
                if (g >= G) continue;
                double S[NAT][3];
                load_cell(tin, t, k, S);
#pragma unroll
                for (int at = 0; at < NAT; ++at) {
                    double H[3];
                    field_at(tin, k, at, S, H);
                    part[t * NR + 3 * at] += S[at][0];
                    part[t * NR + 3 * at + 1] += S[at][1];
                    part[t * NR + 3 * at + 2] += S[at][2];
                    part[t * NR + 3 * NAT] += S[at][0] * (H[0] - cp.field[at][0]) + S[at][1] * (H[1] - cp.field[at][1]) +
                                              S[at][2] * (H[2] - cp.field[at][2]);
                }
            }
        }
        write_traj(row);
        reduce_partials(part);
        __syncthreads();
        finish_raw(row);
    }
    if (a.y_out) {
#pragma unroll
        for (int t = 0; t < TPC; ++t) {
            if (t >= ntr) continue;
            double* dst = a.y_out + (b0 + t) * (long long)G * NAT * 3;
#pragma unroll
            for (int k = 0; k < CPT; ++k) {
                const int g = tid + k * blockDim.x;
                if (g >= G) continue;
#pragma unroll
                for (int at = 0; at < NAT; ++at)
#pragma unroll
                    for (int c = 0; c < 3; ++c) dst[((long long)g * NAT + at) * 3 + c] = y[t][k][at][c];
            }
        }
    }
}

}  // namespace cmd
