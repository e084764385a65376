// rk_global.cuh -- persistent CTA-per-trajectory integrator with the state in
// global memory: controlled Dormand-Prince 5(4), fixed-step Dormand-Prince and
// a global-memory RK4 for lattices too large for the resident kernel.
//
// Same right-hand side and cell layout as rk4_resident.cuh (couplings as
// compile-time-indexed kernel parameters, cell-major SoA vectors
// v[(atom*3 + comp)*G + cell]), but every RK vector lives in a per-trajectory
// global workspace (L2-resident for the lattice sizes of an uneven batch), so
// any number of cells fits and seven stage derivatives can be kept.
//
// A launch is persistent: each CTA pulls trajectory indices from a queue
// (host-sorted longest first) until the batch is drained, so trajectories of
// very different sizes and step counts load-balance.  Two lattice types (two
// coupling sets, e.g. honeycomb and pyrochlore) can be mixed in one launch.
//
// Step control of the controlled mode follows the CPU path of the reference
// (Boost.Odeint make_controlled<runge_kutta_dopri5> driven by
// integrate_adaptive, lattice.h:4072-4078): error
//   max_i |x_err_i| / (abs + rel (|x_i| + dt |dxdt_i|)),
// reject when > 1 with dt *= max(0.9 err^(-1/3), 0.2), otherwise accept and
// when err < 0.5 grow dt *= 0.9 max(err, 5^-5)^(-1/5); the last step is cut to
// land on T_end; FSAL reuse of the last stage.  The error max is a
// per-CTA block reduction, so every thread takes the same decision.
#pragma once

#include "rk4_resident.cuh"
#include "rk_fixed.cuh"

namespace cmd {

// Steps of the fixed-step methods over one CTA: the own elements of a thread are
// its cells' NAT*3 entries, the barrier is the CTA's (rk_fixed.cuh).
template <class R, class E>
struct CtaStepCtx {
    const R& rhs_f;
    const E& each_f;
    __device__ void rhs(const double* Y, double* K, double ts) const { rhs_f(Y, K, ts); }
    template <class F>
    __device__ void each(F&& f) const { each_f(f); }
    __device__ void sync() const { __syncthreads(); }
};

constexpr int kGVectors = 12;   // y, ynew, Ya, Yb, k1..k7, spare

struct GTraj {
    int type;                  // 0 or 1: which coupling set
    int G;                     // cells
    const int* nbr;            // [G][NAT][Z-LZ] offsets (atom*3*G + cell)
    const double* y0;          // AoS [N*3]
    double* yout;              // AoS [N*3] or nullptr
    double* work;              // kGVectors * NAT*3*G doubles
    double* rows;              // [max_rows][11] = {t, M_af, M_loc, M_glob, E/N}
    double* traj;              // [max_rows][N*3] AoS states of the rows, or nullptr
    long long max_rows;
    double T0, T1, dt0;
    long long n_steps;         // fixed-step modes: steps to take
    long long save_every;      // fixed-step modes
    Pulse pulse;               // a1 = a2 = 0: no drive
    long long* stat;           // [4] rows written, accepted, rejected, status (0 ok, 1 failed control)
};

struct GArgs {
    const GTraj* traj;
    int B;
    int* queue;                // zeroed before the launch
    int mode;
    double abs_tol, rel_tol;
    long long max_steps;       // controlled mode: cap on accepted steps (0: none)
    double width, freq;
    const double* frames0; const double* afm0;   // per type [NAT*9], [NAT] (device)
    const double* frames1; const double* afm1;
};

// dS/dt at the stage input Y for cell g (all NAT atoms), written to K.  When
// `part` is non-null it accumulates sum S per atom and S.(H_static - B).
template <int NAT, int Z, int LZ>
__device__ __forceinline__ void rhs_cell(const Couplings<NAT, Z>& cp, const double* __restrict__ Y,
                                         double* __restrict__ K, int G, int g, const int* __restrict__ nbr,
                                         double f1, double f2, bool drive, double* part) {
    constexpr int NL = Z - LZ;
    double S[NAT][3];
#pragma unroll
    for (int at = 0; at < NAT; ++at)
#pragma unroll
        for (int c = 0; c < 3; ++c) S[at][c] = Y[(at * 3 + c) * G + g];
#pragma unroll
    for (int at = 0; at < NAT; ++at) {
        double H[3];
        if (cp.has_field) {
            H[0] = -cp.field[at][0]; H[1] = -cp.field[at][1]; H[2] = -cp.field[at][2];
        } else {
            H[0] = 0.0; H[1] = 0.0; H[2] = 0.0;
        }
        if (cp.has_onsite) {
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                bond_acc(H[d], 2.0 * cp.onsite[at][3 * d], 2.0 * cp.onsite[at][3 * d + 1], 2.0 * cp.onsite[at][3 * d + 2], S[at][0], S[at][1], S[at][2]);
            }
        }
#pragma unroll
        for (int n = 0; n < LZ; ++n) {
            const int pb = (at + 1 + n) % NAT;
#pragma unroll
            for (int d = 0; d < 3; ++d)
                bond_acc(H[d], cp.J[at][n][3 * d], cp.J[at][n][3 * d + 1], cp.J[at][n][3 * d + 2], S[pb][0], S[pb][1], S[pb][2]);
        }
#pragma unroll
        for (int m = 0; m < NL; ++m) {
            const int n = LZ + m;
            if (n < cp.zc[at]) {
                const int p = nbr[((long long)g * NAT + at) * NL + m];
                const double P0 = Y[p], P1 = Y[p + G], P2 = Y[p + 2 * G];
#pragma unroll
                for (int d = 0; d < 3; ++d)
                    bond_acc(H[d], cp.J[at][n][3 * d], cp.J[at][n][3 * d + 1], cp.J[at][n][3 * d + 2], P0, P1, P2);
            }
        }
        if (part) {
            part[3 * at] += S[at][0]; part[3 * at + 1] += S[at][1]; part[3 * at + 2] += S[at][2];
            part[3 * NAT] += S[at][0] * (H[0] - cp.field[at][0]) + S[at][1] * (H[1] - cp.field[at][1]) +
                             S[at][2] * (H[2] - cp.field[at][2]);
        }
        if (drive) {
#pragma unroll
            for (int d = 0; d < 3; ++d) drive_acc(H[d], cp.d1[at][d], cp.d2[at][d], f1, f2);
        }
        K[(at * 3 + 0) * G + g] = H[1] * S[at][2] - H[2] * S[at][1];
        K[(at * 3 + 1) * G + g] = H[2] * S[at][0] - H[0] * S[at][2];
        K[(at * 3 + 2) * G + g] = H[0] * S[at][1] - H[1] * S[at][0];
    }
}

// Block-wide sum of NV per-thread values into out[0..used) (thread 0 only).
// Caller provides red[32][kRedStride]; contains one __syncthreads.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* red, int used, double* out) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const double r = warp_reduce_many<NV>(v);
    constexpr int span = 32 / NV;
    if ((lane % span) == 0) red[warp * kRedStride + lane / span] = r;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int q = 0; q < used; ++q) {
            double s = 0.0;
            for (int w = 0; w < nw; ++w) s += red[w * kRedStride + q];
            out[q] = s;
        }
    }
}

template <int NAT, int Z, int LZ, bool XM>
__device__ void run_trajectory(const Couplings<NAT, Z>& cp, const GTraj& T, const GArgs& a,
                               const double* frames, const double* afm, double* sh) {
    constexpr int NV = NVals<NAT>::value;
    constexpr int NR = NVals<NAT>::used;
    const int G = T.G;
    const long long V = (long long)NAT * 3 * G;
    double* y = T.work;
    double* yn = T.work + V;
    double* Ya = T.work + 2 * V;
    double* Yb = T.work + 3 * V;
    double* k[7];
#pragma unroll
    for (int j = 0; j < 7; ++j) k[j] = T.work + (4 + j) * V;
    double* red = sh;                    // [32][kRedStride]
    double* fin = sh + 32 * kRedStride;  // [16]: finished sums
    double* emx = fin + 16;              // [32]: per-warp error maxima
    const int tid = threadIdx.x, nt = blockDim.x;
    const bool drive = T.pulse.a1 != 0.0 || T.pulse.a2 != 0.0;
    const double N = (double)G * NAT;

    for (int g = tid; g < G; g += nt)
#pragma unroll
        for (int at = 0; at < NAT; ++at)
#pragma unroll
            for (int c = 0; c < 3; ++c) y[(at * 3 + c) * G + g] = T.y0[((long long)g * NAT + at) * 3 + c];
    __syncthreads();

    auto factors = [&](double ts, double& f1, double& f2) {
        f1 = drive ? drive_factor(T.pulse.a1, ts - T.pulse.t1, a.width, a.freq) : 0.0;
        f2 = drive ? drive_factor(T.pulse.a2, ts - T.pulse.t2, a.width, a.freq) : 0.0;
    };
    // RHS over all own cells: K = f(Y, ts); optional observable partial sums.
    auto rhs = [&](const double* Yin, double* K, double ts, double* part) {
        double f1, f2;
        factors(ts, f1, f2);
        for (int g = tid; g < G; g += nt) rhs_cell<NAT, Z, LZ>(cp, Yin, K, G, g, T.nbr, f1, f2, drive, part);
    };
    long long nrow = 0;
    // Records row nrow = {t, observables of Ystate}; every thread calls it.
    auto record = [&](double t, const double* part_total, const double* Ystate) {
        if (nrow < T.max_rows) {
            if (T.traj) {
                double* dst = T.traj + nrow * (long long)G * NAT * 3;
                for (int g = tid; g < G; g += nt)
                    for (int at = 0; at < NAT; ++at)
                        for (int c = 0; c < 3; ++c) dst[((long long)g * NAT + at) * 3 + c] = Ystate[(at * 3 + c) * G + g];
            }
            if (tid == 0) {
                double ml[3] = {0, 0, 0}, mg[3] = {0, 0, 0}, ma[3] = {0, 0, 0};
                for (int at = 0; at < NAT; ++at) {
                    const double* R = frames + 9 * at;
                    const double* m = part_total + 3 * at;
                    for (int d = 0; d < 3; ++d) {
                        ml[d] += m[d];
                        const double v = R[3 * d] * m[0] + R[3 * d + 1] * m[1] + R[3 * d + 2] * m[2];
                        mg[d] += v;
                        ma[d] += afm[at] * v;
                    }
                }
                double* o = T.rows + nrow * 11;
                o[0] = t;
                for (int d = 0; d < 3; ++d) {
                    o[1 + d] = ma[d] / N;
                    o[4 + d] = ml[d] / N;
                    o[7 + d] = mg[d] / N;
                }
                o[10] = 0.5 * part_total[3 * NAT] / N;
            }
        }
        ++nrow;
    };
    auto observe_rhs = [&](const double* Yin, double* K, double ts) {
        double part[NV];
#pragma unroll
        for (int q = 0; q < NV; ++q) part[q] = 0.0;
        rhs(Yin, K, ts, part);
        block_sum<NV>(part, red, NR, fin);
        __syncthreads();
        record(ts, fin, Yin);
    };

    long long acc_steps = 0, rej_steps = 0, status = 0;
    double t = T.T0;

    if (a.mode == kModeRK45) {
        static constexpr double a21 = 1.0 / 5.0;
        static constexpr double a31 = 3.0 / 40.0, a32 = 9.0 / 40.0;
        static constexpr double a41 = 44.0 / 45.0, a42 = -56.0 / 15.0, a43 = 32.0 / 9.0;
        static constexpr double a51 = 19372.0 / 6561.0, a52 = -25360.0 / 2187.0, a53 = 64448.0 / 6561.0,
                                a54 = -212.0 / 729.0;
        static constexpr double a61 = 9017.0 / 3168.0, a62 = -355.0 / 33.0, a63 = 46732.0 / 5247.0,
                                a64 = 49.0 / 176.0, a65 = -5103.0 / 18656.0;
        static constexpr double c2 = 1.0 / 5.0, c3 = 3.0 / 10.0, c4 = 4.0 / 5.0, c5 = 8.0 / 9.0;
        static constexpr double b1 = 35.0 / 384.0, b3 = 500.0 / 1113.0, b4 = 125.0 / 192.0,
                                b5 = -2187.0 / 6784.0, b6 = 11.0 / 84.0;
        static constexpr double dc1 = b1 - 5179.0 / 57600.0, dc3 = b3 - 7571.0 / 16695.0,
                                dc4 = b4 - 393.0 / 640.0, dc5 = b5 - (-92097.0 / 339200.0),
                                dc6 = b6 - 187.0 / 2100.0, dc7 = -1.0 / 40.0;
        const double eps = 2.220446049250313e-16;        // numeric_limits<double>::epsilon
        double dt = T.dt0;
        double* K1 = k[0];
        double* K7 = k[6];
        observe_rhs(y, K1, t);                           // first observer call + FSAL seed
        while (T.T1 - t > eps) {
            if ((t + dt) - T.T1 > eps) dt = T.T1 - t;
            int fails = 0;
            for (;;) {
                // stages 2..6 into alternating Y buffers, stage 7 into yn
                for (int g = tid; g < G; g += nt)
                    for (int e = 0; e < NAT * 3; ++e) {
                        const long long i = (long long)e * G + g;
                        Ya[i] = y[i] + dt * a21 * K1[i];
                    }
                __syncthreads();
                rhs(Ya, k[1], t + dt * c2, nullptr);
                for (int g = tid; g < G; g += nt)
                    for (int e = 0; e < NAT * 3; ++e) {
                        const long long i = (long long)e * G + g;
                        Yb[i] = y[i] + dt * a31 * K1[i] + dt * a32 * k[1][i];
                    }
                __syncthreads();
                rhs(Yb, k[2], t + dt * c3, nullptr);
                for (int g = tid; g < G; g += nt)
                    for (int e = 0; e < NAT * 3; ++e) {
                        const long long i = (long long)e * G + g;
                        Ya[i] = y[i] + dt * a41 * K1[i] + dt * a42 * k[1][i] + dt * a43 * k[2][i];
                    }
                __syncthreads();
                rhs(Ya, k[3], t + dt * c4, nullptr);
                for (int g = tid; g < G; g += nt)
                    for (int e = 0; e < NAT * 3; ++e) {
                        const long long i = (long long)e * G + g;
                        Yb[i] = y[i] + dt * a51 * K1[i] + dt * a52 * k[1][i] + dt * a53 * k[2][i] +
                                dt * a54 * k[3][i];
                    }
                __syncthreads();
                rhs(Yb, k[4], t + dt * c5, nullptr);
                for (int g = tid; g < G; g += nt)
                    for (int e = 0; e < NAT * 3; ++e) {
                        const long long i = (long long)e * G + g;
                        Ya[i] = y[i] + dt * a61 * K1[i] + dt * a62 * k[1][i] + dt * a63 * k[2][i] +
                                dt * a64 * k[3][i] + dt * a65 * k[4][i];
                    }
                __syncthreads();
                rhs(Ya, k[5], t + dt, nullptr);
                for (int g = tid; g < G; g += nt)
                    for (int e = 0; e < NAT * 3; ++e) {
                        const long long i = (long long)e * G + g;
                        yn[i] = y[i] + dt * b1 * K1[i] + dt * b3 * k[2][i] + dt * b4 * k[3][i] +
                                dt * b5 * k[4][i] + dt * b6 * k[5][i];
                    }
                __syncthreads();
                double part[NV];
#pragma unroll
                for (int q = 0; q < NV; ++q) part[q] = 0.0;
                rhs(yn, K7, t + dt, part);                // FSAL stage; observables of yn
                __syncthreads();
                double emax = 0.0;
                for (int g = tid; g < G; g += nt)
                    for (int e = 0; e < NAT * 3; ++e) {
                        const long long i = (long long)e * G + g;
                        const double err = dt * dc1 * K1[i] + dt * dc3 * k[2][i] + dt * dc4 * k[3][i] +
                                           dt * dc5 * k[4][i] + dt * dc6 * k[5][i] + dt * dc7 * K7[i];
                        const double r = fabs(err) / (a.abs_tol + a.rel_tol * (1.0 * fabs(y[i]) +
                                                                                1.0 * dt * fabs(K1[i])));
                        emax = fmax(emax, r);
                    }
                // block max (identical value in every thread) + observable sums
                double ev[NV];
#pragma unroll
                for (int q = 0; q < NV; ++q) ev[q] = part[q];
                block_sum<NV>(ev, red, NR, fin);          // sums in fin[0..NR)
                double wm = emax;
#pragma unroll
                for (int o = 16; o >= 1; o >>= 1) wm = fmax(wm, __shfl_xor_sync(0xffffffffu, wm, o));
                if ((tid & 31) == 0) emx[tid >> 5] = wm;
                __syncthreads();
                double err = 0.0;
                for (int w = 0; w < (nt >> 5); ++w) err = fmax(err, emx[w]);
                if (err > 1.0) {
                    dt *= fmax(0.9 * pow(err, -1.0 / 3.0), 0.2);
                    ++rej_steps;
                    __syncthreads();
                    if (++fails >= 500) { status = 1; break; }
                    continue;
                }
                // accept: t += dt, swap y/yn and K1/K7, observe, grow dt
                t += dt;
                double* tmp = y; y = yn; yn = tmp;
                tmp = K1; K1 = K7; K7 = tmp;
                record(t, fin, y);
                if (err < 0.5) {
                    err = fmax(pow(5.0, -5.0), err);
                    dt *= 0.9 * pow(err, -1.0 / 5.0);
                }
                ++acc_steps;
                __syncthreads();
                break;
            }
            if (status != 0) break;
            if (a.max_steps > 0 && acc_steps >= a.max_steps) break;
        }
    } else {
        // Fixed-step modes follow the reference GPU loop: rows every save_every
        // steps from the k1 evaluation, plus a final observation; the steps are
        // rk_fixed.cuh's (the methods past RK4 / DOPRI5 / Cash-Karp only in the
        // XM instance, so the RK45 kernel keeps its registers).
        auto rhs3 = [&](const double* Yin, double* K, double ts) { rhs(Yin, K, ts, nullptr); };
        auto each = [&](auto&& f) {
            for (int g = tid; g < G; g += nt)
                for (int e = 0; e < NAT * 3; ++e) f((long long)e * G + g);
        };
        const CtaStepCtx<decltype(rhs3), decltype(each)> ctx{rhs3, each};
        const double dt = T.dt0;
        long long save_left = 0;
        for (long long step = 0; step < T.n_steps; ++step) {
            const bool obs = save_left == 0;
            save_left = obs ? T.save_every - 1 : save_left - 1;
            if (obs) observe_rhs(y, k[0], t);
            else rhs(y, k[0], t, nullptr);
            fixed_step<XM>(a.mode, ctx, y, k, Ya, Yb, yn, t, dt);
            t += dt;
            ++acc_steps;
        }
        observe_rhs(y, k[0], t);
    }
    __syncthreads();
    if (T.yout)
        for (int g = tid; g < G; g += nt)
#pragma unroll
            for (int at = 0; at < NAT; ++at)
#pragma unroll
                for (int c = 0; c < 3; ++c) T.yout[((long long)g * NAT + at) * 3 + c] = y[(at * 3 + c) * G + g];
    if (tid == 0 && T.stat) {
        T.stat[0] = nrow;
        T.stat[1] = acc_steps;
        T.stat[2] = rej_steps;
        T.stat[3] = status;
    }
    __syncthreads();
}

template <int NA0, int Z0, int LZ0, int NA1, int Z1, int LZ1, bool XM>
__global__ void __launch_bounds__(256, 1)
rk_global_kernel(const __grid_constant__ Couplings<NA0, Z0> c0, const __grid_constant__ Couplings<NA1, Z1> c1,
                 const __grid_constant__ GArgs a) {
    __shared__ double sh[32 * kRedStride + 16 + 32];
    __shared__ int next;
    for (;;) {
        if (threadIdx.x == 0) next = atomicAdd(a.queue, 1);
        __syncthreads();
        const int b = next;
        __syncthreads();
        if (b >= a.B) break;
        const GTraj& T = a.traj[b];
        if (T.type == 0) run_trajectory<NA0, Z0, LZ0, XM>(c0, T, a, a.frames0, a.afm0, sh);
        else run_trajectory<NA1, Z1, LZ1, XM>(c1, T, a, a.frames1, a.afm1, sh);
    }
}

}  // namespace cmd
