// rk_adjoint.cuh -- discrete adjoint of the RK4 trajectory (no reference
// counterpart: the reference has no gradients).
//
// Loss  L = sum_{n=0..S} |M_local(y_n) - T_n|^2,  M_local(y) = (1/N) sum_i S_i,
// over the RK4 trajectory of the reference GPU stepper's arithmetic
// (integrator.cuh:115-139).  The couplings depend linearly on parameters theta
// (K, Gamma, Gamma', J, h for the Kitaev family): J_n = sum_q theta_q DJ_q,
// B = sum_q theta_q DB_q, A = sum_q theta_q DA_q (+ theta-independent parts),
// with DJ/DB/DA read off lattices built at theta = e_q.
//
// Reverse sweep of one step y' = y + dt/6 (k1 + 2 k2 + 2 k3 + k4) with
// cotangent lam' (stage inputs Y2 = y + dt/2 k1, Y3 = y + dt/2 k2, Y4 = y + dt k3
// recomputed from the stored y):
//   kb4 = dt/6 lam'                      -> Yb4 = f_Y(Y4)^T kb4
//   kb3 = dt/3 lam' + dt Yb4             -> Yb3
//   kb2 = dt/3 lam' + dt/2 Yb3           -> Yb2
//   kb1 = dt/6 lam' + dt/2 Yb2           -> Yb1
//   lam = lam' + Yb4 + Yb3 + Yb2 + Yb1 + dl_n/dy_n
// and the parameter cotangents of the four stages.  The VJP of
// f_i = H_i x S_i with cotangent v:
//   Hbar_i = S_i x v_i
//   Sbar_i = v_i x H_i + 2 A_i^T Hbar_i + sum_n J_n Hbar_p(n)
//   thetabar_q += sum_i Hbar_i . (sum_n DJ_q,n S_p(n) + 2 DA_q S_i - DB_q)
// (the last gather uses site i's own bond list: bond tables hold J at the
// source and J^T at the partner, so sum_{i->p} J^T Hbar_i = sum_{p->i} J Hbar_i).
//
// Memory: checkpoints every C steps (C ~ sqrt(S)); the backward pass re-runs
// each segment forward into a segment buffer, then sweeps it backwards.  All
// vectors are cell-major SoA in global memory, one CTA per trajectory.
#pragma once

#include "rk_global.cuh"

namespace cmd {

template <int NAT, int Z, int NQ>
struct ParamDerivs {
    double DJ[NQ][NAT][Z][9];
    double DB[NQ][NAT][3];
    double DA[NQ][NAT][9];
    int has_DA;
};

struct AdjTraj {
    const double* y0;          // AoS [N*3]
    const double* target;      // [S+1][3]
    double* ckpt;              // [K][V] checkpoints (SoA)
    double* seg;               // [C][V] segment buffer
    double* work;              // 13 * V
    double* mloc;              // [S+1][3] M_local of the forward pass
    double* loss;              // [1]
    double* grad;              // [NQ]
};

struct AdjArgs {
    const AdjTraj* traj;
    int B;
    int G;
    const int* nbr;
    const double* times;       // [S+1] accumulated t_n
    long long n_steps;
    long long ckpt_every;
    double dt;
    Pulse pulse;
    double width, freq;
    int forward_only;
};

// Forward RK4 over own cells: y <- step(y), stage buffers in w.
template <int NAT, int Z, int LZ>
__device__ __forceinline__ void rk4_step_global(const Couplings<NAT, Z>& cp, const AdjArgs& a, double* y,
                                                double* k1, double* k2, double* k3, double* k4, double* Ya,
                                                double* Yb, double t, double* part) {
    const int G = a.G, tid = threadIdx.x, nt = blockDim.x;
    const double dt = a.dt;
    const bool drive = a.pulse.a1 != 0.0 || a.pulse.a2 != 0.0;
    auto rhs = [&](const double* Yin, double* K, double ts, double* pp) {
        const double f1 = drive ? drive_factor(a.pulse.a1, ts - a.pulse.t1, a.width, a.freq) : 0.0;
        const double f2 = drive ? drive_factor(a.pulse.a2, ts - a.pulse.t2, a.width, a.freq) : 0.0;
        for (int g = tid; g < G; g += nt) rhs_cell<NAT, Z, LZ>(cp, Yin, K, G, g, a.nbr, f1, f2, drive, pp);
    };
    rhs(y, k1, t, part);
    __syncthreads();
    for (int g = tid; g < G; g += nt)
        for (int e = 0; e < NAT * 3; ++e) {
            const long long i = (long long)e * G + g;
            Ya[i] = 1.0 * y[i] + (0.5 * dt) * k1[i];
        }
    __syncthreads();
    rhs(Ya, k2, t + 0.5 * dt, nullptr);
    for (int g = tid; g < G; g += nt)
        for (int e = 0; e < NAT * 3; ++e) {
            const long long i = (long long)e * G + g;
            Yb[i] = 1.0 * y[i] + (0.5 * dt) * k2[i];
        }
    __syncthreads();
    rhs(Yb, k3, t + 0.5 * dt, nullptr);
    __syncthreads();
    for (int g = tid; g < G; g += nt)
        for (int e = 0; e < NAT * 3; ++e) {
            const long long i = (long long)e * G + g;
            Ya[i] = 1.0 * y[i] + dt * k3[i];
        }
    __syncthreads();
    rhs(Ya, k4, t + dt, nullptr);
    for (int g = tid; g < G; g += nt)
        for (int e = 0; e < NAT * 3; ++e) {
            const long long i = (long long)e * G + g;
            y[i] += (dt / 6.0) * (k1[i] + 2.0 * k2[i] + 2.0 * k3[i] + k4[i]);
        }
    __syncthreads();
}

// Block sum of 3 values (thread 0 gets the totals).
__device__ __forceinline__ void block_sum3(double (&v)[4], double* red, double* out) {
    block_sum<4>(v, red, 3, out);
}

template <int NAT, int Z, int LZ>
__global__ void __launch_bounds__(256)
adjoint_forward_kernel(const __grid_constant__ Couplings<NAT, Z> cp, const __grid_constant__ AdjArgs a) {
    __shared__ double red[32 * kRedStride];
    __shared__ double tot[4];
    const int b = blockIdx.x;
    const AdjTraj& T = a.traj[b];
    const int G = a.G, tid = threadIdx.x, nt = blockDim.x;
    const long long V = (long long)NAT * 3 * G;
    double* y = T.work;
    double* k1 = T.work + V; double* k2 = T.work + 2 * V; double* k3 = T.work + 3 * V; double* k4 = T.work + 4 * V;
    double* Ya = T.work + 5 * V; double* Yb = T.work + 6 * V;
    const double N = (double)G * NAT;
    for (int g = tid; g < G; g += nt)
        for (int at = 0; at < NAT; ++at)
            for (int c = 0; c < 3; ++c) y[(at * 3 + c) * G + g] = T.y0[((long long)g * NAT + at) * 3 + c];
    __syncthreads();
    double loss = 0.0;
    for (long long n = 0; n <= a.n_steps; ++n) {
        if (!a.forward_only && n % a.ckpt_every == 0 && n < a.n_steps) {
            double* dst = T.ckpt + (n / a.ckpt_every) * V;
            for (int g = tid; g < G; g += nt)
                for (int e = 0; e < NAT * 3; ++e) dst[(long long)e * G + g] = y[(long long)e * G + g];
        }
        double m[4] = {0, 0, 0, 0};
        for (int g = tid; g < G; g += nt)
            for (int at = 0; at < NAT; ++at)
                for (int c = 0; c < 3; ++c) m[c] += y[(at * 3 + c) * G + g];
        block_sum3(m, red, tot);
        if (tid == 0) {
            for (int c = 0; c < 3; ++c) {
                const double mc = tot[c] / N;
                T.mloc[3 * n + c] = mc;
                const double r = mc - T.target[3 * n + c];
                loss += r * r;
            }
        }
        __syncthreads();
        if (n == a.n_steps) break;
        rk4_step_global<NAT, Z, LZ>(cp, a, y, k1, k2, k3, k4, Ya, Yb, a.times[n], nullptr);
    }
    if (tid == 0) T.loss[0] = loss;
}

// Phase A of a stage VJP over own cells: H (forward field at Y), Hbar = S x v,
// parameter cotangents.  Writes H and Hbar (SoA).
template <int NAT, int Z, int LZ, int NQ>
__device__ __forceinline__ void vjp_phase_a(const Couplings<NAT, Z>& cp, const ParamDerivs<NAT, Z, NQ>& pd,
                                            const AdjArgs& a, const double* __restrict__ Y,
                                            const double* __restrict__ v, double* __restrict__ Hout,
                                            double* __restrict__ Hbar, double ts, double (&gq)[NQ]) {
    constexpr int NL = Z - LZ;
    const int G = a.G, tid = threadIdx.x, nt = blockDim.x;
    const bool drive = a.pulse.a1 != 0.0 || a.pulse.a2 != 0.0;
    const double f1 = drive ? drive_factor(a.pulse.a1, ts - a.pulse.t1, a.width, a.freq) : 0.0;
    const double f2 = drive ? drive_factor(a.pulse.a2, ts - a.pulse.t2, a.width, a.freq) : 0.0;
    for (int g = tid; g < G; g += nt) {
        double S[NAT][3];
#pragma unroll
        for (int at = 0; at < NAT; ++at)
#pragma unroll
            for (int c = 0; c < 3; ++c) S[at][c] = Y[(at * 3 + c) * G + g];
#pragma unroll
        for (int at = 0; at < NAT; ++at) {
            double H[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) H[d] = cp.has_field ? -cp.field[at][d] : 0.0;
            if (cp.has_onsite) {
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    H[d] += 2.0 * cp.onsite[at][3 * d + 0] * S[at][0];
                    H[d] += 2.0 * cp.onsite[at][3 * d + 1] * S[at][1];
                    H[d] += 2.0 * cp.onsite[at][3 * d + 2] * S[at][2];
                }
            }
            const double v0 = v[(at * 3 + 0) * G + g], v1 = v[(at * 3 + 1) * G + g], v2 = v[(at * 3 + 2) * G + g];
            const double hb[3] = {S[at][1] * v2 - S[at][2] * v1, S[at][2] * v0 - S[at][0] * v2,
                                  S[at][0] * v1 - S[at][1] * v0};
#pragma unroll
            for (int q = 0; q < NQ; ++q) {
                double acc = -(hb[0] * pd.DB[q][at][0] + hb[1] * pd.DB[q][at][1] + hb[2] * pd.DB[q][at][2]);
                if (pd.has_DA) {
#pragma unroll
                    for (int d = 0; d < 3; ++d)
                        acc += 2.0 * hb[d] * (pd.DA[q][at][3 * d] * S[at][0] + pd.DA[q][at][3 * d + 1] * S[at][1] +
                                              pd.DA[q][at][3 * d + 2] * S[at][2]);
                }
                gq[q] += acc;
            }
            auto bond = [&](int n, double P0, double P1, double P2) {
#pragma unroll
                for (int d = 0; d < 3; ++d)
                    H[d] += cp.J[at][n][3 * d] * P0 + cp.J[at][n][3 * d + 1] * P1 + cp.J[at][n][3 * d + 2] * P2;
#pragma unroll
                for (int q = 0; q < NQ; ++q) {
                    const double* D = pd.DJ[q][at][n];
                    gq[q] += hb[0] * (D[0] * P0 + D[1] * P1 + D[2] * P2) + hb[1] * (D[3] * P0 + D[4] * P1 + D[5] * P2) +
                             hb[2] * (D[6] * P0 + D[7] * P1 + D[8] * P2);
                }
            };
#pragma unroll
            for (int n = 0; n < LZ; ++n) {
                const int pb = (at + 1 + n) % NAT;
                bond(n, S[pb][0], S[pb][1], S[pb][2]);
            }
#pragma unroll
            for (int m = 0; m < NL; ++m) {
                const int n = LZ + m;
                if (n < cp.zc[at]) {
                    const int p = a.nbr[((long long)g * NAT + at) * NL + m];
                    bond(n, Y[p], Y[p + G], Y[p + 2 * G]);
                }
            }
            if (drive) {
#pragma unroll
                for (int d = 0; d < 3; ++d) H[d] -= cp.d1[at][d] * f1 + cp.d2[at][d] * f2;
            }
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                Hout[(at * 3 + d) * G + g] = H[d];
                Hbar[(at * 3 + d) * G + g] = hb[d];
            }
        }
    }
}

// Phase B: Sbar_i = v_i x H_i + 2 A_i^T Hbar_i + sum_n J_n Hbar_p(n); out += scale * Sbar.
template <int NAT, int Z, int LZ>
__device__ __forceinline__ void vjp_phase_b(const Couplings<NAT, Z>& cp, const AdjArgs& a,
                                            const double* __restrict__ v, const double* __restrict__ Hin,
                                            const double* __restrict__ Hbar, double* __restrict__ Sbar) {
    constexpr int NL = Z - LZ;
    const int G = a.G, tid = threadIdx.x, nt = blockDim.x;
    for (int g = tid; g < G; g += nt) {
        double Hb[NAT][3];
#pragma unroll
        for (int at = 0; at < NAT; ++at)
#pragma unroll
            for (int c = 0; c < 3; ++c) Hb[at][c] = Hbar[(at * 3 + c) * G + g];
#pragma unroll
        for (int at = 0; at < NAT; ++at) {
            const double v0 = v[(at * 3 + 0) * G + g], v1 = v[(at * 3 + 1) * G + g], v2 = v[(at * 3 + 2) * G + g];
            const double H0 = Hin[(at * 3 + 0) * G + g], H1 = Hin[(at * 3 + 1) * G + g],
                         H2 = Hin[(at * 3 + 2) * G + g];
            double sb[3] = {v1 * H2 - v2 * H1, v2 * H0 - v0 * H2, v0 * H1 - v1 * H0};
            if (cp.has_onsite) {
#pragma unroll
                for (int d = 0; d < 3; ++d)
                    sb[d] += 2.0 * (cp.onsite[at][d] * Hb[at][0] + cp.onsite[at][3 + d] * Hb[at][1] +
                                    cp.onsite[at][6 + d] * Hb[at][2]);
            }
#pragma unroll
            for (int n = 0; n < LZ; ++n) {
                const int pb = (at + 1 + n) % NAT;
#pragma unroll
                for (int d = 0; d < 3; ++d)
                    sb[d] += cp.J[at][n][3 * d] * Hb[pb][0] + cp.J[at][n][3 * d + 1] * Hb[pb][1] +
                             cp.J[at][n][3 * d + 2] * Hb[pb][2];
            }
#pragma unroll
            for (int m = 0; m < NL; ++m) {
                const int n = LZ + m;
                if (n < cp.zc[at]) {
                    const int p = a.nbr[((long long)g * NAT + at) * NL + m];
                    const double P0 = Hbar[p], P1 = Hbar[p + G], P2 = Hbar[p + 2 * G];
#pragma unroll
                    for (int d = 0; d < 3; ++d)
                        sb[d] += cp.J[at][n][3 * d] * P0 + cp.J[at][n][3 * d + 1] * P1 + cp.J[at][n][3 * d + 2] * P2;
                }
            }
#pragma unroll
            for (int d = 0; d < 3; ++d) Sbar[(at * 3 + d) * G + g] = sb[d];
        }
    }
}

template <int NAT, int Z, int LZ, int NQ>
__global__ void __launch_bounds__(256)
adjoint_backward_kernel(const __grid_constant__ Couplings<NAT, Z> cp, const __grid_constant__ ParamDerivs<NAT, Z, NQ> pd,
                        const __grid_constant__ AdjArgs a) {
    __shared__ double red[32 * kRedStride];
    __shared__ double tot[NQ < 16 ? 16 : NQ];
    const int b = blockIdx.x;
    const AdjTraj& T = a.traj[b];
    const int G = a.G, tid = threadIdx.x, nt = blockDim.x;
    const long long V = (long long)NAT * 3 * G;
    double* y = T.work;
    double* k1 = T.work + 1 * V; double* k2 = T.work + 2 * V; double* k3 = T.work + 3 * V;
    double* Y2 = T.work + 4 * V; double* Y3 = T.work + 5 * V; double* Y4 = T.work + 6 * V;
    double* lam = T.work + 7 * V;
    double* kb = T.work + 8 * V;
    double* Hs = T.work + 9 * V;
    double* Hb = T.work + 10 * V;
    double* Sb = T.work + 11 * V;
    double* tmp = T.work + 12 * V;
    const double N = (double)G * NAT;
    const double dt = a.dt;
    const long long S = a.n_steps;
    double gq[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) gq[q] = 0.0;

    auto dl = [&](long long n, int c) { return 2.0 * (T.mloc[3 * n + c] - T.target[3 * n + c]) / N; };
    // lam_S = dl_S/dy_S (uniform over sites)
    for (int g = tid; g < G; g += nt)
        for (int at = 0; at < NAT; ++at)
            for (int c = 0; c < 3; ++c) lam[(at * 3 + c) * G + g] = dl(S, c);
    __syncthreads();
    const bool drive = a.pulse.a1 != 0.0 || a.pulse.a2 != 0.0;
    auto rhs = [&](const double* Yin, double* K, double ts) {
        const double f1 = drive ? drive_factor(a.pulse.a1, ts - a.pulse.t1, a.width, a.freq) : 0.0;
        const double f2 = drive ? drive_factor(a.pulse.a2, ts - a.pulse.t2, a.width, a.freq) : 0.0;
        for (int g = tid; g < G; g += nt) rhs_cell<NAT, Z, LZ>(cp, Yin, K, G, g, a.nbr, f1, f2, drive, nullptr);
    };
    // one stage VJP: Sb = f_Y(Ystage)^T v
    auto stage_vjp = [&](const double* Ystage, const double* v, double ts) {
        vjp_phase_a<NAT, Z, LZ, NQ>(cp, pd, a, Ystage, v, Hs, Hb, ts, gq);
        __syncthreads();
        vjp_phase_b<NAT, Z, LZ>(cp, a, v, Hs, Hb, Sb);
        __syncthreads();
    };
    const long long C = a.ckpt_every;
    const long long K = (S + C - 1) / C;
    for (long long seg = K - 1; seg >= 0; --seg) {
        const long long n0 = seg * C;
        const long long n1 = (n0 + C < S) ? n0 + C : S;
        // re-run the segment forward from its checkpoint, storing y_n
        for (int g = tid; g < G; g += nt)
            for (int e = 0; e < NAT * 3; ++e) y[(long long)e * G + g] = T.ckpt[seg * V + (long long)e * G + g];
        __syncthreads();
        for (long long n = n0; n < n1; ++n) {
            double* dst = T.seg + (n - n0) * V;
            for (int g = tid; g < G; g += nt)
                for (int e = 0; e < NAT * 3; ++e) dst[(long long)e * G + g] = y[(long long)e * G + g];
            if (n + 1 < n1) rk4_step_global<NAT, Z, LZ>(cp, a, y, k1, k2, k3, Hs, Y2, Y3, a.times[n], nullptr);
        }
        __syncthreads();
        for (long long n = n1 - 1; n >= n0; --n) {
            const double t = a.times[n];
            const double* yn = T.seg + (n - n0) * V;
            // stage inputs of step n
            rhs(yn, k1, t);
            __syncthreads();
            for (int g = tid; g < G; g += nt)
                for (int e = 0; e < NAT * 3; ++e) {
                    const long long i = (long long)e * G + g;
                    Y2[i] = 1.0 * yn[i] + (0.5 * dt) * k1[i];
                }
            __syncthreads();
            rhs(Y2, k2, t + 0.5 * dt);
            __syncthreads();
            for (int g = tid; g < G; g += nt)
                for (int e = 0; e < NAT * 3; ++e) {
                    const long long i = (long long)e * G + g;
                    Y3[i] = 1.0 * yn[i] + (0.5 * dt) * k2[i];
                }
            __syncthreads();
            rhs(Y3, k3, t + 0.5 * dt);
            __syncthreads();
            for (int g = tid; g < G; g += nt)
                for (int e = 0; e < NAT * 3; ++e) {
                    const long long i = (long long)e * G + g;
                    Y4[i] = 1.0 * yn[i] + dt * k3[i];
                    kb[i] = (dt / 6.0) * lam[i];                 // kbar4
                    tmp[i] = lam[i];                             // ybar accumulator
                }
            __syncthreads();
            stage_vjp(Y4, kb, t + dt);                           // Sb = Yb4
            for (int g = tid; g < G; g += nt)
                for (int e = 0; e < NAT * 3; ++e) {
                    const long long i = (long long)e * G + g;
                    tmp[i] += Sb[i];
                    kb[i] = (dt / 3.0) * lam[i] + dt * Sb[i];    // kbar3
                }
            __syncthreads();
            stage_vjp(Y3, kb, t + 0.5 * dt);                     // Sb = Yb3
            for (int g = tid; g < G; g += nt)
                for (int e = 0; e < NAT * 3; ++e) {
                    const long long i = (long long)e * G + g;
                    tmp[i] += Sb[i];
                    kb[i] = (dt / 3.0) * lam[i] + (0.5 * dt) * Sb[i];   // kbar2
                }
            __syncthreads();
            stage_vjp(Y2, kb, t + 0.5 * dt);                     // Sb = Yb2
            for (int g = tid; g < G; g += nt)
                for (int e = 0; e < NAT * 3; ++e) {
                    const long long i = (long long)e * G + g;
                    tmp[i] += Sb[i];
                    kb[i] = (dt / 6.0) * lam[i] + (0.5 * dt) * Sb[i];   // kbar1
                }
            __syncthreads();
            stage_vjp(yn, kb, t);                                // Sb = Yb1
            for (int g = tid; g < G; g += nt)
                for (int at = 0; at < NAT; ++at)
                    for (int c = 0; c < 3; ++c) {
                        const long long i = (long long)(at * 3 + c) * G + g;
                        lam[i] = tmp[i] + Sb[i] + dl(n, c);
                    }
            __syncthreads();
        }
    }
    double v[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = q < NQ ? gq[q] : 0.0;
    block_sum<16>(v, red, NQ, tot);
    if (tid == 0)
        for (int q = 0; q < NQ; ++q) T.grad[q] = tot[q];
}

}  // namespace cmd
