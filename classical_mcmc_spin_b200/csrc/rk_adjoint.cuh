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
// each segment forward, storing the four stage inputs Y_s of every step, then
// sweeps it backwards.  A stage VJP is one pass over own cells: the partner's
// Hbar_p = Y_p x v_p (v = a lam + b Yb_{s+1}, the stage cotangent) is formed
// from the partner's Y, lam and Yb, and the same Y_p gives the forward field
// H_i, so neither H nor Hbar is stored.  The bond parameter terms use the bond
// symmetry (J at the source, J^T at the partner, likewise for dJ/dtheta):
//   sum_i Hbar_i . DJ_n S_p(n) = sum_p S_p . sum_n DJ_n Hbar_partner(n).
// A forward stage is one pass that also forms the next stage input and the
// RK4 sum.  All vectors are cell-major SoA in global memory, one CTA per
// trajectory.
#pragma once

#include "rk_global.cuh"

namespace cmd {

// Threads per trajectory CTA.
constexpr int kAdjThreads = 512;

template <int NAT, int Z, int NQ>
struct ParamDerivs {
    double DJ[NQ][NAT][Z][9];
    double DB[NQ][NAT][3];
    double DA[NQ][NAT][9];
    int has_DA;
    int dj_any[NQ];            // parameter q has a non-zero coupling derivative (resident adjoint skips it if not)
};

struct AdjTraj {
    const double* y0;          // AoS [N*3]
    const double* target;      // [S+1][3]
    double* ckpt;              // [K][V] checkpoints (SoA)
    double* seg;               // [C][V] segment buffer
    double* work;              // 5 * V
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

// One fused RK4 stage s (0..3) for cell g, reading the stage input Yin at
// the neighbours: k = H(Yin) x Yin with the drive factors f1, f2 of the stage
// time; H -> Hout when given;
//   s = 0: acc = k,        Ynext = y + dt/2 k
//   s = 1: acc = acc + 2k, Ynext = y + dt/2 k
//   s = 2: acc = acc + 2k, Ynext = y + dt k
//   s = 3:                 Ynext = y + dt/6 (acc + k)   (Ynext may alias y)
// which is the RK4 step y + dt/6 (k1 + 2 k2 + 2 k3 + k4) of the reference GPU
// stepper (integrator.cuh:115-139) summed in the same order.  Only the cell's
// own entries are written.  Observables of Yin added to obs: OBS = 1: the sum
// of the cell's spins over all atoms, obs[0..2]; OBS = 2: per atom class,
// obs[3*atom + c], and twice the energy, sum_i S_i.(H_i - B_i) (static field,
// before the drive; finish_rows_kernel applies the 1/2), in obs[3*NAT].
template <int NAT, int Z, int LZ, int OBS>
__device__ __forceinline__ void rk4_stage_cell(const Couplings<NAT, Z>& cp, const int* __restrict__ nbr, int G,
                                               int g, double dt, int s, const double* __restrict__ Yin,
                                               const double* y, double* acc, double* Ynext, double* __restrict__ Hout,
                                               double f1, double f2, bool drive, double* obs) {
    constexpr int NL = Z - LZ;
    const double cy = s == 2 ? dt : 0.5 * dt;
    double S[NAT][3];
#pragma unroll
    for (int at = 0; at < NAT; ++at)
#pragma unroll
        for (int c = 0; c < 3; ++c) S[at][c] = Yin[(at * 3 + c) * G + g];
    if (OBS > 0) {
#pragma unroll
        for (int at = 0; at < NAT; ++at)
#pragma unroll
            for (int c = 0; c < 3; ++c) obs[(OBS == 2 ? 3 * at : 0) + c] += S[at][c];
    }
#pragma unroll
    for (int at = 0; at < NAT; ++at) {
        double H[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) H[d] = cp.has_field ? -cp.field[at][d] : 0.0;
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
        for (int mm = 0; mm < NL; ++mm) {
            const int n = LZ + mm;
            if (n < cp.zc[at]) {
                const int p = nbr[((long long)g * NAT + at) * NL + mm];
                const double P0 = Yin[p], P1 = Yin[p + G], P2 = Yin[p + 2 * G];
#pragma unroll
                for (int d = 0; d < 3; ++d)
                    bond_acc(H[d], cp.J[at][n][3 * d], cp.J[at][n][3 * d + 1], cp.J[at][n][3 * d + 2], P0, P1, P2);
            }
        }
        if (OBS == 2) {          // twice the energy: S.(H_static - B), before the drive enters
#pragma unroll
            for (int d = 0; d < 3; ++d) obs[3 * NAT] += S[at][d] * (H[d] - (cp.has_field ? cp.field[at][d] : 0.0));
        }
        if (drive) {
#pragma unroll
            for (int d = 0; d < 3; ++d) drive_acc(H[d], cp.d1[at][d], cp.d2[at][d], f1, f2);
        }
        if (Hout) {
#pragma unroll
            for (int d = 0; d < 3; ++d) Hout[(at * 3 + d) * G + g] = H[d];
        }
        const double k[3] = {H[1] * S[at][2] - H[2] * S[at][1], H[2] * S[at][0] - H[0] * S[at][2],
                             H[0] * S[at][1] - H[1] * S[at][0]};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const long long i = (long long)(at * 3 + c) * G + g;
            const double yi = y[i];
            if (s == 0) {
                acc[i] = k[c];
                Ynext[i] = 1.0 * yi + cy * k[c];
            } else if (s < 3) {
                acc[i] = acc[i] + 2.0 * k[c];
                Ynext[i] = 1.0 * yi + cy * k[c];
            } else if (Ynext) {
                Ynext[i] = yi + (dt / 6.0) * (acc[i] + k[c]);
            }
        }
    }
}

// rk4_stage_cell over this CTA's share of the cells (one CTA per trajectory);
// when m is given, the own-cell sum of Yin over all atoms is added to m[0..2].
template <int NAT, int Z, int LZ>
__device__ __forceinline__ void rk4_stage(const Couplings<NAT, Z>& cp, const AdjArgs& a, int s,
                                          const double* __restrict__ Yin, const double* y, double* acc,
                                          double* Ynext, double* __restrict__ Hout, double ts, double* m) {
    const bool drive = a.pulse.a1 != 0.0 || a.pulse.a2 != 0.0;
    const double f1 = drive ? drive_factor(a.pulse.a1, ts - a.pulse.t1, a.width, a.freq) : 0.0;
    const double f2 = drive ? drive_factor(a.pulse.a2, ts - a.pulse.t2, a.width, a.freq) : 0.0;
    for (int g = threadIdx.x; g < a.G; g += blockDim.x) {
        if (m)
            rk4_stage_cell<NAT, Z, LZ, 1>(cp, a.nbr, a.G, g, a.dt, s, Yin, y, acc, Ynext, Hout, f1, f2, drive, m);
        else
            rk4_stage_cell<NAT, Z, LZ, 0>(cp, a.nbr, a.G, g, a.dt, s, Yin, y, acc, Ynext, Hout, f1, f2, drive,
                                          nullptr);
    }
}

// Block sum of 3 values (thread 0 gets the totals).
__device__ __forceinline__ void block_sum3(double (&v)[4], double* red, double* out) {
    block_sum<4>(v, red, 3, out);
}

template <int NAT, int Z, int LZ>
__global__ void __launch_bounds__(kAdjThreads)
adjoint_forward_kernel(const __grid_constant__ Couplings<NAT, Z> cp, const __grid_constant__ AdjArgs a) {
    __shared__ double red[32 * kRedStride];
    __shared__ double tot[4];
    const int b = blockIdx.x;
    const AdjTraj& T = a.traj[b];
    const int G = a.G, tid = threadIdx.x, nt = blockDim.x;
    const long long V = (long long)NAT * 3 * G;
    double* y = T.work;
    double* acc = T.work + V;
    double* Ya = T.work + 2 * V;
    double* Yb = T.work + 3 * V;
    const double N = (double)G * NAT;
    for (int g = tid; g < G; g += nt)
        for (int at = 0; at < NAT; ++at)
            for (int c = 0; c < 3; ++c) y[(at * 3 + c) * G + g] = T.y0[((long long)g * NAT + at) * 3 + c];
    __syncthreads();
    double loss = 0.0;
    auto record = [&](long long n) {     // after block_sum3: thread 0 holds the sums
        if (tid == 0) {
            for (int c = 0; c < 3; ++c) {
                const double mc = tot[c] / N;
                T.mloc[3 * n + c] = mc;
                const double r = mc - T.target[3 * n + c];
                loss += r * r;
            }
        }
    };
    for (long long n = 0; n < a.n_steps; ++n) {
        if (!a.forward_only && n % a.ckpt_every == 0) {
            double* dst = T.ckpt + (n / a.ckpt_every) * V;
            for (int g = tid; g < G; g += nt)
                for (int e = 0; e < NAT * 3; ++e) dst[(long long)e * G + g] = y[(long long)e * G + g];
        }
        const double t = a.times[n];
        double m[4] = {0, 0, 0, 0};
        rk4_stage<NAT, Z, LZ>(cp, a, 0, y, y, acc, Ya, nullptr, t, m);
        block_sum3(m, red, tot);           // its barrier also ends stage 0
        record(n);
        rk4_stage<NAT, Z, LZ>(cp, a, 1, Ya, y, acc, Yb, nullptr, t + 0.5 * a.dt, nullptr);
        __syncthreads();
        rk4_stage<NAT, Z, LZ>(cp, a, 2, Yb, y, acc, Ya, nullptr, t + 0.5 * a.dt, nullptr);
        __syncthreads();
        rk4_stage<NAT, Z, LZ>(cp, a, 3, Ya, y, acc, y, nullptr, t + a.dt, nullptr);
        __syncthreads();
    }
    double m[4] = {0, 0, 0, 0};
    for (int g = tid; g < G; g += nt)
        for (int at = 0; at < NAT; ++at)
            for (int c = 0; c < 3; ++c) m[c] += y[(at * 3 + c) * G + g];
    block_sum3(m, red, tot);
    record(a.n_steps);
    if (tid == 0) T.loss[0] = loss;
}

// One stage VJP for cell g at stage input Y with cotangent
// v = ca lam + cb Sprev (Sprev unused when cb == 0) and the drive factors
// f1, f2 of the stage time:
//   H_i  = field at Y (static + drive),   Hbar_i = S_i x v_i
//   Yb_i = v_i x H_i + 2 A_i^T Hbar_i + sum_n J_n Hbar_partner(n)
//   thetabar_q += Hbar_i . (2 DA_q S_i - DB_q) + S_i . sum_n DJ_q,n Hbar_partner(n)
// then per own entry  mode 0: Sout = Yb, acc = lam + Yb;  mode 1: Sout = Yb,
// acc += Yb;  mode 2: lam_out = acc + Yb + dl (dl: the loss cotangent at this
// step, per component).  lam, Sprev and Y are read at the partners, so
// lam_out and Sout must be other buffers.  The atoms run in a rolled loop:
// one copy of this large body keeps the instruction cache warm.
template <int NAT, int Z, int LZ, int NQ>
__device__ __forceinline__ void vjp_cell(const Couplings<NAT, Z>& cp, const ParamDerivs<NAT, Z, NQ>& pd,
                                         const int* __restrict__ nbr, int G, int g, const double* __restrict__ Y,
                                         const double* __restrict__ lam, const double* __restrict__ Sprev, double ca,
                                         double cb, double f1, double f2, bool drive, double* __restrict__ Sout,
                                         double* __restrict__ acc, double* __restrict__ lam_out, int mode,
                                         const double* dl, double (&gq)[NQ]) {
    constexpr int NL = Z - LZ;
    auto cot = [&](long long i0, double (&v)[3]) {
        v[0] = ca * lam[i0];
        v[1] = ca * lam[i0 + G];
        v[2] = ca * lam[i0 + 2 * G];
        if (cb != 0.0) {
            v[0] = v[0] + cb * Sprev[i0];
            v[1] = v[1] + cb * Sprev[i0 + G];
            v[2] = v[2] + cb * Sprev[i0 + 2 * G];
        }
    };
    // spin P and Hbar Q of the site at SoA offset p (own site or partner)
    auto partner = [&](long long p, double (&P)[3], double (&Q)[3]) {
        P[0] = Y[p];
        P[1] = Y[p + G];
        P[2] = Y[p + 2 * G];
        double v[3];
        cot(p, v);
        Q[0] = P[1] * v[2] - P[2] * v[1];
        Q[1] = P[2] * v[0] - P[0] * v[2];
        Q[2] = P[0] * v[1] - P[1] * v[0];
    };
#pragma unroll 1
    for (int at = 0; at < NAT; ++at) {
        const long long i0 = (long long)(at * 3) * G + g;
        double Sown[3], hown[3];
        partner(i0, Sown, hown);
        const double S0 = Sown[0], S1 = Sown[1], S2 = Sown[2];
        double H[3], sb[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int d = 0; d < 3; ++d) H[d] = cp.has_field ? -cp.field[at][d] : 0.0;
        if (cp.has_onsite) {
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                bond_acc(H[d], 2.0 * cp.onsite[at][3 * d], 2.0 * cp.onsite[at][3 * d + 1], 2.0 * cp.onsite[at][3 * d + 2], S0, S1, S2);
                sb[d] += 2.0 * (cp.onsite[at][d] * hown[0] + cp.onsite[at][3 + d] * hown[1] +
                                cp.onsite[at][6 + d] * hown[2]);
            }
        }
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            double t = -(hown[0] * pd.DB[q][at][0] + hown[1] * pd.DB[q][at][1] + hown[2] * pd.DB[q][at][2]);
            if (pd.has_DA) {
#pragma unroll
                for (int d = 0; d < 3; ++d)
                    t += 2.0 * hown[d] * (pd.DA[q][at][3 * d] * S0 + pd.DA[q][at][3 * d + 1] * S1 +
                                          pd.DA[q][at][3 * d + 2] * S2);
            }
            gq[q] += t;
        }
        // bond n with partner spin P and partner Hbar Q
        auto bond = [&](int n, const double (&P)[3], const double (&Q)[3]) {
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                bond_acc(H[d], cp.J[at][n][3 * d], cp.J[at][n][3 * d + 1], cp.J[at][n][3 * d + 2], P[0], P[1], P[2]);
                bond_acc(sb[d], cp.J[at][n][3 * d], cp.J[at][n][3 * d + 1], cp.J[at][n][3 * d + 2], Q[0], Q[1], Q[2]);
            }
#pragma unroll
            for (int q = 0; q < NQ; ++q) {
                const double* D = pd.DJ[q][at][n];
                gq[q] += S0 * (D[0] * Q[0] + D[1] * Q[1] + D[2] * Q[2]) +
                         S1 * (D[3] * Q[0] + D[4] * Q[1] + D[5] * Q[2]) +
                         S2 * (D[6] * Q[0] + D[7] * Q[1] + D[8] * Q[2]);
            }
        };
#pragma unroll
        for (int n = 0; n < LZ; ++n) {
            const int pb = (at + 1 + n) % NAT;
            double P[3], Q[3];
            partner((long long)(pb * 3) * G + g, P, Q);
            bond(n, P, Q);
        }
#pragma unroll
        for (int m = 0; m < NL; ++m) {
            const int n = LZ + m;
            if (n < cp.zc[at]) {
                double P[3], Q[3];
                partner(nbr[((long long)g * NAT + at) * NL + m], P, Q);
                bond(n, P, Q);
            }
        }
        if (drive) {
#pragma unroll
            for (int d = 0; d < 3; ++d) drive_acc(H[d], cp.d1[at][d], cp.d2[at][d], f1, f2);
        }
        double v[3];
        cot(i0, v);
        sb[0] += v[1] * H[2] - v[2] * H[1];
        sb[1] += v[2] * H[0] - v[0] * H[2];
        sb[2] += v[0] * H[1] - v[1] * H[0];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const long long i = i0 + d * G;
            if (mode == 0) {
                Sout[i] = sb[d];
                acc[i] = lam[i] + sb[d];
            } else if (mode == 1) {
                Sout[i] = sb[d];
                acc[i] = acc[i] + sb[d];
            } else {
                lam_out[i] = acc[i] + sb[d] + dl[d];
            }
        }
    }
}

// vjp_cell over this CTA's share of the cells (one CTA per trajectory) at the
// stage time ts.
template <int NAT, int Z, int LZ, int NQ>
__device__ __forceinline__ void stage_vjp(const Couplings<NAT, Z>& cp, const ParamDerivs<NAT, Z, NQ>& pd,
                                          const AdjArgs& a, const double* __restrict__ Y,
                                          const double* __restrict__ lam, const double* __restrict__ Sprev,
                                          double ca, double cb, double ts, double* __restrict__ Sout,
                                          double* __restrict__ acc, double* __restrict__ lam_out, int mode,
                                          const double* dl, double (&gq)[NQ]) {
    const bool drive = a.pulse.a1 != 0.0 || a.pulse.a2 != 0.0;
    const double f1 = drive ? drive_factor(a.pulse.a1, ts - a.pulse.t1, a.width, a.freq) : 0.0;
    const double f2 = drive ? drive_factor(a.pulse.a2, ts - a.pulse.t2, a.width, a.freq) : 0.0;
    for (int g = threadIdx.x; g < a.G; g += blockDim.x)
        vjp_cell<NAT, Z, LZ, NQ>(cp, pd, a.nbr, a.G, g, Y, lam, Sprev, ca, cb, f1, f2, drive, Sout, acc, lam_out,
                                 mode, dl, gq);
}

template <int NAT, int Z, int LZ, int NQ>
__global__ void __launch_bounds__(kAdjThreads)
adjoint_backward_kernel(const __grid_constant__ Couplings<NAT, Z> cp, const __grid_constant__ ParamDerivs<NAT, Z, NQ> pd,
                        const __grid_constant__ AdjArgs a) {
    __shared__ double red[32 * kRedStride];
    __shared__ double tot[NQ < 16 ? 16 : NQ];
    const int b = blockIdx.x;
    const AdjTraj& T = a.traj[b];
    const int G = a.G, tid = threadIdx.x, nt = blockDim.x;
    const long long V = (long long)NAT * 3 * G;
    double* lam = T.work;               // cotangent of y_{n+1}; lam2 receives that of y_n
    double* lam2 = T.work + 1 * V;
    double* acc = T.work + 2 * V;       // RK4 sum (recompute) / ybar accumulator (sweep)
    double* Sa = T.work + 3 * V;
    double* Sb = T.work + 4 * V;
    const double N = (double)G * NAT;
    const double dt = a.dt;
    const long long S = a.n_steps;
    double gq[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) gq[q] = 0.0;

    auto dl = [&](long long n, int c) { return 2.0 * (T.mloc[3 * n + c] - T.target[3 * n + c]) / N; };
    for (int g = tid; g < G; g += nt)
        for (int at = 0; at < NAT; ++at)
            for (int c = 0; c < 3; ++c) lam[(at * 3 + c) * G + g] = dl(S, c);
    __syncthreads();
    // Segment slot layout: step j of the segment holds [Y1 Y2 Y3 Y4].
    auto slot = [&](long long j, int q) { return T.seg + (j * 4 + q) * V; };
    const long long C = a.ckpt_every;
    const long long K = (S + C - 1) / C;
    for (long long seg = K - 1; seg >= 0; --seg) {
        const long long n0 = seg * C;
        const long long n1 = (n0 + C < S) ? n0 + C : S;
        // forward recompute of the segment from its checkpoint, keeping every
        // stage input of every step
        {
            double* y1 = slot(0, 0);
            for (int g = tid; g < G; g += nt)
                for (int e = 0; e < NAT * 3; ++e) y1[(long long)e * G + g] = T.ckpt[seg * V + (long long)e * G + g];
        }
        __syncthreads();
        for (long long n = n0; n < n1; ++n) {
            const long long j = n - n0;
            const double t = a.times[n];
            double* y = slot(j, 0);
            rk4_stage<NAT, Z, LZ>(cp, a, 0, y, y, acc, slot(j, 1), nullptr, t, nullptr);
            __syncthreads();
            rk4_stage<NAT, Z, LZ>(cp, a, 1, slot(j, 1), y, acc, slot(j, 2), nullptr, t + 0.5 * dt, nullptr);
            __syncthreads();
            rk4_stage<NAT, Z, LZ>(cp, a, 2, slot(j, 2), y, acc, slot(j, 3), nullptr, t + 0.5 * dt, nullptr);
            __syncthreads();
            rk4_stage<NAT, Z, LZ>(cp, a, 3, slot(j, 3), y, acc, n + 1 < n1 ? slot(j + 1, 0) : nullptr, nullptr,
                                  t + dt, nullptr);
            __syncthreads();
        }
        for (long long n = n1 - 1; n >= n0; --n) {
            const long long j = n - n0;
            const double t = a.times[n];
            // stage 4: kb4 = dt/6 lam -> Yb4 (Sa); acc = lam + Yb4
            stage_vjp<NAT, Z, LZ, NQ>(cp, pd, a, slot(j, 3), lam, nullptr, dt / 6.0, 0.0, t + dt, Sa, acc, nullptr,
                                      0, nullptr, gq);
            __syncthreads();
            // stage 3: kb3 = dt/3 lam + dt Yb4 -> Yb3 (Sb); acc += Yb3
            stage_vjp<NAT, Z, LZ, NQ>(cp, pd, a, slot(j, 2), lam, Sa, dt / 3.0, dt, t + 0.5 * dt, Sb, acc, nullptr,
                                      1, nullptr, gq);
            __syncthreads();
            // stage 2: kb2 = dt/3 lam + dt/2 Yb3 -> Yb2 (Sa); acc += Yb2
            stage_vjp<NAT, Z, LZ, NQ>(cp, pd, a, slot(j, 1), lam, Sb, dt / 3.0, 0.5 * dt, t + 0.5 * dt, Sa, acc,
                                      nullptr, 1, nullptr, gq);
            __syncthreads();
            // stage 1: kb1 = dt/6 lam + dt/2 Yb2 -> Yb1; lam_n = acc + Yb1 + dl_n
            const double dln[3] = {dl(n, 0), dl(n, 1), dl(n, 2)};
            stage_vjp<NAT, Z, LZ, NQ>(cp, pd, a, slot(j, 0), lam, Sa, dt / 6.0, 0.5 * dt, t, nullptr, acc, lam2, 2,
                                      dln, gq);
            __syncthreads();
            double* sw = lam;
            lam = lam2;
            lam2 = sw;
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
