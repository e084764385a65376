// rk_adjoint_cluster.cuh -- the discrete RK4 adjoint of rk_adjoint.cuh (same loss, same
// cotangent recursion, same parameter terms) with each trajectory resident on a
// thread-block cluster of CS CTAs (CS = 1: one CTA), one thread per unit cell.
//
// Phase 1, forward: y_n lives in registers, the RK4 sum in the own slots of shared
// memory and the stage input in shared memory for the partners (double-buffered,
// partners in other CTAs of the cluster through distributed shared memory, as in
// rk4_cluster.cuh).  Every C steps the own cells of y_n go to the checkpoint array;
// M_local(y_n) is summed with the deferred reduction of the forward kernels (stage 0
// accumulates, stage 1 reduces per warp, stage 2 per CTA, stage 3 rank 0 adds the
// CTAs in rank order) and rank 0 accumulates the loss.
//
// Phase 2, backward, segment by segment from the last: re-run the segment from its
// checkpoint (the same arithmetic as phase 1, so the same trajectory) storing the four
// stage inputs of every step in global memory; then sweep it backwards.  A stage VJP
// with cotangent v = ca lam + cb Yb_prev first forms the own Hbar_i = Y_i x v_i and
// publishes it next to Y in shared memory (two pairs of buffers, alternating, so one
// cluster barrier per VJP stage), then gathers the partners' Y (forward field H) and
// Hbar (sum_n J_n Hbar_partner(n), the bond-symmetric form of the transpose) and the
// parameter terms.  The own stage input of the next VJP stage is copied from global
// memory into its buffer pair with cp.async while the current stage computes.  lam,
// the ybar accumulator and the previous stage cotangent live in the own slots of
// shared memory, the parameter cotangents in registers; the gradient is reduced per
// CTA and added over the CTAs in rank order.
#pragma once

#include "rk4_cluster.cuh"
#include "rk_adjoint.cuh"

namespace cmd {

// 8-byte asynchronous global -> shared copy (cp.async, completes in order per thread).
__device__ __forceinline__ void cp_async8(double* smem_dst, const double* gsrc) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

struct AdjClusterArgs {
    const AdjTraj* traj;
    const int* nbr;            // [G][NAT][Z-LZ] partner words (rank << 24) | offset in that CTA's buffer
    const double* drive;       // [S][6] drive factors at t_n, t_n + dt/2, t_n + dt, or nullptr
    int G;                     // cells
    long long n_steps, ckpt_every;
    double dt;
    int forward_only;
};

// Shared memory of one CTA: seven vectors of NAT*3*Gc doubles (two stage-input / Hbar
// pairs, and lam, the ybar accumulator and the previous stage cotangent of the own
// cells), the reduction scratch and the CTA totals.
__host__ __device__ constexpr long long adj_cluster_smem_doubles(int nat, long long gc) {
    return 7LL * nat * 3 * gc + 32LL * kRedStride + 16;
}

template <int NAT, int Z, int LZ, int CS, int MAXT, int NQ>
__global__ void __launch_bounds__(MAXT, 1)
adjoint_cluster_kernel(const __grid_constant__ Couplings<NAT, Z> cp, const __grid_constant__ ParamDerivs<NAT, Z, NQ> pd,
                       const __grid_constant__ AdjClusterArgs a, int Gc) {
    constexpr int NL = Z - LZ;
    constexpr int NQV = NQ <= 4 ? 4 : 8;       // parameter cotangents padded for the warp reduction
    static_assert(NQ <= NAT * 3 && NQ <= 16, "parameter cotangents park in one own-slot vector");
    extern __shared__ double smem[];
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = (int)cluster.block_rank();
    const long long b = blockIdx.x / CS;
    const AdjTraj& T = a.traj[b];
    const int SBc = NAT * 3 * Gc;
    double* acc2 = smem + 4 * SBc;             // ybar accumulator (sweep) / RK4 sum (forward, recompute)
    double* ybp = smem + 5 * SBc;              // cotangent of the previous VJP stage (sweep)
    double* lamv = smem + 6 * SBc;             // lam, the cotangent of y_{n+1} (backward)
    double* red = smem + 7 * SBc;              // [32][kRedStride]
    double* ctot = red + 32 * kRedStride;      // [16] this CTA's totals
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
    const int G = a.G;
    const int g = rank * Gc + tid;
    const bool own = tid < Gc && g < G;
    const long long V = (long long)NAT * 3 * G;
    const double N = (double)G * NAT;
    const double dt = a.dt;
    const long long S = a.n_steps, C = a.ckpt_every;
    const bool drive_on = a.drive != nullptr;

    const double* base[CS];
#pragma unroll
    for (int r = 0; r < CS; ++r) base[r] = r == rank ? smem : cluster.map_shared_rank(smem, r);
    int nb[NAT][NL > 0 ? NL : 1];
#pragma unroll
    for (int at = 0; at < NAT; ++at)
#pragma unroll
        for (int m = 0; m < NL; ++m) nb[at][m] = own ? a.nbr[((long long)g * NAT + at) * NL + m] : 0;

    // global SoA index of (atom, component) of this thread's cell; own slot in a shared vector
    auto gi = [&](int at, int c) { return (long long)(at * 3 + c) * G + g; };
    auto own_i = [&](int at, int c) { return (at * 3 + c) * Gc + tid; };
    // static + drive field of own atom `at` at the stage input in buffer `in` (own cell values Y)
    auto field = [&](int in, int at, const double (&Y)[NAT][3], double f1, double f2, bool drive_now, double (&H)[3]) {
        if (cp.has_field) {
            H[0] = -cp.field[at][0]; H[1] = -cp.field[at][1]; H[2] = -cp.field[at][2];
        } else {
            H[0] = 0.0; H[1] = 0.0; H[2] = 0.0;
        }
        if (cp.has_onsite) {
#pragma unroll
            for (int d = 0; d < 3; ++d)
                bond_acc(H[d], 2.0 * cp.onsite[at][3 * d], 2.0 * cp.onsite[at][3 * d + 1],
                         2.0 * cp.onsite[at][3 * d + 2], Y[at][0], Y[at][1], Y[at][2]);
        }
#pragma unroll
        for (int n = 0; n < LZ; ++n) {
            const int pb = (at + 1 + n) % NAT;
#pragma unroll
            for (int d = 0; d < 3; ++d)
                bond_acc(H[d], cp.J[at][n][3 * d], cp.J[at][n][3 * d + 1], cp.J[at][n][3 * d + 2], Y[pb][0], Y[pb][1],
                         Y[pb][2]);
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
        if (drive_now) {
#pragma unroll
            for (int d = 0; d < 3; ++d) drive_acc(H[d], cp.d1[at][d], cp.d2[at][d], f1, f2);
        }
    };
    // drive factors of stage s of step n (s = 0: t_n, 1 and 2: t_n + dt/2, 3: t_n + dt)
    auto factors = [&](long long n, int s, double& f1, double& f2) {
        if (!drive_on) { f1 = 0.0; f2 = 0.0; return; }
        const int ti = s == 0 ? 0 : (s == 3 ? 2 : 1);
        f1 = a.drive[n * 6 + 2 * ti];
        f2 = a.drive[n * 6 + 2 * ti + 1];
    };

    double y[NAT][3];
    double* const acc = acc2;                  // RK4 sum of the own cells (forward and recompute)
    // One forward RK4 stage s of this thread's cell from the stage input in buffer `in`
    // (the own values re-read from there); the next stage input goes to buffer `out`
    // (integrator.cuh:115-139).
    auto fwd_stage = [&](int s, int in, int out, double f1, double f2) {
        if (!own) return;
        const bool drive_now = drive_on && (f1 != 0.0 || f2 != 0.0);
        double Y[NAT][3];
#pragma unroll
        for (int at = 0; at < NAT; ++at)
#pragma unroll
            for (int c = 0; c < 3; ++c) Y[at][c] = smem[in + own_i(at, c)];
#pragma unroll
        for (int at = 0; at < NAT; ++at) {
            double H[3];
            field(in, at, Y, f1, f2, drive_now, H);
            const double kk[3] = {H[1] * Y[at][2] - H[2] * Y[at][1], H[2] * Y[at][0] - H[0] * Y[at][2],
                                  H[0] * Y[at][1] - H[1] * Y[at][0]};
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const int i = own_i(at, c);
                double v;
                if (s == 0) {
                    acc[i] = kk[c];
                    v = 1.0 * y[at][c] + (0.5 * dt) * kk[c];
                } else if (s == 1) {
                    acc[i] = acc[i] + 2.0 * kk[c];
                    v = 1.0 * y[at][c] + (0.5 * dt) * kk[c];
                } else if (s == 2) {
                    acc[i] = acc[i] + 2.0 * kk[c];
                    v = 1.0 * y[at][c] + dt * kk[c];
                } else {
                    y[at][c] += (dt / 6.0) * (acc[i] + kk[c]);
                    v = y[at][c];
                }
                smem[out + i] = v;
            }
        }
    };
    // M_local partial sums: warp-reduced into red (stage 1), CTA totals into ctot (stage 2)
    auto reduce_m = [&](double (&part)[4]) {
        const double r = warp_reduce_many<4>(part);
        if ((lane & 7) == 0) red[warp * kRedStride + (lane >> 3)] = r;
    };
    auto finish_cta = [&](int nv) {
        for (int q = warp; q < nv; q += nwarps) {
            double s = lane < nwarps ? red[lane * kRedStride + q] : 0.0;
#pragma unroll
            for (int o = 16; o >= 1; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (lane == 0) ctot[q] = s;
        }
    };
    const int ctot_off = 7 * SBc + 32 * kRedStride;
    double loss = 0.0;                         // rank 0, thread 0
    // rank 0, thread 0: M_local(y_n) = sum over the CTAs (rank order) / N, and the loss term
    auto record = [&](long long n) {
        if (rank != 0 || tid != 0) return;
        for (int c = 0; c < 3; ++c) {
            double s = 0.0;
#pragma unroll
            for (int r = 0; r < CS; ++r) s += pick_rank<CS>(base, r)[ctot_off + c];
            const double mc = s / N;
            T.mloc[3 * n + c] = mc;
            const double e = mc - T.target[3 * n + c];
            loss += e * e;
        }
    };

    // ---------------- phase 1: forward ----------------
#pragma unroll
    for (int at = 0; at < NAT; ++at)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double v = own ? T.y0[((long long)g * NAT + at) * 3 + c] : 0.0;
            y[at][c] = v;
            if (own) smem[own_i(at, c)] = v;
        }
    cluster.sync();
    {
        int in = 0, out = SBc;
        double part[4];
        for (long long n = 0; n < S; ++n) {
            if (!a.forward_only && own && n % C == 0) {
                double* dst = T.ckpt + (n / C) * V;
#pragma unroll
                for (int at = 0; at < NAT; ++at)
#pragma unroll
                    for (int c = 0; c < 3; ++c) dst[gi(at, c)] = y[at][c];
            }
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                if (s == 0) {
#pragma unroll
                    for (int q = 0; q < 4; ++q) part[q] = 0.0;
                    if (own)
#pragma unroll
                        for (int at = 0; at < NAT; ++at)
#pragma unroll
                            for (int c = 0; c < 3; ++c) part[c] += y[at][c];
                }
                if (s == 1) reduce_m(part);
                if (s == 2) finish_cta(3);
                if (s == 3) record(n);
                double f1, f2;
                factors(n, s, f1, f2);
                fwd_stage(s, in, out, f1, f2);
                cluster.sync();
                const int tmp = in; in = out; out = tmp;
            }
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) part[q] = 0.0;
        if (own)
#pragma unroll
            for (int at = 0; at < NAT; ++at)
#pragma unroll
                for (int c = 0; c < 3; ++c) part[c] += y[at][c];
        reduce_m(part);
        __syncthreads();
        finish_cta(3);
        cluster.sync();
        record(S);
        if (rank == 0 && tid == 0) T.loss[0] = loss;
        cluster.sync();                        // the remote ctot reads are done
    }
    if (a.forward_only) return;

    // ---------------- phase 2: backward ----------------
    double gq[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) gq[q] = 0.0;
    auto dl = [&](long long n, double (&o)[3]) {
#pragma unroll
        for (int c = 0; c < 3; ++c) o[c] = 2.0 * (T.mloc[3 * n + c] - T.target[3 * n + c]) / N;
    };
    if (own) {
        double d0[3];
        dl(S, d0);
#pragma unroll
        for (int at = 0; at < NAT; ++at)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                lamv[own_i(at, c)] = d0[c];
                ybp[own_i(at, c)] = 0.0;
            }
    }
    auto slot = [&](long long j, int s) { return T.seg + (j * 4 + s) * V; };
    const long long K = (S + C - 1) / C;
    for (long long sg = K - 1; sg >= 0; --sg) {
        const long long n0 = sg * C;
        const long long n1 = (n0 + C < S) ? n0 + C : S;
        // the parameter cotangents wait in the own slots of ybp (idle between sweeps) while
        // the recompute holds y and its temporaries in registers
        if (own) {
#pragma unroll
            for (int q = 0; q < NQ; ++q) ybp[q * Gc + tid] = gq[q];
        }
        // recompute the segment from its checkpoint, storing every stage input
#pragma unroll
        for (int at = 0; at < NAT; ++at)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const double v = own ? T.ckpt[sg * V + gi(at, c)] : 0.0;
                y[at][c] = v;
                if (own) smem[own_i(at, c)] = v;
            }
        cluster.sync();
        int in = 0, out = SBc;
        for (long long n = n0; n < n1; ++n) {
            const long long j = n - n0;
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                if (own) {
                    double* dst = slot(j, s);
#pragma unroll
                    for (int at = 0; at < NAT; ++at)
#pragma unroll
                        for (int c = 0; c < 3; ++c) dst[gi(at, c)] = smem[in + own_i(at, c)];
                }
                double f1, f2;
                factors(n, s, f1, f2);
                fwd_stage(s, in, out, f1, f2);
                cluster.sync();
                const int tmp = in; in = out; out = tmp;
            }
        }
        if (own) {
#pragma unroll
            for (int q = 0; q < NQ; ++q) gq[q] = ybp[q * Gc + tid];
        }
        // reverse sweep.  The own stage input of each VJP stage arrives in the stage's
        // buffer pair by cp.async, issued right after the previous stage's barrier (that
        // pair's last partner reads were two stages ago).
        int vb = 0;
        auto fetch = [&](long long jj, int ss, int dst) {
            if (!own) return;
            const double* src = slot(jj, ss);
#pragma unroll
            for (int at = 0; at < NAT; ++at)
#pragma unroll
                for (int c = 0; c < 3; ++c) cp_async8(smem + dst + own_i(at, c), src + gi(at, c));
            cp_async_commit();
        };
        fetch(n1 - 1 - n0, 3, vb);
        for (long long n = n1 - 1; n >= n0; --n) {
            const long long j = n - n0;
            double dln[3];
            dl(n, dln);
#pragma unroll 1
            for (int s = 3; s >= 0; --s) {
                const double ca = (s == 0 || s == 3) ? dt / 6.0 : dt / 3.0;
                const double cb = s == 3 ? 0.0 : (s == 2 ? dt : 0.5 * dt);
                const int ob = vb == 0 ? 2 * SBc : 0;
                cp_async_wait_all();
                if (own) {              // publish Hbar_i = Y_i x v_i next to Y
#pragma unroll
                    for (int at = 0; at < NAT; ++at) {
                        double Y[3], v[3];
#pragma unroll
                        for (int c = 0; c < 3; ++c) {
                            Y[c] = smem[vb + own_i(at, c)];
                            v[c] = ca * lamv[own_i(at, c)];
                            if (cb != 0.0) v[c] = v[c] + cb * ybp[own_i(at, c)];
                        }
                        smem[vb + SBc + own_i(at, 0)] = Y[1] * v[2] - Y[2] * v[1];
                        smem[vb + SBc + own_i(at, 1)] = Y[2] * v[0] - Y[0] * v[2];
                        smem[vb + SBc + own_i(at, 2)] = Y[0] * v[1] - Y[1] * v[0];
                    }
                }
                cluster.sync();
                if (s > 0) fetch(j, s - 1, ob);
                else if (n > n0) fetch(j - 1, 3, ob);
                if (own) {
                    double f1, f2;
                    factors(n, s, f1, f2);
                    const bool drive_now = drive_on && (f1 != 0.0 || f2 != 0.0);
                    // own Y / Hbar of atom k in this pair
                    auto Yo = [&](int k, int c) { return smem[vb + own_i(k, c)]; };
                    auto Ho = [&](int k, int c) { return smem[vb + SBc + own_i(k, c)]; };
#pragma unroll
                    for (int at = 0; at < NAT; ++at) {
                        const double S0 = Yo(at, 0), S1 = Yo(at, 1), S2 = Yo(at, 2);
                        const double hb[3] = {Ho(at, 0), Ho(at, 1), Ho(at, 2)};
                        double H[3], sb[3] = {0.0, 0.0, 0.0};
#pragma unroll
                        for (int d = 0; d < 3; ++d) H[d] = cp.has_field ? -cp.field[at][d] : 0.0;
                        if (cp.has_onsite) {
#pragma unroll
                            for (int d = 0; d < 3; ++d) {
                                bond_acc(H[d], 2.0 * cp.onsite[at][3 * d], 2.0 * cp.onsite[at][3 * d + 1],
                                         2.0 * cp.onsite[at][3 * d + 2], S0, S1, S2);
                                sb[d] += 2.0 * (cp.onsite[at][d] * hb[0] + cp.onsite[at][3 + d] * hb[1] +
                                                cp.onsite[at][6 + d] * hb[2]);
                            }
                        }
#pragma unroll
                        for (int q = 0; q < NQ; ++q) {
                            double tq = -(hb[0] * pd.DB[q][at][0] + hb[1] * pd.DB[q][at][1] + hb[2] * pd.DB[q][at][2]);
                            if (pd.has_DA) {
#pragma unroll
                                for (int d = 0; d < 3; ++d)
                                    tq += 2.0 * hb[d] * (pd.DA[q][at][3 * d] * S0 + pd.DA[q][at][3 * d + 1] * S1 +
                                                         pd.DA[q][at][3 * d + 2] * S2);
                            }
                            gq[q] += tq;
                        }
                        auto bond = [&](int n_, const double (&P)[3], const double (&Q)[3]) {
#pragma unroll
                            for (int d = 0; d < 3; ++d) {
                                bond_acc(H[d], cp.J[at][n_][3 * d], cp.J[at][n_][3 * d + 1], cp.J[at][n_][3 * d + 2],
                                         P[0], P[1], P[2]);
                                bond_acc(sb[d], cp.J[at][n_][3 * d], cp.J[at][n_][3 * d + 1],
                                         cp.J[at][n_][3 * d + 2], Q[0], Q[1], Q[2]);
                            }
#pragma unroll
                            for (int q = 0; q < NQ; ++q) {
                                if (!pd.dj_any[q]) continue;        // e.g. a field parameter
                                const double* D = pd.DJ[q][at][n_];
                                gq[q] += S0 * (D[0] * Q[0] + D[1] * Q[1] + D[2] * Q[2]) +
                                         S1 * (D[3] * Q[0] + D[4] * Q[1] + D[5] * Q[2]) +
                                         S2 * (D[6] * Q[0] + D[7] * Q[1] + D[8] * Q[2]);
                            }
                        };
#pragma unroll
                        for (int n_ = 0; n_ < LZ; ++n_) {
                            const int pb = (at + 1 + n_) % NAT;
                            const double P[3] = {Yo(pb, 0), Yo(pb, 1), Yo(pb, 2)};
                            const double Q[3] = {Ho(pb, 0), Ho(pb, 1), Ho(pb, 2)};
                            bond(n_, P, Q);
                        }
#pragma unroll
                        for (int m = 0; m < NL; ++m) {
                            const int n_ = LZ + m;
                            if (n_ < cp.zc[at]) {
                                const int w = nb[at][m];
                                const double* src = pick_rank<CS>(base, w >> kClusterRankShift);
                                const int p = vb + (w & kClusterOffsetMask);
                                const double P[3] = {src[p], src[p + Gc], src[p + 2 * Gc]};
                                const double Q[3] = {src[p + SBc], src[p + SBc + Gc], src[p + SBc + 2 * Gc]};
                                bond(n_, P, Q);
                            }
                        }
                        if (drive_now) {
#pragma unroll
                            for (int d = 0; d < 3; ++d) drive_acc(H[d], cp.d1[at][d], cp.d2[at][d], f1, f2);
                        }
                        double v[3];
#pragma unroll
                        for (int c = 0; c < 3; ++c) {
                            v[c] = ca * lamv[own_i(at, c)];
                            if (cb != 0.0) v[c] = v[c] + cb * ybp[own_i(at, c)];
                        }
                        sb[0] += v[1] * H[2] - v[2] * H[1];
                        sb[1] += v[2] * H[0] - v[0] * H[2];
                        sb[2] += v[0] * H[1] - v[1] * H[0];
#pragma unroll
                        for (int d = 0; d < 3; ++d) {
                            const int i = own_i(at, d);
                            if (s == 3) {
                                ybp[i] = sb[d];
                                acc2[i] = lamv[i] + sb[d];
                            } else if (s > 0) {
                                ybp[i] = sb[d];
                                acc2[i] = acc2[i] + sb[d];
                            } else {
                                lamv[i] = acc2[i] + sb[d] + dln[d];
                            }
                        }
                    }
                }
                vb = ob;
            }
        }
        cluster.sync();                        // the last VJP stage's partner reads are done
    }
    // gradient: per-CTA totals, then rank 0 adds the CTAs in rank order
    {
        double v[NQV];
#pragma unroll
        for (int q = 0; q < NQV; ++q) v[q] = q < NQ ? gq[q] : 0.0;
        const double r = warp_reduce_many<NQV>(v);
        constexpr int span = 32 / NQV;
        if ((lane % span) == 0) red[warp * kRedStride + lane / span] = r;
        __syncthreads();
        finish_cta(NQ);
        cluster.sync();
        if (rank == 0 && tid < NQ) {
            double s = 0.0;
#pragma unroll
            for (int r2 = 0; r2 < CS; ++r2) s += pick_rank<CS>(base, r2)[ctot_off + tid];
            T.grad[tid] = s;
        }
        cluster.sync();
    }
}

}  // namespace cmd
