// rk45_onchip.cuh -- controlled Dormand-Prince 5(4) with every RK vector on chip:
// one trajectory per CTA, or per thread-block cluster of CS CTAs (CS SMs), APT
// sites of one unit cell per thread (APT = NAT: a whole cell; APT = 1: one site).
//
// Step control is the CPU path of the reference (Boost.Odeint
// make_controlled<runge_kutta_dopri5> driven by integrate_adaptive,
// lattice.h:4072-4078), with the arithmetic in the same order as the oracle's
// restatement (stage inputs y + dt a_s1 K1 + dt a_s2 K2 + ..., the embedded
// error dt dc1 K1 + ... + dt dc7 K7, the error norm
// max_i |err_i| / (abs + rel (|y_i| + dt |K1_i|)), reject with
// dt *= max(0.9 err^(-1/3), 0.2), accept and grow with
// dt *= 0.9 max(err, 5^-5)^(-1/5) when err < 0.5, the last step cut to land on
// T_end, FSAL reuse of the seventh stage), so accepted / rejected step
// sequences are the oracle's.
//
// Layout (B200: 227 KB shared memory, 64K registers per SM):
//   * CTA `rank` of the cluster owns cells [rank*Gc, rank*Gc + Gc); thread t
//     advances atoms [ag*APT, ag*APT + APT) of cell rank*Gc + t % Gp, atom
//     group ag = t / Gp (Gp = Gc rounded up to a multiple of 32, so ag is
//     uniform per warp and is dispatched to a compile-time constant): every
//     coupling matrix is a compile-time-indexed kernel-parameter (constant-
//     bank) operand, and bonds to atoms of the cell the thread owns read the
//     partner from registers.  APT trades registers per thread (whole cells:
//     ILP, in-cell bonds in registers) against threads per SM (single sites:
//     more warps to hide latency); the autotuner picks;
//   * y, K1 and the current stage input stay in registers; K2..K5 and, from
//     stage 6, the first terms of the embedded error sit in the thread's own
//     slots of shared memory; the stage input other threads read is published
//     in shared memory, double buffered, SoA buf[(atom*3 + comp)*Gp + cell];
//   * the five stage rows of stages 2..5 run as one loop over a constant-memory
//     table (one copy of the right-hand side in the loop body keeps the
//     register footprint small), stage 6 and the FSAL stage 7 explicitly;
//   * a partner in another cell is read through an offset into this CTA's
//     buffer (one CTA) or a 32-bit shared::cluster address of the partner
//     CTA's buffer computed once (cluster), so a partner in another CTA costs
//     one distributed-shared-memory load per component;
//   * one barrier per stage (cluster-scope release/acquire when CS > 1) and
//     one per attempted step for the reduction: every warp stores its error
//     maximum into every CTA of the cluster and its observable partials (sum
//     of S per atom class and sum S.(H - B) of the new state, from the
//     seventh stage's field) into rank 0, so after the barrier each warp forms
//     the error maximum locally -- identical in every thread, so all take the
//     same decision -- and rank 0 adds the observables in a fixed order (warp
//     butterfly, warps in order, CTAs in rank order) and writes the row.
#pragma once

#include <cooperative_groups.h>
#include <stdint.h>

#include "rk4_cluster.cuh"
#include "rk_global.cuh"

namespace cmd {

struct R45Args {
    const GTraj* traj;        // this launch's trajectories (one per CTA / cluster)
    const int* pw;            // [G][NAT][Z-LZ] partner words (rank << 24) | SoA offset in that CTA's buffer
    int G;                    // cells per trajectory
    int Gc;                   // cells per CTA
    int Gp;                   // Gc rounded up to a multiple of 32 (threads per CTA)
    int Gs;                   // row length of the two stage buffers: Gp own cells, then (halo tilings) the
                              // columns of partners owned by other CTAs of the cluster
    const int* push;          // halo tilings: [G][NAT][Z-LZ] words (rank << 24) | slot in that CTA's stage
                              // buffer 0 this site's stage inputs are pushed to, or -1
    double abs_tol, rel_tol;
    int max_steps;            // cap on accepted steps, 1 .. 2^31 - 2 (the host turns "none" into the largest)
    double width, freq;       // pulse envelope
    const double* frames;     // [NAT*9] (device)
    const double* afm;        // [NAT]
};

// Reduction values per warp: the observable partials padded to a power of two.
__host__ __device__ constexpr int r45_nv(int nat) { return 3 * nat + 1 <= 8 ? 8 : 16; }

// Shared memory of one CTA in doubles: two stage buffers of row length gs,
// K2..K5 (and, with yk, y and K1) of row length gp, the per-warp error maxima of
// every CTA [cs][maxt/32], rank 0's per-warp observable partials
// [cs][maxt/32][nv] and the drive factors [12].
__host__ __device__ constexpr long long r45_smem_doubles(int nat, int gp, int gs, int cs, int maxt, bool yk = false) {
    return 2LL * nat * 3 * gs + (yk ? 6LL : 4LL) * nat * 3 * gp + (long long)cs * (maxt / 32) * (1 + r45_nv(nat)) +
           12;
}

__device__ __forceinline__ uint32_t r45_map(uint32_t local, int rank) {
    uint32_t out;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(out) : "r"(local), "r"(rank));
    return out;
}

// Barrier of the trajectory's CTAs (cluster-scope release / acquire when CS > 1).
// Returns 0 in a way the compiler cannot see through: every distributed-shared-
// memory address of the following stage adds it, so no load of a partner's
// stage input moves above the barrier that publishes it.
template <int CS>
__device__ __forceinline__ uint32_t r45_sync() {
    uint32_t tok;
    if constexpr (CS > 1)
        asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;\n\tmov.u32 %0, 0;"
                     : "=r"(tok)::"memory");
    else
        asm volatile("bar.sync 0;\n\tmov.u32 %0, 0;" : "=r"(tok)::"memory");
    return tok;
}

__device__ __forceinline__ double r45_ld_cluster(uint32_t addr) {
    double v;
    asm("ld.shared::cluster.f64 %0, [%1];" : "=d"(v) : "r"(addr));
    return v;
}

__device__ __forceinline__ void r45_st_cluster(uint32_t addr, double v) {
    asm volatile("st.shared::cluster.f64 [%0], %1;" ::"r"(addr), "d"(v) : "memory");
}

// Dormand-Prince 5(4) stage rows (Dormand & Prince 1980): row r forms the
// input of stage r + 2 from K1..K_{r+1}.
__constant__ double kR45A[5][5] = {
    {1.0 / 5.0, 0, 0, 0, 0},
    {3.0 / 40.0, 9.0 / 40.0, 0, 0, 0},
    {44.0 / 45.0, -56.0 / 15.0, 32.0 / 9.0, 0, 0},
    {19372.0 / 6561.0, -25360.0 / 2187.0, 64448.0 / 6561.0, -212.0 / 729.0, 0},
    {9017.0 / 3168.0, -355.0 / 33.0, 46732.0 / 5247.0, 49.0 / 176.0, -5103.0 / 18656.0}};

// k = f(stage input) for the APT atoms of atom group AG of this thread's cell,
// the stage input published in buffer `in` (own atoms also in cur); with OBS
// the atoms' observable partials (S, then S.(H - B) summed) go to part.  Every
// product has a run-time operand, so the couplings stay constant-bank operands
// instead of values held across the step loop: -B as z - B with z = +0 from the
// barrier token, 2 A S as A (2 S) and -d f as d (-f) (all exact rewrites).
template <int NAT, int Z, int LZ, int APT, int CS, bool HALO, bool OBS, int AG>
__device__ __forceinline__ void r45_rhs_group(const Couplings<NAT, Z>& cp, const double* smem, int in, int lc,
                                              int Gp, const uint32_t (&pa)[APT][(Z - LZ) > 0 ? (Z - LZ) : 1],
                                              uint32_t tok, double f1, double f2, bool drive,
                                              const double (&cur)[APT][3], double (&k)[APT][3], double* part) {
    constexpr int NL = Z - LZ;
    const double z = __longlong_as_double((long long)tok);
    const double nf1 = -f1, nf2 = -f2;
#pragma unroll
    for (int a = 0; a < APT; ++a) {
        constexpr int base = AG * APT;
        const int at = base + a;
        double P[NL > 0 ? NL : 1][3];
#pragma unroll
        for (int m = 0; m < NL; ++m)
            if (LZ + m < cp.zc[at]) {
                if constexpr (CS > 1 && !HALO) {
                    const uint32_t p0 = pa[a][m] + 8u * (uint32_t)in + tok, cs = 8u * (uint32_t)Gp;
                    P[m][0] = r45_ld_cluster(p0);
                    P[m][1] = r45_ld_cluster(p0 + cs);
                    P[m][2] = r45_ld_cluster(p0 + 2u * cs);
                } else {
                    const int p0 = (int)pa[a][m] + in;
                    P[m][0] = smem[p0];
                    P[m][1] = smem[p0 + Gp];
                    P[m][2] = smem[p0 + 2 * Gp];
                }
            }
        // partners inside the cell: registers when this thread owns them, else
        // this CTA's buffer
        double L[LZ > 0 ? LZ : 1][3];
#pragma unroll
        for (int n = 0; n < LZ; ++n) {
            const int pb = (at + 1 + n) % NAT;
#pragma unroll
            for (int c = 0; c < 3; ++c)
                L[n][c] = (pb / APT == AG) ? cur[pb % APT][c] : smem[in + (pb * 3 + c) * Gp + lc];
        }
        double H[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) H[d] = cp.has_field ? z - cp.field[at][d] : z;
        if (cp.has_onsite) {
            const double s0 = 2.0 * cur[a][0], s1 = 2.0 * cur[a][1], s2 = 2.0 * cur[a][2];
#pragma unroll
            for (int d = 0; d < 3; ++d)
                bond_acc(H[d], cp.onsite[at][3 * d], cp.onsite[at][3 * d + 1], cp.onsite[at][3 * d + 2], s0, s1, s2);
        }
#pragma unroll
        for (int n = 0; n < LZ; ++n) {
#pragma unroll
            for (int d = 0; d < 3; ++d)
                bond_acc(H[d], cp.J[at][n][3 * d], cp.J[at][n][3 * d + 1], cp.J[at][n][3 * d + 2], L[n][0], L[n][1],
                         L[n][2]);
        }
#pragma unroll
        for (int m = 0; m < NL; ++m)
            if (LZ + m < cp.zc[at]) {
#pragma unroll
                for (int d = 0; d < 3; ++d)
                    bond_acc(H[d], cp.J[at][LZ + m][3 * d], cp.J[at][LZ + m][3 * d + 1], cp.J[at][LZ + m][3 * d + 2],
                             P[m][0], P[m][1], P[m][2]);
            }
        if constexpr (OBS) {
            part[3 * a] = cur[a][0];
            part[3 * a + 1] = cur[a][1];
            part[3 * a + 2] = cur[a][2];
            part[3 * APT] += cur[a][0] * (H[0] - cp.field[at][0]) + cur[a][1] * (H[1] - cp.field[at][1]) +
                             cur[a][2] * (H[2] - cp.field[at][2]);
        }
        if (drive) {
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                H[d] = fma(cp.d1[at][d], nf1, H[d]);
                H[d] = fma(cp.d2[at][d], nf2, H[d]);
            }
        }
        k[a][0] = H[1] * cur[a][2] - H[2] * cur[a][1];
        k[a][1] = H[2] * cur[a][0] - H[0] * cur[a][2];
        k[a][2] = H[0] * cur[a][1] - H[1] * cur[a][0];
    }
}

// r45_rhs_group with the warp-uniform atom group `ag` as a compile-time constant.
template <int NAT, int Z, int LZ, int APT, int CS, bool HALO, bool OBS, int AG = 0>
__device__ __forceinline__ void r45_rhs(int ag, const Couplings<NAT, Z>& cp, const double* smem, int in, int lc,
                                        int Gp, const uint32_t (&pa)[APT][(Z - LZ) > 0 ? (Z - LZ) : 1],
                                        uint32_t tok, double f1, double f2, bool drive, const double (&cur)[APT][3],
                                        double (&k)[APT][3], double* part) {
    if constexpr (AG + 1 < NAT / APT) {
        if (ag != AG) {
            r45_rhs<NAT, Z, LZ, APT, CS, HALO, OBS, AG + 1>(ag, cp, smem, in, lc, Gp, pa, tok, f1, f2, drive, cur, k,
                                                            part);
            return;
        }
    }
    r45_rhs_group<NAT, Z, LZ, APT, CS, HALO, OBS, AG>(cp, smem, in, lc, Gp, pa, tok, f1, f2, drive, cur, k, part);
}

// Observable partials of a thread: S of its APT atoms, then S.(H - B), padded.
__host__ __device__ constexpr int r45_nvl(int apt) { return 3 * apt + 1 <= 4 ? 4 : (3 * apt + 1 <= 8 ? 8 : 16); }

template <int NAT, int Z, int LZ, int APT, int CS, int MAXT, bool YK = false, bool HALO = false>
__global__ void __launch_bounds__(MAXT, 1)
rk45_onchip_kernel(const __grid_constant__ Couplings<NAT, Z> cp, const __grid_constant__ R45Args a) {
    constexpr int NL = Z - LZ;                       // bonds per atom leaving the cell
    constexpr int NR = 3 * NAT + 1;                  // observables per row
    constexpr int NV = r45_nv(NAT);                  // observable slots per warp (rank 0's table)
    constexpr int NVL = r45_nvl(APT);                // observable partials per thread
    constexpr int NWM = MAXT / 32;                   // warps per CTA at most
    static constexpr double c2 = 1.0 / 5.0, c3 = 3.0 / 10.0, c4 = 4.0 / 5.0, c5 = 8.0 / 9.0;
    static constexpr double b1 = 35.0 / 384.0, b3 = 500.0 / 1113.0, b4 = 125.0 / 192.0,
                            b5 = -2187.0 / 6784.0, b6 = 11.0 / 84.0;
    static constexpr double dc1 = b1 - 5179.0 / 57600.0, dc3 = b3 - 7571.0 / 16695.0,
                            dc4 = b4 - 393.0 / 640.0, dc5 = b5 - (-92097.0 / 339200.0),
                            dc6 = b6 - 187.0 / 2100.0, dc7 = -1.0 / 40.0;
    const double eps = 2.220446049250313e-16;        // numeric_limits<double>::epsilon

    extern __shared__ double smem[];
    int rank = 0;
    if constexpr (CS > 1) rank = (int)cooperative_groups::this_cluster().block_rank();
    const GTraj& T = a.traj[blockIdx.x / CS];
    const int Gp = a.Gp, SB = NAT * 3 * Gp;          // K slots (and y, K1): rows of Gp
    const int Gs = a.Gs, SBs = NAT * 3 * Gs;         // stage buffers: rows of Gs
    double* Ks = smem + 2 * SBs;                     // K2, K3, K4, K5: [4][SB], own slots
    double* emx = Ks + (YK ? 6 : 4) * SB;            // [CS][NWM] per-warp error maxima of every CTA
    double* obs = emx + CS * NWM;                    // [CS][NWM][NV] per-warp observable partials (rank 0 reads)
    double* drv = obs + CS * NWM * NV;               // [12] drive factors of stages 2..6 (pulse 1, 2)
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
    const int ag = tid / Gp, lc = tid - ag * Gp;     // atom group (warp-uniform) and cell of this thread
    const int g = rank * a.Gc + lc;
    const bool own = lc < a.Gc && g < a.G;
    const int me = ag * APT * 3 * Gs + lc;           // own stage-buffer slot of atom 0 of the group, component 0
    const int mk = ag * APT * 3 * Gp + lc;           // its K slot
    const bool drive = T.pulse.a1 != 0.0 || T.pulse.a2 != 0.0;
    const double Nsites = (double)a.G * NAT;

    // partners outside the cell: word offset into this CTA's buffer 0 (one CTA)
    // or shared::cluster byte address of the partner's slot in buffer 0 (cluster)
    uint32_t pa[APT][NL > 0 ? NL : 1];
    const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(smem);
#pragma unroll
    for (int i = 0; i < APT; ++i)
#pragma unroll
        for (int m = 0; m < NL; ++m) {
            const int w = own ? a.pw[((long long)g * NAT + ag * APT + i) * NL + m] : ((rank << kClusterRankShift) | lc);
            if constexpr (CS > 1 && !HALO)
                pa[i][m] = r45_map(sbase + 8u * (uint32_t)(w & kClusterOffsetMask), w >> kClusterRankShift);
            else
                pa[i][m] = (uint32_t)(w & kClusterOffsetMask);
        }
    // halo tilings: shared::cluster addresses (buffer 0, component 0) of the
    // other CTAs' halo slots this thread's sites are pushed to (~0: none)
    uint32_t pd[APT][HALO && NL > 0 ? NL : 1];
#pragma unroll
    for (int i = 0; i < APT; ++i)
#pragma unroll
        for (int d = 0; d < (HALO && NL > 0 ? NL : 1); ++d) {
            pd[i][d] = ~0u;
            if constexpr (HALO) {
                const int w = own ? a.push[((long long)g * NAT + ag * APT + i) * NL + d] : -1;
                if (w >= 0) pd[i][d] = r45_map(sbase + 8u * (uint32_t)(w & kClusterOffsetMask), w >> kClusterRankShift);
            }
        }
    // this warp's reduction slots
    const uint32_t emx_slot = (uint32_t)__cvta_generic_to_shared(emx + rank * NWM + warp);
    const uint32_t obs_slot = (uint32_t)__cvta_generic_to_shared(obs + (rank * NWM + warp) * NV);

    // y and K1 of the thread's atoms: registers, or (YK) its own slots of two
    // more shared-memory vectors, which leaves registers to the stages
    double yr[APT][3], k1r[APT][3], cur[APT][3];
    auto yref = [&](int i, int c) __attribute__((always_inline)) -> double& {
        if constexpr (YK) return Ks[4 * SB + mk + (i * 3 + c) * Gp];
        else return yr[i][c];
    };
    auto k1ref = [&](int i, int c) __attribute__((always_inline)) -> double& {
        if constexpr (YK) return Ks[5 * SB + mk + (i * 3 + c) * Gp];
        else return k1r[i][c];
    };
#pragma unroll
    for (int i = 0; i < APT; ++i)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            yref(i, c) = own ? T.y0[((long long)g * NAT + ag * APT + i) * 3 + c] : 0.0;
            cur[i][c] = yref(i, c);
        }

    auto rhs = [&](int in, uint32_t tok, double f1, double f2, double (&k)[APT][3]) __attribute__((always_inline)) {
        r45_rhs<NAT, Z, LZ, APT, CS, HALO, false>(ag, cp, smem, in, lc, Gs, pa, tok, f1, f2, drive, cur, k, nullptr);
    };
    auto rhs_obs = [&](int in, uint32_t tok, double f1, double f2, double (&k)[APT][3], double (&part)[NVL])
        __attribute__((always_inline)) {
        r45_rhs<NAT, Z, LZ, APT, CS, HALO, true>(ag, cp, smem, in, lc, Gs, pa, tok, f1, f2, drive, cur, k, part);
    };
    // Publishes v as the next stage input of own atom i (registers and buffer
    // `out`; halo tilings also store it into the halo slots of the other CTAs
    // that read it, made visible by the cluster barrier that follows).
    auto publish = [&](int out, int i, int c, double v) __attribute__((always_inline)) {
        cur[i][c] = v;
        smem[out + me + (i * 3 + c) * Gs] = v;
        if constexpr (HALO) {
#pragma unroll
            for (int d = 0; d < (NL > 0 ? NL : 1); ++d)
                if (pd[i][d] != ~0u) r45_st_cluster(pd[i][d] + 8u * (uint32_t)(out + c * Gs), v);
        }
    };
    // the initial state is the first stage input (halo tilings store into the
    // other CTAs only once every CTA of the cluster runs)
    if constexpr (HALO) r45_sync<CS>();
#pragma unroll
    for (int i = 0; i < APT; ++i)
#pragma unroll
        for (int c = 0; c < 3; ++c) publish(0, i, c, yref(i, c));

    // One barrier: every warp's error maximum lands in every CTA, its observable
    // partials (placed at their atoms' rows, zeros elsewhere) in rank 0;
    // afterwards every warp forms the maximum over all warps of all CTAs, and
    // rank 0's warp 0 lane q holds observable q (summed over warps in order, CTAs
    // in rank order).
    auto reduce = [&](double (&part)[NVL], double emax, double& obs_q) __attribute__((always_inline)) -> double {
        const double r = warp_reduce_many<NVL>(part);
        constexpr int span = 32 / NVL;               // lane span * j holds partial j
        double m = emax;
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        // lane q < NV: this warp's contribution to observable q
        const int qa = lane / 3;
        int j = -1;
        if (lane < 3 * NAT && qa / APT == ag) j = (qa % APT) * 3 + (lane - 3 * qa);
        else if (lane == 3 * NAT) j = 3 * APT;
        const double vq = __shfl_sync(0xffffffffu, r, (j < 0 ? 0 : j) * span);
        const double val = j < 0 ? 0.0 : vq;
        if constexpr (CS > 1) {
            if (lane < CS) r45_st_cluster(r45_map(emx_slot, lane), m);
            if (lane < NV) r45_st_cluster(r45_map(obs_slot, 0) + 8u * (uint32_t)lane, val);
        } else {
            if (lane == 0) emx[warp] = m;
            if (lane < NV) obs[warp * NV + lane] = val;
        }
        r45_sync<CS>();
        double err = 0.0;
        for (int i = lane; i < CS * NWM; i += 32)
            if ((i % NWM) < nwarps) err = fmax(err, emx[i]);
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) err = fmax(err, __shfl_xor_sync(0xffffffffu, err, o));
        if (rank == 0 && warp == 0) {
            double s = 0.0;
            if (lane < NR)
                for (int r2 = 0; r2 < CS; ++r2)
                    for (int w = 0; w < nwarps; ++w) s += obs[(r2 * NWM + w) * NV + lane];
            obs_q = s;
        }
        return err;
    };

    int nrow = 0;                                    // 32-bit counters: fewer registers held across the steps
    // Row nrow = {t, M_af, M_local, M_global, E/N} from the observable sums held
    // by rank 0's warp 0 (lane q: observable q); states of the row if saved.
    auto record = [&](double t, double obs_q) __attribute__((always_inline)) {
        if (nrow < T.max_rows) {
            if (T.traj && own) {
                double* dst = T.traj + (long long)nrow * a.G * NAT * 3 + ((long long)g * NAT + ag * APT) * 3;
#pragma unroll
                for (int i = 0; i < APT; ++i)
#pragma unroll
                    for (int c = 0; c < 3; ++c) dst[i * 3 + c] = yref(i, c);
            }
            if (rank == 0 && warp == 0) {
                double m[NR];
#pragma unroll
                for (int q = 0; q < NR; ++q) m[q] = __shfl_sync(0xffffffffu, obs_q, q);
                if (lane == 0) {
                    double ml[3] = {0, 0, 0}, mg[3] = {0, 0, 0}, ma[3] = {0, 0, 0};
#pragma unroll
                    for (int a2 = 0; a2 < NAT; ++a2) {
                        const double* R = a.frames + 9 * a2;
#pragma unroll
                        for (int d = 0; d < 3; ++d) {
                            ml[d] += m[3 * a2 + d];
                            const double v = R[3 * d] * m[3 * a2] + R[3 * d + 1] * m[3 * a2 + 1] +
                                             R[3 * d + 2] * m[3 * a2 + 2];
                            mg[d] += v;
                            ma[d] += a.afm[a2] * v;
                        }
                    }
                    double* o = T.rows + (long long)nrow * 11;
                    o[0] = t;
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        o[1 + d] = ma[d] / Nsites;
                        o[4 + d] = ml[d] / Nsites;
                        o[7 + d] = mg[d] / Nsites;
                    }
                    o[10] = 0.5 * m[3 * NAT] / Nsites;
                }
            }
        }
        ++nrow;
    };
    auto factor = [&](int p, double ts) __attribute__((always_inline)) {
        return p == 0 ? drive_factor(T.pulse.a1, ts - T.pulse.t1, a.width, a.freq)
                      : drive_factor(T.pulse.a2, ts - T.pulse.t2, a.width, a.freq);
    };

    double t = T.T0;
    uint32_t tok = r45_sync<CS>();
    int in = 0;                                      // buffer holding the current stage input
    {
        double part[NVL], k[APT][3];
#pragma unroll
        for (int q = 0; q < NVL; ++q) part[q] = 0.0;
        const double f1 = drive ? factor(0, t) : 0.0, f2 = drive ? factor(1, t) : 0.0;
        rhs_obs(in, tok, f1, f2, k, part);
#pragma unroll
        for (int i = 0; i < APT; ++i)
#pragma unroll
            for (int c = 0; c < 3; ++c) k1ref(i, c) = k[i][c];
        if (!own)
#pragma unroll
            for (int q = 0; q < NVL; ++q) part[q] = 0.0;
        double obs_q = 0.0;
        reduce(part, 0.0, obs_q);
        record(t, obs_q);
    }

    int acc_steps = 0, status = 0;
    long long rej_steps = 0;
    double dt = T.dt0;
    while (T.T1 - t > eps) {
        if ((t + dt) - T.T1 > eps) dt = T.T1 - t;
        int fails = 0;
        for (;;) {
            // drive factors of stages 2..6 (stage 7 shares stage 6's time)
            if (drive && warp == 0 && lane < 10) {
                const int sidx = lane >> 1;
                const double cc = sidx == 0 ? c2 : (sidx == 1 ? c3 : (sidx == 2 ? c4 : c5));
                const double ts = sidx == 4 ? t + dt : t + dt * cc;
                drv[lane] = factor(lane & 1, ts);
            }
            double k[APT][3];
            in ^= SBs;
#pragma unroll
            for (int i = 0; i < APT; ++i)
#pragma unroll
                for (int c = 0; c < 3; ++c) publish(in, i, c, yref(i, c) + dt * kR45A[0][0] * k1ref(i, c));
            tok = r45_sync<CS>();
            // stages 2..5: K_{r+2}, then the input of stage r+3 (y + dt a_{r+3,1} K1 + ...
            // + dt a_{r+3,r+2} K_{r+2}, added left to right); K2..K5 in own slots [r]
#pragma unroll 1
            for (int r = 0; r < 4; ++r) {
                rhs(in, tok, drv[2 * r], drv[2 * r + 1], k);
                in ^= SBs;
#pragma unroll
                for (int i = 0; i < APT; ++i)
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        const int s = mk + (i * 3 + c) * Gp;
                        Ks[r * SB + s] = k[i][c];
                        double v = yref(i, c) + dt * kR45A[r + 1][0] * k1ref(i, c);
                        for (int j = 0; j < r; ++j) v = v + dt * kR45A[r + 1][j + 1] * Ks[j * SB + s];
                        publish(in, i, c, v + dt * kR45A[r + 1][r + 1] * k[i][c]);
                    }
                tok = r45_sync<CS>();
            }
            // stage 6: the new solution (published) and the first terms of the error
            rhs(in, tok, drv[8], drv[9], k);
            in ^= SBs;
#pragma unroll
            for (int i = 0; i < APT; ++i)
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const int s = mk + (i * 3 + c) * Gp;
                    const double K3 = Ks[SB + s], K4 = Ks[2 * SB + s], K5 = Ks[3 * SB + s];
                    // the partial error goes to K2's slot (K2 is not read after stage 5)
                    Ks[s] = dt * dc1 * k1ref(i, c) + dt * dc3 * K3 + dt * dc4 * K4 + dt * dc5 * K5 + dt * dc6 * k[i][c];
                    publish(in, i, c,
                            yref(i, c) + dt * b1 * k1ref(i, c) + dt * b3 * K3 + dt * b4 * K4 + dt * b5 * K5 +
                                dt * b6 * k[i][c]);
                }
            tok = r45_sync<CS>();
            // stage 7 (FSAL): K7 = f(yn), observables of yn, error norm
            double part[NVL];
#pragma unroll
            for (int q = 0; q < NVL; ++q) part[q] = 0.0;
            rhs_obs(in, tok, drv[8], drv[9], k, part);
            double emax = 0.0;
#pragma unroll
            for (int i = 0; i < APT; ++i)
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const double ec = Ks[mk + (i * 3 + c) * Gp] + dt * dc7 * k[i][c];
                    const double r =
                        fabs(ec) / (a.abs_tol + a.rel_tol * (1.0 * fabs(yref(i, c)) + 1.0 * dt * fabs(k1ref(i, c))));
                    emax = fmax(emax, r);
                }
            if (!own) {
                emax = 0.0;
#pragma unroll
                for (int q = 0; q < NVL; ++q) part[q] = 0.0;
            }
            double obs_q = 0.0;
            double err = reduce(part, emax, obs_q);
            if (err > 1.0) {
                dt *= fmax(0.9 * pow(err, -1.0 / 3.0), 0.2);
                ++rej_steps;
                if (++fails >= 500) {
                    status = 1;
                    break;
                }
                continue;
            }
            t += dt;
#pragma unroll
            for (int i = 0; i < APT; ++i)
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    yref(i, c) = cur[i][c];                 // the new solution, published in stage 6
                    k1ref(i, c) = k[i][c];
                }
            record(t, obs_q);
            if (err < 0.5) {
                err = fmax(pow(5.0, -5.0), err);
                dt *= 0.9 * pow(err, -1.0 / 5.0);
            }
            ++acc_steps;
            break;
        }
        if (status != 0) break;
        if (acc_steps >= a.max_steps) break;
    }
    if (T.yout && own)
#pragma unroll
        for (int i = 0; i < APT; ++i)
#pragma unroll
            for (int c = 0; c < 3; ++c) T.yout[((long long)g * NAT + ag * APT + i) * 3 + c] = yref(i, c);
    if (rank == 0 && tid == 0 && T.stat) {
        T.stat[0] = nrow;
        T.stat[1] = acc_steps;
        T.stat[2] = rej_steps;
        T.stat[3] = status;
    }
    r45_sync<CS>();                                  // no CTA leaves while others may read its shared memory
}

}  // namespace cmd
