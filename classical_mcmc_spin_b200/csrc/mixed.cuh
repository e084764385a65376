// mixed.cuh -- Landau-Lifshitz dynamics of a mixed SU(2) / SU(3) lattice (the
// reference's second GPU MD path, src/gpu/mixed_lattice_gpu.cu): SU(2) sites
// carry 3-component spins, SU(3) sites 8-component Gell-Mann vectors.
//
// Local fields (mixed_lattice_gpu.cu:54-187), per site i of either kind:
//   H_i = -B_i + 2 A_i S_i + sum_n J_n S_p(n) + sum_m M_m S'_q(m) - drive(t),
// where J couples like sites (3x3 or 8x8) and M the other kind (3x8 seen from an
// SU(2) site, 8x3 from an SU(3) site; both directions are supplied, as in the
// reference), and the drive is each kind's own two-pulse field
// (gpu_common_helpers.cuh:355-377).  Equations of motion
// (gpu_common_helpers.cuh:386-399): dS/dt = H x S for SU(2) and
// (dS/dt)_a = f_abc H_b S_c for SU(3), f the totally antisymmetric structure
// constants of su(3).  Partners outside the lattice are skipped, as in the
// reference.
//
// One trajectory per launch, persistent for the whole run: a thread-block cluster
// of CS CTAs (up to 16, a non-portable size the host checks before using), one
// site per thread (more when the lattice is larger), the state and
// the stage vectors in global memory (L2-resident at these sizes), the distinct
// couplings in shared memory, the cluster barrier between stages; the steps are
// rk_fixed.cuh's.  The reference launches
// two RHS kernels and an update kernel per stage with a device synchronisation
// after each.
#pragma once

#include "drive.cuh"
#include "rk_fixed.cuh"

#include <cooperative_groups.h>

namespace cmd {

namespace mcg = cooperative_groups;

// Couplings are stored once per distinct value: `tab` holds the distinct fields,
// on-site matrices, like-site and mixed bond matrices of each kind (offsets off_*),
// and per-site / per-(slot, site) indices pick them (index arrays site-minor, so a
// warp's loads coalesce).  The kernel copies `tab` into shared memory when it fits.
struct MixedDev {
    int N2, N3, NA2, NA3;                  // sites and atoms per cell of each kind
    int z2, z3, zm2, zm3;                  // ELL widths: like-site bonds, mixed bonds
    const double* tab;                     // distinct couplings (global memory), block strides kStride*
    int tab_doubles, tab_in_smem;
    const int* order;                      // [N2 + N3] site of each work slot: the kinds alternate by warp
    int off_f2, off_o2, off_b2, off_m2;    // offsets in tab: fields [3], on-site [9], bonds [9], mixed [3*8]
    int off_f3, off_o3, off_b3, off_m3;    //                 fields [8], on-site [64], bonds [64], mixed [8*3]
    const int* f2i;                        // [N2] field index
    const int* o2i;                        // [N2] on-site index
    const int* b2i;                        // [z2][N2] bond matrix index
    const int* part2;                      // [z2][N2] SU(2) partner or -1
    const int* cnt2;                       // [N2]
    const int* m2i;                        // [zm2][N2] mixed matrix index
    const int* mpart2;                     // [zm2][N2] SU(3) partner or -1
    const int* mcnt2;                      // [N2]
    const int* f3i;
    const int* o3i;
    const int* b3i;                        // [z3][N3]
    const int* part3;
    const int* cnt3;
    const int* m3i;                        // [zm3][N3]
    const int* mpart3;                     // SU(2) partner or -1
    const int* mcnt3;
    const double* drive2;                  // [2][NA2][3]
    const double* drive3;                  // [2][NA3][8]
    double amp2, width2, freq2, t1_2, t2_2;
    double amp3, width3, freq3, t1_3, t2_3;
};

// Doubles between consecutive distinct blocks of each table: odd, so lanes reading
// different blocks at the same offset fall in different shared-memory banks.
constexpr int kStrideF2 = 3, kStrideO2 = 9, kStrideB2 = 9, kStrideM = 25;
constexpr int kStrideF3 = 9, kStrideO3 = 65, kStrideB3 = 65;

struct MixedRun {
    double* work;              // 11 vectors of V doubles: y, k[0..6], Ya, Yb, yn
    const double* y0;          // [V] initial state
    double* y_out;             // [V] final state
    double* rows;              // [max_rows][V] saved states, or nullptr
    long long max_rows;
    double T0, dt;
    long long n_steps, save_every;
    int mode;
};

// r = f_abc a_b b_c from the nine independent non-zero structure constants
// f_123 = 1, f_147 = f_246 = f_257 = f_345 = 1/2, f_156 = f_367 = -1/2,
// f_458 = f_678 = sqrt(3)/2 (1-based), each contributing to its three cyclic slots.
__device__ __forceinline__ void su3_cross(double (&r)[8], const double (&a)[8], const double (&b)[8]) {
    constexpr double h = 0.5, q = 0.86602540378443864676;
    constexpr int T[9][3] = {{0, 1, 2}, {0, 3, 6}, {0, 4, 5}, {1, 3, 5}, {1, 4, 6},
                             {2, 3, 4}, {2, 5, 6}, {3, 4, 7}, {5, 6, 7}};
    constexpr double F[9] = {1.0, h, -h, h, h, h, -h, q, q};
#pragma unroll
    for (int c = 0; c < 8; ++c) r[c] = 0.0;
#pragma unroll
    for (int t = 0; t < 9; ++t) {
        const int x = T[t][0], y = T[t][1], z = T[t][2];
        r[x] += F[t] * (a[y] * b[z] - a[z] * b[y]);
        r[y] += F[t] * (a[z] * b[x] - a[x] * b[z]);
        r[z] += F[t] * (a[x] * b[y] - a[y] * b[x]);
    }
}

// dS/dt of site s (SU(2) sites first, then SU(3)) at state Y; T = the distinct-coupling
// table (shared or global memory); f = drive factors (SU(2) pulse 1, pulse 2, SU(3)
// pulse 1, pulse 2) of the stage time.
__device__ __forceinline__ void mixed_rhs_site(const MixedDev& m, const double* T, const double* __restrict__ Y,
                                               double* __restrict__ K, int s, const double (&f)[4]) {
    const double* Y3 = Y + 3LL * m.N2;
    if (s < m.N2) {
        double S[3], H[3];
        const double* B = T + m.off_f2 + kStrideF2 * m.f2i[s];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            S[d] = Y[3LL * s + d];
            H[d] = -B[d];
        }
        const double* A = T + m.off_o2 + kStrideO2 * m.o2i[s];
#pragma unroll
        for (int i = 0; i < 3; ++i) H[i] += 2.0 * (A[3 * i] * S[0] + A[3 * i + 1] * S[1] + A[3 * i + 2] * S[2]);
        const int nb = min(m.cnt2[s], m.z2);
        for (int n = 0; n < nb; ++n) {
            const int p = m.part2[(long long)n * m.N2 + s];
            if (p < 0) continue;
            const double* J = T + m.off_b2 + kStrideB2 * m.b2i[(long long)n * m.N2 + s];
            const double P0 = Y[3LL * p], P1 = Y[3LL * p + 1], P2 = Y[3LL * p + 2];
#pragma unroll
            for (int i = 0; i < 3; ++i) H[i] += J[3 * i] * P0 + J[3 * i + 1] * P1 + J[3 * i + 2] * P2;
        }
        const int nm = min(m.mcnt2[s], m.zm2);
        for (int n = 0; n < nm; ++n) {
            const int p = m.mpart2[(long long)n * m.N2 + s];
            if (p < 0) continue;
            const double* M = T + m.off_m2 + kStrideM * m.m2i[(long long)n * m.N2 + s];
            double P[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) P[j] = Y3[8LL * p + j];
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                double t = 0.0;
#pragma unroll
                for (int j = 0; j < 8; ++j) t += M[8 * i + j] * P[j];
                H[i] += t;
            }
        }
        if (m.amp2 != 0.0) {
            const int at = s % m.NA2;
#pragma unroll
            for (int i = 0; i < 3; ++i)
                H[i] -= f[0] * m.drive2[3 * at + i] + f[1] * m.drive2[3 * (m.NA2 + at) + i];
        }
        K[3LL * s] = H[1] * S[2] - H[2] * S[1];
        K[3LL * s + 1] = H[2] * S[0] - H[0] * S[2];
        K[3LL * s + 2] = H[0] * S[1] - H[1] * S[0];
    } else {
        const int s3 = s - m.N2;
        double S[8], H[8];
        const double* B = T + m.off_f3 + kStrideF3 * m.f3i[s3];
#pragma unroll
        for (int d = 0; d < 8; ++d) {
            S[d] = Y3[8LL * s3 + d];
            H[d] = -B[d];
        }
        const double* A = T + m.off_o3 + kStrideO3 * m.o3i[s3];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            double t = 0.0;
#pragma unroll
            for (int j = 0; j < 8; ++j) t += A[8 * i + j] * S[j];
            H[i] += 2.0 * t;
        }
        const int nb = min(m.cnt3[s3], m.z3);
        for (int n = 0; n < nb; ++n) {
            const int p = m.part3[(long long)n * m.N3 + s3];
            if (p < 0) continue;
            const double* J = T + m.off_b3 + kStrideB3 * m.b3i[(long long)n * m.N3 + s3];
            double P[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) P[j] = Y3[8LL * p + j];
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                double t = 0.0;
#pragma unroll
                for (int j = 0; j < 8; ++j) t += J[8 * i + j] * P[j];
                H[i] += t;
            }
        }
        const int nm = min(m.mcnt3[s3], m.zm3);
        for (int n = 0; n < nm; ++n) {
            const int p = m.mpart3[(long long)n * m.N3 + s3];
            if (p < 0) continue;
            const double* M = T + m.off_m3 + kStrideM * m.m3i[(long long)n * m.N3 + s3];
            const double P0 = Y[3LL * p], P1 = Y[3LL * p + 1], P2 = Y[3LL * p + 2];
#pragma unroll
            for (int i = 0; i < 8; ++i) H[i] += M[3 * i] * P0 + M[3 * i + 1] * P1 + M[3 * i + 2] * P2;
        }
        if (m.amp3 != 0.0) {
            const int at = s3 % m.NA3;
#pragma unroll
            for (int i = 0; i < 8; ++i)
                H[i] -= f[2] * m.drive3[8 * at + i] + f[3] * m.drive3[8 * (m.NA3 + at) + i];
        }
        double r[8];
        su3_cross(r, H, S);
#pragma unroll
        for (int d = 0; d < 8; ++d) K[3LL * m.N2 + 8LL * s3 + d] = r[d];
    }
}

// Steps over one cluster: every thread of the cluster owns the elements of a strided
// share of the work slots (sites through MixedDev::order), the barrier is the cluster's.
template <class R, class E>
struct ClusterStepCtx {
    const R& rhs_f;
    const E& each_f;
    __device__ void rhs(const double* Y, double* K, double ts) const { rhs_f(Y, K, ts); }
    template <class F>
    __device__ void each(F&& f) const { each_f(f); }
    __device__ void sync() const { mcg::this_cluster().sync(); }
};

constexpr int kMixedThreads = 512;

template <int CS>
__global__ void __launch_bounds__(kMixedThreads, 1)
mixed_integrate_kernel(const __grid_constant__ MixedDev m, const __grid_constant__ MixedRun r) {
    mcg::cluster_group cluster = mcg::this_cluster();
    extern __shared__ double stab[];       // the distinct couplings, when they fit
    const int nt = (int)blockDim.x * CS;
    const int gt = (int)cluster.block_rank() * (int)blockDim.x + (int)threadIdx.x;
    const long long V = 3LL * m.N2 + 8LL * m.N3;
    const int sites = m.N2 + m.N3;
    const bool driven = m.amp2 != 0.0 || m.amp3 != 0.0;
    double* y = r.work;
    double* k[7];
#pragma unroll
    for (int j = 0; j < 7; ++j) k[j] = r.work + (1 + j) * V;
    double* Ya = r.work + 8 * V;
    double* Yb = r.work + 9 * V;
    double* yn = r.work + 10 * V;

    const double* T = m.tab_in_smem ? stab : m.tab;
    // drive factors of the stage time: lanes 0-3 of every warp compute one each and the
    // warp shares them (no CTA barrier)
    auto rhs = [&](const double* Yin, double* K, double ts) {
        double f[4] = {0.0, 0.0, 0.0, 0.0};
        if (driven) {
            const int q = threadIdx.x & 3;
            const double v = q == 0   ? drive_factor(m.amp2, ts - m.t1_2, m.width2, m.freq2)
                             : q == 1 ? drive_factor(m.amp2, ts - m.t2_2, m.width2, m.freq2)
                             : q == 2 ? drive_factor(m.amp3, ts - m.t1_3, m.width3, m.freq3)
                                      : drive_factor(m.amp3, ts - m.t2_3, m.width3, m.freq3);
#pragma unroll
            for (int k = 0; k < 4; ++k) f[k] = __shfl_sync(0xffffffffu, v, k);
        }
        for (int q = gt; q < sites; q += nt) mixed_rhs_site(m, T, Yin, K, m.order[q], f);
    };
    // the elements of the thread's own sites: the ones its rhs writes (rk_fixed.cuh reads
    // a stage derivative right after the rhs that wrote it, without a barrier)
    auto each = [&](auto&& f) {
        for (int q = gt; q < sites; q += nt) {
            const int s = m.order[q];
            if (s < m.N2) {
                const long long b = 3LL * s;
                f(b);
                f(b + 1);
                f(b + 2);
            } else {
                const long long b = 3LL * m.N2 + 8LL * (s - m.N2);
#pragma unroll
                for (int d = 0; d < 8; ++d) f(b + d);
            }
        }
    };
    const ClusterStepCtx<decltype(rhs), decltype(each)> ctx{rhs, each};

    if (m.tab_in_smem)
        for (int i = threadIdx.x; i < m.tab_doubles; i += blockDim.x) stab[i] = m.tab[i];
    each([&](long long i) { y[i] = r.y0[i]; });
    cluster.sync();
    double t = r.T0;
    long long row = 0, save_left = 0;
    auto save = [&]() {
        if (r.rows && row < r.max_rows) each([&](long long i) { r.rows[row * V + i] = y[i]; });
        ++row;
    };
    for (long long step = 0; step < r.n_steps; ++step) {
        const bool obs = save_left == 0;
        save_left = obs ? r.save_every - 1 : save_left - 1;
        if (obs) save();
        rhs(y, k[0], t);
        fixed_step<true>(r.mode, ctx, y, k, Ya, Yb, yn, t, r.dt);
        t += r.dt;
    }
    save();
    each([&](long long i) { r.y_out[i] = y[i]; });
}

// Means of each kind's components and their (-1)^(site mod atoms) staggered means
// (gpu_common_helpers.cu:163-211): out = [m2 (3), ms2 (3), m3 (8), ms3 (8)].  One
// CTA per (kind, component), partial sums in a fixed order.
__global__ void mixed_magnetization_kernel(const double* __restrict__ Y, int N2, int N3, int NA2, int NA3,
                                           double* __restrict__ out) {
    __shared__ double sl[256], ss[256];
    const int b = blockIdx.x;
    const bool su3 = b >= 3;
    const int comp = su3 ? b - 3 : b, dim = su3 ? 8 : 3;
    const int N = su3 ? N3 : N2, NA = su3 ? NA3 : NA2;
    const double* base = su3 ? Y + 3LL * N2 : Y;
    double a = 0.0, c = 0.0;
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        const double v = base[(long long)i * dim + comp];
        a += v;
        c += ((i % NA) & 1) ? -v : v;
    }
    sl[threadIdx.x] = a;
    ss[threadIdx.x] = c;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            sl[threadIdx.x] += sl[threadIdx.x + w];
            ss[threadIdx.x] += ss[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double inv = N > 0 ? 1.0 / (double)N : 0.0;
        out[su3 ? 6 + comp : comp] = sl[0] * inv;
        out[su3 ? 14 + comp : 3 + comp] = ss[0] * inv;
    }
}

// Each site rescaled to `len` when its norm exceeds 1e-10
// (gpu_common_helpers.cu:139-160).
__global__ void mixed_normalize_kernel(double* __restrict__ Y, int N2, int N3, double len2, double len3) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= N2 + N3) return;
    const bool su3 = s >= N2;
    const int dim = su3 ? 8 : 3;
    double* v = su3 ? Y + 3LL * N2 + 8LL * (s - N2) : Y + 3LL * s;
    double nrm = 0.0;
    for (int d = 0; d < dim; ++d) nrm += v[d] * v[d];
    nrm = sqrt(nrm);
    if (nrm > 1e-10) {
        const double len = su3 ? len3 : len2;
        for (int d = 0; d < dim; ++d) v[d] = v[d] * len / nrm;
    }
}

}  // namespace cmd
