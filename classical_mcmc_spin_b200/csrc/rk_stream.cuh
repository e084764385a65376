// rk_stream.cuh -- RK4 and its discrete adjoint for lattices too large for a
// resident CTA (e.g. the 65536-spin conventional-cubic pyrochlore), with state
// streamed through L2 / HBM.
//
// Every RK4 stage is ONE launch over a (cell tile, trajectory) grid; each
// thread advances one site (cell, atom) with rk4_stage_site, the atom uniform
// per warp, so all SMs work on every trajectory and the kernel boundary is the
// only barrier between stages (no device-side waits anywhere).  The adjoint
// uses the same launches for its segment recompute and one vjp_cell launch per
// stage for the reverse sweep (one cell per thread).
//
// Vectors are cell-major SoA per trajectory, v[(atom*3 + c)*G + g], trajectory
// b at p + b*stride (SVec).  Per stage a cell reads its stage input (own and
// partners'), y and the RK4 sum, and writes the sum and the next stage input:
// per spin 72 B (stage 0: y in, sum and next input out), 120 B (stages 1, 2)
// and 96 B (stage 3: y written in place), 408 B per spin-step when the
// partners' reads hit in cache.
//
// Observables, in a fixed summation order without atomics: the stage-0 launch
// of step n leaves one partial per (trajectory, tile) (spin sums per atom class
// and the energy), and the first CTA of each trajectory in the stage-1 launch
// of the same step sums them over the tiles in a fixed order.  That CTA writes the
// raw row (as rk4_resident's rows: finished by finish_rows_kernel) and/or the
// M_local loss terms.  The state after the last step is summed by
// stream_obs_kernel + stream_reduce_kernel.
#pragma once

#include "rk_adjoint.cuh"

namespace cmd {

constexpr int kStreamTile = 256;     // cells per CTA (one cell per thread)
constexpr int kPart = 16;            // doubles per partial slot

struct SVec {
    double* p;
    long long stride;                // doubles between trajectories
    __device__ __forceinline__ double* at(int b) const { return p ? p + (long long)b * stride : nullptr; }
};

struct StreamArgs {
    int G;                           // cells per trajectory
    int tiles;                       // ceil(G / kStreamTile)
    int B;
    const int* nbr;
    double dt;
    long long n_steps;
    const double* times;             // [n_steps + 1] accumulated t_n
    const double* drive;             // [B][n_steps][6] envelope factors (drive_table_kernel) or null
    double* part;                    // [B][tiles][kPart]
    // raw rows [B][rows][raw_stride] (3*NAT spin sums + energy), or null
    double* raw;
    long long raw_stride, save_every, rows;
    // M_local loss: target / mloc [B][n_steps+1][3], loss [B], or null
    const double* target;
    double* mloc;
    double* loss;
    double n_sites;
    // checkpoints [B][n_ckpt][V] every ckpt_every steps, or null
    double* ckpt;
    long long ckpt_every, n_ckpt, V;
    // step base added to every stage launch's step argument, or null (base 0):
    // a replayed launch sequence (CUDA graph) advances it on the device
    const long long* nbase;
};

// Threads of a CTA: NAT groups of kStreamTile/NAT consecutive threads, group
// a advancing atom a of the CTA's kStreamTile/NAT cells (the atom is uniform
// per warp for NAT in {1, 2, 4, 8}).
template <int NAT>
constexpr int stream_cells() { return kStreamTile / NAT; }

template <int NAT>
__device__ __forceinline__ void stream_site(int& at, int& g) {
    constexpr int CPT = stream_cells<NAT>();
    at = (int)threadIdx.x / CPT;
    g = (int)blockIdx.x * CPT + ((int)threadIdx.x - at * CPT);
}

// rk4_stage_cell for site (cell g, atom AT) alone.  Every load comes before
// the first store (acc / Ynext may alias y), so a thread's loads are all in
// flight together.
template <int NAT, int Z, int LZ, int AT, int OBS>
__device__ __forceinline__ void rk4_stage_site(const Couplings<NAT, Z>& cp, const int* __restrict__ nbr, int G,
                                               int g, double dt, int s, const double* __restrict__ Yin,
                                               const double* y, double* acc, double* Ynext, double f1, double f2,
                                               bool drive, double* obs) {
    constexpr int NL = Z - LZ;
    const long long i0 = (long long)(AT * 3) * G + g;
    double S[3], yv[3], av[3], H[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) S[c] = Yin[i0 + c * G];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        yv[c] = s == 0 ? S[c] : y[i0 + c * G];
        av[c] = (s == 0 || !acc) ? 0.0 : acc[i0 + c * G];
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) H[d] = cp.has_field ? -cp.field[AT][d] : 0.0;
    if (cp.has_onsite) {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            bond_acc(H[d], 2.0 * cp.onsite[AT][3 * d], 2.0 * cp.onsite[AT][3 * d + 1], 2.0 * cp.onsite[AT][3 * d + 2], S[0], S[1], S[2]);
        }
    }
#pragma unroll
    for (int n = 0; n < LZ; ++n) {
        const long long ip = (long long)(((AT + 1 + n) % NAT) * 3) * G + g;
        const double P0 = Yin[ip], P1 = Yin[ip + G], P2 = Yin[ip + 2 * G];
#pragma unroll
        for (int d = 0; d < 3; ++d)
            bond_acc(H[d], cp.J[AT][n][3 * d], cp.J[AT][n][3 * d + 1], cp.J[AT][n][3 * d + 2], P0, P1, P2);
    }
#pragma unroll
    for (int m = 0; m < NL; ++m) {
        const int n = LZ + m;
        if (n < cp.zc[AT]) {
            const int p = nbr[((long long)g * NAT + AT) * NL + m];
            const double P0 = Yin[p], P1 = Yin[p + G], P2 = Yin[p + 2 * G];
#pragma unroll
            for (int d = 0; d < 3; ++d)
                bond_acc(H[d], cp.J[AT][n][3 * d], cp.J[AT][n][3 * d + 1], cp.J[AT][n][3 * d + 2], P0, P1, P2);
        }
    }
    if (OBS == 2) {
#pragma unroll
        for (int c = 0; c < 3; ++c) obs[3 * AT + c] += S[c];
#pragma unroll
        for (int d = 0; d < 3; ++d) obs[3 * NAT] += S[d] * (H[d] - (cp.has_field ? cp.field[AT][d] : 0.0));
    }
    if (drive) {
#pragma unroll
        for (int d = 0; d < 3; ++d) drive_acc(H[d], cp.d1[AT][d], cp.d2[AT][d], f1, f2);
    }
    const double k[3] = {H[1] * S[2] - H[2] * S[1], H[2] * S[0] - H[0] * S[2], H[0] * S[1] - H[1] * S[0]};
    const double cy = s == 2 ? dt : 0.5 * dt;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const long long i = i0 + c * G;
        if (s == 0) {
            acc[i] = k[c];
            Ynext[i] = 1.0 * yv[c] + cy * k[c];
        } else if (s < 3) {
            acc[i] = av[c] + 2.0 * k[c];
            Ynext[i] = 1.0 * yv[c] + cy * k[c];
        } else if (Ynext) {
            Ynext[i] = yv[c] + (dt / 6.0) * (av[c] + k[c]);
        }
    }
}

// Envelope factors of trajectory b for stage s of step n.
__device__ __forceinline__ void stream_drive(const StreamArgs& a, int b, long long n, int s, double& f1,
                                             double& f2) {
    if (!a.drive) {
        f1 = f2 = 0.0;
        return;
    }
    const int q = s == 0 ? 0 : (s < 3 ? 2 : 4);
    const double* d = a.drive + ((long long)b * a.n_steps + n) * 6 + q;
    f1 = d[0];
    f2 = d[1];
}

// Sums the tile partials of step n of trajectory b and writes its raw row
// and / or loss terms.  Called by a whole CTA: warp w sums values w, w+nwarps,
// ...; lane l adds tiles l, l+32, ... in order, then a fixed butterfly adds
// the lanes, so the order never depends on timing.
template <int NAT>
__device__ void stream_reduce(const StreamArgs& a, int b, long long n, double* sh) {
    constexpr int NR = 3 * NAT + 1;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    const double* p = a.part + (long long)b * a.tiles * kPart;
    for (int q = warp; q < NR; q += nw) {
        double s = 0.0;
        for (int t = lane; t < a.tiles; t += 32) s += p[(long long)t * kPart + q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) sh[q] = s;
    }
    __syncthreads();
    if (a.raw && tid < NR) {
        long long r = -1;
        if (n % a.save_every == 0) r = n / a.save_every;
        else if (n == a.n_steps) r = a.rows - 1;
        if (r >= 0) a.raw[((long long)b * a.rows + r) * a.raw_stride + tid] = sh[tid];
    }
    if (a.mloc && tid == 0) {
        double l = 0.0;
        for (int c = 0; c < 3; ++c) {
            double m = 0.0;
            for (int at = 0; at < NAT; ++at) m += sh[3 * at + c];
            m /= a.n_sites;
            const long long i = ((long long)b * (a.n_steps + 1) + n) * 3 + c;
            a.mloc[i] = m;
            const double r = m - a.target[i];
            l += r * r;
        }
        a.loss[b] = (n == 0 ? 0.0 : a.loss[b]) + l;
    }
    __syncthreads();
}

// Block sum of v[0..used) in a fixed order (lanes by the butterfly, then the
// warps in order), finished in parallel: thread q < used gets the total of
// value q and returns it in *out (other threads: false).
template <int NV>
__device__ __forceinline__ bool block_sum_par(double (&v)[NV], double* red, int used, double* out) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const double r = warp_reduce_many<NV>(v);
    constexpr int span = 32 / NV;
    if ((lane % span) == 0) red[warp * kRedStride + lane / span] = r;
    __syncthreads();
    if ((int)threadIdx.x >= used) return false;
    double s = 0.0;
    for (int w = 0; w < nw; ++w) s += red[w * kRedStride + threadIdx.x];
    *out = s;
    return true;
}

// Block-reduces this thread's partial o[NR] and stores it in the tile's slot.
template <int NR>
__device__ __forceinline__ void stream_store_partial(const StreamArgs& a, int b, const double (&o)[NR],
                                                     double* red) {
    double v[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = q < NR ? o[q] : 0.0;
    double t;
    if (block_sum_par<16>(v, red, NR, &t)) a.part[((long long)b * a.tiles + blockIdx.x) * kPart + threadIdx.x] = t;
}

// One RK4 stage s of step n for every (tile, trajectory).  Stage 0 also leaves
// the observables' partials of Yin (= y_n) and the checkpoint of y_n; the
// first tile of stage 1 finishes step n's observables.
template <int NAT, int Z, int LZ>
__global__ void __launch_bounds__(kStreamTile, 4)
stream_stage_kernel(const __grid_constant__ Couplings<NAT, Z> cp, const __grid_constant__ StreamArgs a, int s,
                    long long n_arg, SVec Yin, SVec y, SVec acc, SVec Ynext, int with_obs) {
    constexpr int NR = 3 * NAT + 1;
    const long long n = (a.nbase ? *a.nbase : 0) + n_arg;
    __shared__ double red[32 * kRedStride];
    __shared__ double tot[16];
    const int b = blockIdx.y;
    int at, g;
    stream_site<NAT>(at, g);
    if (s == 1 && with_obs && blockIdx.x == 0) stream_reduce<NAT>(a, b, n, tot);
    double f1, f2;
    stream_drive(a, b, n, s, f1, f2);
    const bool drive = a.drive != nullptr && (f1 != 0.0 || f2 != 0.0);
    double o[NR];
#pragma unroll
    for (int q = 0; q < NR; ++q) o[q] = 0.0;
    if (g < a.G) {
        const double* yin = Yin.at(b);
        with_atom<NAT>(at, [&](auto tag) {
            constexpr int AT = decltype(tag)::value;
            if (s == 0 && with_obs)
                rk4_stage_site<NAT, Z, LZ, AT, 2>(cp, a.nbr, a.G, g, a.dt, s, yin, y.at(b), acc.at(b), Ynext.at(b),
                                                  f1, f2, drive, o);
            else
                rk4_stage_site<NAT, Z, LZ, AT, 0>(cp, a.nbr, a.G, g, a.dt, s, yin, y.at(b), acc.at(b), Ynext.at(b),
                                                  f1, f2, drive, nullptr);
            if (s == 0 && a.ckpt && n % a.ckpt_every == 0) {
                double* dst = a.ckpt + ((long long)b * a.n_ckpt + n / a.ckpt_every) * a.V;
#pragma unroll
                for (int c = 0; c < 3; ++c) dst[(long long)(AT * 3 + c) * a.G + g] = yin[(long long)(AT * 3 + c) * a.G + g];
            }
        });
    }
    if (s == 0 && with_obs) stream_store_partial<NR>(a, b, o, red);
}

// Advances the step base of a replayed launch sequence by k steps.
static __global__ void stream_advance_kernel(long long* nbase, long long k) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *nbase += k;
}

// Sets the step base of a replayed launch sequence.
static __global__ void stream_set_base_kernel(long long* nbase, long long v) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *nbase = v;
}

// Observables' partials of y (the state after the last step).
template <int NAT, int Z, int LZ>
__global__ void __launch_bounds__(kStreamTile)
stream_obs_kernel(const __grid_constant__ Couplings<NAT, Z> cp, const __grid_constant__ StreamArgs a, SVec y) {
    constexpr int NR = 3 * NAT + 1;
    __shared__ double red[32 * kRedStride];
    const int b = blockIdx.y;
    int at, g;
    stream_site<NAT>(at, g);
    double o[NR];
#pragma unroll
    for (int q = 0; q < NR; ++q) o[q] = 0.0;
    if (g < a.G) {
        // a stage-3 pass with no output: only the observables of y are kept
        with_atom<NAT>(at, [&](auto tag) {
            rk4_stage_site<NAT, Z, LZ, decltype(tag)::value, 2>(cp, a.nbr, a.G, g, a.dt, 3, y.at(b), y.at(b), nullptr,
                                                                nullptr, 0.0, 0.0, false, o);
        });
    }
    stream_store_partial<NR>(a, b, o, red);
}

// Finishes step n's observables (one CTA per trajectory).
template <int NAT>
__global__ void __launch_bounds__(kStreamTile) stream_reduce_kernel(const __grid_constant__ StreamArgs a, long long n) {
    __shared__ double sh[16];
    stream_reduce<NAT>(a, blockIdx.x, n, sh);
}

// AoS state [B][N][3] (site = cell*NAT + atom; y0_stride doubles between
// trajectories, 0 = shared) -> SoA vector, and back.
template <int NAT>
__global__ void stream_load_kernel(const double* __restrict__ y0, long long y0_stride, int G, SVec y) {
    const int b = blockIdx.y;
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= G) return;
    const double* src = y0 + (long long)b * y0_stride;
    double* dst = y.at(b);
#pragma unroll
    for (int at = 0; at < NAT; ++at)
#pragma unroll
        for (int c = 0; c < 3; ++c) dst[(at * 3 + c) * G + g] = src[((long long)g * NAT + at) * 3 + c];
}

template <int NAT>
__global__ void stream_store_kernel(SVec y, int G, double* __restrict__ out) {
    const int b = blockIdx.y;
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= G) return;
    const double* src = y.at(b);
    double* dst = out + (long long)b * G * NAT * 3;
#pragma unroll
    for (int at = 0; at < NAT; ++at)
#pragma unroll
        for (int c = 0; c < 3; ++c) dst[((long long)g * NAT + at) * 3 + c] = src[(at * 3 + c) * G + g];
}

// ---------------------------------------------------------------------------
// Adjoint sweep.

struct StreamVjpArgs {
    int G, tiles;                    // tiles of kStreamTile cells
    const int* nbr;
    double dt;
    long long n_steps;
    const double* drive;             // as StreamArgs::drive
    const double* target;            // [B][n_steps+1][3]
    const double* mloc;              // [B][n_steps+1][3]
    double n_sites;
    double* gpart;                   // [B][tiles][kPart] gradient partials (accumulated)
    const long long* nbase;          // step base of a replayed launch sequence (step = *nbase + n), or nullptr
};

// lam_b = dl_S (the loss cotangent of the last state) on every site.
template <int NAT>
__global__ void stream_lam_init_kernel(const __grid_constant__ StreamVjpArgs a, SVec lam) {
    const int b = blockIdx.y;
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= a.G) return;
    const long long i = ((long long)b * (a.n_steps + 1) + a.n_steps) * 3;
    double* l = lam.at(b);
#pragma unroll
    for (int at = 0; at < NAT; ++at)
#pragma unroll
        for (int c = 0; c < 3; ++c) l[(at * 3 + c) * a.G + g] = 2.0 * (a.mloc[i + c] - a.target[i + c]) / a.n_sites;
}

// One stage VJP (stage s of step n) for every (tile of kStreamTile cells,
// trajectory), one cell per thread: mode and buffers as vjp_cell; the tile's
// parameter cotangents are added to its slot.
template <int NAT, int Z, int LZ, int NQ>
__global__ void __launch_bounds__(kStreamTile, 3)
stream_vjp_kernel(const __grid_constant__ Couplings<NAT, Z> cp, const __grid_constant__ ParamDerivs<NAT, Z, NQ> pd,
                  const __grid_constant__ StreamVjpArgs a, int s, long long n_arg, SVec Y, SVec lam, SVec Sprev,
                  double ca, double cb, SVec Sout, SVec acc, SVec lam_out, int mode) {
    const long long n = (a.nbase ? *a.nbase : 0) + n_arg;
    __shared__ double red[32 * kRedStride];
    const int b = blockIdx.y;
    const int g = blockIdx.x * kStreamTile + threadIdx.x;    // one cell per thread
    double f1 = 0.0, f2 = 0.0;
    if (a.drive) {
        const int q = s == 0 ? 0 : (s < 3 ? 2 : 4);
        const double* d = a.drive + ((long long)b * a.n_steps + n) * 6 + q;
        f1 = d[0];
        f2 = d[1];
    }
    const bool drive = a.drive != nullptr && (f1 != 0.0 || f2 != 0.0);
    double dl[3] = {0.0, 0.0, 0.0};
    if (mode == 2) {
        const long long i = ((long long)b * (a.n_steps + 1) + n) * 3;
#pragma unroll
        for (int c = 0; c < 3; ++c) dl[c] = 2.0 * (a.mloc[i + c] - a.target[i + c]) / a.n_sites;
    }
    double gq[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) gq[q] = 0.0;
    if (g < a.G) {
        vjp_cell<NAT, Z, LZ, NQ>(cp, pd, a.nbr, a.G, g, Y.at(b), lam.at(b), Sprev.at(b), ca, cb, f1, f2, drive,
                                 Sout.at(b), acc.at(b), lam_out.at(b), mode, dl, gq);
    }
    double v[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = q < NQ ? gq[q] : 0.0;
    double t;
    if (block_sum_par<16>(v, red, NQ, &t)) a.gpart[((long long)b * a.tiles + blockIdx.x) * kPart + threadIdx.x] += t;
}

// grad[b][q] = sum over tiles of the partials (tile order); one CTA per trajectory.
static __global__ void stream_grad_kernel(const double* __restrict__ gpart, int tiles, int nq, double* __restrict__ out,
                                   long long out_stride) {
    const int b = blockIdx.x;
    const int q = threadIdx.x;
    if (q >= nq) return;
    double s = 0.0;
    for (int t = 0; t < tiles; ++t) s += gpart[((long long)b * tiles + t) * kPart + q];
    out[(long long)b * out_stride + q] = s;
}

}  // namespace cmd
