// cmd_core.h -- definitions shared by the translation units of the C ABI (not
// installed): the handle, the compiled lattice layout, the run descriptions and
// the launch entry points of each kernel family.
//
//   cmd_api.cu   public entry points, lattice compilation, small kernels
//   resident.cu  resident RK4 (one CTA or a 2-/4-CTA cluster per trajectory),
//                variant table, autotuner support
//   stream.cu    streamed RK4 stages and the streamed adjoint
//   global.cu    global-state integrator (fixed-step methods; controlled
//                Dormand-Prince where no on-chip tiling holds the lattice) and
//                the dispatch of controlled batches
//   rk45.cu      on-chip controlled Dormand-Prince tilings and their launches
//   adjoint.cu   resident and per-trajectory discrete adjoint, cmd_adjoint_rk4
//   noalloc.cu   allocation-free batch entry point and its static scratch
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstring>
#include <functional>
#include <string>
#include <vector>

#include "cmd.h"
#include "cmd_internal.h"
#include "rk4_resident.cuh"
#include "rk_global.cuh"

#define CUDA_TRY(expr)                                                                   \
    do {                                                                                 \
        cudaError_t e_ = (expr);                                                         \
        if (e_ != cudaSuccess)                                                           \
            return ::cmd::fail(e_ == cudaErrorMemoryAllocation ? CMD_ERR_OOM : CMD_ERR_CUDA, \
                               std::string(#expr) + ": " + cudaGetErrorString(e_));      \
    } while (0)

namespace cmd {

constexpr size_t kMaxSmem = 232448;   // 227 KB dynamic shared memory per CTA on sm_100

// Per-unit-cell description of the lattice, derived from the flat tables.
struct Layout {
    int NA = 0;                 // sites per cell (= classes)
    int64_t G = 0;              // cells
    int Z = 0;                  // slots per atom (max over atoms)
    int LZ = 0;                 // leading "local" slots (partner in the same cell)
    std::vector<int> zc;        // slots per atom
    std::vector<double> J;      // [NA][Z][9]
    std::vector<int> nbr;       // [G][NA][Z-LZ] shared-memory offsets
    std::vector<int> slot_entry;  // [NA][Z] ELL entry at cell 0 each slot came from
    bool uniform = false;
    std::string why;            // reason when not uniform
    // halo columns of the RK45 cluster partition into cs CTAs (index cs; -1: not
    // computed yet), filled on first use
    mutable std::vector<int64_t> halo_cols = std::vector<int64_t>(17, -1);
};

}  // namespace cmd

struct cmd_handle {
    int64_t N = 0;
    int NA = 0;                 // sites per group (classes) used by the kernels
    int n_atoms_ref = 0;        // the caller's n_atoms when it differs from NA
    int zmax = 0;
    std::vector<double> field, onsite, frames, afm;   // per atom
    bool has_field = false, has_onsite = false;
    cmd::Layout lay;
    cudaStream_t stream = nullptr;
    cmd::DevBuf state, nbr, obs, traj, batch_states, batch_out, pulses, scratch;
    cmd::DevBuf dframes, dafm, times, drive, raw, tune_states, tune_obs;
    cmd::DevBuf gwork, gmeta, gstat, grows, gqueue;
    cmd::DevBuf awork, ackpt, aseg, amloc, aout, ameta, ain;
    cmd::DevBuf sbuf, spart, sgpart;  // streamed RK4 / adjoint: stage vectors, tile partials
    cmd::DevBuf chunk_states, chunk_rows;   // cmd_run_batch: ping-pong states and row buffers of time chunks
    cmd::DevBuf cnbr2, cnbr4, cnbr8, cnbr16;  // partner tables of the 2-, 4-, 8- and 16-CTA cluster kernels
    cmd::DevBuf cnbr_all;       // RK45 on-chip kernels: every slot's partner word per site (built on first use)
    cmd::DevBuf cpush;          // RK45 halo tilings: every site's push words
    int cnbr_all_cs = 0;        // 2 * cluster size (+1 for halo words) cnbr_all / cpush were built for
    cudaStream_t copy_stream = nullptr;  // cmd_run_batch: device-to-host copies of finished chunks
    cmd::HostBuf hstage;        // cmd_run_uneven: page-locked staging of the rows and final states
    std::vector<cudaStream_t> aux_streams;   // concurrent launches of an uneven batch (created on first use)
    // streamed RK4: the stage launches of one chunk of steps captured as a CUDA
    // graph, replayed per chunk; rebuilt when any launch parameter changes
    bool graphs = true;
    cudaGraphExec_t stream_graph = nullptr;
    std::vector<unsigned char> stream_graph_key;
    // batched resident run / uneven batch: each call's launches captured and
    // replayed as one graph, the executable graph updated in place per call
    cudaGraphExec_t call_graph[2] = {nullptr, nullptr};
    std::vector<unsigned char> call_sig[2];   // kernels and launch shapes of call_graph[i]
    // streamed adjoint: one full checkpoint segment (recompute and reverse
    // sweep) per starting order of the two cotangent buffers, keyed like stream_graph
    cudaGraphExec_t adj_graph[2] = {nullptr, nullptr};
    std::vector<unsigned char> adj_graph_key[2];
    cmd::DevBuf snbase;         // device step base of the replayed chunks
    std::vector<cudaEvent_t> aux_events;
    bool has_state = false;
    int device = -1;            // device current at cmd_create (owns the stream and buffers)
    double* noalloc_base = nullptr;   // device address of the allocation-free scratch on `device`
    int variant = -1;           // resident-kernel variant; -1 = heuristic default
    int rk45_variant = -1;      // on-chip RK45 tiling; -1 = heuristic default, -2 = global-memory kernel
    // pulse (set_gpu_pulse)
    std::vector<double> fd;     // [2][NA*3]
    double amp = 0.0, width = 1.0, freq = 0.0, t1 = 0.0, t2 = 0.0;
    // controlled stepper
    double abs_tol = 1e-6, rel_tol = 1e-6;
    int64_t max_steps = 0;
};

namespace cmd {

// Everything one resident run needs besides the handle.
struct RunSpec {
    int64_t B = 1;
    const double* y0 = nullptr;       // device
    int64_t y0_stride = 0;
    double* y_out = nullptr;          // device
    double* obs = nullptr;            // device [B][rows][10]
    double* traj = nullptr;           // device [B][rows][N*3]
    double T0 = 0.0, dt = 0.0;
    int64_t n_steps = 0, save = 1;
    const Pulse* pulses = nullptr;    // device [B]
    double width = 1.0, freq = 0.0;
    const double* d1 = nullptr;       // host [NA*3]
    const double* d2 = nullptr;
    const double* frames = nullptr;   // device [NA*9]
    const double* afm = nullptr;      // device [NA]
    double n_sites = 1.0;
    int variant = -1;                 // -1: handle's choice
};

// One trajectory of the global-state / on-chip controlled integrators.
struct GJob {
    cmd_handle* h = nullptr;
    const double* y0 = nullptr;     // device AoS
    double* yout = nullptr;         // device AoS or null
    double* rows = nullptr;         // device [max_rows][11]
    double* traj = nullptr;         // device [max_rows][N*3] or null
    int64_t max_rows = 0;
    double T0 = 0, T1 = 0, dt0 = 0;
    int64_t n_steps = 0, save_every = 1;
    Pulse pulse{0, 0, 0, 0};
};

using LaunchFn = int (*)(const cmd_handle*, const ResidentArgs&, const double*, const double*, int64_t,
                         cudaStream_t);

// Resident-kernel variants compiled into the library: (atoms/cell, bonds/atom,
// in-cell bonds) x (cells per thread, max threads, min CTAs per SM, own stage
// input kept in registers, trajectories per CTA).  The autotuner times the
// ones that fit a lattice.
struct Variant {
    int NAT, Z, LZ, CPT, MAXT, MINB;
    bool YREG;
    int TPC;
    int CS;                       // CTAs per trajectory (thread-block cluster), 1 = one CTA
    bool lean;                    // rk4_lean_kernel (compile-time strides; every atom carries Z bonds)
    LaunchFn fn;
    const char* name;
};

// Streamed adjoint (rk_stream.cuh) for batches too small to fill the GPU with
// one CTA per trajectory: every stage (forward, recompute, VJP) is one launch
// over (cell tile, trajectory).
struct StreamAdjJob {
    int64_t B, S, C, K;
    bool fwd_only;
    const double* y0;          // device AoS [B][N*3]
    const double* target;      // device [B][S+1][3]
    const double* times;       // device [S+1]
    double* mloc;              // device [B][S+1][3]
    double* out;               // device [B][1 + kAdjParams]: loss, grad
    double dt;
};

constexpr int kAdjParams = 5;

inline int64_t rows_for(int64_t n_steps, int64_t save) { return (n_steps + save - 1) / save + 1; }

template <int NAT, int Z>
void fill_couplings(const cmd_handle* h, const double* d1, const double* d2, Couplings<NAT, Z>& cp) {
    std::memset(&cp, 0, sizeof(cp));
    const Layout& L = h->lay;
    for (int a = 0; a < NAT; ++a) {
        for (int s = 0; s < Z && s < L.zc[a]; ++s)
            std::memcpy(cp.J[a][s], &L.J[((size_t)a * L.Z + s) * 9], 9 * sizeof(double));
        cp.zc[a] = L.zc[a];
        std::memcpy(cp.field[a], &h->field[3 * a], 3 * sizeof(double));
        std::memcpy(cp.onsite[a], &h->onsite[9 * a], 9 * sizeof(double));
        if (d1) std::memcpy(cp.d1[a], d1 + 3 * a, 3 * sizeof(double));
        if (d2) std::memcpy(cp.d2[a], d2 + 3 * a, 3 * sizeof(double));
    }
    cp.has_field = h->has_field;
    cp.has_onsite = h->has_onsite;
}

// Shared memory of the resident kernel: two stage buffers per trajectory of a
// CTA, the reduction rows and the staged envelopes.
inline size_t resident_smem(int NA, int64_t G, int tpc = 1) {
    return (size_t)tpc * 2 * NA * 3 * G * sizeof(double) + (32 * kRedStride + 12 * tpc) * sizeof(double);
}

inline int64_t cluster_cells(int64_t G, int cs) { return (G + cs - 1) / cs; }

inline size_t cluster_smem(int NA, int64_t G, int cs) {
    return ((size_t)2 * NA * 3 * cluster_cells(G, cs) + 32 * kRedStride + 12 + 16) * sizeof(double);
}

template <int NAT>
void launch_finish(const double* raw, int64_t stride, int64_t n, const double* fr, const double* afm,
                   double n_sites, double* obs, cudaStream_t st) {
    const int blocks = (int)std::min<int64_t>((n + 255) / 256, 4096);
    finish_rows_kernel<NAT><<<std::max(blocks, 1), 256, 0, st>>>(raw, stride, n, fr, afm, n_sites, obs);
}

// Unit-cell types compiled into the global-state, streamed and on-chip RK45
// kernels: type 0 = 2-atom cells with 3 bonds per site (honeycomb), type 1 =
// 4-atom cells with 6 bonds per site (nearest-neighbour pyrochlore).
inline int global_type(const Layout& L) {
    if (!L.uniform) return -1;
    if (L.NA == 2 && L.Z == 3 && L.LZ == 1) return 0;
    if (L.NA == 4 && L.Z == 6 && L.LZ == 3) return 1;
    return -1;
}

// ---- cmd_api.cu
int sync(cmd_handle* h);
int caller_atoms(const cmd_handle* h);
int check_handle(cmd_handle* h, bool need_state);
int validate_batch(const cmd_handle* h, const cmd_batch_desc* d);
int no_instance(const Layout& L);

// ---- resident.cu
const Variant* variant_table();
int variant_count();
bool variant_fits(const Variant& v, const Layout& L);
int default_variant(const Layout& L);
int pick_variant(const cmd_handle* h);
int run_resident(cmd_handle* h, const RunSpec& r, cudaStream_t st, int32_t* launches);
int upload_cluster_table(cmd_handle* h, int cs);
const int* cluster_table(const cmd_handle* h, int cs);
void variant_shape(const Variant& V, const Layout& L, int64_t* threads, int64_t* smem);

// ---- stream.cu
// Drops the handle's captured launch sequences (after its stream is idle).
void release_stream_graph(cmd_handle* h);
// Graph slots of graph_call.
constexpr int kGraphResident = 0, kGraphUneven = 1;
// Runs enqueue() (stream-ordered work on st and on streams that join st; no
// synchronous calls) through a CUDA graph when the handle's graphs are on and
// st can be captured (not a default stream, not already capturing): the
// launches are captured, the handle's executable graph of `slot` is updated
// with them (instantiated when the launch topology changed) and launched on st.
// Otherwise enqueue() runs directly.  Either way the same kernels run with the
// same arguments.
int graph_call(cmd_handle* h, int slot, cudaStream_t st, const std::function<int()>& enqueue);
int run_streamed(cmd_handle* h, const RunSpec& r, cudaStream_t st, int32_t* launches);
int run_stream_adjoint(cmd_handle* h, const StreamAdjJob& j, int n_params, const std::vector<double>& DJ,
                       const std::vector<double>& DB, const std::vector<double>& DA, bool has_DA);

// ---- global.cu
// Runs the jobs on `owner`'s stream and synchronises; stats [B][4] out (rows
// written, accepted, rejected, status).  Controlled RK45 jobs run on the
// on-chip kernels where a tiling holds their lattice, the rest on the
// global-state kernel.
int run_global(cmd_handle* owner, std::vector<GJob>& jobs, int mode, double abs_tol, double rel_tol,
               int64_t max_steps, std::vector<long long>& stats);

// ---- rk45.cu: on-chip controlled Dormand-Prince tilings
int rk45_variant_count();
const char* rk45_variant_name(int i);
bool rk45_fits(int i, const Layout& L);
// The tiling a handle's trajectories use: its tuned pick, else the first that
// holds the lattice; -1 when none does (or the handle forces the global-state kernel).
int rk45_pick(const cmd_handle* h);
// Uploads the partner words tiling `variant` reads (synchronous; a no-op when
// they are current).  rk45_launch does it too; call it first where the launch
// must not synchronise (inside a stream capture).
int rk45_prepare(cmd_handle* h, int variant);
// Launches trajectories d_traj[0..B) (all on h's lattice) with tiling `variant` on `st`.
int rk45_launch(cmd_handle* h, int variant, const GTraj* d_traj, int64_t B, double abs_tol, double rel_tol,
                int64_t max_steps, cudaStream_t st);

// ---- noalloc.cu
int noalloc_lookup(double** out);

}  // namespace cmd
