// cmd_api.cu -- C-ABI implementation of the B200 Landau-Lifshitz MD path.
//
// Replaces the reference's gpu:: host API (include/classical_spin/gpu/
// lattice_gpu_api.h; implementation src/gpu/lattice_gpu.cu:586-791).  The
// reference keeps the lattice as an ELL table of per-entry 3x3 matrices and
// runs each RK stage as separate kernel launches with a device-wide sync in
// between (integrator.cuh:115-139: 8 launches + 4 syncs per step).  Here the
// lattice is compiled once at cmd_create into a per-unit-cell coupling table
// (identical for every cell, so it lives in kernel parameters) plus int32
// neighbour offsets, and a whole trajectory -- every stage of every step and
// the per-step observables -- runs inside one CTA of one launch.
#include "cmd.h"
#include "cmd_internal.h"
#include "rk4_resident.cuh"
#include "rk4_cluster.cuh"
#include "rk_global.cuh"
#include "rk_adjoint.cuh"
#include "rk_adjoint_cluster.cuh"
#include "rk_stream.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

namespace cmd {

static thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}
void clear_error() { g_last_error.clear(); }

}  // namespace cmd

using cmd::fail;

namespace {

constexpr size_t kMaxSmem = 232448;   // 227 KB dynamic shared memory per CTA on sm_100

#define CUDA_TRY(expr)                                                                   \
    do {                                                                                 \
        cudaError_t e_ = (expr);                                                         \
        if (e_ != cudaSuccess)                                                           \
            return fail(e_ == cudaErrorMemoryAllocation ? CMD_ERR_OOM : CMD_ERR_CUDA,    \
                        std::string(#expr) + ": " + cudaGetErrorString(e_));             \
    } while (0)

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
};

using cmd::DevBuf;

// Scratch of the allocation-free entry point (cmd_run_batch_device_noalloc):
// 2^22 doubles (32 MiB) per device.  The array is part of this file's device
// module, so every GPU that loads the module (at cmd_create at the latest, see
// noalloc_lookup) holds it until the process exits.  In host code
// `g_noalloc_scratch` is only a stand-in for the symbol; its device address
// comes from cudaGetSymbolAddress.
constexpr int64_t kNoAllocScratchDoubles = (int64_t)1 << 22;
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

// Device address of g_noalloc_scratch on the current device.  cmd_create calls
// it with the handle's device current and keeps the address in the handle, so
// the module (and the 32 MiB with it) is loaded at handle creation, never
// inside an allocation-free call, and a handle created after a context
// teardown looks the address up afresh.
int noalloc_lookup(double** out) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
        return fail(e == cudaErrorMemoryAllocation ? CMD_ERR_OOM : CMD_ERR_CUDA,
                    std::string("cudaGetSymbolAddress(allocation-free scratch): ") + cudaGetErrorString(e));
    *out = static_cast<double*>(p);
    return CMD_OK;
}

}  // namespace

struct cmd_handle {
    int64_t N = 0;
    int NA = 0;                 // sites per group (classes) used by the kernels
    int n_atoms_ref = 0;        // the caller's n_atoms when it differs from NA
    int zmax = 0;
    std::vector<double> field, onsite, frames, afm;   // per atom
    bool has_field = false, has_onsite = false;
    Layout lay;
    cudaStream_t stream = nullptr;
    DevBuf state, nbr, obs, traj, batch_states, batch_out, pulses, scratch;
    DevBuf dframes, dafm, times, drive, raw, tune_states, tune_obs;
    DevBuf gwork, gmeta, gstat, grows, gqueue;
    DevBuf awork, ackpt, aseg, amloc, aout, ameta, ain;
    DevBuf sbuf, spart, sgpart;  // streamed RK4 / adjoint: stage vectors, tile partials
    DevBuf chunk_states, chunk_rows;   // cmd_run_batch: ping-pong states and row buffers of time chunks
    DevBuf cnbr2, cnbr4;         // partner tables of the 2- and 4-CTA cluster kernels (built at create)
    cudaStream_t copy_stream = nullptr;  // cmd_run_batch: device-to-host copies of finished chunks
    bool has_state = false;
    int device = -1;            // device current at cmd_create (owns the stream and buffers)
    double* noalloc_base = nullptr;   // device address of the allocation-free scratch on `device`
    int variant = -1;           // resident-kernel variant; -1 = heuristic default
    // pulse (set_gpu_pulse)
    std::vector<double> fd;     // [2][NA*3]
    double amp = 0.0, width = 1.0, freq = 0.0, t1 = 0.0, t2 = 0.0;
    // controlled stepper
    double abs_tol = 1e-6, rel_tol = 1e-6;
    int64_t max_steps = 0;
};

namespace {

bool mat_equal(const double* a, const double* b) { return std::memcmp(a, b, 9 * sizeof(double)) == 0; }
bool mat_zero(const double* a) {
    for (int i = 0; i < 9; ++i)
        if (a[i] != 0.0) return false;
    return true;
}

// Compile the flat ELL tables into the per-cell layout.  Requirements (every
// lattice the reference builds from a UnitCell satisfies them): N = NA * G,
// field/onsite depend on the atom only, and after dropping all-zero coupling
// entries (which add exactly 0.0) each site of atom a carries the same
// multiset of (J, partner atom) as the site of atom a in cell 0.
//
// `NA` is the group size: n_atoms itself, or a divisor of it when a large unit
// cell is a union of identical smaller groups (the 16-site cubic pyrochlore cell
// = 4 FCC translations of the 4-site group).  Sites are then grouped as
// consecutive runs of NA, and everything per atom must depend on atom % NA.
void analyse_as(const cmd_lattice_desc& d, int NA, Layout& L) {
    L = Layout{};
    const int64_t N = d.lattice_size;
    const int zmax = d.max_bilinear;
    if (NA <= 0 || N % NA != 0) { L.why = "lattice_size is not a multiple of n_atoms"; return; }
    if (d.n_atoms % NA != 0) { L.why = "group size does not divide n_atoms"; return; }
    for (int a = NA; a < d.n_atoms; ++a) {
        if ((d.frames && std::memcmp(d.frames + 9 * a, d.frames + 9 * (a % NA), 9 * sizeof(double)) != 0) ||
            (d.afm_signs && d.afm_signs[a] != d.afm_signs[a % NA])) {
            L.why = "sublattice frames differ within a group class";
            return;
        }
    }
    L.NA = NA;
    L.G = N / NA;
    for (int64_t i = 0; i < N; ++i) {
        const int a = (int)(i % NA);
        if (std::memcmp(&d.field[3 * i], &d.field[3 * a], 3 * sizeof(double)) != 0 ||
            std::memcmp(&d.onsite[9 * i], &d.onsite[9 * a], 9 * sizeof(double)) != 0) {
            L.why = "field or onsite term differs between cells";
            return;
        }
    }
    // canonical (cell 0) slot lists per atom
    struct Slot { const double* J; int b; int64_t p0; int e; };   // p0: partner seen from cell 0; e: ELL entry
    std::vector<std::vector<Slot>> canon(NA);
    for (int a = 0; a < NA; ++a) {
        for (int64_t n = 0; n < d.counts[a]; ++n) {
            const double* J = &d.bilinear[9 * (a * (int64_t)zmax + n)];
            if (mat_zero(J)) continue;
            const int64_t p = d.partners[a * (int64_t)zmax + n];
            canon[a].push_back(Slot{J, (int)(p % NA), p, (int)n});
        }
    }
    // Try local-first ordering: slot n < NA-1 of atom a bonds to atom (a+1+n)%NA
    // inside the same cell.
    auto attempt = [&](bool local_first) -> bool {
        int LZ = 0;
        std::vector<std::vector<Slot>> order(NA);
        if (local_first) {
            LZ = NA - 1;
            for (int a = 0; a < NA; ++a) {
                std::vector<char> used(canon[a].size(), 0);
                for (int n = 0; n < NA - 1; ++n) {
                    const int want = (a + 1 + n) % NA;
                    int pick = -1;
                    for (size_t q = 0; q < canon[a].size(); ++q) {
                        if (used[q] || canon[a][q].b != want) continue;
                        if (canon[a][q].p0 / NA != 0) continue;   // must stay inside cell 0
                        pick = (int)q;
                        break;
                    }
                    if (pick < 0) return false;
                    used[pick] = 1;
                    order[a].push_back(canon[a][pick]);
                }
                for (size_t q = 0; q < canon[a].size(); ++q)
                    if (!used[q]) order[a].push_back(canon[a][q]);
            }
        } else {
            order = canon;
        }
        // Non-local slots in a size-independent order (partner atom, then the
        // coupling matrix), so lattices of one unit cell share one coupling table.
        for (int a = 0; a < NA; ++a)
            std::stable_sort(order[a].begin() + LZ, order[a].end(), [](const Slot& x, const Slot& y) {
                if (x.b != y.b) return x.b < y.b;
                return std::memcmp(x.J, y.J, 9 * sizeof(double)) < 0;
            });
        int Z = 0;
        for (int a = 0; a < NA; ++a) Z = std::max(Z, (int)order[a].size());
        const int NL = Z - LZ;
        const int64_t G = L.G;
        std::vector<int> nbr((size_t)G * NA * std::max(NL, 1), 0);
        std::vector<char> taken(zmax);
        for (int64_t g = 0; g < G; ++g) {
            for (int a = 0; a < NA; ++a) {
                const int64_t i = g * NA + a;
                std::fill(taken.begin(), taken.end(), 0);
                const int64_t cnt = d.counts[i];
                int nz = 0;
                for (int64_t n = 0; n < cnt; ++n)
                    if (!mat_zero(&d.bilinear[9 * (i * zmax + n)])) ++nz;
                if (nz != (int)order[a].size()) return false;
                for (int s = 0; s < (int)order[a].size(); ++s) {
                    const Slot& sl = order[a][s];
                    int pick = -1;
                    for (int64_t n = 0; n < cnt; ++n) {
                        if (taken[n]) continue;
                        const int64_t p = d.partners[i * zmax + n];
                        if (p < 0 || p >= d.lattice_size) return false;
                        if ((int)(p % NA) != sl.b) continue;
                        if (!mat_equal(&d.bilinear[9 * (i * zmax + n)], sl.J)) continue;
                        if (s < LZ && p / NA != g) continue;   // local slot: same cell
                        pick = (int)n;
                        break;
                    }
                    if (pick < 0) return false;
                    taken[pick] = 1;
                    if (s >= LZ) {
                        const int64_t p = d.partners[i * zmax + pick];
                        const int64_t off = (int64_t)(p % NA) * 3 * G + p / NA;
                        if (off > INT32_MAX) return false;
                        nbr[((size_t)g * NA + a) * NL + (s - LZ)] = (int)off;
                    }
                }
            }
        }
        L.LZ = LZ;
        L.Z = Z;
        L.zc.resize(NA);
        L.J.assign((size_t)NA * std::max(Z, 1) * 9, 0.0);
        L.slot_entry.assign((size_t)NA * std::max(Z, 1), -1);
        for (int a = 0; a < NA; ++a) {
            L.zc[a] = (int)order[a].size();
            for (int s2 = 0; s2 < (int)order[a].size(); ++s2) L.slot_entry[(size_t)a * Z + s2] = order[a][s2].e;
            for (int s = 0; s < (int)order[a].size(); ++s)
                std::memcpy(&L.J[((size_t)a * Z + s) * 9], order[a][s].J, 9 * sizeof(double));
        }
        L.nbr.swap(nbr);
        return true;
    };
    if (attempt(true) || attempt(false)) {
        L.uniform = true;
        return;
    }
    L.why = "coupling table is not identical in every unit cell";
}

int64_t rows_for(int64_t n_steps, int64_t save) { return (n_steps + save - 1) / save + 1; }

bool layout_has_kernel(const Layout& L);

// Chooses the group size: the whole unit cell when a kernel covers it,
// otherwise the largest of 4, 2, 1 dividing n_atoms that gives a uniform
// layout some kernel covers.
void analyse(const cmd_lattice_desc& d, Layout& L) {
    analyse_as(d, d.n_atoms, L);
    if (L.uniform && layout_has_kernel(L)) return;
    Layout first = L;
    for (int na : {4, 2, 1}) {
        if (na >= d.n_atoms || d.n_atoms % na != 0) continue;
        Layout alt;
        analyse_as(d, na, alt);
        if (alt.uniform && layout_has_kernel(alt)) {
            L = std::move(alt);
            return;
        }
    }
    L = std::move(first);
}

template <int NAT, int Z>
void fill_couplings(const cmd_handle* h, const double* d1, const double* d2, cmd::Couplings<NAT, Z>& cp) {
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
size_t resident_smem(int NA, int64_t G, int tpc = 1) {
    return (size_t)tpc * 2 * NA * 3 * G * sizeof(double) + (32 * cmd::kRedStride + 12 * tpc) * sizeof(double);
}

using LaunchFn = int (*)(const cmd_handle*, const cmd::ResidentArgs&, const double*, const double*, int64_t,
                         cudaStream_t);

template <int NAT, int Z, int LZ, int CPT, int MAXT, int MINB, bool YREG, int TPC>
int launch_one(const cmd_handle* h, const cmd::ResidentArgs& args, const double* d1, const double* d2,
               int64_t B, cudaStream_t st) {
    auto kern = cmd::rk4_resident_kernel<NAT, Z, LZ, CPT, MAXT, MINB, YREG, TPC>;
    const int64_t G = h->lay.G;
    int threads = (int)((G + CPT - 1) / CPT);
    threads = ((threads + 31) / 32) * 32;
    if (threads > MAXT) return fail(CMD_ERR_UNSUPPORTED, "lattice too large for this kernel variant");
    const size_t smem = resident_smem(NAT, G, TPC);
    if (smem > kMaxSmem) return fail(CMD_ERR_UNSUPPORTED, "stage buffers exceed shared memory");
    // Function attributes belong to the current device's context: set on every
    // launch (a host-side call of about a microsecond), so handles on several
    // devices, several host threads and a re-created context all see it.
    CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMaxSmem));
    cmd::Couplings<NAT, Z> cp;
    fill_couplings<NAT, Z>(h, d1, d2, cp);
    cmd::ResidentArgs a = args;
    a.B = B;
    kern<<<(unsigned)((B + TPC - 1) / TPC), threads, smem, st>>>(cp, a);
    CUDA_TRY(cudaGetLastError());
    return CMD_OK;
}

// Partner table of the CS-CTA cluster kernel: the resident table's offsets
// (atom*3)*G + cell become (rank << 24) | ((atom*3)*Gc + cell - rank*Gc) with
// Gc = ceil(G / CS) cells per CTA.  Built once per handle.
int64_t cluster_cells(int64_t G, int cs) { return (G + cs - 1) / cs; }

int upload_cluster_table(cmd_handle* h, int cs) {
    const Layout& L = h->lay;
    const int64_t G = L.G, Gc = cluster_cells(G, cs);
    if ((int64_t)L.NA * 3 * Gc >= (1 << cmd::kClusterRankShift)) return CMD_OK;   // never launched
    std::vector<int> t(L.nbr.size(), 0);
    for (size_t i = 0; i < L.nbr.size(); ++i) {
        const int64_t off = L.nbr[i];
        const int64_t at = off / (3 * G), c = off - at * 3 * G;     // partner atom*3 block and cell
        const int64_t gp = c % G, comp = c / G;                     // comp is 0 for the offsets stored
        const int64_t r = gp / Gc, l = gp - r * Gc;
        t[i] = (int)((r << cmd::kClusterRankShift) | ((at * 3 + comp) * Gc + l));
    }
    DevBuf& d = cs == 2 ? h->cnbr2 : h->cnbr4;
    if (int rc = d.ensure(std::max<size_t>(t.size(), 1) * sizeof(int))) return rc;
    if (!t.empty() && cudaMemcpy(d.p, t.data(), t.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(CMD_ERR_CUDA, "cluster neighbour table upload failed");
    return CMD_OK;
}

size_t cluster_smem(int NA, int64_t G, int cs) {
    return ((size_t)2 * NA * 3 * cluster_cells(G, cs) + 32 * cmd::kRedStride + 12 + 16) * sizeof(double);
}

template <int NAT, int Z, int LZ, int CS, int MAXT>
int launch_cluster(const cmd_handle* h, const cmd::ResidentArgs& args, const double* d1, const double* d2,
                   int64_t B, cudaStream_t st) {
    auto kern = cmd::rk4_cluster_kernel<NAT, Z, LZ, CS, MAXT>;
    const int64_t G = h->lay.G, Gc = cluster_cells(G, CS);
    const int threads = (int)((Gc + 31) / 32 * 32);
    if (threads > MAXT) return fail(CMD_ERR_UNSUPPORTED, "lattice too large for this cluster variant");
    const size_t smem = cluster_smem(NAT, G, CS);
    if (smem > kMaxSmem) return fail(CMD_ERR_UNSUPPORTED, "stage buffers exceed shared memory");
    const DevBuf& tab = CS == 2 ? h->cnbr2 : h->cnbr4;
    if (!tab.p) return fail(CMD_ERR_UNSUPPORTED, "no cluster neighbour table for this lattice");
    // Function attributes belong to the current device's context: set on every
    // launch (a host-side call of about a microsecond), so handles on several
    // devices, several host threads and a re-created context all see it.
    CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMaxSmem));
    cmd::Couplings<NAT, Z> cp;
    fill_couplings<NAT, Z>(h, d1, d2, cp);
    cmd::ResidentArgs a = args;
    a.B = B;
    a.nbr = static_cast<const int*>(tab.p);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(B * CS));
    cfg.blockDim = dim3((unsigned)threads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = CS;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    CUDA_TRY(cudaLaunchKernelEx(&cfg, kern, cp, a, (int)Gc));
    return CMD_OK;
}

// Resident-kernel variants compiled into the library: (atoms/cell, bonds/atom,
// in-cell bonds) x (cells per thread, max threads, min CTAs per SM, own stage
// input kept in registers, trajectories per CTA).  The autotuner times the
// ones that fit a lattice.
struct Variant {
    int NAT, Z, LZ, CPT, MAXT, MINB;
    bool YREG;
    int TPC;
    int CS;                       // CTAs per trajectory (thread-block cluster), 1 = one CTA
    LaunchFn fn;
    const char* name;
};

#define CMD_VARIANT(NAT, Z, LZ, CPT, MAXT, MINB, YREG, TPC) \
    Variant{NAT, Z, LZ, CPT, MAXT, MINB, YREG, TPC, 1, &launch_one<NAT, Z, LZ, CPT, MAXT, MINB, YREG, TPC>, \
            "rk4_resident<" #NAT "," #Z "," #LZ "> cpt=" #CPT " maxt=" #MAXT " minb=" #MINB " yreg=" #YREG \
            " tpc=" #TPC}
#define CMD_CLUSTER(NAT, Z, LZ, CS, MAXT) \
    Variant{NAT, Z, LZ, 1, MAXT, 1, true, 1, CS, &launch_cluster<NAT, Z, LZ, CS, MAXT>, \
            "rk4_cluster<" #NAT "," #Z "," #LZ "> cs=" #CS " maxt=" #MAXT}

const Variant kVariants[] = {
    // 2-atom cells with 3 bonds per site (Kitaev / Heisenberg honeycomb)
    CMD_VARIANT(2, 3, 1, 1, 640, 1, true, 1),
    CMD_VARIANT(2, 3, 1, 2, 320, 2, false, 1),
    CMD_VARIANT(2, 3, 1, 3, 192, 3, false, 1),
    CMD_VARIANT(2, 3, 1, 4, 160, 3, false, 1),
    CMD_VARIANT(2, 3, 1, 4, 160, 3, true, 1),
    CMD_VARIANT(2, 3, 1, 6, 96, 3, true, 1),
    CMD_VARIANT(2, 3, 1, 2, 512, 1, true, 1),
    CMD_VARIANT(2, 3, 1, 4, 256, 2, false, 1),
    // two trajectories per CTA: twice the independent work between barriers
    CMD_VARIANT(2, 3, 1, 1, 640, 1, false, 2),
    CMD_VARIANT(2, 3, 1, 1, 640, 1, true, 2),
    CMD_VARIANT(2, 3, 1, 2, 320, 1, false, 2),
    // one trajectory over a cluster of 2 or 4 CTAs (distributed shared memory)
    CMD_CLUSTER(2, 3, 1, 2, 640),
    CMD_CLUSTER(2, 3, 1, 4, 640),
    // 4-atom cells with 6 bonds per site (nearest-neighbour pyrochlore)
    CMD_VARIANT(4, 6, 3, 1, 512, 1, true, 1),
    CMD_VARIANT(4, 6, 3, 2, 256, 2, false, 1),
    CMD_VARIANT(4, 6, 3, 2, 512, 1, false, 1),
    CMD_CLUSTER(4, 6, 3, 2, 512),
    CMD_CLUSTER(4, 6, 3, 4, 512),
};
constexpr int kNumVariants = (int)(sizeof(kVariants) / sizeof(kVariants[0]));

bool variant_fits(const Variant& v, const Layout& L) {
    if (!L.uniform || v.NAT != L.NA || v.Z != L.Z || v.LZ != L.LZ) return false;
    if (v.CS > 1) {
        const int64_t Gc = cluster_cells(L.G, v.CS);
        return Gc >= 32 && (Gc + 31) / 32 * 32 <= v.MAXT && cluster_smem(v.NAT, L.G, v.CS) <= kMaxSmem &&
               (int64_t)v.NAT * 3 * Gc < (1 << cmd::kClusterRankShift);
    }
    const int64_t threads = ((L.G + v.CPT - 1) / v.CPT + 31) / 32 * 32;
    if (threads > v.MAXT) return false;
    const size_t smem = resident_smem(v.NAT, L.G, v.TPC);
    if (smem > kMaxSmem) return false;
    return true;
}

// Variant used when the caller did not pick one: the first fitting entry of
// the table (entries are ordered by preference for a lone trajectory).
int default_variant(const Layout& L) {
    for (int i = 0; i < kNumVariants; ++i)
        if (variant_fits(kVariants[i], L)) return i;
    return -1;
}

int no_instance(const Layout& L) {
    if (!L.uniform) return fail(CMD_ERR_UNSUPPORTED, "lattice layout not supported: " + L.why);
    char buf[200];
    std::snprintf(buf, sizeof(buf),
                  "no resident kernel for %d atoms/cell, %d bonds/site, %d local, %lld cells",
                  L.NA, L.Z, L.LZ, (long long)L.G);
    return fail(CMD_ERR_UNSUPPORTED, buf);
}

int pick_variant(const cmd_handle* h) {
    if (h->variant >= 0 && h->variant < kNumVariants && variant_fits(kVariants[h->variant], h->lay))
        return h->variant;
    return default_variant(h->lay);
}

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
    const cmd::Pulse* pulses = nullptr;   // device [B]
    double width = 1.0, freq = 0.0;
    const double* d1 = nullptr;       // host [NA*3]
    const double* d2 = nullptr;
    const double* frames = nullptr;   // device [NA*9]
    const double* afm = nullptr;      // device [NA]
    double n_sites = 1.0;
    int variant = -1;                 // -1: handle's choice
};

template <int NAT>
void launch_finish(const double* raw, int64_t stride, int64_t n, const double* fr, const double* afm,
                   double n_sites, double* obs, cudaStream_t st) {
    const int blocks = (int)std::min<int64_t>((n + 255) / 256, 4096);
    cmd::finish_rows_kernel<NAT><<<std::max(blocks, 1), 256, 0, st>>>(raw, stride, n, fr, afm, n_sites, obs);
}

// Launches drive-table pre-pass (when driven), the resident kernel and the
// row-finishing post-pass on `st`.  Asynchronous; returns the launch count.
int run_resident(cmd_handle* h, const RunSpec& r, cudaStream_t st, int32_t* launches) {
    int32_t nl = 0;
    const int vi = r.variant >= 0 ? r.variant : pick_variant(h);
    if (vi < 0 || !variant_fits(kVariants[vi], h->lay)) return no_instance(h->lay);
    const Variant& V = kVariants[vi];
    const int64_t rows = rows_for(r.n_steps, r.save);
    const int NR = 3 * V.NAT + 1;
    cmd::ResidentArgs a{};
    a.G = (int)h->lay.G;
    a.n_steps = r.n_steps;
    a.save_every = r.save;
    a.T0 = r.T0;
    a.dt = r.dt;
    a.nbr = h->nbr.as<int>();
    a.y0 = r.y0;
    a.y0_stride = r.y0_stride;
    a.y_out = r.y_out;
    a.rows = rows;
    a.traj = r.traj;
    a.drive = nullptr;
    if (r.obs) {
        if (NR <= 10) {
            a.raw = r.obs;
            a.raw_stride = 10;
        } else {
            if (int rc = h->raw.ensure((size_t)r.B * rows * NR * sizeof(double))) return rc;
            a.raw = h->raw.as<double>();
            a.raw_stride = NR;
        }
    }
    if (r.pulses && r.n_steps > 0) {
        std::vector<double> grid;
        grid.reserve(r.n_steps + 1);
        double t = r.T0;
        for (int64_t k = 0; k < r.n_steps; ++k) {     // t_k of the reference loop (t += dt)
            grid.push_back(t);
            t += r.dt;
        }
        if (int rc = h->times.ensure(grid.size() * sizeof(double))) return rc;
        if (int rc = h->drive.ensure((size_t)r.B * r.n_steps * 6 * sizeof(double))) return rc;
        CUDA_TRY(cudaMemcpyAsync(h->times.p, grid.data(), grid.size() * sizeof(double), cudaMemcpyHostToDevice, st));
        const int64_t total = r.B * r.n_steps * 6;
        const int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 32);
        cmd::drive_table_kernel<<<blocks, 256, 0, st>>>(r.pulses, h->times.as<double>(), r.n_steps, r.dt, r.width,
                                                       r.freq, r.B, h->drive.as<double>());
        CUDA_TRY(cudaGetLastError());
        ++nl;
        a.drive = h->drive.as<double>();
    }
    static const std::vector<double> zeros(3 * 64, 0.0);
    if (int rc = V.fn(h, a, r.d1 ? r.d1 : zeros.data(), r.d2 ? r.d2 : zeros.data(), r.B, st)) return rc;
    ++nl;
    if (r.obs) {
        const int64_t n = r.B * rows;
        const double* fr = r.frames ? r.frames : h->dframes.as<double>();
        const double* af = r.afm ? r.afm : h->dafm.as<double>();
        switch (V.NAT) {
            case 2: launch_finish<2>(a.raw, a.raw_stride, n, fr, af, r.n_sites, r.obs, st); break;
            case 4: launch_finish<4>(a.raw, a.raw_stride, n, fr, af, r.n_sites, r.obs, st); break;
            default: return fail(CMD_ERR_UNSUPPORTED, "no row finisher for this cell size");
        }
        CUDA_TRY(cudaGetLastError());
        ++nl;
    }
    if (launches) *launches = nl;
    return CMD_OK;
}

// ---------------------------------------------------------------------------
// Streamed RK4 (rk_stream.cuh): lattices no resident variant holds.  One launch
// per stage over (cell tile, trajectory); same RunSpec contract and outputs as
// run_resident.

template <int NAT, int Z, int LZ>
int stream_forward(cmd_handle* h, const RunSpec& r, cudaStream_t st, int32_t* launches) {
    constexpr int NR = 3 * NAT + 1;
    int32_t nl = 0;
    const int G = (int)h->lay.G;
    const int tiles = (G + cmd::stream_cells<NAT>() - 1) / cmd::stream_cells<NAT>();
    const int64_t V = (int64_t)NAT * 3 * G;
    const int64_t B = r.B;
    if (B > 65535) return fail(CMD_ERR_UNSUPPORTED, "streamed batches are limited to 65535 trajectories");
    if (r.traj && B != 1) return fail(CMD_ERR_UNSUPPORTED, "streamed state saving is for single trajectories");
    const int64_t rows = rows_for(r.n_steps, r.save);
    if (int rc = h->sbuf.ensure((size_t)4 * B * V * sizeof(double))) return rc;
    if (int rc = h->spart.ensure((size_t)B * tiles * cmd::kPart * sizeof(double))) return rc;
    double* base = h->sbuf.as<double>();
    const cmd::SVec y{base, V}, acc{base + B * V, V}, Ya{base + 2 * B * V, V}, Yb{base + 3 * B * V, V};
    cmd::StreamArgs a{};
    a.G = G;
    a.tiles = tiles;
    a.B = (int)B;
    a.nbr = h->nbr.as<int>();
    a.dt = r.dt;
    a.n_steps = r.n_steps;
    a.part = h->spart.as<double>();
    a.n_sites = r.n_sites;
    a.save_every = r.save;
    a.rows = rows;
    a.V = V;
    if (r.obs) {
        if (NR <= 10) {
            a.raw = r.obs;
            a.raw_stride = 10;
        } else {
            if (int rc = h->raw.ensure((size_t)B * rows * NR * sizeof(double))) return rc;
            a.raw = h->raw.as<double>();
            a.raw_stride = NR;
        }
    }
    if (r.pulses && r.n_steps > 0) {
        std::vector<double> grid;
        grid.reserve(r.n_steps);
        double t = r.T0;
        for (int64_t k = 0; k < r.n_steps; ++k) {     // t_k of the reference loop (t += dt)
            grid.push_back(t);
            t += r.dt;
        }
        if (int rc = h->times.ensure(grid.size() * sizeof(double))) return rc;
        if (int rc = h->drive.ensure((size_t)B * r.n_steps * 6 * sizeof(double))) return rc;
        CUDA_TRY(cudaMemcpyAsync(h->times.p, grid.data(), grid.size() * sizeof(double), cudaMemcpyHostToDevice, st));
        const int64_t total = B * r.n_steps * 6;
        const int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 32);
        cmd::drive_table_kernel<<<blocks, 256, 0, st>>>(r.pulses, h->times.as<double>(), r.n_steps, r.dt, r.width,
                                                       r.freq, B, h->drive.as<double>());
        CUDA_TRY(cudaGetLastError());
        ++nl;
        a.times = h->times.as<double>();
        a.drive = h->drive.as<double>();
    }
    static const std::vector<double> zeros(3 * 64, 0.0);
    cmd::Couplings<NAT, Z> cp;
    fill_couplings<NAT, Z>(h, r.d1 ? r.d1 : zeros.data(), r.d2 ? r.d2 : zeros.data(), cp);
    const dim3 grid(tiles, (unsigned)B), gridc((G + 255) / 256, (unsigned)B);
    const int64_t N3 = (int64_t)G * NAT * 3;
    auto save_traj = [&](int64_t row) {
        const cmd::SVec src = y;
        cmd::stream_store_kernel<NAT><<<gridc, 256, 0, st>>>(src, G, r.traj + row * N3);
        ++nl;
    };
    cmd::stream_load_kernel<NAT><<<gridc, 256, 0, st>>>(r.y0, r.y0_stride, G, y);
    CUDA_TRY(cudaGetLastError());
    ++nl;
    const int with_obs = r.obs ? 1 : 0;
    for (int64_t n = 0; n < r.n_steps; ++n) {
        if (r.traj && n % r.save == 0) save_traj(n / r.save);
        cmd::stream_stage_kernel<NAT, Z, LZ><<<grid, cmd::kStreamTile, 0, st>>>(cp, a, 0, n, y, y, acc, Ya, with_obs);
        cmd::stream_stage_kernel<NAT, Z, LZ><<<grid, cmd::kStreamTile, 0, st>>>(cp, a, 1, n, Ya, y, acc, Yb, with_obs);
        cmd::stream_stage_kernel<NAT, Z, LZ><<<grid, cmd::kStreamTile, 0, st>>>(cp, a, 2, n, Yb, y, acc, Ya, with_obs);
        cmd::stream_stage_kernel<NAT, Z, LZ><<<grid, cmd::kStreamTile, 0, st>>>(cp, a, 3, n, Ya, y, acc, y, with_obs);
        nl += 4;
        if ((n & 1023) == 0) CUDA_TRY(cudaGetLastError());
    }
    CUDA_TRY(cudaGetLastError());
    if (r.traj) save_traj(rows - 1);
    if (r.obs) {
        cmd::stream_obs_kernel<NAT, Z, LZ><<<grid, cmd::kStreamTile, 0, st>>>(cp, a, y);
        cmd::stream_reduce_kernel<NAT><<<(unsigned)B, cmd::kStreamTile, 0, st>>>(a, r.n_steps);
        CUDA_TRY(cudaGetLastError());
        nl += 2;
    }
    if (r.y_out) {
        cmd::stream_store_kernel<NAT><<<gridc, 256, 0, st>>>(y, G, r.y_out);
        CUDA_TRY(cudaGetLastError());
        ++nl;
    }
    if (r.obs) {
        const double* fr = r.frames ? r.frames : h->dframes.as<double>();
        const double* af = r.afm ? r.afm : h->dafm.as<double>();
        launch_finish<NAT>(a.raw, a.raw_stride, B * rows, fr, af, r.n_sites, r.obs, st);
        CUDA_TRY(cudaGetLastError());
        ++nl;
    }
    if (launches) *launches = nl;
    return CMD_OK;
}

// ---------------------------------------------------------------------------
// Global-state integrator (rk_global.cuh): controlled / fixed Dormand-Prince and
// global-memory RK4, persistent over a queue of trajectories.

// Unit-cell types compiled into rk_global_kernel: type 0 = 2-atom cells with 3
// bonds per site (honeycomb), type 1 = 4-atom cells with 6 bonds per site
// (nearest-neighbour pyrochlore).
int global_type(const Layout& L) {
    if (!L.uniform) return -1;
    if (L.NA == 2 && L.Z == 3 && L.LZ == 1) return 0;
    if (L.NA == 4 && L.Z == 6 && L.LZ == 3) return 1;
    return -1;
}

bool layout_has_kernel(const Layout& L) { return default_variant(L) >= 0 || global_type(L) >= 0; }

// RK4 over the handle's lattice: the resident kernel when a variant holds the
// lattice (or one is named), else the streamed stage kernels.
int run_rk4(cmd_handle* h, const RunSpec& r, cudaStream_t st, int32_t* launches) {
    if (r.variant >= 0 || pick_variant(h) >= 0) return run_resident(h, r, st, launches);
    switch (global_type(h->lay)) {
        case 0: return stream_forward<2, 3, 1>(h, r, st, launches);
        case 1: return stream_forward<4, 6, 3>(h, r, st, launches);
        default: return no_instance(h->lay);
    }
}

struct GJob {
    cmd_handle* h = nullptr;
    const double* y0 = nullptr;     // device AoS
    double* yout = nullptr;         // device AoS or null
    double* rows = nullptr;         // device [max_rows][11]
    double* traj = nullptr;         // device [max_rows][N*3] or null
    int64_t max_rows = 0;
    double T0 = 0, T1 = 0, dt0 = 0;
    int64_t n_steps = 0, save_every = 1;
    cmd::Pulse pulse{0, 0, 0, 0};
};

bool same_couplings(const cmd_handle* a, const cmd_handle* b) {
    return a->lay.J == b->lay.J && a->lay.zc == b->lay.zc && a->field == b->field && a->onsite == b->onsite &&
           a->fd == b->fd && a->width == b->width && a->freq == b->freq && a->frames == b->frames &&
           a->afm == b->afm;
}

int sync(cmd_handle* h);

// Runs the jobs in one persistent launch on `owner`'s stream; stats [B][4] out.
int run_global(cmd_handle* owner, std::vector<GJob>& jobs, int mode, double abs_tol, double rel_tol,
               int64_t max_steps, std::vector<long long>& stats) {
    const int64_t B = (int64_t)jobs.size();
    if (B <= 0) return fail(CMD_ERR_INVALID_ARG, "empty batch");
    const cmd_handle* src[2] = {nullptr, nullptr};
    for (const GJob& j : jobs) {
        const int ty = global_type(j.h->lay);
        if (ty < 0) return no_instance(j.h->lay);
        if (!src[ty]) src[ty] = j.h;
        else if (!same_couplings(src[ty], j.h))
            return fail(CMD_ERR_UNSUPPORTED, "lattices of one unit-cell type must share couplings and pulse settings");
    }
    if (src[0] && src[1] && (src[0]->width != src[1]->width || src[0]->freq != src[1]->freq))
        return fail(CMD_ERR_UNSUPPORTED, "pulse width / frequency must agree across the batch");
    // longest first (cells x expected steps)
    std::vector<int64_t> order(B);
    for (int64_t i = 0; i < B; ++i) order[i] = i;
    auto cost = [&](int64_t i) {
        const GJob& j = jobs[i];
        const double steps = j.n_steps > 0 ? (double)j.n_steps : (j.T1 - j.T0) / std::max(j.dt0, 1e-300);
        return (double)j.h->N * steps;
    };
    std::stable_sort(order.begin(), order.end(), [&](int64_t x, int64_t y) { return cost(x) > cost(y); });
    size_t work_total = 0;
    std::vector<size_t> woff(B);
    for (int64_t i = 0; i < B; ++i) {
        woff[i] = work_total;
        work_total += (size_t)cmd::kGVectors * 3 * jobs[i].h->N;
    }
    if (int rc = owner->gwork.ensure(work_total * sizeof(double))) return rc;
    if (int rc = owner->gmeta.ensure((size_t)B * sizeof(cmd::GTraj))) return rc;
    if (int rc = owner->gstat.ensure((size_t)B * 4 * sizeof(long long))) return rc;
    if (int rc = owner->gqueue.ensure(sizeof(int))) return rc;
    std::vector<cmd::GTraj> tr(B);
    long long* dstat = owner->gstat.as<long long>();
    for (int64_t q = 0; q < B; ++q) {
        const int64_t i = order[q];
        const GJob& j = jobs[i];
        cmd::GTraj& T = tr[q];
        T.type = global_type(j.h->lay);
        T.G = (int)j.h->lay.G;
        T.nbr = j.h->nbr.as<int>();
        T.y0 = j.y0;
        T.yout = j.yout;
        T.work = owner->gwork.as<double>() + woff[i];
        T.rows = j.rows;
        T.traj = j.traj;
        T.max_rows = j.max_rows;
        T.T0 = j.T0; T.T1 = j.T1; T.dt0 = j.dt0;
        T.n_steps = j.n_steps;
        T.save_every = j.save_every;
        T.pulse = j.pulse;
        T.stat = dstat + 4 * i;
    }
    cudaStream_t st = owner->stream;
    CUDA_TRY(cudaMemcpyAsync(owner->gmeta.p, tr.data(), B * sizeof(cmd::GTraj), cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemsetAsync(owner->gqueue.p, 0, sizeof(int), st));
    CUDA_TRY(cudaMemsetAsync(owner->gstat.p, 0, B * 4 * sizeof(long long), st));
    cmd::GArgs a{};
    a.traj = owner->gmeta.as<cmd::GTraj>();
    a.B = (int)B;
    a.queue = owner->gqueue.as<int>();
    a.mode = mode;
    a.abs_tol = abs_tol;
    a.rel_tol = rel_tol;
    a.max_steps = max_steps;
    const cmd_handle* any = src[0] ? src[0] : src[1];
    a.width = any->width;
    a.freq = any->freq;
    cmd::Couplings<2, 3> c0;
    cmd::Couplings<4, 6> c1;
    std::memset(&c0, 0, sizeof(c0));
    std::memset(&c1, 0, sizeof(c1));
    if (src[0]) {
        fill_couplings<2, 3>(src[0], src[0]->fd.data(), src[0]->fd.data() + 3 * src[0]->NA, c0);
        a.frames0 = src[0]->dframes.as<double>();
        a.afm0 = src[0]->dafm.as<double>();
    }
    if (src[1]) {
        fill_couplings<4, 6>(src[1], src[1]->fd.data(), src[1]->fd.data() + 3 * src[1]->NA, c1);
        a.frames1 = src[1]->dframes.as<double>();
        a.afm1 = src[1]->dafm.as<double>();
    }
    auto kern = mode >= cmd::kModeEuler ? cmd::rk_global_kernel<2, 3, 1, 4, 6, 3, true>
                                        : cmd::rk_global_kernel<2, 3, 1, 4, 6, 3, false>;
    int dev = 0, nsm = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, 0);
    const int grid = (int)std::min<int64_t>(B, (int64_t)nsm * std::max(per_sm, 1));
    kern<<<grid, 256, 0, st>>>(c0, c1, a);
    CUDA_TRY(cudaGetLastError());
    stats.assign((size_t)B * 4, 0);
    CUDA_TRY(cudaMemcpyAsync(stats.data(), owner->gstat.p, B * 4 * sizeof(long long), cudaMemcpyDeviceToHost, st));
    return sync(owner);
}

// Reference GPU loop (integrator.cuh:477-483): number of steps and times.
int64_t count_steps(double T0, double T1, double dt, double margin, std::vector<double>* times) {
    int64_t n = 0;
    double t = T0;
    while (t < T1 - margin) {
        if (times) times->push_back(t);
        t += dt;
        ++n;
        if (n > (int64_t)1 << 40) break;
    }
    if (times) times->push_back(t);
    return n;
}

int sync(cmd_handle* h) {
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return fail(CMD_ERR_CUDA, std::string("kernel execution: ") + cudaGetErrorString(e));
    return CMD_OK;
}

__global__ void normalize_kernel(double* s, double len, int64_t N) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const double x = s[3 * i], y = s[3 * i + 1], z = s[3 * i + 2];
    const double n = sqrt(x * x + y * y + z * z);
    if (n > 0.0) {
        s[3 * i] = len * x / n;
        s[3 * i + 1] = len * y / n;
        s[3 * i + 2] = len * z / n;
    }
}

// compute_magnetization_gpu semantics: mean and (-1)^i staggered mean.  One CTA,
// fixed-order tree reduction.
__global__ void magnetization_kernel(const double* s, int64_t N, double* out) {
    __shared__ double sh[6][256];
    double v[6] = {0, 0, 0, 0, 0, 0};
    for (int64_t i = threadIdx.x; i < N; i += blockDim.x) {
        const double sg = (i % 2 == 0) ? 1.0 : -1.0;
        for (int c = 0; c < 3; ++c) {
            v[c] += s[3 * i + c];
            v[3 + c] += sg * s[3 * i + c];
        }
    }
    for (int q = 0; q < 6; ++q) sh[q][threadIdx.x] = v[q];
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int q = 0; q < 6; ++q) sh[q][threadIdx.x] += sh[q][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int q = 0; q < 6; ++q) out[q] = sh[q][0] / (double)N;
}

int upload_frames(cmd_handle* h, const double* frames, const double* afm) {
    if (int rc = h->dframes.ensure(9 * (size_t)h->NA * sizeof(double))) return rc;
    if (int rc = h->dafm.ensure((size_t)h->NA * sizeof(double))) return rc;
    CUDA_TRY(cudaMemcpyAsync(h->dframes.p, frames, 9 * h->NA * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(cudaMemcpyAsync(h->dafm.p, afm, h->NA * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    return sync(h);
}

int caller_atoms(const cmd_handle* h) { return h->n_atoms_ref ? h->n_atoms_ref : h->NA; }

// Per-atom array of the caller's unit cell [caller atoms][w] -> per class [NA][w].
int reduce_per_class(const cmd_handle* h, const double* in, int w, std::vector<double>& out, const char* what) {
    const int ca = caller_atoms(h);
    out.assign(in, in + (size_t)w * h->NA);
    for (int a = h->NA; a < ca; ++a)
        for (int c = 0; c < w; ++c)
            if (in[a * w + c] != out[(a % h->NA) * w + c])
                return fail(CMD_ERR_UNSUPPORTED, std::string(what) + " must be uniform per sublattice class");
    return CMD_OK;
}

int check_handle(cmd_handle* h, bool need_state) {
    if (!h) return fail(CMD_ERR_INVALID_ARG, "NULL handle");
    if (need_state && !h->has_state) return fail(CMD_ERR_STATE, "spins not set (call cmd_set_spins first)");
    return CMD_OK;
}

}  // namespace

extern "C" {

const char* cmd_last_error(void) { return cmd::g_last_error.c_str(); }
const char* cmd_version(void) { return "classical_mcmc_spin_b200 0.1 (sm_100a, fp64)"; }

int cmd_create(const cmd_lattice_desc* d, cmd_handle** out) {
    cmd::clear_error();
    if (!out) return fail(CMD_ERR_INVALID_ARG, "output pointer is NULL");
    *out = nullptr;
    if (!d) return fail(CMD_ERR_INVALID_ARG, "NULL lattice description");
    if (d->spin_dim != 3) return fail(CMD_ERR_UNSUPPORTED, "only spin_dim = 3 is supported");
    if (d->lattice_size <= 0 || d->n_atoms <= 0 || d->max_bilinear < 0)
        return fail(CMD_ERR_INVALID_ARG, "bad lattice sizes");
    if (d->lattice_size > ((int64_t)1 << 30)) return fail(CMD_ERR_INVALID_ARG, "lattice too large");
    if (!d->field || !d->onsite || !d->counts || (d->max_bilinear > 0 && (!d->bilinear || !d->partners)))
        return fail(CMD_ERR_INVALID_ARG, "NULL lattice array");
    for (int64_t i = 0; i < d->lattice_size; ++i)
        if (d->counts[i] < 0 || d->counts[i] > d->max_bilinear)
            return fail(CMD_ERR_INVALID_ARG, "bilinear count out of range");
    for (int64_t i = 0; i < d->lattice_size * 3; ++i)
        if (!std::isfinite(d->field[i])) return fail(CMD_ERR_NONFINITE, "non-finite field");
    for (int64_t i = 0; i < d->lattice_size * d->max_bilinear * 9; ++i)
        if (!std::isfinite(d->bilinear[i])) return fail(CMD_ERR_NONFINITE, "non-finite coupling");
    cmd_handle* h = new (std::nothrow) cmd_handle();
    if (!h) return fail(CMD_ERR_OOM, "host allocation failed");
    h->N = d->lattice_size;
    h->NA = d->n_atoms;
    h->zmax = d->max_bilinear;
    h->field.assign(d->field, d->field + 3 * d->n_atoms);
    h->onsite.assign(d->onsite, d->onsite + 9 * d->n_atoms);
    h->frames.assign(9 * (size_t)d->n_atoms, 0.0);
    h->afm.assign(d->n_atoms, 1.0);
    for (int a = 0; a < d->n_atoms; ++a) {
        if (d->frames) std::memcpy(&h->frames[9 * a], d->frames + 9 * a, 9 * sizeof(double));
        else h->frames[9 * a] = h->frames[9 * a + 4] = h->frames[9 * a + 8] = 1.0;
        if (d->afm_signs) h->afm[a] = d->afm_signs[a];
    }
    for (double v : h->field) h->has_field |= (v != 0.0);
    for (double v : h->onsite) h->has_onsite |= (v != 0.0);
    h->fd.assign(2 * 3 * (size_t)d->n_atoms, 0.0);
    analyse(*d, h->lay);
    if (h->lay.uniform && h->lay.NA != d->n_atoms) {
        // grouped cell: per-class tables are the first NA atoms' (checked uniform)
        const int na = h->lay.NA;
        h->NA = na;
        h->field.resize(3 * na);
        h->onsite.resize(9 * na);
        h->frames.resize(9 * na);
        h->afm.resize(na);
        h->fd.assign(6 * (size_t)na, 0.0);
        h->n_atoms_ref = d->n_atoms;
    }
    int rc = CMD_OK;
    if (cudaGetDevice(&h->device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
        rc = fail(CMD_ERR_CUDA, "cudaStreamCreate failed (no CUDA device?)");
    } else if ((rc = noalloc_lookup(&h->noalloc_base)) != CMD_OK) {
        // the device module (with the allocation-free scratch) could not be loaded
    } else if (h->lay.uniform) {
        rc = h->nbr.ensure(std::max<size_t>(h->lay.nbr.size(), 1) * sizeof(int));
        if (rc == CMD_OK && !h->lay.nbr.empty() &&
            cudaMemcpy(h->nbr.p, h->lay.nbr.data(), h->lay.nbr.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess)
            rc = fail(CMD_ERR_CUDA, "neighbour table upload failed");
        for (int cs : {2, 4})
            if (rc == CMD_OK) rc = upload_cluster_table(h, cs);
    }
    if (rc == CMD_OK) rc = h->state.ensure((size_t)h->N * 3 * sizeof(double));
    if (rc == CMD_OK) rc = upload_frames(h, h->frames.data(), h->afm.data());
    if (rc != CMD_OK) {
        cmd_destroy(h);
        return rc;
    }
    *out = h;
    return CMD_OK;
}

int cmd_destroy(cmd_handle* h) {
    if (!h) return CMD_OK;
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (DevBuf* b : {&h->state, &h->nbr, &h->obs, &h->traj, &h->batch_states, &h->batch_out,
                      &h->pulses, &h->scratch, &h->dframes, &h->dafm, &h->times, &h->drive, &h->raw,
                      &h->tune_states, &h->tune_obs, &h->gwork, &h->gmeta, &h->gstat, &h->grows, &h->gqueue,
                      &h->awork, &h->ackpt, &h->aseg, &h->amloc, &h->aout, &h->ameta, &h->ain,
                      &h->sbuf, &h->spart, &h->sgpart, &h->chunk_states, &h->chunk_rows, &h->cnbr2, &h->cnbr4})
        b->release();
    if (h->copy_stream) cudaStreamDestroy(h->copy_stream);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return CMD_OK;
}

int cmd_set_pulse(cmd_handle* h, const double* fd, double amp, double width, double freq, double t1,
                  double t2) {
    cmd::clear_error();
    if (int rc = check_handle(h, false)) return rc;
    if (!fd) return fail(CMD_ERR_INVALID_ARG, "NULL field_drive");
    if (!(width != 0.0) || !std::isfinite(amp) || !std::isfinite(width) || !std::isfinite(freq))
        return fail(CMD_ERR_INVALID_ARG, "bad pulse parameters");
    // field_drive is [2][caller atoms][3]; a grouped cell needs it uniform per class
    const int ca = caller_atoms(h);
    std::vector<double> v(6 * (size_t)h->NA);
    for (int p = 0; p < 2; ++p)
        for (int a = 0; a < ca; ++a)
            for (int c = 0; c < 3; ++c) {
                const double x = fd[(p * ca + a) * 3 + c];
                if (a < h->NA) v[(p * h->NA + a) * 3 + c] = x;
                else if (x != v[(p * h->NA + a % h->NA) * 3 + c])
                    return fail(CMD_ERR_UNSUPPORTED, "pulse directions must be uniform per sublattice class");
            }
    h->fd.swap(v);
    h->amp = amp; h->width = width; h->freq = freq; h->t1 = t1; h->t2 = t2;
    return CMD_OK;
}

int cmd_set_spins(cmd_handle* h, const double* s, int64_t n) {
    cmd::clear_error();
    if (int rc = check_handle(h, false)) return rc;
    if (!s || n != h->N * 3) return fail(CMD_ERR_INVALID_ARG, "spin array must hold N*3 doubles");
    for (int64_t i = 0; i < n; ++i)
        if (!std::isfinite(s[i])) return fail(CMD_ERR_NONFINITE, "non-finite spin component");
    CUDA_TRY(cudaMemcpyAsync(h->state.p, s, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    if (int rc = sync(h)) return rc;
    h->has_state = true;
    return CMD_OK;
}

int cmd_get_spins(cmd_handle* h, double* s, int64_t n) {
    cmd::clear_error();
    if (int rc = check_handle(h, true)) return rc;
    if (!s || n != h->N * 3) return fail(CMD_ERR_INVALID_ARG, "spin array must hold N*3 doubles");
    CUDA_TRY(cudaMemcpyAsync(s, h->state.p, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    return sync(h);
}

int cmd_set_tolerances(cmd_handle* h, double abs_tol, double rel_tol, int64_t max_steps) {
    cmd::clear_error();
    if (int rc = check_handle(h, false)) return rc;
    if (!(abs_tol >= 0.0) || !(rel_tol >= 0.0) || (abs_tol == 0.0 && rel_tol == 0.0) || max_steps < 0)
        return fail(CMD_ERR_INVALID_ARG, "bad tolerances");
    h->abs_tol = abs_tol; h->rel_tol = rel_tol; h->max_steps = max_steps;
    return CMD_OK;
}

namespace {

// Runs `n_steps` RK4 steps of the handle's trajectory on device, saving rows.
int run_single(cmd_handle* h, double T0, double dt, int64_t n_steps, int64_t save, double n_sites,
               bool want_obs, bool want_traj, bool with_pulse) {
    const int64_t rows = rows_for(n_steps, save);
    if (want_obs)
        if (int rc = h->obs.ensure((size_t)rows * 10 * sizeof(double))) return rc;
    if (want_traj)
        if (int rc = h->traj.ensure((size_t)rows * h->N * 3 * sizeof(double))) return rc;
    const bool driven = with_pulse && h->amp != 0.0;
    cmd::Pulse pl{h->t1, h->t2, h->amp, h->amp};
    if (driven) {
        if (int rc = h->pulses.ensure(sizeof(cmd::Pulse))) return rc;
        CUDA_TRY(cudaMemcpyAsync(h->pulses.p, &pl, sizeof(pl), cudaMemcpyHostToDevice, h->stream));
    }
    RunSpec r;
    r.B = 1;
    r.y0 = h->state.as<double>();
    r.y_out = h->state.as<double>();
    r.obs = want_obs ? h->obs.as<double>() : nullptr;
    r.traj = want_traj ? h->traj.as<double>() : nullptr;
    r.T0 = T0;
    r.dt = dt;
    r.n_steps = n_steps;
    r.save = save;
    r.pulses = driven ? h->pulses.as<cmd::Pulse>() : nullptr;
    r.width = h->width;
    r.freq = h->freq;
    r.d1 = h->fd.data();
    r.d2 = h->fd.data() + 3 * h->NA;
    r.n_sites = n_sites;
    if (int rc = run_rk4(h, r, h->stream, nullptr)) return rc;
    return sync(h);
}

}  // namespace

namespace {

int mode_of(int method) {
    switch (method) {
        case CMD_RK45: return cmd::kModeRK45;
        case CMD_DOPRI5_FIXED: return cmd::kModeDopri5Fixed;
        case CMD_CASH_KARP_FIXED: return cmd::kModeCashKarpFixed;
        case CMD_EULER: return cmd::kModeEuler;
        case CMD_MIDPOINT: return cmd::kModeMidpoint;
        case CMD_SSPRK53: return cmd::kModeSSPRK53;
        case CMD_RK78: return cmd::kModeRK78;
        case CMD_BULIRSCH_STOER: return cmd::kModeBulirschStoer;
        default: return cmd::kModeRK4;
    }
}

bool fixed_method(int method) { return method >= CMD_RK4 && method <= CMD_BULIRSCH_STOER && method != CMD_RK45; }
bool known_method(int method) { return method >= CMD_RK4 && method <= CMD_BULIRSCH_STOER; }

// One trajectory of the handle through the global-state integrator.
int run_global_single(cmd_handle* h, int method, double T0, double T1, double dt, int64_t n_steps, int64_t save,
                      int64_t max_rows, bool want_traj, int64_t* rows_needed) {
    GJob j;
    j.h = h;
    j.y0 = h->state.as<double>();
    j.yout = h->state.as<double>();
    if (int rc = h->grows.ensure((size_t)std::max<int64_t>(max_rows, 1) * 11 * sizeof(double))) return rc;
    j.rows = h->grows.as<double>();
    if (want_traj) {
        if (int rc = h->traj.ensure((size_t)std::max<int64_t>(max_rows, 1) * h->N * 3 * sizeof(double))) return rc;
        j.traj = h->traj.as<double>();
    }
    j.max_rows = max_rows;
    j.T0 = T0; j.T1 = T1; j.dt0 = dt;
    j.n_steps = n_steps;
    j.save_every = save;
    if (h->amp != 0.0) j.pulse = cmd::Pulse{h->t1, h->t2, h->amp, h->amp};
    std::vector<GJob> jobs{j};
    std::vector<long long> stats;
    if (int rc = run_global(h, jobs, mode_of(method), h->abs_tol, h->rel_tol, h->max_steps, stats)) return rc;
    if (rows_needed) *rows_needed = stats[0];
    if (stats[3] != 0) return fail(CMD_ERR_NONFINITE, "step-size control failed (500 consecutive rejections)");
    return CMD_OK;
}

bool resident_fits(const cmd_handle* h) { return pick_variant(h) >= 0; }
bool rk4_fits(const cmd_handle* h) { return resident_fits(h) || global_type(h->lay) >= 0; }

}  // namespace

int cmd_step(cmd_handle* h, double t, double dt, int method) {
    cmd::clear_error();
    if (int rc = check_handle(h, true)) return rc;
    if (!fixed_method(method))
        return fail(CMD_ERR_INVALID_ARG, "cmd_step takes a fixed-step method (any but CMD_RK45)");
    if (!std::isfinite(t) || !std::isfinite(dt)) return fail(CMD_ERR_INVALID_ARG, "non-finite t or dt");
    if (method == CMD_RK4 && resident_fits(h)) return run_single(h, t, dt, 1, 1, (double)h->N, false, false, true);
    return run_global_single(h, method, t, t + dt, dt, 1, 1, 0, false, nullptr);
}

int cmd_integrate(cmd_handle* h, double T0, double T1, double dt, int64_t save_interval, int method,
                  double* times, double* obs, double* states, int64_t max_rows, int64_t* rows_out) {
    cmd::clear_error();
    if (int rc = check_handle(h, true)) return rc;
    if (!known_method(method)) return fail(CMD_ERR_INVALID_ARG, "unknown integration method");
    if (save_interval <= 0 || !(dt > 0.0) || !std::isfinite(T0) || !std::isfinite(T1))
        return fail(CMD_ERR_INVALID_ARG, "bad integration window");
    if (method == CMD_RK45) {
        // rows = accepted steps + 1, known only afterwards
        if (max_rows <= 0) {
            if (rows_out) *rows_out = (h->max_steps > 0 ? h->max_steps : (int64_t)((T1 - T0) / dt) * 4 + 16) + 1;
            return fail(CMD_ERR_INVALID_ARG, "max_rows too small");
        }
        int64_t needed = 0;
        if (int rc = run_global_single(h, method, T0, T1, dt, 0, 1, max_rows, states != nullptr, &needed)) return rc;
        if (rows_out) *rows_out = needed;
        if (needed > max_rows) return fail(CMD_ERR_INVALID_ARG, "max_rows too small");
        std::vector<double> rows((size_t)needed * 11);
        CUDA_TRY(cudaMemcpy(rows.data(), h->grows.p, rows.size() * sizeof(double), cudaMemcpyDeviceToHost));
        for (int64_t r = 0; r < needed; ++r) {
            if (times) times[r] = rows[11 * r];
            if (obs) std::memcpy(obs + 10 * r, &rows[11 * r + 1], 10 * sizeof(double));
        }
        if (states)
            CUDA_TRY(cudaMemcpy(states, h->traj.p, needed * h->N * 3 * sizeof(double), cudaMemcpyDeviceToHost));
        return CMD_OK;
    }
    std::vector<double> grid;
    const int64_t n = count_steps(T0, T1, dt, 0.0, &grid);
    const int64_t rows = rows_for(n, save_interval);
    if (rows_out) *rows_out = rows;
    if (max_rows < rows) return fail(CMD_ERR_INVALID_ARG, "max_rows too small");
    if (method == CMD_RK4 && rk4_fits(h)) {
        if (int rc = run_single(h, T0, dt, n, save_interval, (double)h->N, obs != nullptr, states != nullptr, true))
            return rc;
        if (obs) CUDA_TRY(cudaMemcpy(obs, h->obs.p, rows * 10 * sizeof(double), cudaMemcpyDeviceToHost));
    } else {
        if (int rc = run_global_single(h, method, T0, T1, dt, n, save_interval, rows, states != nullptr, nullptr))
            return rc;
        if (obs) {
            std::vector<double> r11((size_t)rows * 11);
            CUDA_TRY(cudaMemcpy(r11.data(), h->grows.p, r11.size() * sizeof(double), cudaMemcpyDeviceToHost));
            for (int64_t r = 0; r < rows; ++r) std::memcpy(obs + 10 * r, &r11[11 * r + 1], 10 * sizeof(double));
        }
    }
    if (times) {
        int64_t r = 0;
        for (int64_t k = 0; k < n; k += save_interval) times[r++] = grid[k];
        times[r] = grid[n];
    }
    if (states)
        CUDA_TRY(cudaMemcpy(states, h->traj.p, rows * h->N * 3 * sizeof(double), cudaMemcpyDeviceToHost));
    return CMD_OK;
}

int cmd_run_uneven(cmd_traj_spec* specs, int64_t B, int method, double abs_tol, double rel_tol,
                   int64_t max_steps) {
    cmd::clear_error();
    if (!specs || B <= 0) return fail(CMD_ERR_INVALID_ARG, "empty batch");
    if (!known_method(method)) return fail(CMD_ERR_INVALID_ARG, "unknown integration method");
    if (method == CMD_RK45 && (!(abs_tol >= 0.0) || !(rel_tol >= 0.0) || (abs_tol == 0.0 && rel_tol == 0.0)))
        return fail(CMD_ERR_INVALID_ARG, "bad tolerances");
    cmd_handle* owner = specs[0].lattice;
    size_t in_total = 0, row_total = 0;
    std::vector<size_t> ioff(B), roff(B);
    std::vector<int64_t> nsteps(B, 0);
    for (int64_t b = 0; b < B; ++b) {
        cmd_traj_spec& sp = specs[b];
        if (!sp.lattice || !sp.state || !sp.rows || sp.max_rows <= 0 || !(sp.dt > 0.0) || !(sp.T1 >= sp.T0))
            return fail(CMD_ERR_INVALID_ARG, "bad trajectory spec");
        for (int64_t i = 0; i < sp.lattice->N * 3; ++i)
            if (!std::isfinite(sp.state[i])) return fail(CMD_ERR_NONFINITE, "non-finite initial spin");
        ioff[b] = in_total;
        in_total += (size_t)sp.lattice->N * 3;
        roff[b] = row_total;
        row_total += (size_t)sp.max_rows * 11;
        if (method != CMD_RK45) nsteps[b] = count_steps(sp.T0, sp.T1, sp.dt, 0.0, nullptr);
    }
    if (int rc = owner->batch_states.ensure(2 * in_total * sizeof(double))) return rc;
    if (int rc = owner->batch_out.ensure(row_total * sizeof(double))) return rc;
    double* din = owner->batch_states.as<double>();
    double* dout = din + in_total;
    double* drows = owner->batch_out.as<double>();
    std::vector<GJob> jobs(B);
    for (int64_t b = 0; b < B; ++b) {
        cmd_traj_spec& sp = specs[b];
        CUDA_TRY(cudaMemcpyAsync(din + ioff[b], sp.state, sp.lattice->N * 3 * sizeof(double), cudaMemcpyHostToDevice,
                                 owner->stream));
        GJob& j = jobs[b];
        j.h = sp.lattice;
        j.y0 = din + ioff[b];
        j.yout = dout + ioff[b];
        j.rows = drows + roff[b];
        j.max_rows = sp.max_rows;
        j.T0 = sp.T0; j.T1 = sp.T1; j.dt0 = sp.dt;
        j.n_steps = nsteps[b];
        j.save_every = 1;
        if (sp.a1 != 0.0 || sp.a2 != 0.0) j.pulse = cmd::Pulse{sp.t1, sp.t2, sp.a1, sp.a2};
    }
    std::vector<long long> stats;
    if (int rc = run_global(owner, jobs, mode_of(method), abs_tol, rel_tol, max_steps, stats)) return rc;
    bool overflow = false;
    for (int64_t b = 0; b < B; ++b) {
        cmd_traj_spec& sp = specs[b];
        for (int q = 0; q < 4; ++q) sp.stats[q] = stats[4 * b + q];
        const int64_t n = std::min<int64_t>(sp.stats[0], sp.max_rows);
        overflow |= sp.stats[0] > sp.max_rows;
        CUDA_TRY(cudaMemcpyAsync(sp.rows, drows + roff[b], n * 11 * sizeof(double), cudaMemcpyDeviceToHost, owner->stream));
        if (sp.final_state)
            CUDA_TRY(cudaMemcpyAsync(sp.final_state, dout + ioff[b], sp.lattice->N * 3 * sizeof(double),
                                     cudaMemcpyDeviceToHost, owner->stream));
    }
    if (int rc = sync(owner)) return rc;
    if (overflow) return fail(CMD_ERR_INVALID_ARG, "max_rows too small for some trajectory");
    for (int64_t b = 0; b < B; ++b)
        if (specs[b].stats[3] != 0) return fail(CMD_ERR_NONFINITE, "step-size control failed for some trajectory");
    return CMD_OK;
}

int cmd_observables(cmd_handle* h, double* row) {
    cmd::clear_error();
    if (int rc = check_handle(h, true)) return rc;
    if (!row) return fail(CMD_ERR_INVALID_ARG, "NULL row");
    if (int rc = run_single(h, 0.0, 0.0, 0, 1, (double)h->N, true, false, false)) return rc;
    CUDA_TRY(cudaMemcpy(row, h->obs.p, 10 * sizeof(double), cudaMemcpyDeviceToHost));
    return CMD_OK;
}

int cmd_energy(cmd_handle* h, double* energy) {
    cmd::clear_error();
    if (int rc = check_handle(h, true)) return rc;
    if (!energy) return fail(CMD_ERR_INVALID_ARG, "NULL energy");
    if (int rc = run_single(h, 0.0, 0.0, 0, 1, 1.0, true, false, false)) return rc;
    double row[10];
    CUDA_TRY(cudaMemcpy(row, h->obs.p, sizeof(row), cudaMemcpyDeviceToHost));
    *energy = row[9];
    return CMD_OK;
}

}  // extern "C"

namespace {

// max_c |(H_i x S_i)_c| over all sites with the drive off (Lattice::
// max_dSdt_norm_no_drive, lattice_md.cpp:235-279): one thread per site (cell g,
// atom at) of the AoS state; partners from the resident table's SoA offsets.
// Non-negative doubles order like their bit patterns, so an integer atomicMax
// gives the exact maximum in any order.
template <int NAT, int Z, int LZ>
__global__ void dsdt_max_kernel(const __grid_constant__ cmd::Couplings<NAT, Z> cp, const double* __restrict__ y,
                                const int* __restrict__ nbr, int64_t G, unsigned long long* out) {
    constexpr int NL = Z - LZ;
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double m = 0.0;
    if (e < G * NAT) {
        const int64_t g = e / NAT;
        const int at = (int)(e - g * NAT);
        auto spin = [&](int64_t gg, int aa, double (&P)[3]) {
            const double* q = y + (gg * NAT + aa) * 3;
            P[0] = q[0];
            P[1] = q[1];
            P[2] = q[2];
        };
        double S[3], H[3];
        spin(g, at, S);
        for (int d = 0; d < 3; ++d) H[d] = cp.has_field ? -cp.field[at][d] : 0.0;
        if (cp.has_onsite)
            for (int d = 0; d < 3; ++d)
                cmd::bond_acc(H[d], 2.0 * cp.onsite[at][3 * d], 2.0 * cp.onsite[at][3 * d + 1],
                              2.0 * cp.onsite[at][3 * d + 2], S[0], S[1], S[2]);
        for (int n = 0; n < LZ; ++n) {
            double P[3];
            spin(g, (at + 1 + n) % NAT, P);
            for (int d = 0; d < 3; ++d)
                cmd::bond_acc(H[d], cp.J[at][n][3 * d], cp.J[at][n][3 * d + 1], cp.J[at][n][3 * d + 2], P[0], P[1],
                              P[2]);
        }
        for (int mm = 0; mm < NL; ++mm) {
            const int n = LZ + mm;
            if (n >= cp.zc[at]) continue;
            const int64_t off = nbr[(g * NAT + at) * NL + mm];
            const int64_t ap = off / (3 * G), gp = off - ap * 3 * G;
            double P[3];
            spin(gp, (int)ap, P);
            for (int d = 0; d < 3; ++d)
                cmd::bond_acc(H[d], cp.J[at][n][3 * d], cp.J[at][n][3 * d + 1], cp.J[at][n][3 * d + 2], P[0], P[1],
                              P[2]);
        }
        const double k0 = H[1] * S[2] - H[2] * S[1], k1 = H[2] * S[0] - H[0] * S[2], k2 = H[0] * S[1] - H[1] * S[0];
        m = fmax(fabs(k0), fmax(fabs(k1), fabs(k2)));
    }
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m > 0.0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

template <int NAT, int Z, int LZ>
int launch_dsdt_max(cmd_handle* h, unsigned long long* out) {
    static const std::vector<double> zeros(3 * 64, 0.0);
    cmd::Couplings<NAT, Z> cp;
    fill_couplings<NAT, Z>(h, zeros.data(), zeros.data(), cp);
    const int64_t n = h->lay.G * NAT;
    dsdt_max_kernel<NAT, Z, LZ><<<(unsigned)((n + 255) / 256), 256, 0, h->stream>>>(
        cp, h->state.as<double>(), h->nbr.as<int>(), h->lay.G, out);
    CUDA_TRY(cudaGetLastError());
    return CMD_OK;
}

}  // namespace

extern "C" {

int cmd_max_dsdt_no_drive(cmd_handle* h, double* out) {
    cmd::clear_error();
    if (int rc = check_handle(h, true)) return rc;
    if (!out) return fail(CMD_ERR_INVALID_ARG, "NULL output");
    if (h->NA > 64) return fail(CMD_ERR_UNSUPPORTED, "cells limited to 64 atoms");
    if (int rc = h->scratch.ensure(sizeof(unsigned long long))) return rc;
    auto* d = static_cast<unsigned long long*>(h->scratch.p);
    CUDA_TRY(cudaMemsetAsync(d, 0, sizeof(unsigned long long), h->stream));
    int rc = CMD_OK;
    switch (global_type(h->lay)) {
        case 0: rc = launch_dsdt_max<2, 3, 1>(h, d); break;
        case 1: rc = launch_dsdt_max<4, 6, 3>(h, d); break;
        default: return no_instance(h->lay);
    }
    if (rc != CMD_OK) return rc;
    if (int rc2 = sync(h)) return rc2;
    unsigned long long bits = 0;
    CUDA_TRY(cudaMemcpy(&bits, d, sizeof(bits), cudaMemcpyDeviceToHost));
    std::memcpy(out, &bits, sizeof(double));
    return CMD_OK;
}

int cmd_normalize(cmd_handle* h, double spin_length) {
    cmd::clear_error();
    if (int rc = check_handle(h, true)) return rc;
    if (!std::isfinite(spin_length)) return fail(CMD_ERR_INVALID_ARG, "bad spin length");
    const int64_t N = h->N;
    normalize_kernel<<<(unsigned)((N + 255) / 256), 256, 0, h->stream>>>(h->state.as<double>(), spin_length, N);
    CUDA_TRY(cudaGetLastError());
    return sync(h);
}

int cmd_magnetization(cmd_handle* h, double* ml, double* ms) {
    cmd::clear_error();
    if (int rc = check_handle(h, true)) return rc;
    if (!ml || !ms) return fail(CMD_ERR_INVALID_ARG, "NULL output");
    if (int rc = h->scratch.ensure(6 * sizeof(double))) return rc;
    magnetization_kernel<<<1, 256, 0, h->stream>>>(h->state.as<double>(), h->N, h->scratch.as<double>());
    CUDA_TRY(cudaGetLastError());
    if (int rc = sync(h)) return rc;
    double v[6];
    CUDA_TRY(cudaMemcpy(v, h->scratch.p, sizeof(v), cudaMemcpyDeviceToHost));
    std::memcpy(ml, v, 3 * sizeof(double));
    std::memcpy(ms, v + 3, 3 * sizeof(double));
    return CMD_OK;
}

int64_t cmd_batch_rows(int64_t n_steps, int64_t save_interval) {
    if (n_steps < 0 || save_interval <= 0) return -1;
    return rows_for(n_steps, save_interval);
}

namespace {

int validate_batch(const cmd_handle* h, const cmd_batch_desc* d) {
    if (!d) return fail(CMD_ERR_INVALID_ARG, "NULL batch description");
    if (d->B <= 0 || d->B > (1 << 24)) return fail(CMD_ERR_INVALID_ARG, "bad batch size");
    if (d->method != CMD_RK4) return fail(CMD_ERR_UNSUPPORTED, "batched path implements CMD_RK4 only");
    if (!d->states || !d->obs) return fail(CMD_ERR_INVALID_ARG, "NULL states or obs");
    if (d->n_steps < 0 || d->save_interval <= 0 || !(d->dt > 0.0) || !std::isfinite(d->T0))
        return fail(CMD_ERR_INVALID_ARG, "bad time grid");
    const bool drive = d->d1 || d->d2;
    if (drive && !d->pulse4 && (!d->t1 || !d->t2 || !d->a1 || !d->a2))
        return fail(CMD_ERR_INVALID_ARG, "pulse arrays required when a drive direction is given");
    if (drive && !(d->width != 0.0)) return fail(CMD_ERR_INVALID_ARG, "pulse width must be non-zero");
    (void)h;
    return CMD_OK;
}

int run_batch_device(cmd_handle* h, const cmd_batch_desc* d, const cmd::Pulse* d_pulses,
                     cudaStream_t st, int32_t* launches) {
    RunSpec r;
    r.B = d->B;
    r.y0 = d->states;
    r.y0_stride = d->shared_initial ? 0 : h->N * 3;
    r.y_out = d->final_states;
    r.obs = d->obs;
    r.T0 = d->T0;
    r.dt = d->dt;
    r.n_steps = d->n_steps;
    r.save = d->save_interval;
    r.pulses = d_pulses;
    r.width = d->width;
    r.freq = d->freq;
    std::vector<double> d1c, d2c;
    if (d->d1)
        if (int rc = reduce_per_class(h, d->d1, 3, d1c, "pulse directions")) return rc;
    if (d->d2)
        if (int rc = reduce_per_class(h, d->d2, 3, d2c, "pulse directions")) return rc;
    r.d1 = d->d1 ? d1c.data() : nullptr;
    r.d2 = d->d2 ? d2c.data() : nullptr;
    r.n_sites = (double)h->N;
    return run_rk4(h, r, st, launches);
}

// Long host-buffer batches run in time chunks so that the observable rows of
// chunk c travel to the host (second stream) while chunk c+1 computes.  Chunk
// c starts from chunk c-1's final states at the exact accumulated time of the
// single-run loop (t += dt from T0), so every step and every row is what one
// launch would produce; chunk lengths are multiples of save_interval, and a
// chunk's last row (the next chunk's first) is copied once.
constexpr int64_t kChunkMinSteps = 4096;
constexpr int64_t kChunks = 8;

int run_batch_chunked(cmd_handle* h, const cmd_batch_desc* d, const double* d_init, const cmd::Pulse* d_pulses) {
    const int64_t B = d->B, N3 = h->N * 3, S = d->n_steps, sv = d->save_interval;
    const int64_t rows_total = rows_for(S, sv);
    int64_t chunk = (S + kChunks - 1) / kChunks;
    chunk = (chunk + sv - 1) / sv * sv;
    const int64_t rows_chunk = rows_for(chunk, sv);
    if (!h->copy_stream) CUDA_TRY(cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking));
    if (int rc = h->chunk_states.ensure((size_t)2 * B * N3 * sizeof(double))) return rc;
    if (int rc = h->chunk_rows.ensure((size_t)2 * B * rows_chunk * 10 * sizeof(double))) return rc;
    double* st[2] = {h->chunk_states.as<double>(), h->chunk_states.as<double>() + B * N3};
    double* rb[2] = {h->chunk_rows.as<double>(), h->chunk_rows.as<double>() + B * rows_chunk * 10};
    cudaEvent_t done[2] = {nullptr, nullptr}, copied[2] = {nullptr, nullptr};
    int rc = CMD_OK;
    auto cuda_ok = [&](cudaError_t e, const char* what) {
        if (e == cudaSuccess) return true;
        rc = fail(CMD_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
        return false;
    };
    for (int i = 0; i < 2 && rc == CMD_OK; ++i) {
        cuda_ok(cudaEventCreateWithFlags(&done[i], cudaEventDisableTiming), "cudaEventCreate");
        if (rc == CMD_OK) cuda_ok(cudaEventCreateWithFlags(&copied[i], cudaEventDisableTiming), "cudaEventCreate");
    }
    double t = d->T0;
    int64_t k0 = 0, c = 0, last = 0;
    while (rc == CMD_OK && k0 < S) {
        const int64_t n = std::min(chunk, S - k0);
        const int slot = (int)(c & 1);
        const bool final_chunk = k0 + n == S;
        const int64_t rows_c = rows_for(n, sv);
        if (c >= 2 && !cuda_ok(cudaStreamWaitEvent(h->stream, copied[slot], 0), "cudaStreamWaitEvent")) break;
        cmd_batch_desc dd = *d;
        dd.states = c == 0 ? d_init : st[1 - slot];
        dd.shared_initial = c == 0 ? d->shared_initial : 0;
        dd.final_states = st[slot];
        dd.obs = rb[slot];
        dd.T0 = t;
        dd.n_steps = n;
        if ((rc = run_batch_device(h, &dd, d_pulses, h->stream, nullptr)) != CMD_OK) break;
        if (!cuda_ok(cudaEventRecord(done[slot], h->stream), "cudaEventRecord")) break;
        if (!cuda_ok(cudaStreamWaitEvent(h->copy_stream, done[slot], 0), "cudaStreamWaitEvent")) break;
        const int64_t ncopy = final_chunk ? rows_c : rows_c - 1;
        if (!cuda_ok(cudaMemcpy2DAsync(d->obs + (k0 / sv) * 10, (size_t)rows_total * 10 * sizeof(double), rb[slot],
                                       (size_t)rows_c * 10 * sizeof(double), (size_t)ncopy * 10 * sizeof(double),
                                       (size_t)B, cudaMemcpyDeviceToHost, h->copy_stream),
                     "cudaMemcpy2DAsync"))
            break;
        if (!cuda_ok(cudaEventRecord(copied[slot], h->copy_stream), "cudaEventRecord")) break;
        for (int64_t k = 0; k < n; ++k) t += d->dt;     // the single-run loop's accumulated time
        last = slot;
        k0 += n;
        ++c;
    }
    if (rc == CMD_OK && d->final_states)
        cuda_ok(cudaMemcpyAsync(d->final_states, st[last], B * N3 * sizeof(double), cudaMemcpyDeviceToHost,
                                h->stream),
                "cudaMemcpyAsync");
    const cudaError_t e1 = cudaStreamSynchronize(h->copy_stream);
    const cudaError_t e2 = cudaStreamSynchronize(h->stream);
    for (int i = 0; i < 2; ++i) {
        if (done[i]) cudaEventDestroy(done[i]);
        if (copied[i]) cudaEventDestroy(copied[i]);
    }
    if (rc != CMD_OK) return rc;
    if (e1 != cudaSuccess) return fail(CMD_ERR_CUDA, std::string("copy stream: ") + cudaGetErrorString(e1));
    if (e2 != cudaSuccess) return fail(CMD_ERR_CUDA, std::string("stream: ") + cudaGetErrorString(e2));
    return CMD_OK;
}

}  // namespace

int cmd_run_batch(cmd_handle* h, const cmd_batch_desc* d) {
    cmd::clear_error();
    if (int rc = check_handle(h, false)) return rc;
    if (int rc = validate_batch(h, d)) return rc;
    if (d->d1 || d->d2)
        if (h->NA > 64) return fail(CMD_ERR_UNSUPPORTED, "drive directions limited to 64 atoms");
    const int64_t B = d->B, N3 = h->N * 3;
    const int64_t n_init = d->shared_initial ? 1 : B;
    const int64_t rows = rows_for(d->n_steps, d->save_interval);
    for (int64_t i = 0; i < n_init * N3; ++i)
        if (!std::isfinite(d->states[i])) return fail(CMD_ERR_NONFINITE, "non-finite initial spin");
    const bool chunked = d->n_steps >= kChunkMinSteps;
    if (int rc = h->batch_states.ensure((size_t)(n_init + (d->final_states && !chunked ? B : 0)) * N3 *
                                        sizeof(double)))
        return rc;
    if (!chunked)
        if (int rc = h->batch_out.ensure((size_t)B * rows * 10 * sizeof(double))) return rc;
    double* d_init = h->batch_states.as<double>();
    double* d_final = d->final_states && !chunked ? d_init + n_init * N3 : nullptr;
    CUDA_TRY(cudaMemcpyAsync(d_init, d->states, n_init * N3 * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    const bool drive = d->d1 || d->d2;
    cmd::Pulse* d_pulses = nullptr;
    std::vector<cmd::Pulse> hp;
    if (drive) {
        hp.resize(B);
        for (int64_t b = 0; b < B; ++b) hp[b] = cmd::Pulse{d->t1[b], d->t2[b], d->a1[b], d->a2[b]};
        if (int rc = h->pulses.ensure(B * sizeof(cmd::Pulse))) return rc;
        d_pulses = h->pulses.as<cmd::Pulse>();
        CUDA_TRY(cudaMemcpyAsync(d_pulses, hp.data(), B * sizeof(cmd::Pulse), cudaMemcpyHostToDevice, h->stream));
    }
    if (chunked) return run_batch_chunked(h, d, d_init, d_pulses);
    cmd_batch_desc dd = *d;
    dd.states = d_init;
    dd.obs = h->batch_out.as<double>();
    dd.final_states = d_final;
    if (int rc = run_batch_device(h, &dd, d_pulses, h->stream, nullptr)) return rc;
    CUDA_TRY(cudaMemcpyAsync(d->obs, dd.obs, B * rows * 10 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    if (d->final_states)
        CUDA_TRY(cudaMemcpyAsync(d->final_states, d_final, B * N3 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    return sync(h);
}

int cmd_run_batch_device(cmd_handle* h, const cmd_batch_desc* d, void* stream, int32_t* launches) {
    cmd::clear_error();
    if (launches) *launches = 0;
    if (int rc = check_handle(h, false)) return rc;
    if (int rc = validate_batch(h, d)) return rc;
    cudaStream_t st = stream ? (cudaStream_t)stream : h->stream;
    if ((d->d1 || d->d2) && !d->pulse4)
        return fail(CMD_ERR_INVALID_ARG, "driven device batch needs pulse4");
    if ((d->d1 || d->d2) && h->NA > 64) return fail(CMD_ERR_UNSUPPORTED, "drive directions limited to 64 atoms");
    const cmd::Pulse* d_pulses = (d->d1 || d->d2) ? reinterpret_cast<const cmd::Pulse*>(d->pulse4) : nullptr;
    return run_batch_device(h, d, d_pulses, st, launches);
}


}  // extern "C"

namespace {

constexpr int kAdjParams = 5;

// Derivative tables [q][atom][slot][9], [q][atom][3], [q][atom][9] into the kernel parameter block.
template <int NAT, int Z, int NQ>
void fill_param_derivs(const std::vector<double>& DJ, const std::vector<double>& DB, const std::vector<double>& DA,
                       bool has_DA, cmd::ParamDerivs<NAT, Z, NQ>& pd) {
    std::memset(&pd, 0, sizeof(pd));
    for (int q = 0; q < NQ; ++q)
        for (int at = 0; at < NAT; ++at) {
            for (int s = 0; s < Z; ++s)
                std::memcpy(pd.DJ[q][at][s], &DJ[(((size_t)q * NAT + at) * Z + s) * 9], 9 * sizeof(double));
            std::memcpy(pd.DB[q][at], &DB[((size_t)q * NAT + at) * 3], 3 * sizeof(double));
            std::memcpy(pd.DA[q][at], &DA[((size_t)q * NAT + at) * 9], 9 * sizeof(double));
        }
    pd.has_DA = has_DA;
    for (int q = 0; q < NQ; ++q) {
        pd.dj_any[q] = 0;
        for (int at = 0; at < NAT; ++at)
            for (int s = 0; s < Z; ++s)
                for (int e = 0; e < 9; ++e) pd.dj_any[q] |= pd.DJ[q][at][s][e] != 0.0;
    }
}

template <int NAT, int Z, int LZ>
int launch_adjoint(cmd_handle* h, const cmd::AdjArgs& a, const std::vector<double>& DJ, const std::vector<double>& DB,
                   const std::vector<double>& DA, bool has_DA, int64_t B) {
    cmd::Couplings<NAT, Z> cp;
    fill_couplings<NAT, Z>(h, h->fd.data(), h->fd.data() + 3 * h->NA, cp);
    cmd::adjoint_forward_kernel<NAT, Z, LZ><<<(unsigned)B, cmd::kAdjThreads, 0, h->stream>>>(cp, a);
    CUDA_TRY(cudaGetLastError());
    if (a.forward_only) return CMD_OK;
    cmd::ParamDerivs<NAT, Z, kAdjParams> pd;
    fill_param_derivs<NAT, Z, kAdjParams>(DJ, DB, DA, has_DA, pd);
    cmd::adjoint_backward_kernel<NAT, Z, LZ, kAdjParams><<<(unsigned)B, cmd::kAdjThreads, 0, h->stream>>>(cp, pd, a);
    CUDA_TRY(cudaGetLastError());
    return CMD_OK;
}

// Resident adjoint (rk_adjoint_cluster.cuh): one CTA or one cluster of CS CTAs per
// trajectory, one thread per unit cell.
using AdjClusterFn = int (*)(cmd_handle*, cmd::AdjClusterArgs, const std::vector<double>&, const std::vector<double>&,
                             const std::vector<double>&, bool, int64_t);

// Partner words of the cluster layout with CS CTAs (CS = 1: the global offsets, rank 0).
const int* cluster_table(const cmd_handle* h, int cs) {
    return cs == 1 ? h->nbr.as<int>() : static_cast<const int*>((cs == 2 ? h->cnbr2 : h->cnbr4).p);
}

template <int NAT, int Z, int LZ, int CS, int MAXT>
int launch_adjoint_cluster(cmd_handle* h, cmd::AdjClusterArgs a, const std::vector<double>& DJ,
                           const std::vector<double>& DB, const std::vector<double>& DA, bool has_DA, int64_t B) {
    auto kern = cmd::adjoint_cluster_kernel<NAT, Z, LZ, CS, MAXT, kAdjParams>;
    const int64_t G = h->lay.G, Gc = cluster_cells(G, CS);
    const int threads = (int)((Gc + 31) / 32 * 32);
    const size_t smem = (size_t)cmd::adj_cluster_smem_doubles(NAT, Gc) * sizeof(double);
    if (threads > MAXT || smem > kMaxSmem) return fail(CMD_ERR_UNSUPPORTED, "lattice too large for this adjoint variant");
    a.nbr = cluster_table(h, CS);
    if (!a.nbr && !h->lay.nbr.empty()) return fail(CMD_ERR_UNSUPPORTED, "no cluster neighbour table for this lattice");
    // Function attributes belong to the current device's context: set on every
    // launch (a host-side call of about a microsecond), so handles on several
    // devices, several host threads and a re-created context all see it.
    CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMaxSmem));
    cmd::Couplings<NAT, Z> cp;
    fill_couplings<NAT, Z>(h, h->fd.data(), h->fd.data() + 3 * h->NA, cp);
    cmd::ParamDerivs<NAT, Z, kAdjParams> pd;
    fill_param_derivs<NAT, Z, kAdjParams>(DJ, DB, DA, has_DA, pd);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(B * CS));
    cfg.blockDim = dim3((unsigned)threads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = h->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = CS;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    CUDA_TRY(cudaLaunchKernelEx(&cfg, kern, cp, pd, a, (int)Gc));
    return CMD_OK;
}

struct AdjClusterVariant {
    int NAT, Z, LZ, CS, MAXT;
    AdjClusterFn fn;
};

const AdjClusterVariant kAdjClusterVariants[] = {
    {2, 3, 1, 1, 576, &launch_adjoint_cluster<2, 3, 1, 1, 576>},
    {2, 3, 1, 2, 576, &launch_adjoint_cluster<2, 3, 1, 2, 576>},
    {2, 3, 1, 4, 576, &launch_adjoint_cluster<2, 3, 1, 4, 576>},
    {4, 6, 3, 1, 256, &launch_adjoint_cluster<4, 6, 3, 1, 256>},
    {4, 6, 3, 2, 256, &launch_adjoint_cluster<4, 6, 3, 2, 256>},
    {4, 6, 3, 4, 256, &launch_adjoint_cluster<4, 6, 3, 4, 256>},
};

// The resident adjoint variant for h's lattice: the smallest cluster whose CTAs hold
// the cells; -1 if none does.
int pick_adjoint_cluster(const cmd_handle* h) {
    const Layout& L = h->lay;
    const int ty = global_type(L);
    if (ty < 0) return -1;
    for (int i = 0; i < (int)(sizeof(kAdjClusterVariants) / sizeof(kAdjClusterVariants[0])); ++i) {
        const AdjClusterVariant& v = kAdjClusterVariants[i];
        if ((ty == 0) != (v.NAT == 2)) continue;
        const int64_t Gc = cluster_cells(L.G, v.CS);
        if ((Gc + 31) / 32 * 32 > v.MAXT) continue;
        if ((size_t)cmd::adj_cluster_smem_doubles(v.NAT, Gc) * sizeof(double) > kMaxSmem) continue;
        if ((int64_t)v.NAT * 3 * Gc >= (1 << cmd::kClusterRankShift)) continue;
        if (v.CS > 1 && !cluster_table(h, v.CS)) continue;
        return i;
    }
    return -1;
}


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

template <int NAT, int Z, int LZ, int NQ>
int stream_adjoint(cmd_handle* h, const StreamAdjJob& j, const std::vector<double>& DJ, const std::vector<double>& DB,
                   const std::vector<double>& DA, bool has_DA) {
    cudaStream_t st = h->stream;
    const int G = (int)h->lay.G;
    const int tiles = (G + cmd::stream_cells<NAT>() - 1) / cmd::stream_cells<NAT>();
    const int64_t V = (int64_t)NAT * 3 * G, B = j.B, S = j.S, C = j.C, K = j.K;
    if (int rc = h->sbuf.ensure((size_t)5 * B * V * sizeof(double))) return rc;
    if (int rc = h->spart.ensure(((size_t)B * tiles * cmd::kPart + B) * sizeof(double))) return rc;
    const int vtiles = (G + cmd::kStreamTile - 1) / cmd::kStreamTile;     // VJP: one cell per thread
    if (int rc = h->sgpart.ensure((size_t)B * vtiles * cmd::kPart * sizeof(double))) return rc;
    double* base = h->sbuf.as<double>();
    double* d_loss = h->spart.as<double>() + (size_t)B * tiles * cmd::kPart;
    const bool driven = h->amp != 0.0;
    if (driven) {
        std::vector<cmd::Pulse> pl((size_t)B, cmd::Pulse{h->t1, h->t2, h->amp, h->amp});
        if (int rc = h->pulses.ensure((size_t)B * sizeof(cmd::Pulse))) return rc;
        if (int rc = h->drive.ensure((size_t)B * S * 6 * sizeof(double))) return rc;
        CUDA_TRY(cudaMemcpyAsync(h->pulses.p, pl.data(), pl.size() * sizeof(cmd::Pulse), cudaMemcpyHostToDevice, st));
        const int64_t total = B * S * 6;
        const int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 32);
        cmd::drive_table_kernel<<<blocks, 256, 0, st>>>(h->pulses.as<cmd::Pulse>(), j.times, S, j.dt, h->width,
                                                       h->freq, B, h->drive.as<double>());
        CUDA_TRY(cudaGetLastError());
    }
    cmd::Couplings<NAT, Z> cp;
    fill_couplings<NAT, Z>(h, h->fd.data(), h->fd.data() + 3 * h->NA, cp);
    cmd::StreamArgs a{};
    a.G = G;
    a.tiles = tiles;
    a.B = (int)B;
    a.nbr = h->nbr.as<int>();
    a.dt = j.dt;
    a.n_steps = S;
    a.times = j.times;
    a.drive = driven ? h->drive.as<double>() : nullptr;
    a.part = h->spart.as<double>();
    a.save_every = 1;
    a.rows = S + 1;
    a.target = j.target;
    a.mloc = j.mloc;
    a.loss = d_loss;
    a.n_sites = (double)h->N;
    a.ckpt = j.fwd_only ? nullptr : h->ackpt.as<double>();
    a.ckpt_every = C;
    a.n_ckpt = K;
    a.V = V;
    const dim3 grid(tiles, (unsigned)B), gridc((G + 255) / 256, (unsigned)B);
    const cmd::SVec none{nullptr, 0};
    // forward: loss terms every step, checkpoints every C steps
    {
        const cmd::SVec y{base, V}, acc{base + B * V, V}, Ya{base + 2 * B * V, V}, Yb{base + 3 * B * V, V};
        cmd::stream_load_kernel<NAT><<<gridc, 256, 0, st>>>(j.y0, (long long)G * NAT * 3, G, y);
        for (int64_t n = 0; n < S; ++n) {
            cmd::stream_stage_kernel<NAT, Z, LZ><<<grid, cmd::kStreamTile, 0, st>>>(cp, a, 0, n, y, y, acc, Ya, 1);
            cmd::stream_stage_kernel<NAT, Z, LZ><<<grid, cmd::kStreamTile, 0, st>>>(cp, a, 1, n, Ya, y, acc, Yb, 1);
            cmd::stream_stage_kernel<NAT, Z, LZ><<<grid, cmd::kStreamTile, 0, st>>>(cp, a, 2, n, Yb, y, acc, Ya, 1);
            cmd::stream_stage_kernel<NAT, Z, LZ><<<grid, cmd::kStreamTile, 0, st>>>(cp, a, 3, n, Ya, y, acc, y, 1);
            if ((n & 1023) == 0) CUDA_TRY(cudaGetLastError());
        }
        cmd::stream_obs_kernel<NAT, Z, LZ><<<grid, cmd::kStreamTile, 0, st>>>(cp, a, y);
        cmd::stream_reduce_kernel<NAT><<<(unsigned)B, cmd::kStreamTile, 0, st>>>(a, S);
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaMemcpy2DAsync(j.out, (1 + kAdjParams) * sizeof(double), d_loss, sizeof(double), sizeof(double),
                                   (size_t)B, cudaMemcpyDeviceToDevice, st));
    }
    if (j.fwd_only) return CMD_OK;
    cmd::ParamDerivs<NAT, Z, NQ> pd;
    std::memset(&pd, 0, sizeof(pd));
    for (int q = 0; q < NQ; ++q)
        for (int at = 0; at < NAT; ++at) {
            for (int sl = 0; sl < Z; ++sl)
                std::memcpy(pd.DJ[q][at][sl], &DJ[(((size_t)q * NAT + at) * Z + sl) * 9], 9 * sizeof(double));
            std::memcpy(pd.DB[q][at], &DB[((size_t)q * NAT + at) * 3], 3 * sizeof(double));
            std::memcpy(pd.DA[q][at], &DA[((size_t)q * NAT + at) * 9], 9 * sizeof(double));
        }
    pd.has_DA = has_DA;
    cmd::StreamVjpArgs v{};
    v.G = G;
    v.tiles = vtiles;
    v.nbr = a.nbr;
    v.dt = j.dt;
    v.n_steps = S;
    v.drive = a.drive;
    v.target = j.target;
    v.mloc = j.mloc;
    v.n_sites = a.n_sites;
    v.gpart = h->sgpart.as<double>();
    cmd::StreamArgs ar = a;              // recompute: no observables, no checkpoints
    ar.ckpt = nullptr;
    CUDA_TRY(cudaMemsetAsync(v.gpart, 0, (size_t)B * vtiles * cmd::kPart * sizeof(double), st));
    const dim3 vgrid(vtiles, (unsigned)B);
    cmd::SVec lam{base, V}, lam2{base + B * V, V};
    const cmd::SVec acc{base + 2 * B * V, V}, Sa{base + 3 * B * V, V}, Sb{base + 4 * B * V, V};
    cmd::stream_lam_init_kernel<NAT><<<gridc, 256, 0, st>>>(v, lam);
    double* seg = h->aseg.as<double>();
    auto slot = [&](int64_t jj, int q) { return cmd::SVec{seg + (jj * 4 + q) * V, C * 4 * V}; };
    const double dt = j.dt;
    for (int64_t sg = K - 1; sg >= 0; --sg) {
        const int64_t n0 = sg * C, n1 = std::min(n0 + C, S);
        CUDA_TRY(cudaMemcpy2DAsync(seg, (size_t)C * 4 * V * sizeof(double), h->ackpt.as<double>() + sg * V,
                                   (size_t)K * V * sizeof(double), (size_t)V * sizeof(double), (size_t)B,
                                   cudaMemcpyDeviceToDevice, st));
        for (int64_t n = n0; n < n1; ++n) {
            const int64_t jj = n - n0;
            const cmd::SVec y = slot(jj, 0);
            const cmd::SVec last = n + 1 < n1 ? slot(jj + 1, 0) : none;
            cmd::stream_stage_kernel<NAT, Z, LZ><<<grid, cmd::kStreamTile, 0, st>>>(cp, ar, 0, n, y, y, acc,
                                                                                   slot(jj, 1), 0);
            cmd::stream_stage_kernel<NAT, Z, LZ><<<grid, cmd::kStreamTile, 0, st>>>(cp, ar, 1, n, slot(jj, 1), y, acc,
                                                                                   slot(jj, 2), 0);
            cmd::stream_stage_kernel<NAT, Z, LZ><<<grid, cmd::kStreamTile, 0, st>>>(cp, ar, 2, n, slot(jj, 2), y, acc,
                                                                                   slot(jj, 3), 0);
            cmd::stream_stage_kernel<NAT, Z, LZ><<<grid, cmd::kStreamTile, 0, st>>>(cp, ar, 3, n, slot(jj, 3), y, acc,
                                                                                   last, 0);
        }
        for (int64_t n = n1 - 1; n >= n0; --n) {
            const int64_t jj = n - n0;
            auto vjp = cmd::stream_vjp_kernel<NAT, Z, LZ, NQ>;
            vjp<<<vgrid, cmd::kStreamTile, 0, st>>>(cp, pd, v, 3, n, slot(jj, 3), lam, none, dt / 6.0, 0.0, Sa, acc,
                                                   none, 0);
            vjp<<<vgrid, cmd::kStreamTile, 0, st>>>(cp, pd, v, 2, n, slot(jj, 2), lam, Sa, dt / 3.0, dt, Sb, acc,
                                                   none, 1);
            vjp<<<vgrid, cmd::kStreamTile, 0, st>>>(cp, pd, v, 1, n, slot(jj, 1), lam, Sb, dt / 3.0, 0.5 * dt, Sa, acc,
                                                   none, 1);
            vjp<<<vgrid, cmd::kStreamTile, 0, st>>>(cp, pd, v, 0, n, slot(jj, 0), lam, Sa, dt / 6.0, 0.5 * dt, none,
                                                   acc, lam2, 2);
            std::swap(lam, lam2);
        }
        CUDA_TRY(cudaGetLastError());
    }
    cmd::stream_grad_kernel<<<(unsigned)B, 32, 0, st>>>(v.gpart, vtiles, NQ, j.out + 1, 1 + kAdjParams);
    CUDA_TRY(cudaGetLastError());
    return CMD_OK;
}

// Threads per CTA and shared memory per CTA of variant V on layout L.
void variant_shape(const Variant& V, const Layout& L, int64_t* threads, int64_t* smem) {
    if (V.CS > 1) {
        *threads = (cluster_cells(L.G, V.CS) + 31) / 32 * 32;
        *smem = (int64_t)cluster_smem(L.NA, L.G, V.CS);
    } else {
        *threads = ((L.G + V.CPT - 1) / V.CPT + 31) / 32 * 32;
        *smem = (int64_t)resident_smem(L.NA, L.G, V.TPC);
    }
}

}  // namespace

extern "C" {

int cmd_adjoint_rk4(cmd_handle* h, const cmd_adjoint_desc* d) {
    cmd::clear_error();
    if (int rc = check_handle(h, false)) return rc;
    if (!d || d->B <= 0 || !d->states || !d->target || !d->loss || d->n_steps <= 0 || !(d->dt > 0.0))
        return fail(CMD_ERR_INVALID_ARG, "bad adjoint description");
    if (d->n_params < 0 || d->n_params > kAdjParams || (d->n_params > 0 && (!d->dparams || !d->grad)))
        return fail(CMD_ERR_INVALID_ARG, "n_params must be 0..5 with derivative lattices and a grad buffer");
    if (d->path < CMD_ADJ_AUTO || d->path > CMD_ADJ_GLOBAL) return fail(CMD_ERR_INVALID_ARG, "unknown adjoint path");
    const int ty = global_type(h->lay);
    if (ty < 0) return no_instance(h->lay);
    const int NA = h->NA, Z = h->lay.Z;
    // derivative tables per (parameter, atom class, slot) from the theta = e_q lattices
    std::vector<double> DJ((size_t)kAdjParams * NA * Z * 9, 0.0), DB((size_t)kAdjParams * NA * 3, 0.0),
        DA((size_t)kAdjParams * NA * 9, 0.0);
    bool has_DA = false;
    for (int q = 0; q < d->n_params; ++q) {
        const cmd_lattice_desc& p = d->dparams[q];
        if (p.lattice_size != h->N || !p.counts || !p.partners || !p.bilinear || !p.field || !p.onsite)
            return fail(CMD_ERR_INVALID_ARG, "derivative lattice does not match the handle's lattice");
        for (int a = 0; a < NA; ++a) {
            for (int s = 0; s < h->lay.zc[a]; ++s) {
                const int e = h->lay.slot_entry[(size_t)a * Z + s];
                if (e < 0 || e >= p.counts[a]) return fail(CMD_ERR_INVALID_ARG, "derivative lattice bond tables differ");
                std::memcpy(&DJ[(((size_t)q * NA + a) * Z + s) * 9], &p.bilinear[((int64_t)a * p.max_bilinear + e) * 9],
                            9 * sizeof(double));
            }
            std::memcpy(&DB[((size_t)q * NA + a) * 3], &p.field[3 * a], 3 * sizeof(double));
            std::memcpy(&DA[((size_t)q * NA + a) * 9], &p.onsite[9 * a], 9 * sizeof(double));
            for (int k = 0; k < 9; ++k) has_DA |= p.onsite[9 * a + k] != 0.0;
        }
    }
    const int64_t B = d->B, S = d->n_steps, N3 = h->N * 3, V = N3;
    int64_t C = d->checkpoint_every > 0 ? d->checkpoint_every : (int64_t)std::ceil(std::sqrt((double)S));
    C = std::max<int64_t>(1, std::min(C, S));
    const int64_t K = (S + C - 1) / C;
    const bool fwd_only = d->forward_only != 0;
    if (int rc = h->awork.ensure((size_t)B * 5 * V * sizeof(double))) return rc;
    if (!fwd_only) {
        if (int rc = h->ackpt.ensure((size_t)B * K * V * sizeof(double))) return rc;
        if (int rc = h->aseg.ensure((size_t)B * C * 4 * V * sizeof(double))) return rc;
    }
    if (int rc = h->amloc.ensure((size_t)B * (S + 1) * 3 * sizeof(double))) return rc;
    if (int rc = h->aout.ensure((size_t)B * (1 + kAdjParams) * sizeof(double))) return rc;
    if (int rc = h->ain.ensure(((size_t)B * N3 + (size_t)B * (S + 1) * 3 + (S + 1)) * sizeof(double))) return rc;
    if (int rc = h->ameta.ensure((size_t)B * sizeof(cmd::AdjTraj))) return rc;
    for (int64_t i = 0; i < B * N3; ++i)
        if (!std::isfinite(d->states[i])) return fail(CMD_ERR_NONFINITE, "non-finite initial spin");
    double* din = h->ain.as<double>();
    double* dtgt = din + B * N3;
    double* dtimes = dtgt + B * (S + 1) * 3;
    std::vector<double> times((size_t)S + 1);
    double t = d->T0;
    for (int64_t n = 0; n <= S; ++n) { times[n] = t; t += d->dt; }
    CUDA_TRY(cudaMemcpyAsync(din, d->states, B * N3 * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(cudaMemcpyAsync(dtgt, d->target, B * (S + 1) * 3 * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(cudaMemcpyAsync(dtimes, times.data(), times.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    std::vector<cmd::AdjTraj> tr(B);
    double* dout = h->aout.as<double>();
    for (int64_t b = 0; b < B; ++b) {
        cmd::AdjTraj& T = tr[b];
        T.y0 = din + b * N3;
        T.target = dtgt + b * (S + 1) * 3;
        T.ckpt = fwd_only ? nullptr : h->ackpt.as<double>() + b * K * V;
        T.seg = fwd_only ? nullptr : h->aseg.as<double>() + b * C * 4 * V;
        T.work = h->awork.as<double>() + b * 5 * V;
        T.mloc = h->amloc.as<double>() + b * (S + 1) * 3;
        T.loss = dout + b * (1 + kAdjParams);
        T.grad = dout + b * (1 + kAdjParams) + 1;
    }
    CUDA_TRY(cudaMemcpyAsync(h->ameta.p, tr.data(), B * sizeof(cmd::AdjTraj), cudaMemcpyHostToDevice, h->stream));
    cmd::AdjArgs a{};
    a.traj = h->ameta.as<cmd::AdjTraj>();
    a.B = (int)B;
    a.G = (int)h->lay.G;
    a.nbr = h->nbr.as<int>();
    a.times = dtimes;
    a.n_steps = S;
    a.ckpt_every = C;
    a.dt = d->dt;
    if (h->amp != 0.0) a.pulse = cmd::Pulse{h->t1, h->t2, h->amp, h->amp};
    a.width = h->width;
    a.freq = h->freq;
    a.forward_only = fwd_only;
    // resident (one CTA or cluster per trajectory) when a variant holds the lattice; else one
    // CTA per trajectory in global memory when the batch fills the GPU, else streamed stages
    const int cpt = cmd::kStreamTile / std::max(1, h->NA);
    const int tiles = (int)((h->lay.G + cpt - 1) / cpt);
    const int resident = (d->path == CMD_ADJ_AUTO || d->path == CMD_ADJ_RESIDENT) ? pick_adjoint_cluster(h) : -1;
    if (d->path == CMD_ADJ_RESIDENT && resident < 0)
        return fail(CMD_ERR_UNSUPPORTED, "no resident adjoint variant holds this lattice");
    const bool streamed = resident < 0 && B <= 65535 &&
                          (d->path == CMD_ADJ_STREAMED || (d->path == CMD_ADJ_AUTO && B < 148 && tiles >= 2));
    int rc = CMD_OK;
    if (resident >= 0) {
        cmd::AdjClusterArgs ca{};
        ca.traj = a.traj;
        ca.G = a.G;
        ca.n_steps = S;
        ca.ckpt_every = C;
        ca.dt = d->dt;
        ca.forward_only = fwd_only;
        if (h->amp != 0.0) {
            const cmd::Pulse pl{h->t1, h->t2, h->amp, h->amp};
            if (int rc2 = h->pulses.ensure(sizeof(cmd::Pulse))) return rc2;
            if (int rc2 = h->drive.ensure((size_t)S * 6 * sizeof(double))) return rc2;
            CUDA_TRY(cudaMemcpyAsync(h->pulses.p, &pl, sizeof(pl), cudaMemcpyHostToDevice, h->stream));
            const int blocks = (int)std::min<int64_t>((S * 6 + 255) / 256, 148 * 32);
            cmd::drive_table_kernel<<<blocks, 256, 0, h->stream>>>(h->pulses.as<cmd::Pulse>(), dtimes, S, d->dt,
                                                                 h->width, h->freq, 1, h->drive.as<double>());
            CUDA_TRY(cudaGetLastError());
            ca.drive = h->drive.as<double>();
        }
        rc = kAdjClusterVariants[resident].fn(h, ca, DJ, DB, DA, has_DA, B);
    } else if (streamed) {
        StreamAdjJob j{B, S, C, K, fwd_only, din, dtgt, dtimes, h->amloc.as<double>(), dout, d->dt};
        // the VJP carries as many parameter cotangents as requested (4 or 5)
        if (d->n_params <= 4)
            rc = ty == 0 ? stream_adjoint<2, 3, 1, 4>(h, j, DJ, DB, DA, has_DA)
                         : stream_adjoint<4, 6, 3, 4>(h, j, DJ, DB, DA, has_DA);
        else
            rc = ty == 0 ? stream_adjoint<2, 3, 1, 5>(h, j, DJ, DB, DA, has_DA)
                         : stream_adjoint<4, 6, 3, 5>(h, j, DJ, DB, DA, has_DA);
    } else {
        rc = ty == 0 ? launch_adjoint<2, 3, 1>(h, a, DJ, DB, DA, has_DA, B)
                     : launch_adjoint<4, 6, 3>(h, a, DJ, DB, DA, has_DA, B);
    }
    if (rc != CMD_OK) return rc;
    std::vector<double> out((size_t)B * (1 + kAdjParams));
    CUDA_TRY(cudaMemcpyAsync(out.data(), dout, out.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    if (d->m_local)
        CUDA_TRY(cudaMemcpyAsync(d->m_local, h->amloc.p, B * (S + 1) * 3 * sizeof(double), cudaMemcpyDeviceToHost,
                                 h->stream));
    if (int rc2 = sync(h)) return rc2;
    for (int64_t b = 0; b < B; ++b) {
        d->loss[b] = out[b * (1 + kAdjParams)];
        if (!fwd_only)
            for (int q = 0; q < d->n_params; ++q) d->grad[b * d->n_params + q] = out[b * (1 + kAdjParams) + 1 + q];
    }
    return CMD_OK;
}

int cmd_plan_layout(const cmd_lattice_desc* d, int64_t* info) {
    cmd::clear_error();
    if (!d || !info) return fail(CMD_ERR_INVALID_ARG, "NULL argument");
    for (int i = 0; i < 7; ++i) info[i] = 0;
    if (d->spin_dim != 3 || d->lattice_size <= 0 || d->n_atoms <= 0 || !d->counts || !d->field || !d->onsite)
        return fail(CMD_ERR_INVALID_ARG, "bad lattice description");
    cmd_handle tmp;                    // host-side fields only; no stream, no device memory
    tmp.N = d->lattice_size;
    tmp.NA = d->n_atoms;
    tmp.zmax = d->max_bilinear;
    analyse(*d, tmp.lay);
    info[0] = tmp.lay.NA;
    info[1] = tmp.lay.G;
    info[2] = tmp.lay.Z;
    info[6] = tmp.lay.LZ;
    const Layout& L = tmp.lay;
    const int vi = default_variant(L);
    if (vi < 0) return no_instance(L);
    const Variant& V = kVariants[vi];
    variant_shape(V, L, &info[3], &info[5]);
    info[4] = V.CPT;
    return CMD_OK;
}

int cmd_layout_info(cmd_handle* h, int64_t* info) {
    cmd::clear_error();
    if (int rc = check_handle(h, false)) return rc;
    if (!info) return fail(CMD_ERR_INVALID_ARG, "NULL info");
    for (int i = 0; i < 6; ++i) info[i] = 0;
    info[0] = h->lay.NA;
    info[1] = h->lay.G;
    info[2] = h->lay.Z;
    const int vi = pick_variant(h);
    if (vi < 0) return no_instance(h->lay);
    const Variant& V = kVariants[vi];
    variant_shape(V, h->lay, &info[3], &info[5]);
    info[4] = V.CPT;
    return CMD_OK;
}

int cmd_variant_count(void) { return kNumVariants; }

int cmd_variant_info(cmd_handle* h, int32_t idx, char* name, int32_t name_len, int32_t* fits) {
    cmd::clear_error();
    if (idx < 0 || idx >= kNumVariants) return fail(CMD_ERR_INVALID_ARG, "variant index out of range");
    if (name && name_len > 0) {
        std::strncpy(name, kVariants[idx].name, (size_t)name_len - 1);
        name[name_len - 1] = 0;
    }
    if (fits) *fits = (h && variant_fits(kVariants[idx], h->lay)) ? 1 : 0;
    return CMD_OK;
}

int cmd_set_variant(cmd_handle* h, int32_t idx) {
    cmd::clear_error();
    if (int rc = check_handle(h, false)) return rc;
    if (idx < -1 || idx >= kNumVariants) return fail(CMD_ERR_INVALID_ARG, "variant index out of range");
    if (idx >= 0 && !variant_fits(kVariants[idx], h->lay))
        return fail(CMD_ERR_UNSUPPORTED, "variant does not fit this lattice");
    h->variant = idx;
    return CMD_OK;
}

int cmd_get_variant(cmd_handle* h, int32_t* idx) {
    cmd::clear_error();
    if (int rc = check_handle(h, false)) return rc;
    if (!idx) return fail(CMD_ERR_INVALID_ARG, "NULL output");
    *idx = pick_variant(h);
    return CMD_OK;
}

// Times every fitting variant on a B-trajectory, n_steps-step RK4 batch from the
// handle's current state (observables every step, no drive) and keeps the
// fastest.  ms[kNumVariants] (may be NULL) gets the times, -1 for variants that
// do not fit.
int cmd_autotune(cmd_handle* h, int64_t B, int64_t n_steps, int32_t* best, double* ms) {
    cmd::clear_error();
    if (int rc = check_handle(h, true)) return rc;
    if (B <= 0 || n_steps <= 0) return fail(CMD_ERR_INVALID_ARG, "bad autotune size");
    const int64_t rows = rows_for(n_steps, 1);
    if (int rc = h->tune_obs.ensure((size_t)B * rows * 10 * sizeof(double))) return rc;
    cudaEvent_t e0, e1;
    CUDA_TRY(cudaEventCreate(&e0));
    CUDA_TRY(cudaEventCreate(&e1));
    int win = -1;
    float best_ms = 0.0f;
    int rc = CMD_OK;
    for (int i = 0; i < kNumVariants && rc == CMD_OK; ++i) {
        if (ms) ms[i] = -1.0;
        if (!variant_fits(kVariants[i], h->lay)) continue;
        RunSpec r;
        r.B = B;
        r.y0 = h->state.as<double>();
        r.obs = h->tune_obs.as<double>();
        r.dt = 0.01;
        r.n_steps = n_steps;
        r.save = 1;
        r.n_sites = (double)h->N;
        r.variant = i;
        float t = 0.0f;
        for (int rep = 0; rep < 2 && rc == CMD_OK; ++rep) {     // first run warms up
            cudaEventRecord(e0, h->stream);
            rc = run_resident(h, r, h->stream, nullptr);
            cudaEventRecord(e1, h->stream);
            if (rc == CMD_OK) rc = sync(h);
            if (rc == CMD_OK) cudaEventElapsedTime(&t, e0, e1);
        }
        if (rc != CMD_OK) break;
        if (ms) ms[i] = t;
        if (win < 0 || t < best_ms) { win = i; best_ms = t; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc != CMD_OK) return rc;
    if (win < 0) return no_instance(h->lay);
    h->variant = win;
    if (best) *best = win;
    return CMD_OK;
}

int cmd_integrate_batched(cmd_handle* h, const double* init, const double* tau2, int64_t B,
                          const double* afm_signs, const double* frames, double T0, double T1,
                          double dt, int64_t save_interval, int method, double* times, double* mags,
                          int64_t max_rows, int64_t* rows_out) {
    cmd::clear_error();
    if (int rc = check_handle(h, false)) return rc;
    if (!init || !tau2 || B <= 0) return fail(CMD_ERR_INVALID_ARG, "bad batch arguments");
    if (method != CMD_RK4) return fail(CMD_ERR_UNSUPPORTED, "batched mode supports rk4 only (lattice_gpu.cu:781-784)");
    if (save_interval <= 0 || !(dt > 0.0)) return fail(CMD_ERR_INVALID_ARG, "bad time grid");
    std::vector<double> grid;
    const int64_t n = count_steps(T0, T1, dt, 1e-12, &grid);
    const int64_t rows = rows_for(n, save_interval);
    if (rows_out) *rows_out = rows;
    if (max_rows < rows) return fail(CMD_ERR_INVALID_ARG, "max_rows too small");
    std::vector<double> t1(B, h->t1), a(B, h->amp), obs((size_t)B * rows * 10);
    // Frames / AFM signs of the call override the lattice's for the observables.
    std::vector<double> frc, afc;
    if (frames)
        if (int rc = reduce_per_class(h, frames, 9, frc, "sublattice frames")) return rc;
    if (afm_signs)
        if (int rc = reduce_per_class(h, afm_signs, 1, afc, "AFM signs")) return rc;
    if (int rc = upload_frames(h, frames ? frc.data() : h->frames.data(), afm_signs ? afc.data() : h->afm.data()))
        return rc;
    cmd_batch_desc d{};
    d.B = B;
    d.states = init;
    d.shared_initial = 1;
    d.method = CMD_RK4;
    d.t1 = t1.data(); d.t2 = tau2; d.a1 = a.data(); d.a2 = a.data();
    // h->fd is per class; expand to the caller's atoms for cmd_run_batch
    const int ca = caller_atoms(h);
    std::vector<double> e1(3 * (size_t)ca), e2(3 * (size_t)ca);
    for (int at = 0; at < ca; ++at)
        for (int c = 0; c < 3; ++c) {
            e1[3 * at + c] = h->fd[3 * (at % h->NA) + c];
            e2[3 * at + c] = h->fd[3 * h->NA + 3 * (at % h->NA) + c];
        }
    d.d1 = e1.data(); d.d2 = e2.data();
    d.width = h->width; d.freq = h->freq;
    d.T0 = T0; d.dt = dt;
    d.n_steps = n; d.save_interval = save_interval;
    d.obs = obs.data();
    d.final_states = nullptr;
    const int rc = cmd_run_batch(h, &d);
    const int rc2 = upload_frames(h, h->frames.data(), h->afm.data());
    if (rc != CMD_OK) return rc;
    if (rc2 != CMD_OK) return rc2;
    if (times) {
        int64_t r = 0;
        for (int64_t k = 0; k < n; k += save_interval) times[r++] = grid[k];
        times[r] = grid[n];
    }
    if (mags)
        for (int64_t r = 0; r < rows; ++r)
            for (int64_t b = 0; b < B; ++b)
                std::memcpy(mags + (r * B + b) * 9, &obs[((size_t)b * rows + r) * 10], 9 * sizeof(double));
    return CMD_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free batch entry point (no reference counterpart).
//
// Some callers cannot call cudaMalloc: code whose device memory belongs to
// another allocator that has already reserved the GPU (a caching allocator
// holding the whole device, a pre-partitioned serving pool), and loops that
// cannot take the device-wide synchronisation that cudaMalloc / cudaFree may
// imply.  cmd_run_batch_device grows handle-owned scratch buffers on demand
// (the step-time grid, the pulse-envelope table and, for cells of more than 3
// atoms, the raw observable rows); cmd_run_batch_device_noalloc runs the same
// kernels with that scratch carved out of one file-scope device array instead.
namespace {

// t_k of the reference loop (t = T0; t += dt) for k < n, by one thread: the
// same sequence of IEEE additions as the host-built grid of run_resident.
__global__ void time_grid_kernel(double T0, double dt, int64_t n, double* out) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    double t = T0;
    for (int64_t k = 0; k < n; ++k) {
        out[k] = t;
        t += dt;
    }
}

constexpr int64_t noalloc_round(int64_t n) { return (n + 31) / 32 * 32; }   // 256-byte regions

// run_resident with its scratch in g_noalloc_scratch.  Every scratch element
// a launch reads is written earlier in the same call (time grid, envelope
// table, raw rows), so nothing needs clearing between calls.
int run_resident_noalloc(cmd_handle* h, const RunSpec& r, cudaStream_t st, int32_t* launches) {
    int32_t nl = 0;
    const int vi = pick_variant(h);
    if (vi < 0 || !variant_fits(kVariants[vi], h->lay)) {
        if (!h->lay.uniform) return no_instance(h->lay);
        return fail(CMD_ERR_UNSUPPORTED, "cmd_run_batch_device_noalloc runs resident lattices only (one CTA or a "
                                         "2- or 4-CTA cluster per trajectory); this lattice needs the streamed "
                                         "kernels: use cmd_run_batch_device");
    }
    const Variant& V = kVariants[vi];
    if (r.n_steps > kNoAllocScratchDoubles)
        return fail(CMD_ERR_INVALID_ARG, "cmd_run_batch_device_noalloc: n_steps beyond the static scratch");
    const int64_t rows = rows_for(r.n_steps, r.save);
    const int NR = 3 * V.NAT + 1;
    const bool driven = r.pulses && r.n_steps > 0;
    const bool raw_in_scratch = r.obs && NR > 10;
    const int64_t n_times = driven ? noalloc_round(r.n_steps) : 0;
    const int64_t n_drive = driven ? noalloc_round(r.B * r.n_steps * 6) : 0;
    const int64_t n_raw = raw_in_scratch ? noalloc_round(r.B * rows * NR) : 0;
    const int64_t need = n_times + n_drive + n_raw;
    if (need > kNoAllocScratchDoubles) {
        char buf[320];
        std::snprintf(buf, sizeof(buf),
                      "cmd_run_batch_device_noalloc: this batch needs %lld doubles of scratch (time grid %lld + "
                      "envelope table B*n_steps*6 = %lld + raw rows %lld), the static scratch holds %lld (32 MiB); "
                      "split the batch",
                      (long long)need, (long long)n_times, (long long)n_drive, (long long)n_raw,
                      (long long)kNoAllocScratchDoubles);
        return fail(CMD_ERR_INVALID_ARG, buf);
    }
    int dev = -1;
    CUDA_TRY(cudaGetDevice(&dev));
    if (dev != h->device || !h->noalloc_base)
        return fail(CMD_ERR_INVALID_ARG, "cmd_run_batch_device_noalloc: make the handle's device current (the "
                                         "scratch address belongs to the device the handle was created on)");
    double* base = h->noalloc_base;
    double* s_times = base;
    double* s_drive = base + n_times;
    double* s_raw = base + n_times + n_drive;

    cmd::ResidentArgs a{};
    a.G = (int)h->lay.G;
    a.n_steps = r.n_steps;
    a.save_every = r.save;
    a.T0 = r.T0;
    a.dt = r.dt;
    a.nbr = h->nbr.as<int>();
    a.y0 = r.y0;
    a.y0_stride = r.y0_stride;
    a.y_out = r.y_out;
    a.rows = rows;
    a.traj = r.traj;
    a.drive = nullptr;
    if (r.obs) {
        a.raw = raw_in_scratch ? s_raw : r.obs;
        a.raw_stride = raw_in_scratch ? NR : 10;
    }
    if (driven) {
        time_grid_kernel<<<1, 32, 0, st>>>(r.T0, r.dt, r.n_steps, s_times);
        CUDA_TRY(cudaGetLastError());
        ++nl;
        const int64_t total = r.B * r.n_steps * 6;
        const int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 32);
        cmd::drive_table_kernel<<<blocks, 256, 0, st>>>(r.pulses, s_times, r.n_steps, r.dt, r.width, r.freq, r.B,
                                                       s_drive);
        CUDA_TRY(cudaGetLastError());
        ++nl;
        a.drive = s_drive;
    }
    static const double zeros[3 * 64] = {};
    if (int rc = V.fn(h, a, r.d1 ? r.d1 : zeros, r.d2 ? r.d2 : zeros, r.B, st)) return rc;
    ++nl;
    if (r.obs) {
        const int64_t n = r.B * rows;
        const double* fr = r.frames ? r.frames : h->dframes.as<double>();
        const double* af = r.afm ? r.afm : h->dafm.as<double>();
        switch (V.NAT) {
            case 2: launch_finish<2>(a.raw, a.raw_stride, n, fr, af, r.n_sites, r.obs, st); break;
            case 4: launch_finish<4>(a.raw, a.raw_stride, n, fr, af, r.n_sites, r.obs, st); break;
            default: return fail(CMD_ERR_UNSUPPORTED, "no row finisher for this cell size");
        }
        CUDA_TRY(cudaGetLastError());
        ++nl;
    }
    if (launches) *launches = nl;
    return CMD_OK;
}

}  // namespace

extern "C" {

int cmd_run_batch_device_noalloc(cmd_handle* h, const cmd_batch_desc* d, void* stream, int32_t* launches) {
    cmd::clear_error();
    if (launches) *launches = 0;
    if (int rc = check_handle(h, false)) return rc;
    if (int rc = validate_batch(h, d)) return rc;
    cudaStream_t st = stream ? (cudaStream_t)stream : h->stream;
    const bool drive = d->d1 || d->d2;
    if (drive && !d->pulse4) return fail(CMD_ERR_INVALID_ARG, "driven device batch needs pulse4");
    if (drive && h->NA > 64)
        return fail(CMD_ERR_UNSUPPORTED, "cmd_run_batch_device_noalloc: pulse directions limited to 64 atoms per cell");
    RunSpec r;
    r.B = d->B;
    r.y0 = d->states;
    r.y0_stride = d->shared_initial ? 0 : h->N * 3;
    r.y_out = d->final_states;
    r.obs = d->obs;
    r.T0 = d->T0;
    r.dt = d->dt;
    r.n_steps = d->n_steps;
    r.save = d->save_interval;
    r.pulses = drive ? reinterpret_cast<const cmd::Pulse*>(d->pulse4) : nullptr;
    r.width = d->width;
    r.freq = d->freq;
    // per-class pulse directions in fixed host arrays (no heap)
    double d1c[3 * 64], d2c[3 * 64];
    const int ca = caller_atoms(h);
    const double* dirs[2] = {d->d1, d->d2};
    double* outs[2] = {d1c, d2c};
    for (int k = 0; k < 2; ++k) {
        if (!dirs[k]) continue;
        for (int a = 0; a < 3 * h->NA; ++a) outs[k][a] = dirs[k][a];
        for (int a = h->NA; a < ca; ++a)
            for (int c = 0; c < 3; ++c)
                if (dirs[k][a * 3 + c] != outs[k][(a % h->NA) * 3 + c])
                    return fail(CMD_ERR_UNSUPPORTED, "pulse directions must be uniform per sublattice class");
    }
    r.d1 = d->d1 ? d1c : nullptr;
    r.d2 = d->d2 ? d2c : nullptr;
    r.n_sites = (double)h->N;
    return run_resident_noalloc(h, r, st, launches);
}

}  // extern "C"
