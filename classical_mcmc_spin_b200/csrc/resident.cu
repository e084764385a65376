// resident.cu -- resident RK4 launches: one CTA, or one thread-block cluster of
// 2 or 4 CTAs, per trajectory (rk4_resident.cuh, rk4_cluster.cuh), the variant
// table the autotuner chooses from, and the partner tables of the cluster
// layouts.
#include "cmd_core.h"
#include "rk4_cluster.cuh"
#include "rk4_lean.cuh"

namespace cmd {
namespace {

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

template <int NAT, int Z, int LZ, int MAXT, int MINB>
int launch_lean(const cmd_handle* h, const cmd::ResidentArgs& args, const double* d1, const double* d2,
                int64_t B, cudaStream_t st) {
    auto kern = cmd::rk4_lean_kernel<NAT, Z, LZ, MAXT, MINB>;
    const int64_t G = h->lay.G;
    const int threads = (int)((G + 31) / 32 * 32);
    if (threads > MAXT) return fail(CMD_ERR_UNSUPPORTED, "lattice too large for this kernel variant");
    const size_t smem = (size_t)cmd::lean_smem_doubles(NAT, MAXT) * sizeof(double);
    CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMaxSmem));
    cmd::Couplings<NAT, Z> cp;
    fill_couplings<NAT, Z>(h, d1, d2, cp);
    cmd::ResidentArgs a = args;
    a.B = B;
    kern<<<(unsigned)B, threads, smem, st>>>(cp, a);
    CUDA_TRY(cudaGetLastError());
    return CMD_OK;
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

#define CMD_VARIANT(NAT, Z, LZ, CPT, MAXT, MINB, YREG, TPC) \
    Variant{NAT, Z, LZ, CPT, MAXT, MINB, YREG, TPC, 1, false, &launch_one<NAT, Z, LZ, CPT, MAXT, MINB, YREG, TPC>, \
            "rk4_resident<" #NAT "," #Z "," #LZ "> cpt=" #CPT " maxt=" #MAXT " minb=" #MINB " yreg=" #YREG \
            " tpc=" #TPC}
#define CMD_LEAN(NAT, Z, LZ, MAXT, MINB) \
    Variant{NAT, Z, LZ, 1, MAXT, MINB, true, 1, 1, true, &launch_lean<NAT, Z, LZ, MAXT, MINB>, \
            "rk4_lean<" #NAT "," #Z "," #LZ "> maxt=" #MAXT " minb=" #MINB}
#define CMD_CLUSTER(NAT, Z, LZ, CS, MAXT) \
    Variant{NAT, Z, LZ, 1, MAXT, 1, true, 1, CS, false, &launch_cluster<NAT, Z, LZ, CS, MAXT>, \
            "rk4_cluster<" #NAT "," #Z "," #LZ "> cs=" #CS " maxt=" #MAXT}

const Variant kVariants[] = {
    // 2-atom cells with 3 bonds per site (Kitaev / Heisenberg honeycomb)
    CMD_LEAN(2, 3, 1, 640, 1),
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
    CMD_LEAN(4, 6, 3, 256, 1),
    CMD_VARIANT(4, 6, 3, 1, 512, 1, true, 1),
    CMD_VARIANT(4, 6, 3, 2, 256, 2, false, 1),
    CMD_VARIANT(4, 6, 3, 2, 512, 1, false, 1),
    CMD_CLUSTER(4, 6, 3, 2, 512),
    CMD_CLUSTER(4, 6, 3, 4, 512),
};
constexpr int kNumVariants = (int)(sizeof(kVariants) / sizeof(kVariants[0]));

}  // namespace

const Variant* variant_table() { return kVariants; }
int variant_count() { return kNumVariants; }

// Partner table of the CS-CTA cluster kernel: the resident table's offsets
// (atom*3)*G + cell become (rank << 24) | ((atom*3)*Gc + cell - rank*Gc) with
// Gc = ceil(G / CS) cells per CTA.  Built once per handle.
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

// Partner words of the cluster layout with CS CTAs (CS = 1: the global offsets, rank 0).
const int* cluster_table(const cmd_handle* h, int cs) {
    return cs == 1 ? h->nbr.as<int>() : static_cast<const int*>((cs == 2 ? h->cnbr2 : h->cnbr4).p);
}

bool variant_fits(const Variant& v, const Layout& L) {
    if (!L.uniform || v.NAT != L.NA || v.Z != L.Z || v.LZ != L.LZ) return false;
    if (v.lean) {
        for (int a = 0; a < L.NA; ++a)
            if (L.zc[a] != L.Z) return false;
        return (L.G + 31) / 32 * 32 <= v.MAXT &&
               (size_t)lean_smem_doubles(v.NAT, v.MAXT) * sizeof(double) <= kMaxSmem;
    }
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
        a.drive = h->drive.as<double>();
    }
    if (r.obs && V.NAT != 2 && V.NAT != 4) return fail(CMD_ERR_UNSUPPORTED, "no row finisher for this cell size");
    static const std::vector<double> zeros(3 * 64, 0.0);
    const double* d1 = r.d1 ? r.d1 : zeros.data();
    const double* d2 = r.d2 ? r.d2 : zeros.data();
    // drive table, the resident kernel and the row finisher: one graph
    const int rc = graph_call(h, kGraphResident, st, [&]() -> int {
        if (a.drive) {
            const int64_t total = r.B * r.n_steps * 6;
            const int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 32);
            cmd::drive_table_kernel<<<blocks, 256, 0, st>>>(r.pulses, h->times.as<double>(), r.n_steps, r.dt,
                                                           r.width, r.freq, r.B, h->drive.as<double>());
            CUDA_TRY(cudaGetLastError());
            ++nl;
        }
        if (int rc2 = V.fn(h, a, d1, d2, r.B, st)) return rc2;
        ++nl;
        if (r.obs) {
            const int64_t n = r.B * rows;
            const double* fr = r.frames ? r.frames : h->dframes.as<double>();
            const double* af = r.afm ? r.afm : h->dafm.as<double>();
            if (V.NAT == 2) launch_finish<2>(a.raw, a.raw_stride, n, fr, af, r.n_sites, r.obs, st);
            else launch_finish<4>(a.raw, a.raw_stride, n, fr, af, r.n_sites, r.obs, st);
            CUDA_TRY(cudaGetLastError());
            ++nl;
        }
        return CMD_OK;
    });
    if (rc != CMD_OK) return rc;
    if (launches) *launches = nl;
    return CMD_OK;
}

void variant_shape(const Variant& V, const Layout& L, int64_t* threads, int64_t* smem) {
    if (V.lean) {
        *threads = (L.G + 31) / 32 * 32;
        *smem = (int64_t)lean_smem_doubles(V.NAT, V.MAXT) * (int64_t)sizeof(double);
    } else if (V.CS > 1) {
        *threads = (cluster_cells(L.G, V.CS) + 31) / 32 * 32;
        *smem = (int64_t)cluster_smem(L.NA, L.G, V.CS);
    } else {
        *threads = ((L.G + V.CPT - 1) / V.CPT + 31) / 32 * 32;
        *smem = (int64_t)resident_smem(L.NA, L.G, V.TPC);
    }
}

}  // namespace cmd
