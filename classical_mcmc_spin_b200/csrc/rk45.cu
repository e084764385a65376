// rk45.cu -- launches of the on-chip controlled Dormand-Prince kernels
// (rk45_onchip.cuh): the tilings compiled into the library (CTAs per
// trajectory x threads per CTA), the partner-word tables of each tiling, and
// the choice between them (the handle's pick, made by cmd_autotune_rk45, or
// the smallest cluster that holds the lattice).
#include "cmd_core.h"
#include "rk45_onchip.cuh"

#include <cstdio>

namespace cmd {
namespace {

using R45Fn = int (*)(const cmd_handle*, const R45Args&, int64_t, cudaStream_t);

struct R45Variant {
    int NAT, Z, LZ, APT, CS, MAXT;
    bool YK;                  // y and K1 in shared memory instead of registers
    bool HALO;                // partners in other CTAs pushed into halo columns (else read remotely)
    R45Fn fn;
    const char* name;
};

// Cells per CTA and the padded per-atom row of a tiling.
void r45_shape(const R45Variant& v, int64_t G, int64_t* Gc, int64_t* Gp) {
    *Gc = (G + v.CS - 1) / v.CS;
    *Gp = (*Gc + 31) / 32 * 32;
}

// Halo columns of a cluster partition: for every CTA r, the distinct sites of
// other CTAs its sites bond to get one column each in the row of their atom,
// numbered in the order of the partner table.  col[(r * G + cell) * NA + atom]
// = the column (>= 0) of that remote site in CTA r's rows, or -1.  Returns the
// largest number of columns any atom row of any CTA needs.
int64_t halo_columns(const Layout& L, int cs, int64_t Gc, std::vector<int>* col) {
    const int NA = L.NA, NL = L.Z - L.LZ;
    const int64_t G = L.G;
    if (col) col->assign((size_t)cs * G * NA, -1);
    std::vector<int> seen((size_t)G * NA, -1), count((size_t)NA, 0);
    int64_t most = 0;
    for (int r = 0; r < cs; ++r) {
        std::fill(count.begin(), count.end(), 0);
        for (int64_t g = r * Gc; g < std::min<int64_t>((r + 1) * Gc, G); ++g)
            for (int at = 0; at < NA; ++at)
                for (int m = 0; m < NL; ++m) {
                    const int64_t off = L.nbr[((size_t)g * NA + at) * NL + m];
                    const int64_t pat = off / (3 * G), pc = off - pat * 3 * G;
                    if (pc / Gc == r) continue;
                    const size_t site = (size_t)pc * NA + pat;
                    if (seen[site] == r) continue;
                    seen[site] = r;
                    const int c = count[pat]++;
                    if (col) (*col)[((size_t)r * G + pc) * NA + pat] = c;
                    most = std::max<int64_t>(most, c + 1);
                }
    }
    return most;
}

// Row length of a tiling's stage buffers: Gp own cells, then the halo columns.
int64_t r45_row(const R45Variant& v, const Layout& L, int64_t Gc, int64_t Gp) {
    if (!v.HALO || v.CS == 1) return Gp;
    int64_t& cols = L.halo_cols[v.CS];
    if (cols < 0) cols = halo_columns(L, v.CS, Gc, nullptr);
    return Gp + (cols + 1) / 2 * 2;
}

template <int NAT, int Z, int LZ, int APT, int CS, int MAXT, bool YK, bool HALO>
int launch_r45(const cmd_handle* h, const R45Args& a, int64_t B, cudaStream_t st) {
    auto kern = rk45_onchip_kernel<NAT, Z, LZ, APT, CS, MAXT, YK, HALO>;
    const int threads = NAT / APT * a.Gp;
    const size_t smem = (size_t)r45_smem_doubles(NAT, a.Gp, a.Gs, CS, MAXT, YK) * sizeof(double);
    if (threads > MAXT || smem > kMaxSmem) return fail(CMD_ERR_UNSUPPORTED, "lattice does not fit this RK45 tiling");
    // Function attributes belong to the current device's context: set on every launch.
    CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMaxSmem));
    if (CS > 8) CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    Couplings<NAT, Z> cp;
    fill_couplings<NAT, Z>(h, h->fd.data(), h->fd.data() + 3 * h->NA, cp);
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
    cfg.numAttrs = CS > 1 ? 1 : 0;
    CUDA_TRY(cudaLaunchKernelEx(&cfg, kern, cp, a));
    return CMD_OK;
}

#define CMD_R45(NAT, Z, LZ, APT, CS, MAXT) \
    R45Variant{NAT, Z, LZ, APT, CS, MAXT, false, false, &launch_r45<NAT, Z, LZ, APT, CS, MAXT, false, false>, \
               "rk45_onchip<" #NAT "," #Z "," #LZ "> apt=" #APT " cs=" #CS " maxt=" #MAXT}
#define CMD_R45_YK(NAT, Z, LZ, APT, CS, MAXT) \
    R45Variant{NAT, Z, LZ, APT, CS, MAXT, true, false, &launch_r45<NAT, Z, LZ, APT, CS, MAXT, true, false>, \
               "rk45_onchip<" #NAT "," #Z "," #LZ "> apt=" #APT " cs=" #CS " maxt=" #MAXT " yk"}
#define CMD_R45_HALO(NAT, Z, LZ, APT, CS, MAXT) \
    R45Variant{NAT, Z, LZ, APT, CS, MAXT, false, true, &launch_r45<NAT, Z, LZ, APT, CS, MAXT, false, true>, \
               "rk45_onchip<" #NAT "," #Z "," #LZ "> apt=" #APT " cs=" #CS " maxt=" #MAXT " halo"}
#define CMD_R45_HALO_YK(NAT, Z, LZ, APT, CS, MAXT) \
    R45Variant{NAT, Z, LZ, APT, CS, MAXT, true, true, &launch_r45<NAT, Z, LZ, APT, CS, MAXT, true, true>, \
               "rk45_onchip<" #NAT "," #Z "," #LZ "> apt=" #APT " cs=" #CS " maxt=" #MAXT " halo yk"}

// Tilings: atoms per thread (a whole cell, or fewer for more threads per SM) x
// CTAs per trajectory x thread bound (registers per thread = 64K / bound), where
// y and K1 live ("yk": the thread's own shared-memory slots, which frees
// registers for the stages) and how partners in other CTAs are read ("halo":
// their owners store them into halo columns of this CTA's stage buffers before
// the stage barrier, so every partner read is a local shared-memory load;
// otherwise each is a distributed-shared-memory load).  Ordered by preference
// when nothing was tuned: the first that holds a lattice is its default.  The
// order follows the uneven batch's lattices measured on a B200 (accepted
// spin-steps per second, tol 1e-10): honeycomb up to 16x16 on one CTA with a
// site per thread, 24x24 and 32x32 on 2-CTA clusters with a cell per thread (y,
// K1 in shared memory); pyrochlore 4^3 conventional cells on 2-CTA clusters,
// 6^3 and 8^3 on 4- and 8-CTA clusters with halo columns, two sites per thread.
const R45Variant kR45[] = {
    // honeycomb (2-atom cells, 3 bonds per site)
    CMD_R45(2, 3, 1, 1, 1, 512),
    CMD_R45_YK(2, 3, 1, 2, 2, 512),
    CMD_R45(2, 3, 1, 2, 2, 512),
    CMD_R45(2, 3, 1, 2, 1, 256),
    CMD_R45(2, 3, 1, 2, 4, 256),
    CMD_R45(2, 3, 1, 2, 8, 256),
    CMD_R45(2, 3, 1, 1, 2, 1024),
    // pyrochlore (4-atom groups, 6 bonds per site)
    CMD_R45(4, 6, 3, 2, 2, 256),
    CMD_R45_HALO(4, 6, 3, 2, 4, 512),
    CMD_R45_HALO(4, 6, 3, 2, 8, 512),
    CMD_R45(4, 6, 3, 2, 4, 512),
    CMD_R45_YK(4, 6, 3, 4, 8, 256),
    CMD_R45(4, 6, 3, 2, 8, 512),
    CMD_R45(4, 6, 3, 2, 1, 512),
    CMD_R45(4, 6, 3, 2, 16, 256),
    CMD_R45(4, 6, 3, 4, 1, 256),
    CMD_R45(4, 6, 3, 4, 4, 256),
    CMD_R45(4, 6, 3, 4, 8, 256),
    CMD_R45(4, 6, 3, 1, 2, 512),
    CMD_R45_YK(4, 6, 3, 2, 4, 512),
    CMD_R45_YK(4, 6, 3, 4, 4, 256),
    CMD_R45_HALO_YK(4, 6, 3, 2, 4, 512),
};
constexpr int kNumR45 = (int)(sizeof(kR45) / sizeof(kR45[0]));

// Partner words [G][NA][Z-LZ] of a tiling (the bonds that leave the cell).
// Remote reads: slot m of site (g, at) holds (rank << 24) | ((partner atom * 3)
// * Gp + partner cell - rank * Gc), the partner's slot in its CTA's stage
// buffer.  Halo tilings: the partner's slot in this CTA's own stage buffer (its
// cell, or its halo column), and push words: for each site, the halo slots
// (rank << 24) | slot of the other CTAs that read it, -1 for the rest.
int upload_partner_words(cmd_handle* h, const R45Variant& v, int64_t Gc, int64_t Gp, int64_t Gs) {
    const int key = v.CS * 2 + (v.HALO ? 1 : 0);
    if (h->cnbr_all_cs == key && h->cnbr_all.p) return CMD_OK;
    const Layout& L = h->lay;
    const int NA = L.NA, NL = L.Z - L.LZ;
    const int64_t G = L.G;
    const size_t n = std::max<size_t>((size_t)G * NA * NL, 1);
    std::vector<int> w(n, 0), push;
    std::vector<int> col;
    if (v.HALO && v.CS > 1) {
        halo_columns(L, v.CS, Gc, &col);
        push.assign(n, -1);
    }
    for (size_t i = 0; i < L.nbr.size(); ++i) {
        const int64_t off = L.nbr[i];                 // (atom*3)*G + cell of the resident layout
        const int64_t pat = off / (3 * G), gp = off - pat * 3 * G;
        const int64_t r = gp / Gc, l = gp - r * Gc;
        if (col.empty()) {
            w[i] = (int)((r << kClusterRankShift) | (pat * 3 * Gp + l));
            continue;
        }
        const int64_t site = (int64_t)(i / NL);       // g * NA + at of the reading site
        const int64_t own_r = (site / NA) / Gc;
        if (r == own_r) {
            w[i] = (int)(pat * 3 * Gs + l);
        } else {
            const int c = col[((size_t)own_r * G + gp) * NA + pat];
            w[i] = (int)(pat * 3 * Gs + Gp + c);
            // the partner pushes its value into this column of CTA own_r (once per CTA)
            int* slots = &push[((size_t)gp * NA + pat) * NL];
            const int word = (int)((own_r << kClusterRankShift) | (pat * 3 * Gs + Gp + c));
            int k = 0;
            while (k < NL && slots[k] >= 0 && slots[k] != word) ++k;
            if (k == NL) return fail(CMD_ERR_UNSUPPORTED, "a site is read by more CTAs than it has bonds");
            slots[k] = word;
        }
    }
    h->cnbr_all_cs = 0;
    if (int rc = h->cnbr_all.ensure(w.size() * sizeof(int))) return rc;
    CUDA_TRY(cudaMemcpy(h->cnbr_all.p, w.data(), w.size() * sizeof(int), cudaMemcpyHostToDevice));
    if (!push.empty()) {
        if (int rc = h->cpush.ensure(push.size() * sizeof(int))) return rc;
        CUDA_TRY(cudaMemcpy(h->cpush.p, push.data(), push.size() * sizeof(int), cudaMemcpyHostToDevice));
    }
    h->cnbr_all_cs = key;
    return CMD_OK;
}

}  // namespace

int rk45_variant_count() { return kNumR45; }
const char* rk45_variant_name(int i) { return (i >= 0 && i < kNumR45) ? kR45[i].name : ""; }

bool rk45_fits(int i, const Layout& L) {
    if (i < 0 || i >= kNumR45) return false;
    const R45Variant& v = kR45[i];
    if (!L.uniform || v.NAT != L.NA || v.Z != L.Z || v.LZ != L.LZ) return false;
    int64_t Gc, Gp;
    r45_shape(v, L.G, &Gc, &Gp);
    if (v.CS > 1 && Gc < 32) return false;                      // a cluster only for lattices one CTA cannot hold well
    if (v.NAT / v.APT * Gp > v.MAXT) return false;
    const int64_t Gs = r45_row(v, L, Gc, Gp);
    if ((size_t)r45_smem_doubles(v.NAT, (int)Gp, (int)Gs, v.CS, v.MAXT, v.YK) * sizeof(double) > kMaxSmem) return false;
    if (6 * (int64_t)v.NAT * 3 * Gs >= (1 << kClusterRankShift)) return false;
    return true;
}

int rk45_pick(const cmd_handle* h) {
    if (h->rk45_variant == -2) return -1;                      // forced onto the global-state kernel
    if (h->rk45_variant >= 0 && rk45_fits(h->rk45_variant, h->lay)) return h->rk45_variant;
    for (int i = 0; i < kNumR45; ++i)
        if (rk45_fits(i, h->lay)) return i;
    return -1;
}

int rk45_prepare(cmd_handle* h, int variant) {
    if (!rk45_fits(variant, h->lay)) return fail(CMD_ERR_UNSUPPORTED, "RK45 tiling does not hold this lattice");
    const R45Variant& v = kR45[variant];
    int64_t Gc, Gp;
    r45_shape(v, h->lay.G, &Gc, &Gp);
    return upload_partner_words(h, v, Gc, Gp, r45_row(v, h->lay, Gc, Gp));
}

int rk45_launch(cmd_handle* h, int variant, const GTraj* d_traj, int64_t B, double abs_tol, double rel_tol,
                int64_t max_steps, cudaStream_t st) {
    if (int rc = rk45_prepare(h, variant)) return rc;
    const R45Variant& v = kR45[variant];
    int64_t Gc, Gp;
    r45_shape(v, h->lay.G, &Gc, &Gp);
    R45Args a{};
    a.traj = d_traj;
    a.pw = h->cnbr_all.as<int>();
    a.G = (int)h->lay.G;
    a.Gc = (int)Gc;
    a.Gp = (int)Gp;
    a.Gs = (int)r45_row(v, h->lay, Gc, Gp);
    a.push = v.HALO ? h->cpush.as<int>() : nullptr;
    a.abs_tol = abs_tol;
    a.rel_tol = rel_tol;
    // the kernel counts accepted steps in 32 bits: "no cap" becomes 2^31 - 2
    constexpr int64_t kMaxCap = 2147483646;
    a.max_steps = (int)((max_steps <= 0 || max_steps > kMaxCap) ? kMaxCap : max_steps);
    a.width = h->width;
    a.freq = h->freq;
    a.frames = h->dframes.as<double>();
    a.afm = h->dafm.as<double>();
    return v.fn(h, a, B, st);
}

}  // namespace cmd
