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
#include "cmd_core.h"
#include "rk4_cluster.cuh"
#include "rk_global.cuh"

#include <chrono>
#include <thread>
#include <cmath>
#include <cstdio>

namespace cmd {

static thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}
void clear_error() { g_last_error.clear(); }

}  // namespace cmd

using namespace cmd;

bool layout_has_kernel(const Layout& L);

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

}  // namespace

bool layout_has_kernel(const Layout& L) { return default_variant(L) >= 0 || global_type(L) >= 0; }

namespace {

// RK4 over the handle's lattice: the resident kernel when a variant holds the
// lattice (or one is named), else the streamed stage kernels.
int run_rk4(cmd_handle* h, const RunSpec& r, cudaStream_t st, int32_t* launches) {
    if (r.variant >= 0 || pick_variant(h) >= 0) return run_resident(h, r, st, launches);
    return run_streamed(h, r, st, launches);
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

}  // namespace

int cmd::sync(cmd_handle* h) {
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return fail(CMD_ERR_CUDA, std::string("kernel execution: ") + cudaGetErrorString(e));
    return CMD_OK;
}

namespace {


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

}  // namespace

int cmd::caller_atoms(const cmd_handle* h) { return h->n_atoms_ref ? h->n_atoms_ref : h->NA; }

namespace {


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

}  // namespace

int cmd::check_handle(cmd_handle* h, bool need_state) {
    if (!h) return fail(CMD_ERR_INVALID_ARG, "NULL handle");
    if (need_state && !h->has_state) return fail(CMD_ERR_STATE, "spins not set (call cmd_set_spins first)");
    return CMD_OK;
}

namespace {


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
    release_stream_graph(h);
    for (DevBuf* b : {&h->state, &h->nbr, &h->obs, &h->traj, &h->batch_states, &h->batch_out,
                      &h->pulses, &h->scratch, &h->dframes, &h->dafm, &h->times, &h->drive, &h->raw,
                      &h->tune_states, &h->tune_obs, &h->gwork, &h->gmeta, &h->gstat, &h->grows, &h->gqueue,
                      &h->awork, &h->ackpt, &h->aseg, &h->amloc, &h->aout, &h->ameta, &h->ain,
                      &h->sbuf, &h->spart, &h->sgpart, &h->snbase, &h->chunk_states, &h->chunk_rows, &h->cnbr2, &h->cnbr4, &h->cnbr8, &h->cnbr16, &h->cnbr_all, &h->cpush})
        b->release();
    h->hstage.release();
    for (cudaStream_t s2 : h->aux_streams) cudaStreamSynchronize(s2);
    for (cudaEvent_t e2 : h->aux_events) cudaEventDestroy(e2);
    for (cudaStream_t s2 : h->aux_streams) cudaStreamDestroy(s2);
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
    // Rows and final states: device -> page-locked staging (one asynchronous copy
    // each), then into the caller's arrays on a few host threads; where the
    // staging cannot be had, straight into the caller's arrays.
    std::vector<size_t> hoff(B), foff(B);
    size_t hs_total = 0;
    for (int64_t b = 0; b < B; ++b) {
        cmd_traj_spec& sp = specs[b];
        for (int q = 0; q < 4; ++q) sp.stats[q] = stats[4 * b + q];
        overflow |= sp.stats[0] > sp.max_rows;
        hoff[b] = hs_total;
        hs_total += (size_t)std::min<int64_t>(sp.stats[0], sp.max_rows) * 11;
    }
    for (int64_t b = 0; b < B; ++b) {
        foff[b] = hs_total;
        if (specs[b].final_state) hs_total += (size_t)specs[b].lattice->N * 3;
    }
    const bool staged = owner->hstage.ensure(std::max<size_t>(hs_total, 1) * sizeof(double)) == CMD_OK;
    cmd::clear_error();
    double* hst = staged ? owner->hstage.as<double>() : nullptr;
    for (int64_t b = 0; b < B; ++b) {
        cmd_traj_spec& sp = specs[b];
        const int64_t n = std::min<int64_t>(sp.stats[0], sp.max_rows);
        CUDA_TRY(cudaMemcpyAsync(staged ? hst + hoff[b] : sp.rows, drows + roff[b], n * 11 * sizeof(double),
                                 cudaMemcpyDeviceToHost, owner->stream));
        if (sp.final_state)
            CUDA_TRY(cudaMemcpyAsync(staged ? hst + foff[b] : sp.final_state, dout + ioff[b],
                                     sp.lattice->N * 3 * sizeof(double), cudaMemcpyDeviceToHost, owner->stream));
    }
    if (int rc = sync(owner)) return rc;
    if (staged) {
        const int nt = (int)std::max<int64_t>(1, std::min<int64_t>(B, 8));
        auto part = [&](int k) {
            for (int64_t b = k; b < B; b += nt) {
                cmd_traj_spec& sp = specs[b];
                const int64_t n = std::min<int64_t>(sp.stats[0], sp.max_rows);
                std::memcpy(sp.rows, hst + hoff[b], (size_t)n * 11 * sizeof(double));
                if (sp.final_state)
                    std::memcpy(sp.final_state, hst + foff[b], (size_t)sp.lattice->N * 3 * sizeof(double));
            }
        };
        std::vector<std::thread> pool;
        for (int k = 1; k < nt; ++k) pool.emplace_back(part, k);
        part(0);
        for (std::thread& t : pool) t.join();
    }
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

}  // namespace
}  // extern "C"

int cmd::validate_batch(const cmd_handle* h, const cmd_batch_desc* d) {
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

extern "C" {
namespace {


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

extern "C" {

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
    const Variant& V = variant_table()[vi];
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
    const Variant& V = variant_table()[vi];
    variant_shape(V, h->lay, &info[3], &info[5]);
    info[4] = V.CPT;
    return CMD_OK;
}

int cmd_variant_count(void) { return variant_count(); }

int cmd_variant_info(cmd_handle* h, int32_t idx, char* name, int32_t name_len, int32_t* fits) {
    cmd::clear_error();
    if (idx < 0 || idx >= variant_count()) return fail(CMD_ERR_INVALID_ARG, "variant index out of range");
    if (name && name_len > 0) {
        std::strncpy(name, variant_table()[idx].name, (size_t)name_len - 1);
        name[name_len - 1] = 0;
    }
    if (fits) *fits = (h && variant_fits(variant_table()[idx], h->lay)) ? 1 : 0;
    return CMD_OK;
}

int cmd_set_variant(cmd_handle* h, int32_t idx) {
    cmd::clear_error();
    if (int rc = check_handle(h, false)) return rc;
    if (idx < -1 || idx >= variant_count()) return fail(CMD_ERR_INVALID_ARG, "variant index out of range");
    if (idx >= 0 && !variant_fits(variant_table()[idx], h->lay))
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
// fastest.  ms[variant_count()] (may be NULL) gets the times, -1 for variants that
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
    for (int i = 0; i < variant_count() && rc == CMD_OK; ++i) {
        if (ms) ms[i] = -1.0;
        if (!variant_fits(variant_table()[i], h->lay)) continue;
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

int cmd_set_graphs(cmd_handle* h, int32_t enable) {
    cmd::clear_error();
    if (int rc = check_handle(h, false)) return rc;
    h->graphs = enable != 0;
    if (!h->graphs) release_stream_graph(h);
    return CMD_OK;
}

int cmd_rk45_variant_count(void) { return rk45_variant_count(); }

int cmd_rk45_variant_info(cmd_handle* h, int32_t idx, char* name, int32_t name_len, int32_t* fits) {
    cmd::clear_error();
    if (idx < 0 || idx >= rk45_variant_count()) return fail(CMD_ERR_INVALID_ARG, "tiling index out of range");
    if (name && name_len > 0) {
        std::strncpy(name, rk45_variant_name(idx), (size_t)name_len - 1);
        name[name_len - 1] = 0;
    }
    if (fits) *fits = (h && rk45_fits(idx, h->lay)) ? 1 : 0;
    return CMD_OK;
}

int cmd_set_rk45_variant(cmd_handle* h, int32_t idx) {
    cmd::clear_error();
    if (int rc = check_handle(h, false)) return rc;
    if (idx < -2 || idx >= rk45_variant_count()) return fail(CMD_ERR_INVALID_ARG, "tiling index out of range");
    if (idx >= 0 && !rk45_fits(idx, h->lay))
        return fail(CMD_ERR_UNSUPPORTED, std::string(rk45_variant_name(idx)) + " does not hold this lattice");
    h->rk45_variant = idx;
    return CMD_OK;
}

int cmd_get_rk45_variant(cmd_handle* h, int32_t* idx) {
    cmd::clear_error();
    if (int rc = check_handle(h, false)) return rc;
    if (!idx) return fail(CMD_ERR_INVALID_ARG, "NULL output");
    const int v = rk45_pick(h);
    *idx = v < 0 ? -2 : v;
    return CMD_OK;
}

int cmd_autotune_rk45(cmd_handle* h, int64_t B, int64_t n_steps, int32_t* best, double* ms) {
    cmd::clear_error();
    if (int rc = check_handle(h, true)) return rc;
    if (B <= 0 || B > (1 << 20) || n_steps <= 0) return fail(CMD_ERR_INVALID_ARG, "bad autotune size");
    const int64_t max_rows = n_steps + 2, N3 = h->N * 3;
    if (int rc = h->tune_obs.ensure((size_t)B * (max_rows * 11 + N3) * sizeof(double))) return rc;
    double* rows = h->tune_obs.as<double>();
    double* yout = rows + B * max_rows * 11;
    std::vector<GJob> jobs(B);
    for (int64_t b = 0; b < B; ++b) {
        GJob& j = jobs[b];
        j.h = h;
        j.y0 = h->state.as<double>();
        j.yout = yout + b * N3;
        j.rows = rows + b * max_rows * 11;
        j.max_rows = max_rows;
        j.T0 = 0.0;
        j.T1 = 1e300;
        j.dt0 = 0.01;
    }
    const int saved = h->rk45_variant;
    int win = -1;
    double best_ms = 0.0;
    int rc = CMD_OK;
    for (int i = 0; i < rk45_variant_count() && rc == CMD_OK; ++i) {
        if (ms) ms[i] = -1.0;
        if (!rk45_fits(i, h->lay)) continue;
        h->rk45_variant = i;
        double t = 0.0;
        std::vector<long long> stats;
        for (int rep = 0; rep < 3 && rc == CMD_OK; ++rep) {     // first run warms up, best of the other two
            const auto t0 = std::chrono::steady_clock::now();
            rc = run_global(h, jobs, kModeRK45, h->abs_tol, h->rel_tol, n_steps, stats);
            const double tr = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            if (rep == 1 || (rep > 1 && tr < t)) t = tr;
        }
        if (rc != CMD_OK) break;
        if (ms) ms[i] = t;
        if (win < 0 || t < best_ms) { win = i; best_ms = t; }
    }
    h->rk45_variant = saved;
    if (rc != CMD_OK) return rc;
    if (win < 0) return fail(CMD_ERR_UNSUPPORTED, "no on-chip RK45 tiling holds this lattice");
    h->rk45_variant = win;
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

