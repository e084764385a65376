// noalloc.cu -- the allocation-free batch entry point and its static scratch.
#include "cmd_core.h"

#include <cstdio>

namespace cmd {

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

}  // namespace cmd

using namespace cmd;

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
    if (vi < 0 || !variant_fits(variant_table()[vi], h->lay)) {
        if (!h->lay.uniform) return no_instance(h->lay);
        return fail(CMD_ERR_UNSUPPORTED, "cmd_run_batch_device_noalloc runs resident lattices only (one CTA or a "
                                         "2- or 4-CTA cluster per trajectory); this lattice needs the streamed "
                                         "kernels: use cmd_run_batch_device");
    }
    const Variant& V = variant_table()[vi];
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

