/*
 * cmd.h -- C ABI of the B200 Landau-Lifshitz molecular-dynamics path.
 *
 * Drop-in replacement for the reference's host-side GPU boundary
 * `namespace gpu` in include/classical_spin/gpu/lattice_gpu_api.h
 * (ze-bang/Classical_MCMC_Spin).  That header passes std::vector / std::string
 * and an opaque C++ handle; this one takes plain pointers and sizes, returns an
 * int status from every call and never lets an exception cross the boundary.
 *
 * Conventions
 *   - spin_dim is 3 (SU(2) spins); state arrays are the reference's flat
 *     layout [site*3 + component], sites ordered ((i*d2+j)*d3+k)*n_atoms+atom.
 *   - All numbers are FP64.
 *   - A handle is not thread safe; different handles may be driven from
 *     different host threads.  Each handle owns one CUDA stream.
 *   - Observable rows are 10 doubles: {M_af[3], M_local[3], M_global[3], E/N}
 *     with every magnetisation divided by N (the reference observers'
 *     normalisation, src/core/lattice_md.cpp:406-422) and E/N the energy per
 *     site of the static Hamiltonian (lattice.h:1485 total_energy_flat / N).
 */
#ifndef CMD_H
#define CMD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes (the reference throws std::runtime_error or silently no-ops,
 * lattice_gpu.cu:660-723 and gpu_common_helpers.cuh:15-32). */
enum {
    CMD_OK = 0,
    CMD_ERR_INVALID_ARG = 1,
    CMD_ERR_UNSUPPORTED = 2,
    CMD_ERR_CUDA = 3,
    CMD_ERR_NONFINITE = 4,
    CMD_ERR_WATCHDOG = 5,
    CMD_ERR_OOM = 6,
    CMD_ERR_STATE = 7
};

/* Integration methods.  The reference GPU API takes a method string
 * (lattice_gpu_api.h:101-125); "rk4" and "dopri5" are the ones on this path.
 *   CMD_RK4          classic fixed-step RK4 (integrator.cuh:115-139)
 *   CMD_DOPRI5_FIXED Dormand-Prince 5 tableau, fixed step, no error control
 *                    (the reference GPU "dopri5", integrator.cuh:186-228)
 *   CMD_RK45         controlled Dormand-Prince 5(4) with the CPU path's
 *                    Boost.Odeint step control (lattice.h:4072-4078)
 *   CMD_CASH_KARP_FIXED  Cash-Karp 5 tableau, fixed step (the reference GPU
 *                    "rk5" / "rkck54", integrator.cuh:141-185)
 * and the reference GPU's other fixed-step methods, same tableaux:
 *   CMD_EULER        "euler" (integrator.cuh:91-99)
 *   CMD_MIDPOINT     "rk2" / "midpoint" (integrator.cuh:100-114)
 *   CMD_SSPRK53      "ssprk53", five-stage third-order SSP RK, the reference
 *                    GPU API's default method (integrator.cuh:406-448)
 *   CMD_RK78         "rk78" / "rkf78": the first 11 Fehlberg 7(8) stages with
 *                    the 7th-order weights (integrator.cuh:230-370)
 *   CMD_BULIRSCH_STOER  "bulirsch_stoer" / "bs": modified midpoint over four
 *                    substeps plus smoothing, no extrapolation
 *                    (integrator.cuh:371-405)
 * ("rk54" / "rkf54" is CMD_DOPRI5_FIXED, integrator.cuh:450-452.)          */
enum {
    CMD_RK4 = 0, CMD_DOPRI5_FIXED = 1, CMD_RK45 = 2, CMD_CASH_KARP_FIXED = 3,
    CMD_EULER = 4, CMD_MIDPOINT = 5, CMD_SSPRK53 = 6, CMD_RK78 = 7, CMD_BULIRSCH_STOER = 8
};

typedef struct cmd_handle cmd_handle;

/*
 * Lattice in the reference's flattened GPU-boundary form
 * (create_gpu_lattice_data, lattice_gpu_api.h:47-57; filled by
 * Lattice::ensure_gpu_data_initialized, lattice.h:5429-5497), plus the
 * sublattice frames and AFM signs that the reference passes separately to
 * integrate_gpu_batched (lattice_gpu_api.h:205-214).
 */
typedef struct cmd_lattice_desc {
    int64_t lattice_size;        /* N                                          */
    int32_t spin_dim;            /* must be 3                                  */
    int32_t n_atoms;             /* atoms per unit cell                        */
    int32_t max_bilinear;        /* ELL width                                  */
    int32_t reserved;
    const double* field;         /* [N*3]                                      */
    const double* onsite;        /* [N*9]                                      */
    const double* bilinear;      /* [N*max_bilinear*9] row-major J per entry   */
    const int64_t* partners;     /* [N*max_bilinear]                           */
    const int64_t* counts;       /* [N] valid entries per site                 */
    const double* frames;        /* [n_atoms*9] or NULL (identity)             */
    const double* afm_signs;     /* [n_atoms]   or NULL (all +1)               */
} cmd_lattice_desc;

/* create_gpu_lattice_data (lattice_gpu_api.h:47-57). */
int cmd_create(const cmd_lattice_desc* desc, cmd_handle** out);
/* destroy_gpu_lattice_data (lattice_gpu_api.h:62). */
int cmd_destroy(cmd_handle* h);

/* set_gpu_pulse (lattice_gpu_api.h:67-75): field_drive [2*n_atoms*3], already
 * rotated by the sublattice frames (Lattice::set_pulse, lattice_md.cpp:210-224). */
int cmd_set_pulse(cmd_handle* h, const double* field_drive, double amp, double width,
                  double freq, double t_pulse_1, double t_pulse_2);

/* set_gpu_spins / get_gpu_spins (lattice_gpu_api.h:83-97); n = N*3. */
int cmd_set_spins(cmd_handle* h, const double* spins, int64_t n);
int cmd_get_spins(cmd_handle* h, double* spins, int64_t n);

/* step_gpu (lattice_gpu_api.h:135-140): one step of `method` from time t. */
int cmd_step(cmd_handle* h, double t, double dt, int method);

/*
 * integrate_gpu (lattice_gpu_api.h:117-125).  Fixed-step methods follow the
 * reference loop: t = T0; while (t < T1) { if (k % save_interval == 0) save;
 * step; t += dt; ++k; } save.  CMD_RK45 follows the CPU controller and saves
 * every accepted step (dt is the initial step, tolerances from
 * cmd_set_tolerances).  Per saved row: times[r], obs[r*10..], and, when
 * `states` is non-NULL, the full state states[r*N*3..] (the reference's
 * trajectory vector).  *rows_out gets the number of rows; CMD_ERR_INVALID_ARG
 * if max_rows is too small (rows_out still gets the count needed).
 */
int cmd_integrate(cmd_handle* h, double T0, double T1, double dt, int64_t save_interval,
                  int method, double* times, double* obs, double* states, int64_t max_rows,
                  int64_t* rows_out);

/* Controlled-stepper tolerances (SpinConfig md_abs_tol / md_rel_tol) and the
 * accepted-step cap for CMD_RK45. */
int cmd_set_tolerances(cmd_handle* h, double abs_tol, double rel_tol, int64_t max_steps);

/* compute_energy_gpu (lattice_gpu_api.h:145; unimplemented in the reference):
 * total energy of the current state, same terms as total_energy_flat. */
int cmd_energy(cmd_handle* h, double* energy);

/* normalize_spins_gpu (lattice_gpu_api.h:150). */
int cmd_normalize(cmd_handle* h, double spin_length);

/* compute_magnetization_gpu (lattice_gpu_api.h:155-159): mean spin and the
 * (-1)^i staggered mean (lattice_gpu.cu:729-760), each [3]. */
int cmd_magnetization(cmd_handle* h, double* mag_local, double* mag_staggered);

/* Lattice::max_dSdt_norm_no_drive (lattice_md.cpp:235-279): the largest
 * component |dS/dt| of the current state with the drive off -- the
 * stationarity check that gates reusing M0 for M1(tau) in 2DCS. */
int cmd_max_dsdt_no_drive(cmd_handle* h, double* out);

/* Observables of the current state: one 10-double row (see top of file). */
int cmd_observables(cmd_handle* h, double* row);

/*
 * integrate_gpu_batched (lattice_gpu_api.h:171-214): B replicas of this
 * lattice from one initial state, replica b with second-pulse time tau2[b]
 * and every other pulse parameter from cmd_set_pulse.  Loop:
 * while (t < T1 - 1e-12), saving every save_interval steps and at the end.
 * mags[r][b][m][d] (m = 0 M_af, 1 M_local, 2 M_global), each / N.
 * afm_signs / frames may be NULL to use the lattice's own.
 */
int cmd_integrate_batched(cmd_handle* h, const double* initial_state, const double* tau2,
                          int64_t B, const double* afm_signs, const double* frames,
                          double T0, double T1, double dt, int64_t save_interval,
                          int method, double* times, double* mags, int64_t max_rows,
                          int64_t* rows_out);

/*
 * Generalised batch (no reference counterpart; it is the batched 2DCS scan
 * with pump-only / probe-only / pump+probe trajectories in one launch).
 * Trajectory b starts from states[b] (or from states[0] for every b when
 * shared_initial != 0), with drive
 *   H -= a1[b] env(t - t1[b]) d1 + a2[b] env(t - t2[b]) d2,
 *   env(x) = exp(-(x / (2 width))^2) cos(freq x)
 * where d1/d2 are the frame-rotated pulse directions [n_atoms*3] (NULL: no
 * drive).  RK4, `n_steps` steps of dt from T0 (t += dt), one row of obs every
 * `save_interval` steps plus the final state: obs[b][row][10].  Final states
 * are written back into `final_states` when non-NULL.  Host pointers.
 */
typedef struct cmd_batch_desc {
    int64_t B;
    const double* states;        /* [B or 1][N*3]                              */
    int32_t shared_initial;
    int32_t method;              /* CMD_RK4                                    */
    const double* t1; const double* t2;   /* [B]                               */
    const double* a1; const double* a2;   /* [B] pulse amplitudes              */
    const double* d1; const double* d2;   /* [n_atoms*3] or NULL               */
    double width, freq;
    double T0, dt;
    int64_t n_steps, save_interval;
    double* obs;                 /* [B][rows][10]; rows = n_steps/save + 1 (+1 if n_steps%save) */
    double* final_states;        /* [B][N*3] or NULL                           */
    const double* pulse4;        /* cmd_run_batch_device only: device [B][4] =
                                    {t1, t2, a1, a2} (t1..a2 above are unused) */
} cmd_batch_desc;
int cmd_run_batch(cmd_handle* h, const cmd_batch_desc* d);
/* Rows cmd_run_batch writes per trajectory. */
int64_t cmd_batch_rows(int64_t n_steps, int64_t save_interval);

/*
 * Device-resident variant of cmd_run_batch for callers that keep their data
 * on the GPU (the torch layer, the benchmark): states, obs, final_states and
 * pulse4 are device pointers; d1/d2 stay host arrays (they become kernel
 * parameters).  The call is asynchronous on `stream` (a cudaStream_t, NULL =
 * the handle's stream).  `launches` (may be NULL) gets the number of kernels
 * launched.
 */
int cmd_run_batch_device(cmd_handle* h, const cmd_batch_desc* d, void* stream, int32_t* launches);

/*
 * Allocation-free variant of cmd_run_batch_device.  It has no counterpart in
 * the reference.  It is for callers that cannot call cudaMalloc: their device
 * memory already belongs to another allocator (a caching allocator that has
 * reserved the GPU, a pre-partitioned serving pool), or they run loops that
 * cannot take the device-wide synchronisation cudaMalloc / cudaFree may imply.
 * Same arguments and results as cmd_run_batch_device, for resident lattices
 * only (those one CTA or a 2- or 4-CTA cluster holds: cmd_layout_info reports
 * the path); a lattice that needs the streamed kernels is rejected with
 * CMD_ERR_UNSUPPORTED, and cmd_run_batch_device runs it.
 * The scratch that cmd_run_batch_device allocates on demand lives here in one
 * static device array of 2^22 doubles (32 MiB).  It is part of the library's
 * device module, which is loaded (and the 32 MiB taken) at cmd_create at the
 * latest; every GPU that loads it holds it until the process exits:
 *     scratch doubles = [driven] n_steps + B*n_steps*6
 *                     + [cells of more than 3 atoms] B*rows*(3*atoms+1)
 * (each term rounded up to a multiple of 32).  A batch needing more is
 * rejected with CMD_ERR_INVALID_ARG; split it into smaller batches.
 * The call allocates no device memory: cmd_create looks up the array's device
 * address (cudaGetSymbolAddress) with the handle's device current and keeps it
 * in the handle, so call this with the handle's device current.  Every call
 * shares the one array, so calls whose work overlaps on the GPU (other
 * streams, other handles, other threads) race: order them on one stream, or
 * synchronise between them.  Everything a call reads from the array it first
 * writes itself, so nothing carries over between calls.
 */
int cmd_run_batch_device_noalloc(cmd_handle* h, const cmd_batch_desc* d, void* stream, int32_t* launches);

/*
 * 2DCS analysis step (restates util/readers_new/reader_honeycomb.py:459-553,
 * which the reference runs offline after pump_probe_spectroscopy).  Inputs are
 * host arrays of one magnetisation kind (the reader uses M_local): M0 [n_t][3]
 * (pump only), M1 and M01 [n_tau][n_t][3] (probe only, pump + probe at delay
 * tau_k).  For component `component`:
 *   m_nl[k][t]     = M01[k][t] - M0[t] - M1[k][t]
 *   spectrum[k][t] = | fftshift(fft2(m_nl - mean(m_nl))) | with the omega_t
 *                    axis flipped, axes (omega_tau, omega_t) as in the reader.
 * The 2-D FFT runs on the device (cuFFT); either output may be NULL.
 */
int cmd_nonlinear_spectrum(const double* M0, const double* M1, const double* M01, int64_t n_tau, int64_t n_t,
                           int32_t component, double* m_nl, double* spectrum);

/* Lattice layout chosen at cmd_create (for diagnostics and the autotuner):
 * info[0] = sites per group (unit-cell atoms), info[1] = groups,
 * info[2] = max bonds per site kept, info[3] = threads per block of the
 * resident RK4 kernel, info[4] = groups per thread, info[5] = shared-memory
 * bytes per trajectory. */
int cmd_layout_info(cmd_handle* h, int64_t* info);

/*
 * Uneven batch (no reference counterpart): trajectories on different lattices
 * (different sizes, and up to two unit-cell types, e.g. Kitaev honeycomb and
 * non-Kramers pyrochlore) in one call.  Controlled RK45 runs each lattice's
 * trajectories on the on-chip Dormand-Prince kernel with that handle's tiling
 * (cmd_set_rk45_variant / cmd_autotune_rk45), the lattices' launches running
 * concurrently; everything else runs in one persistent launch that pulls
 * trajectories from a work queue, longest first.  Lattices of one unit-cell
 * type must share their couplings, pulse directions, width and frequency
 * (cmd_set_pulse).  The rows and final states come back through a page-locked
 * host buffer held by the first spec's handle (as large as the rows returned;
 * kept for later calls and freed by cmd_destroy).
 * method: CMD_RK45 (controlled, T0..T1 from dt, tolerances below, at most
 * max_steps accepted steps when > 0; a row after every accepted step) or
 * CMD_RK4 / CMD_DOPRI5_FIXED (fixed dt, reference loop, a row every step).
 * Host pointers.  stats: rows produced (may exceed max_rows: then only
 * max_rows are written and the call returns CMD_ERR_INVALID_ARG), accepted
 * steps, rejected steps, status (0 ok, 1 step-size control failed).
 */
typedef struct cmd_traj_spec {
    cmd_handle* lattice;
    const double* state;         /* [N*3] initial spins                          */
    double T0, T1, dt;
    double t1, t2, a1, a2;       /* pulse pair; a1 = a2 = 0: no drive            */
    double* rows;                /* [max_rows][11] = {t, M_af, M_local, M_global, E/N} */
    int64_t max_rows;
    double* final_state;         /* [N*3] or NULL                                */
    int64_t stats[4];
} cmd_traj_spec;
int cmd_run_uneven(cmd_traj_spec* specs, int64_t B, int method, double abs_tol, double rel_tol,
                   int64_t max_steps);

/*
 * Discrete adjoint of the RK4 trajectory (no reference counterpart; the
 * reference has no gradients).  For each of B initial states, RK4 (the
 * reference GPU stepper's arithmetic, t += dt) for n_steps steps from T0 under
 * h's couplings and pulse, and the loss
 *     L_b = sum_{n=0..n_steps} |M_local(t_n) - target_b[n]|^2,
 * with its gradient with respect to n_params (<= 5) coupling parameters.  The
 * couplings must depend linearly on the parameters; parameter q is described
 * by the lattice built with theta = e_q (same bond tables as h's lattice):
 * its couplings are dJ/dtheta_q, its field dB/dtheta_q, its onsite terms
 * dA/dtheta_q.  Checkpoints every checkpoint_every steps (0: ~sqrt(n_steps));
 * the backward sweep recomputes each segment.  forward_only != 0 runs only the
 * forward pass (loss, m_local; grad untouched).  Host pointers.
 * path: CMD_ADJ_AUTO picks the resident kernel (one CTA or one thread-block
 * cluster per trajectory, state on chip) when one holds the lattice, else one
 * CTA per trajectory with the state in global memory when the batch fills the
 * GPU, else streamed stages; the others force a path (CMD_ERR_UNSUPPORTED when
 * CMD_ADJ_RESIDENT does not fit).
 */
enum { CMD_ADJ_AUTO = 0, CMD_ADJ_RESIDENT = 1, CMD_ADJ_STREAMED = 2, CMD_ADJ_GLOBAL = 3 };
typedef struct cmd_adjoint_desc {
    int64_t B;
    const double* states;              /* [B][N*3]                               */
    double T0, dt;
    int64_t n_steps;
    const double* target;              /* [B][n_steps+1][3]                      */
    int64_t checkpoint_every;
    int32_t n_params;
    int32_t forward_only;
    const cmd_lattice_desc* dparams;   /* [n_params]                             */
    double* loss;                      /* [B] out                                */
    double* grad;                      /* [B][n_params] out                      */
    double* m_local;                   /* [B][n_steps+1][3] out, or NULL          */
    int32_t path;                      /* CMD_ADJ_*                               */
    int32_t reserved;
} cmd_adjoint_desc;
int cmd_adjoint_rk4(cmd_handle* h, const cmd_adjoint_desc* d);

/*
 * Autotuner over the resident-kernel variants compiled into the library
 * (cells per thread x threads per CTA x CTAs per SM x own stage input kept in
 * registers or re-read from shared memory).  No reference counterpart.
 *   cmd_variant_count     number of variants in the library
 *   cmd_variant_info      name of variant idx and whether it fits h's lattice
 *   cmd_set_variant       pin a variant for h (-1: back to the default choice)
 *   cmd_get_variant       variant h uses now
 *   cmd_autotune          time every fitting variant on a B-trajectory,
 *                         n_steps-step batch from h's current spins, pin the
 *                         fastest; ms[cmd_variant_count()] gets the times
 *                         (-1 for variants that do not fit), may be NULL
 */
int cmd_variant_count(void);
int cmd_variant_info(cmd_handle* h, int32_t idx, char* name, int32_t name_len, int32_t* fits);
int cmd_set_variant(cmd_handle* h, int32_t idx);
int cmd_get_variant(cmd_handle* h, int32_t* idx);
int cmd_autotune(cmd_handle* h, int64_t B, int64_t n_steps, int32_t* best, double* ms);

/*
 * CUDA graphs, on by default.  Streamed RK4 (lattices no resident kernel
 * holds; one launch per RK stage): the stage launches of a chunk of 128 steps
 * are captured once as a CUDA graph, kept in the handle and replayed, so a
 * 2x10^4-step run makes 157 graph launches instead of 8x10^4 kernel launches.
 * Batched resident runs (drive table, resident kernel, row finisher) and
 * uneven batches (the per-lattice launches on the handle's auxiliary streams,
 * forked from and joined to the call's stream): each call is captured and
 * launched as one graph, the handle's executable graph updated in place when
 * only arguments change.  Calls on a default stream launch directly.  The
 * library does not capture a stream that is already being captured; its calls
 * also upload host data (time grids, trajectory tables) with ordinary copies,
 * so they are not meant to be recorded into a caller's own graph.  The results
 * are the same with graphs on or off.  No
 * reference counterpart (the reference launches and synchronises every stage,
 * integrator.cuh:115-139).  enable = 0 launches everything directly.
 */
int cmd_set_graphs(cmd_handle* h, int32_t enable);

/*
 * Tilings of the on-chip controlled Dormand-Prince kernel (CMD_RK45 in
 * cmd_integrate and cmd_run_uneven): CTAs per trajectory (one CTA or a
 * thread-block cluster of 2..16) x threads per CTA x sites per thread, with y
 * and K1 in registers or shared memory ("yk") and partners in other CTAs read
 * remotely or pushed into halo columns ("halo").  No reference counterpart;
 * the reference's controlled stepper is the CPU path's Boost.Odeint
 * make_controlled<runge_kutta_dopri5> (lattice.h:4072-4078), which every
 * tiling follows step for step.
 *   cmd_rk45_variant_count  number of tilings in the library
 *   cmd_rk45_variant_info   name of tiling idx and whether it holds h's lattice
 *   cmd_set_rk45_variant    pin a tiling for h (-1: the default choice, the
 *                           smallest cluster that holds the lattice; -2: the
 *                           global-memory kernel, which holds any size)
 *   cmd_get_rk45_variant    tiling h uses now (-2: global-memory kernel)
 *   cmd_autotune_rk45       time every tiling that holds h's lattice on B
 *                           trajectories from h's current spins for n_steps
 *                           accepted steps at h's tolerances (cmd_set_tolerances;
 *                           one warm-up run, then the best of two), pin the
 *                           fastest; ms[cmd_rk45_variant_count()] gets the times
 *                           (-1 where a tiling does not fit), may be NULL
 */
int cmd_rk45_variant_count(void);
int cmd_rk45_variant_info(cmd_handle* h, int32_t idx, char* name, int32_t name_len, int32_t* fits);
int cmd_set_rk45_variant(cmd_handle* h, int32_t idx);
int cmd_get_rk45_variant(cmd_handle* h, int32_t* idx);
int cmd_autotune_rk45(cmd_handle* h, int64_t B, int64_t n_steps, int32_t* best, double* ms);

/* Host-only version of the layout analysis cmd_create performs (no CUDA
 * call): fills info[0..5] like cmd_layout_info, info[6] = leading local slots
 * per atom; returns CMD_ERR_UNSUPPORTED with the reason when no resident
 * kernel covers the lattice. */
int cmd_plan_layout(const cmd_lattice_desc* desc, int64_t* info);

/* Message for the last non-OK status on this host thread. */
const char* cmd_last_error(void);
/* Library version string. */
const char* cmd_version(void);

#ifdef __cplusplus
}
#endif
#endif
