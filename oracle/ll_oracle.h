/*
 * ll_oracle.h -- CPU restatement of the reference Landau-Lifshitz MD path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it.
 * The product (classical_mcmc_spin_b200) never links or calls it.
 *
 * What it restates (reference = ze-bang/Classical_MCMC_Spin, ClassicalSpin_Cpp):
 *   - UnitCell / builders   include/classical_spin/core/unitcell.h:102-356,
 *                           src/core/unitcell_builders.cpp:178-283 (Kitaev),
 *                           :370-471 (non-Kramers pyrochlore)
 *   - Lattice bond tables   include/classical_spin/lattice/lattice.h:601-855
 *                           (neighbour order, reverse J^T, periodic wrap),
 *                           :868-903 (flat CSR), :1057-1059 (site index)
 *   - RHS                   src/core/lattice_md.cpp:39-103 (SU(2) branch),
 *                           :178-191 (drive), :210-224 (set_pulse, R*B)
 *                           lattice.h:1653-1711 (get_local_field_flat)
 *   - Energy                lattice.h:1485-1555 (total_energy_flat)
 *   - Magnetisations        lattice.h:4461-4512, lattice_md.cpp:383-436
 *   - Time stepping         lattice.h:4014-4084 -> Boost.Odeint (third party,
 *                           version unpinned: CMakeLists.txt:74 asks for
 *                           Boost >= 1.65, not vendored).  Restated from the
 *                           published algorithms: classic RK4 and the
 *                           Dormand-Prince 5(4) pair with odeint's default
 *                           error checker / step adjuster and its
 *                           integrate_const / integrate_adaptive drivers.
 *   - GPU-API time loop     include/classical_spin/gpu/ode/integrator.cuh:470-488
 *                           (t += dt while t < T_end), lattice_gpu.cu:557
 *   - Pulse segmentation    include/classical_spin/lattice/pulse_chunking.h:82-161
 *
 * Parity status: the reference CPU path needs Eigen3, Boost, HDF5 and MPI and
 * cannot be built here, and the reference ships no golden vectors for this
 * path.  This restatement is pinned against (a) the reference's own GPU
 * integrator (src/gpu/lattice_gpu.cu, which compiles standalone) built into
 * oracle/_ref and run on a B200, whose outputs are committed as fixtures under
 * tests/golden/, and (b) the reference's pulse_chunking.h compiled directly.
 */
#ifndef LL_ORACLE_H
#define LL_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORA_MAX_ATOMS 32
#define ORA_MAX_BONDS 512

/* One UnitCell::bilinear_interaction entry (unitcell.h:14-30). */
typedef struct ora_bond {
    int src, dst;
    int off[3];
    double J[9];          /* row-major 3x3 */
} ora_bond;

/* UnitCell restricted to spin_dim = 3 (unitcell.h:102-239). */
typedef struct ora_unitcell {
    int n_atoms;
    double pos[ORA_MAX_ATOMS * 3];
    double lattice_vectors[9];
    double field[ORA_MAX_ATOMS * 3];
    double onsite[ORA_MAX_ATOMS * 9];
    double frames[ORA_MAX_ATOMS * 9];
    double afm[ORA_MAX_ATOMS];
    int n_bonds;          /* insertion order; multimap order per source atom */
    ora_bond bonds[ORA_MAX_BONDS];
} ora_unitcell;

typedef struct ora_lattice ora_lattice;

/* Builders.  kp = {K, Gamma, Gammap, J, J2_A, J2_B, J3, J_perp, Ka, Kb, Kc}. */
void ora_uc_kitaev(const double* kp, double h, const double* dir, const double* g,
                   ora_unitcell* uc);
/* pp = {Jpm, Jzz, Jpmpm, J2, delta1, delta2}. */
void ora_uc_pyrochlore_nk(const double* pp, double h, const double* dir, ora_unitcell* uc);
/* 16-site conventional cubic cell built from the primitive non-Kramers cell. */
void ora_uc_pyrochlore_nk_cubic(const double* pp, double h, const double* dir, ora_unitcell* uc);

ora_lattice* ora_lattice_create(const ora_unitcell* uc, int d1, int d2, int d3);
void   ora_lattice_destroy(ora_lattice* L);
size_t ora_lattice_size(const ora_lattice* L);
size_t ora_lattice_nnz(const ora_lattice* L);
int    ora_lattice_max_bilinear(const ora_lattice* L);
/* Flat CSR mirror (lattice.h:868-903): offsets[N+1], partners[nnz], J[nnz*9]. */
void ora_lattice_csr(const ora_lattice* L, int64_t* offsets, int64_t* partners, double* J);
/* Reference GPU-boundary ELL arrays (lattice.h:5441-5487). */
void ora_lattice_ell(const ora_lattice* L, double* field, double* onsite, double* bilinear,
                     int64_t* partners, int64_t* counts);
void ora_lattice_frames(const ora_lattice* L, double* frames, double* afm);

/* Drive (lattice_md.cpp:210-224): field_in1/2 [n_atoms*3] in the global frame. */
void ora_set_pulse(ora_lattice* L, const double* field_in1, double t1,
                   const double* field_in2, double t2, double amp, double width, double freq);
void ora_clear_pulse(ora_lattice* L);
void ora_set_gilbert(ora_lattice* L, double alpha);
void ora_set_threads(int n);

void   ora_rhs(const ora_lattice* L, const double* state, double t, double* dsdt);
void   ora_local_field(const ora_lattice* L, const double* state, double* H);
double ora_energy(const ora_lattice* L, const double* state);
/* out[9] = {M_af(3), M_local(3), M_global(3)}, each divided by N. */
void   ora_magnetizations(const ora_lattice* L, const double* state, double* out);
double ora_max_dsdt_no_drive(ora_lattice* L, const double* state);

/* One classic RK4 step (odeint runge_kutta4). */
void ora_rk4_step(const ora_lattice* L, double* state, double t, double dt);
/* One step of the reference GPU stepper (integrator.cuh:115-139 arithmetic). */
void ora_rk4_step_gpu_form(const ora_lattice* L, double* state, double t, double dt);

/*
 * Fixed-step RK4 driven like odeint integrate_const (t_k = T0 + k*dt).
 * Observer at every step; records {t, M_af, M_loc, M_glob, E} rows (11
 * doubles) when (observer_call % save_interval == 0).  Returns rows written
 * (at most max_rows).  state is advanced in place.
 */
long ora_md_rk4_const(const ora_lattice* L, double* state, double T0, double T1, double dt,
                      long save_interval, double* rows, long max_rows);
/* Same arithmetic, reference GPU-API time loop (t += dt while t < T1). */
long ora_md_rk4_gpu_loop(const ora_lattice* L, double* state, double T0, double T1, double dt,
                         long save_interval, double* rows, long max_rows);

/*
 * Controlled Dormand-Prince 5(4) driven like odeint integrate_adaptive.
 * Records a row at every observer call (each accepted step + start + end).
 * stats[0] = accepted, stats[1] = rejected, stats[2] = RHS evaluations.
 * Returns rows written, or -1 if more than 500 consecutive rejections.
 */
long ora_md_dopri5_adaptive(const ora_lattice* L, double* state, double T0, double T1,
                            double dt0, double abs_tol, double rel_tol, long max_accepted,
                            double* rows, long max_rows, long* stats);
/* Controlled Dormand-Prince driven like odeint integrate_const (observer grid). */
long ora_md_dopri5_const(const ora_lattice* L, double* state, double T0, double T1,
                         double dt, double abs_tol, double rel_tol,
                         double* rows, long max_rows, long* stats);

/* pulse_chunking.h:82-161; segs gets {t0, t1, dt_init} triples, returns count. */
int ora_pulse_segments(double T_start, double T_end, const double* centers, int n_centers,
                       double window, double T_step, double free_dt_factor,
                       double* segs, int max_segs);

/*
 * single/double_pulse_drive CPU semantics (lattice_md.cpp:493-680).  rows get
 * {t, M_af, M_loc, M_glob} (10 doubles).  method: 0 = rk4, 1 = dopri5.
 */
long ora_pulse_drive(ora_lattice* L, const double* state0, const double* field_in1, double t1,
                     const double* field_in2, double t2, int n_pulses, double amp,
                     double width, double freq, double T0, double T1, double step,
                     int method, int chunking, double abs_tol, double rel_tol,
                     double* rows, long max_rows);

/* ---- CPU baseline timing helpers (OpenMP) ---- */
/* Batched RK4 over B independent trajectories of the same lattice, each with its
 * own pulse pair (t1[b], t2[b], s1[b], s2[b] amplitude scales).  Trajectory-
 * parallel like the reference's W2 loop (lattice_md.cpp:809-904).  Writes final
 * states in place and obs [B][nsteps+1][10] = {M_af, M_loc, M_glob, E}. */
void ora_batch_rk4(const ora_lattice* L, double* states, int B, const double* t1,
                   const double* t2, const double* s1, const double* s2, double amp,
                   double width, double freq, const double* dir1, const double* dir2,
                   double T0, double dt, long nsteps, double* obs, int with_energy);

/* ---- gradient references for the discrete adjoint (tests only) ----
 * Loss L = sum_{r=0..nsteps} |M_local(y_r) - target_r|^2 over the GPU-form RK4
 * trajectory (t_r accumulated, t += dt) from state0 under L's couplings and
 * drive.  dparam[q] are lattices with the same bond tables built at theta = e_q:
 * their coupling entries are dJ/dtheta_q and their fields dB/dtheta_q.
 * Forward-mode tangent linear model: grad[q] = dL/dtheta_q.  Returns L. */
double ora_loss_grad_tlm(const ora_lattice* L, const ora_lattice* const* dparam, int nq,
                         const double* state0, double T0, double dt, long nsteps,
                         const double* target, double* grad);
/* The loss alone (for finite differences). */
double ora_loss(const ora_lattice* L, const double* state0, double T0, double dt, long nsteps,
                const double* target);

#ifdef __cplusplus
}
#endif
#endif
