/*
 * cmd_mixed.h -- C ABI of the B200 mixed SU(2) / SU(3) Landau-Lifshitz path,
 * the drop-in for the reference's host GPU API `namespace mixed_gpu`
 * (include/classical_spin/gpu/mixed_lattice_gpu_api.h:25-214 of
 * ze-bang/Classical_MCMC_Spin), implemented by libcmd_b200.so.
 *
 * The lattice: n_su2 SU(2) sites (3-component spins) and n_su3 SU(3) sites
 * (8-component Gell-Mann vectors), in the reference's flattened per-site ELL
 * form (MixedLattice's GPU upload).  The state is one vector: the SU(2) spins,
 * site-major, then the SU(3) spins, site-major (n_su2*3 + n_su3*8 doubles).
 * All functions return a cmd status (cmd.h); cmd_last_error() gives the text.
 * Host pointers throughout.
 */
#ifndef CMD_MIXED_H
#define CMD_MIXED_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct cmd_mixed cmd_mixed;

typedef struct cmd_mixed_desc {
    int64_t n_su2, n_su3;                  /* sites of each kind                        */
    int32_t spin_dim_su2, spin_dim_su3;    /* must be 3 and 8                           */
    int32_t n_atoms_su2, n_atoms_su3;      /* atoms per unit cell (drive, staggering)   */
    int32_t max_bilinear_su2, max_bilinear_su3;   /* ELL widths of like-site bonds      */
    int32_t max_mixed_su2, max_mixed_su3;         /* ELL widths of mixed bonds          */
    const double* field_su2;               /* [n_su2][3]                                */
    const double* onsite_su2;              /* [n_su2][9]                                */
    const double* bilinear_su2;            /* [n_su2][max_bilinear_su2][9]              */
    const int64_t* partners_su2;           /* [n_su2][max_bilinear_su2]                 */
    const int64_t* counts_su2;             /* [n_su2]                                   */
    const double* field_su3;               /* [n_su3][8]                                */
    const double* onsite_su3;              /* [n_su3][64]                               */
    const double* bilinear_su3;            /* [n_su3][max_bilinear_su3][64]             */
    const int64_t* partners_su3;
    const int64_t* counts_su3;
    const double* mixed_su2;               /* [n_su2][max_mixed_su2][3*8], row-major     */
    const int64_t* mixed_partners_su3;     /* [n_su2][max_mixed_su2] SU(3) partner       */
    const int64_t* mixed_counts_su2;       /* [n_su2]                                   */
    const double* mixed_su3;               /* [n_su3][max_mixed_su3][8*3], row-major     */
    const int64_t* mixed_partners_su2;     /* [n_su3][max_mixed_su3] SU(2) partner       */
    const int64_t* mixed_counts_su3;       /* [n_su3]                                   */
} cmd_mixed_desc;

/* create_gpu_mixed_lattice_data (mixed_lattice_gpu_api.h:66-90).  Partners
 * outside the lattice are skipped, as in the reference's local fields
 * (mixed_lattice_gpu.cu:92-118, 157-185). */
int cmd_mixed_create(const cmd_mixed_desc* desc, cmd_mixed** out);
/* destroy_gpu_mixed_lattice_data (:92). */
int cmd_mixed_destroy(cmd_mixed* h);

/* set_gpu_pulse_SU2 / set_gpu_pulse_SU3 (:97-115): sublattice 2 or 3;
 * field_drive [2][n_atoms][spin_dim] (pulse 1, then pulse 2). */
int cmd_mixed_set_pulse(cmd_mixed* h, int32_t sublattice, const double* field_drive, double amp, double width,
                        double freq, double t_pulse_1, double t_pulse_2);

/* set_gpu_mixed_spins / get_gpu_mixed_spins (:120-134); n = n_su2*3 + n_su3*8. */
int cmd_mixed_set_spins(cmd_mixed* h, const double* spins, int64_t n);
int cmd_mixed_get_spins(cmd_mixed* h, double* spins, int64_t n);

/* step_mixed_gpu (:172-177): one step of a fixed-step method (cmd.h's CMD_*
 * except CMD_RK45, which the reference's mixed path does not have). */
int cmd_mixed_step(cmd_mixed* h, double t, double dt, int method);

/* integrate_mixed_gpu (:154-162): the reference loop t = T0; while (t < T1)
 * { if (k % save_interval == 0) save; step; t += dt; ++k; } save.  times[r]
 * and, when non-NULL, states[r][n] per saved row; *rows_out gets the row
 * count (CMD_ERR_INVALID_ARG when max_rows is too small). */
int cmd_mixed_integrate(cmd_mixed* h, double T0, double T1, double dt, int64_t save_interval, int method,
                        double* times, double* states, int64_t max_rows, int64_t* rows_out);

/* compute_magnetization_mixed_gpu (:188-194): means and staggered means
 * (sign (-1)^(site mod n_atoms)) of each kind; m_su2/ms_su2 [3], m_su3/ms_su3 [8]. */
int cmd_mixed_magnetization(cmd_mixed* h, double* m_su2, double* ms_su2, double* m_su3, double* ms_su3);

/* normalize_spins_mixed_gpu (:199-203). */
int cmd_mixed_normalize(cmd_mixed* h, double spin_length_su2, double spin_length_su3);

/* get_mixed_lattice_dims (:208-212): dims = {n_su2, 3, n_atoms_su2, n_su3, 8, n_atoms_su3}. */
int cmd_mixed_dims(cmd_mixed* h, int64_t* dims);

#ifdef __cplusplus
}
#endif

#endif /* CMD_MIXED_H */
