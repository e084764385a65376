/*
 * cmd_lattice.h -- host-side lattice construction for the B200 LL MD path.
 *
 * Mirrors the part of the reference's `Lattice` / `UnitCell` that produces the
 * arrays its GPU boundary consumes (include/classical_spin/lattice/lattice.h:
 * 601-855 constructor, 5429-5497 ensure_gpu_data_initialized), with the
 * builders the MD runs use (src/core/unitcell_builders.cpp:178-283 Kitaev
 * honeycomb, :370-471 non-Kramers pyrochlore).  The bond tables come out in
 * the reference's neighbour order: forward bond at the source, J^T at the
 * partner, single periodic wrap, sites ((i*d2+j)*d3+k)*n_atoms+atom.
 */
#ifndef CMD_LATTICE_H
#define CMD_LATTICE_H

#include <stdint.h>
#include "cmd.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct cmd_lattice cmd_lattice;

/* build_kitaev_honeycomb; kp = {K, Gamma, Gammap, J, J2_A, J2_B, J3, J_perp,
 * Ka, Kb, Kc}; field = g .* (h * dir) on both sublattices. */
int cmd_lattice_kitaev(const double* kp, double h, const double* dir, const double* g,
                       int32_t d1, int32_t d2, int32_t d3, cmd_lattice** out);

/* build_pyrochlore_non_kramer; pp = {Jpm, Jzz, Jpmpm, J2, delta1, delta2}.
 * cubic = 0: the reference's 4-site primitive FCC cell; cubic = 1: the same
 * Hamiltonian on a 16-site conventional cubic cell (no reference counterpart;
 * gives 16*d1*d2*d3 spins in a cube of d1 x d2 x d3 cubic cells). */
int cmd_lattice_pyrochlore_nk(const double* pp, double h, const double* dir, int32_t d1,
                              int32_t d2, int32_t d3, int32_t cubic, cmd_lattice** out);

/* Generic unit cell: bonds[n_bonds] = {src, dst, off0, off1, off2} (ints) with
 * J[n_bonds*9]; field/onsite/frames/afm per atom (frames/afm may be NULL). */
int cmd_lattice_generic(int32_t n_atoms, const int32_t* bonds, const double* J,
                        int32_t n_bonds, const double* field, const double* onsite,
                        const double* frames, const double* afm, int32_t d1, int32_t d2,
                        int32_t d3, cmd_lattice** out);

/* Sizes: N, n_atoms, max_bilinear (ELL width), dims[3]. */
int cmd_lattice_sizes(const cmd_lattice* L, int64_t* N, int32_t* n_atoms,
                      int32_t* max_bilinear, int32_t* dims);

/* Copies of the ELL arrays of ensure_gpu_data_initialized and the per-atom
 * frames / AFM signs (each pointer may be NULL to skip). */
int cmd_lattice_export(const cmd_lattice* L, double* field, double* onsite, double* bilinear,
                       int64_t* partners, int64_t* counts, double* frames, double* afm);

/* Atom positions of the unit cell [n_atoms*3] and lattice vectors [9]. */
int cmd_lattice_geometry(const cmd_lattice* L, double* positions, double* lattice_vectors);

/* Fills `desc` with pointers into L (valid while L lives). */
int cmd_lattice_desc_of(const cmd_lattice* L, cmd_lattice_desc* desc);

/* Lattice::set_pulse rotation (lattice_md.cpp:210-224): out[p][atom] =
 * R_atom * in_p[atom]; in1/in2/out are [n_atoms*3] / [2*n_atoms*3]. */
int cmd_lattice_rotate_pulse(const cmd_lattice* L, const double* in1, const double* in2,
                             double* field_drive);

/* Seeded initial state (no reference counterpart: Lattice::init_random seeds
 * from the clock, lattice.h:649): n spins uniform on the sphere of radius
 * spin_length, Marsaglia's method as in lattice.h:1115-1124, driven by
 * splitmix64(seed); out [n*3]. */
int cmd_lattice_random_spins(int64_t n, uint64_t seed, double spin_length, double* out);

void cmd_lattice_free(cmd_lattice* L);

#ifdef __cplusplus
}
#endif
#endif
