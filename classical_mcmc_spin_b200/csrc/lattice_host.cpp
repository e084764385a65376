// lattice_host.cpp -- host-side unit cells and bond tables for the LL MD path.
//
// Produces exactly the arrays that the reference's Lattice hands to its GPU
// boundary (lattice.h:5429-5497), built the way its constructor builds them
// (lattice.h:601-855): sites in ((i*d2+j)*d3+k)*n_atoms+atom order, each
// unit-cell bond pushed forward at the source and as J^T at the partner, in
// the order the source sites are visited, with a single periodic wrap.
#include "cmd_lattice.h"
#include "cmd_internal.h"

#include <array>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

namespace {

using Mat3 = std::array<double, 9>;

struct CellBond {
    int src, dst;
    int off[3];
    Mat3 J;
};

struct UnitCell {
    int n_atoms = 0;
    std::vector<double> pos;            // [n_atoms*3]
    Mat3 lv{1, 0, 0, 0, 1, 0, 0, 0, 1};
    std::vector<double> field, onsite, frames, afm;
    std::vector<CellBond> bonds;        // insertion order

    explicit UnitCell(int na) : n_atoms(na), pos(3 * na, 0.0), field(3 * na, 0.0),
                                onsite(9 * na, 0.0), frames(9 * na, 0.0), afm(na, 1.0) {
        for (int a = 0; a < na; ++a) frames[9 * a] = frames[9 * a + 4] = frames[9 * a + 8] = 1.0;
    }
    void bond(const Mat3& J, int s, int d, int o0, int o1, int o2) {
        bonds.push_back(CellBond{s, d, {o0, o1, o2}, J});
    }
};

Mat3 diag(double v) { return Mat3{v, 0, 0, 0, v, 0, 0, 0, v}; }

// HoneyComb(3) + build_kitaev_honeycomb (unitcell.h:283-289; unitcell_builders.cpp:178-283).
UnitCell kitaev_cell(const double* kp, double h, const double* dir, const double* g) {
    const double K = kp[0], Gm = kp[1], Gp = kp[2], J = kp[3];
    UnitCell uc(2);
    uc.pos[4] = 1 / std::sqrt(3.0);
    uc.lv = Mat3{1, 0, 0, 0.5, std::sqrt(3.0) / 2, 0, 0, 0, 1};
    const Mat3 Jx{J + K, Gp, Gp, Gp, J, Gm, Gp, Gm, J};
    const Mat3 Jy{J, Gp, Gm, Gp, J + K, Gp, Gm, Gp, J};
    const Mat3 Jz{J, Gm, Gp, Gm, J, Gp, Gp, Gp, J + K};
    uc.bond(Jx, 0, 1, 0, -1, 0);
    uc.bond(Jy, 0, 1, 1, -1, 0);
    uc.bond(Jz, 0, 1, 0, 0, 0);
    const double J2A = kp[4], J2B = kp[5], J3 = kp[6], Jperp = kp[7];
    if (std::abs(J2A) > 1e-12 || std::abs(J2B) > 1e-12) {
        const Mat3 A = diag(J2A), B = diag(J2B);
        uc.bond(A, 0, 0, 1, 0, 0); uc.bond(A, 0, 0, 0, 1, 0); uc.bond(A, 0, 0, 1, -1, 0);
        uc.bond(B, 1, 1, 1, 0, 0); uc.bond(B, 1, 1, 0, 1, 0); uc.bond(B, 1, 1, 1, -1, 0);
    }
    if (std::abs(J3) > 1e-12) {
        const Mat3 M = diag(J3);
        uc.bond(M, 0, 1, 1, -2, 0); uc.bond(M, 0, 1, -1, 0, 0); uc.bond(M, 0, 1, 1, 0, 0);
    }
    if (std::abs(Jperp) > 1e-12) {
        const Mat3 M = diag(Jperp);
        uc.bond(M, 0, 0, 0, 0, 1); uc.bond(M, 1, 1, 0, 0, 1);
    }
    const double Ka = kp[8], Kb = kp[9], Kc = kp[10];
    if (std::abs(Ka) > 1e-12 || std::abs(Kb) > 1e-12 || std::abs(Kc) > 1e-12)
        for (int a = 0; a < 2; ++a) {
            uc.onsite[9 * a] = Ka; uc.onsite[9 * a + 4] = Kb; uc.onsite[9 * a + 8] = Kc;
        }
    const Mat3 R{1.0 / std::sqrt(6.0), -1.0 / std::sqrt(2.0), 1.0 / std::sqrt(3.0),
                 1.0 / std::sqrt(6.0), 1.0 / std::sqrt(2.0), 1.0 / std::sqrt(3.0),
                 -2.0 / std::sqrt(6.0), 0.0, 1.0 / std::sqrt(3.0)};
    for (int a = 0; a < 2; ++a) {
        std::memcpy(&uc.frames[9 * a], R.data(), sizeof(double) * 9);
        for (int d = 0; d < 3; ++d) uc.field[3 * a + d] = g[d] * h * dir[d];
    }
    return uc;
}

// Pyrochlore(3) + build_pyrochlore_non_kramer (unitcell.h:312-356; unitcell_builders.cpp:370-471).
UnitCell pyrochlore_nk_cell(const double* pp, double h, const double* dir) {
    const double Jpm = pp[0], Jzz = pp[1], Jpmpm = pp[2], J2 = pp[3], dl1 = pp[4], dl2 = pp[5];
    UnitCell uc(4);
    const double P[12] = {0.125, 0.125, 0.125, 0.125, -0.125, -0.125,
                          -0.125, 0.125, -0.125, -0.125, -0.125, 0.125};
    uc.pos.assign(P, P + 12);
    uc.lv = Mat3{0, 0.5, 0.5, 0.5, 0, 0.5, 0.5, 0.5, 0};
    // Sublattice frames of the Pyrochlore class: columns x_a, y_a, z_a.
    const double r3 = 1 / std::sqrt(3.0), r2 = 1 / std::sqrt(2.0);
    const double r6a = 2 / std::sqrt(6.0), r6b = 1 / std::sqrt(6.0);
    const double fx[4][3] = {{-r6a, r6b, r6b}, {-r6a, -r6b, -r6b}, {r6a, r6b, -r6b}, {r6a, -r6b, r6b}};
    const double fy[4][3] = {{0, -r2, r2}, {0, r2, -r2}, {0, -r2, -r2}, {0, r2, r2}};
    const double fz[4][3] = {{r3, r3, r3}, {r3, -r3, -r3}, {-r3, r3, -r3}, {-r3, -r3, r3}};
    for (int a = 0; a < 4; ++a)
        for (int r = 0; r < 3; ++r) {
            uc.frames[9 * a + 3 * r + 0] = fx[a][r];
            uc.frames[9 * a + 3 * r + 1] = fy[a][r];
            uc.frames[9 * a + 3 * r + 2] = fz[a][r];
        }
    auto exch = [&](double th) {
        return Mat3{-2 * Jpm + 2 * Jpmpm * std::cos(th), -2 * Jpmpm * std::sin(th), 0,
                    -2 * Jpmpm * std::sin(th), -2 * Jpm - 2 * Jpmpm * std::cos(th), 0, 0, 0, Jzz};
    };
    const Mat3 Jx = exch(2 * M_PI / 3), Jy = exch(4 * M_PI / 3), Jz = exch(0);
    uc.bond(Jz, 0, 1, 0, 0, 0); uc.bond(Jx, 0, 2, 0, 0, 0); uc.bond(Jy, 0, 3, 0, 0, 0);
    uc.bond(Jy, 1, 2, 0, 0, 0); uc.bond(Jx, 1, 3, 0, 0, 0); uc.bond(Jz, 2, 3, 0, 0, 0);
    uc.bond(Jz, 0, 1, 1, 0, 0); uc.bond(Jx, 0, 2, 0, 1, 0); uc.bond(Jy, 0, 3, 0, 0, 1);
    uc.bond(Jy, 1, 2, -1, 1, 0); uc.bond(Jx, 1, 3, -1, 0, 1); uc.bond(Jz, 2, 3, 0, 1, -1);
    const Mat3 M2 = diag(J2);                     // present even when J2 == 0
    for (int s = 0; s < 4; ++s) {
        uc.bond(M2, s, s, 1, 0, 0); uc.bond(M2, s, s, 0, 1, 0); uc.bond(M2, s, s, 0, 0, 1);
    }
    // Builder's local axes (divided by the norm, as in the builder).
    double ax[4][3] = {{-2, 1, 1}, {-2, -1, -1}, {2, 1, -1}, {2, -1, 1}};
    double ay[4][3] = {{0, -1, 1}, {0, 1, -1}, {0, -1, -1}, {0, 1, 1}};
    double az[4][3] = {{1, 1, 1}, {1, -1, -1}, {-1, 1, -1}, {-1, -1, 1}};
    const double hg[3] = {dir[0] * h, dir[1] * h, dir[2] * h};
    for (int a = 0; a < 4; ++a) {
        for (int d = 0; d < 3; ++d) {
            ax[a][d] /= std::sqrt(6.0); ay[a][d] /= std::sqrt(2.0); az[a][d] /= std::sqrt(3.0);
        }
        const double hx = hg[0] * ax[a][0] + hg[1] * ax[a][1] + hg[2] * ax[a][2];
        const double hy = hg[0] * ay[a][0] + hg[1] * ay[a][1] + hg[2] * ay[a][2];
        const double hz = hg[0] * az[a][0] + hg[1] * az[a][1] + hg[2] * az[a][2];
        uc.field[3 * a + 0] = dl1 * hx * hz + dl2 * (hy * hy - hx * hx);
        uc.field[3 * a + 1] = dl1 * hy * hz + 2 * dl2 * hx * hy;
        uc.field[3 * a + 2] = hz;
    }
    return uc;
}

// Re-express a primitive FCC cell on the 16-site conventional cube: atom 4q+s
// is sublattice s shifted by the FCC translation t_q.
UnitCell cubic_from_fcc(const UnitCell& p) {
    static const int tq2[4][3] = {{0, 0, 0}, {0, 1, 1}, {1, 0, 1}, {1, 1, 0}};   // 2*t_q
    static const int a2[3][3] = {{0, 1, 1}, {1, 0, 1}, {1, 1, 0}};               // 2*a_i
    UnitCell c(16);
    c.lv = Mat3{1, 0, 0, 0, 1, 0, 0, 0, 1};
    for (int q = 0; q < 4; ++q)
        for (int s = 0; s < 4; ++s) {
            const int at = 4 * q + s;
            for (int d = 0; d < 3; ++d) {
                c.pos[3 * at + d] = 0.5 * tq2[q][d] + p.pos[3 * s + d];
                c.field[3 * at + d] = p.field[3 * s + d];
            }
            for (int d = 0; d < 9; ++d) {
                c.frames[9 * at + d] = p.frames[9 * s + d];
                c.onsite[9 * at + d] = p.onsite[9 * s + d];
            }
            c.afm[at] = p.afm[s];
        }
    for (int q = 0; q < 4; ++q)
        for (const CellBond& b : p.bonds) {
            int T[3];                                   // 2 * translation
            for (int d = 0; d < 3; ++d)
                T[d] = tq2[q][d] + b.off[0] * a2[0][d] + b.off[1] * a2[1][d] + b.off[2] * a2[2][d];
            for (int r = 0; r < 4; ++r) {
                int m[3];
                bool ok = true;
                for (int d = 0; d < 3; ++d) {
                    const int diff = T[d] - tq2[r][d];
                    if (diff % 2 != 0) { ok = false; break; }
                    m[d] = diff / 2;
                }
                if (ok) { c.bond(b.J, 4 * q + b.src, 4 * r + b.dst, m[0], m[1], m[2]); break; }
            }
        }
    return c;
}

}  // namespace

struct cmd_lattice {
    UnitCell uc{1};
    int d[3] = {0, 0, 0};
    int64_t N = 0;
    int32_t zmax = 0;
    std::vector<double> field, onsite, bil;
    std::vector<int64_t> part, cnt;
};

namespace {

int build(UnitCell&& uc, int d1, int d2, int d3, cmd_lattice** out) {
    if (!out) return cmd::fail(CMD_ERR_INVALID_ARG, "output pointer is NULL");
    *out = nullptr;
    if (d1 <= 0 || d2 <= 0 || d3 <= 0) return cmd::fail(CMD_ERR_INVALID_ARG, "lattice dims must be positive");
    const int NA = uc.n_atoms;
    const int64_t N = (int64_t)NA * d1 * d2 * d3;
    const int dims[3] = {d1, d2, d3};
    for (const CellBond& b : uc.bonds)
        for (int k = 0; k < 3; ++k)
            if (b.off[k] < -dims[k] || b.off[k] > dims[k])
                return cmd::fail(CMD_ERR_INVALID_ARG, "bond offset exceeds the lattice box (single periodic wrap)");
    // partner cell coordinate with the constructor's single wrap
    auto wrap = [](int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); };
    auto site_of = [&](int i, int j, int k, int atom) {
        return (((int64_t)i * d2 + j) * d3 + k) * NA + atom;
    };
    // pass 1: count entries per site (forward + reverse)
    std::vector<int64_t> cnt(N, 0);
    for (int i = 0; i < d1; ++i)
        for (int j = 0; j < d2; ++j)
            for (int k = 0; k < d3; ++k)
                for (const CellBond& b : uc.bonds) {
                    cnt[site_of(i, j, k, b.src)]++;
                    cnt[site_of(wrap(i + b.off[0], d1), wrap(j + b.off[1], d2), wrap(k + b.off[2], d3), b.dst)]++;
                }
    int64_t zmax = 0;
    for (int64_t c : cnt) zmax = std::max(zmax, c);
    cmd_lattice* L = new (std::nothrow) cmd_lattice();
    if (!L) return cmd::fail(CMD_ERR_OOM, "host allocation failed");
    L->d[0] = d1; L->d[1] = d2; L->d[2] = d3;
    L->N = N;
    L->zmax = (int32_t)zmax;
    L->field.resize(3 * N);
    L->onsite.resize(9 * N);
    L->bil.assign((size_t)N * zmax * 9, 0.0);
    L->part.assign((size_t)N * zmax, 0);
    L->cnt.assign(N, 0);
    // pass 2: fill in the constructor's order (sites visited in index order,
    // bonds of each source atom in insertion order)
    for (int i = 0; i < d1; ++i)
        for (int j = 0; j < d2; ++j)
            for (int k = 0; k < d3; ++k)
                for (int atom = 0; atom < NA; ++atom) {
                    const int64_t s = site_of(i, j, k, atom);
                    std::memcpy(&L->field[3 * s], &uc.field[3 * atom], 3 * sizeof(double));
                    std::memcpy(&L->onsite[9 * s], &uc.onsite[9 * atom], 9 * sizeof(double));
                    for (const CellBond& b : uc.bonds) {
                        if (b.src != atom) continue;
                        const int64_t p = site_of(wrap(i + b.off[0], d1), wrap(j + b.off[1], d2),
                                                  wrap(k + b.off[2], d3), b.dst);
                        int64_t e = s * zmax + L->cnt[s]++;
                        L->part[e] = p;
                        std::memcpy(&L->bil[9 * e], b.J.data(), 9 * sizeof(double));
                        e = p * zmax + L->cnt[p]++;
                        L->part[e] = s;
                        for (int r = 0; r < 3; ++r)
                            for (int c = 0; c < 3; ++c) L->bil[9 * e + 3 * r + c] = b.J[3 * c + r];
                    }
                }
    L->uc = std::move(uc);
    *out = L;
    return CMD_OK;
}

}  // namespace

extern "C" {

int cmd_lattice_kitaev(const double* kp, double h, const double* dir, const double* g, int32_t d1,
                       int32_t d2, int32_t d3, cmd_lattice** out) {
    if (!kp || !dir || !g) return cmd::fail(CMD_ERR_INVALID_ARG, "NULL parameter array");
    return build(kitaev_cell(kp, h, dir, g), d1, d2, d3, out);
}

int cmd_lattice_pyrochlore_nk(const double* pp, double h, const double* dir, int32_t d1, int32_t d2,
                              int32_t d3, int32_t cubic, cmd_lattice** out) {
    if (!pp || !dir) return cmd::fail(CMD_ERR_INVALID_ARG, "NULL parameter array");
    UnitCell p = pyrochlore_nk_cell(pp, h, dir);
    if (cubic) return build(cubic_from_fcc(p), d1, d2, d3, out);
    return build(std::move(p), d1, d2, d3, out);
}

int cmd_lattice_generic(int32_t n_atoms, const int32_t* bonds, const double* J, int32_t n_bonds,
                        const double* field, const double* onsite, const double* frames,
                        const double* afm, int32_t d1, int32_t d2, int32_t d3, cmd_lattice** out) {
    if (n_atoms <= 0 || n_bonds < 0 || (n_bonds > 0 && (!bonds || !J)))
        return cmd::fail(CMD_ERR_INVALID_ARG, "bad unit-cell description");
    UnitCell uc(n_atoms);
    for (int b = 0; b < n_bonds; ++b) {
        const int32_t* q = bonds + 5 * b;
        if (q[0] < 0 || q[0] >= n_atoms || q[1] < 0 || q[1] >= n_atoms)
            return cmd::fail(CMD_ERR_INVALID_ARG, "bond atom index out of range");
        Mat3 M;
        std::memcpy(M.data(), J + 9 * b, 9 * sizeof(double));
        uc.bond(M, q[0], q[1], q[2], q[3], q[4]);
    }
    if (field) uc.field.assign(field, field + 3 * n_atoms);
    if (onsite) uc.onsite.assign(onsite, onsite + 9 * n_atoms);
    if (frames) uc.frames.assign(frames, frames + 9 * n_atoms);
    if (afm) uc.afm.assign(afm, afm + n_atoms);
    return build(std::move(uc), d1, d2, d3, out);
}

int cmd_lattice_sizes(const cmd_lattice* L, int64_t* N, int32_t* n_atoms, int32_t* max_bilinear,
                      int32_t* dims) {
    if (!L) return cmd::fail(CMD_ERR_INVALID_ARG, "NULL lattice");
    if (N) *N = L->N;
    if (n_atoms) *n_atoms = L->uc.n_atoms;
    if (max_bilinear) *max_bilinear = L->zmax;
    if (dims) { dims[0] = L->d[0]; dims[1] = L->d[1]; dims[2] = L->d[2]; }
    return CMD_OK;
}

int cmd_lattice_export(const cmd_lattice* L, double* field, double* onsite, double* bilinear,
                       int64_t* partners, int64_t* counts, double* frames, double* afm) {
    if (!L) return cmd::fail(CMD_ERR_INVALID_ARG, "NULL lattice");
    auto cp = [](void* dst, const void* src, size_t bytes) { if (dst) std::memcpy(dst, src, bytes); };
    cp(field, L->field.data(), L->field.size() * sizeof(double));
    cp(onsite, L->onsite.data(), L->onsite.size() * sizeof(double));
    cp(bilinear, L->bil.data(), L->bil.size() * sizeof(double));
    cp(partners, L->part.data(), L->part.size() * sizeof(int64_t));
    cp(counts, L->cnt.data(), L->cnt.size() * sizeof(int64_t));
    cp(frames, L->uc.frames.data(), L->uc.frames.size() * sizeof(double));
    cp(afm, L->uc.afm.data(), L->uc.afm.size() * sizeof(double));
    return CMD_OK;
}

int cmd_lattice_geometry(const cmd_lattice* L, double* positions, double* lattice_vectors) {
    if (!L) return cmd::fail(CMD_ERR_INVALID_ARG, "NULL lattice");
    if (positions) std::memcpy(positions, L->uc.pos.data(), L->uc.pos.size() * sizeof(double));
    if (lattice_vectors) std::memcpy(lattice_vectors, L->uc.lv.data(), 9 * sizeof(double));
    return CMD_OK;
}

int cmd_lattice_desc_of(const cmd_lattice* L, cmd_lattice_desc* d) {
    if (!L || !d) return cmd::fail(CMD_ERR_INVALID_ARG, "NULL argument");
    d->lattice_size = L->N;
    d->spin_dim = 3;
    d->n_atoms = L->uc.n_atoms;
    d->max_bilinear = L->zmax;
    d->reserved = 0;
    d->field = L->field.data();
    d->onsite = L->onsite.data();
    d->bilinear = L->bil.data();
    d->partners = L->part.data();
    d->counts = L->cnt.data();
    d->frames = L->uc.frames.data();
    d->afm_signs = L->uc.afm.data();
    return CMD_OK;
}

int cmd_lattice_rotate_pulse(const cmd_lattice* L, const double* in1, const double* in2, double* fd) {
    if (!L || !in1 || !in2 || !fd) return cmd::fail(CMD_ERR_INVALID_ARG, "NULL argument");
    const int NA = L->uc.n_atoms;
    for (int a = 0; a < NA; ++a) {
        const double* R = &L->uc.frames[9 * a];
        for (int r = 0; r < 3; ++r) {
            fd[3 * a + r] = R[3 * r] * in1[3 * a] + R[3 * r + 1] * in1[3 * a + 1] + R[3 * r + 2] * in1[3 * a + 2];
            fd[3 * NA + 3 * a + r] = R[3 * r] * in2[3 * a] + R[3 * r + 1] * in2[3 * a + 1] + R[3 * r + 2] * in2[3 * a + 2];
        }
    }
    return CMD_OK;
}

void cmd_lattice_free(cmd_lattice* L) { delete L; }

// Seeded spins uniform on the sphere of radius spin_length: splitmix64 drives
// Marsaglia's (1972) rejection method, the method of Lattice::init_random
// (lattice.h:1115-1124), whose generator the reference seeds from the clock.
int cmd_lattice_random_spins(int64_t n, uint64_t seed, double spin_length, double* out) {
    if (n < 0 || (n > 0 && !out) || !(spin_length > 0.0)) return cmd::fail(CMD_ERR_INVALID_ARG, "bad argument");
    uint64_t state = seed;
    auto next = [&]() {
        uint64_t z = (state += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    };
    auto uniform = [&]() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); };   // [0, 1)
    for (int64_t i = 0; i < n; ++i) {
        double u, v, s;
        do {
            u = 2.0 * uniform() - 1.0;
            v = 2.0 * uniform() - 1.0;
            s = u * u + v * v;
        } while (s >= 1.0);
        const double f = 2.0 * std::sqrt(1.0 - s);
        out[3 * i] = spin_length * f * u;
        out[3 * i + 1] = spin_length * f * v;
        out[3 * i + 2] = spin_length * (1.0 - 2.0 * s);
    }
    return CMD_OK;
}

}  // extern "C"
