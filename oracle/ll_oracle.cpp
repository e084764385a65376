/*
 * ll_oracle.cpp -- CPU restatement of the reference LL MD path (test
 * infrastructure only; see ll_oracle.h for the scope and the parity pins).
 *
 * Loops, summation orders and drive arithmetic follow the reference CPU code
 * line by line so that this library can stand in for the reference's own CPU
 * integrator (which cannot be built here: Eigen3/Boost/HDF5/MPI are absent).
 */
#include "ll_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <utility>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

struct ora_lattice {
    int n_atoms = 0, d1 = 0, d2 = 0, d3 = 0;
    size_t N = 0;
    std::vector<double> field;          // [N*3]   per-site copy of uc.field (lattice.h:755)
    std::vector<double> onsite;         // [N*9]
    std::vector<double> frames;         // [n_atoms*9] row-major R (columns = local axes)
    std::vector<double> afm;            // [n_atoms]
    std::vector<std::vector<size_t>> partners;   // lattice.h:480, construction order
    std::vector<std::vector<double>> Jlist;      // 9 doubles per entry of partners[i]
    std::vector<size_t> off, part;      // flat CSR mirror (lattice.h:868-903)
    std::vector<double> J;
    size_t num_bi = 0;
    // time-dependent drive (lattice.h:556-560)
    std::vector<double> fd[2];
    double t_pulse[2] = {0.0, 0.0};
    double amp = 0.0, width = 1.0, freq = 0.0;
    double alpha = 0.0;                 // Gilbert damping (lattice.h:563)
};

namespace {

inline void set3x3(double* m, double a, double b, double c, double d, double e, double f,
                   double g, double h, double i) {
    m[0] = a; m[1] = b; m[2] = c; m[3] = d; m[4] = e; m[5] = f; m[6] = g; m[7] = h; m[8] = i;
}

inline void add_bond(ora_unitcell* uc, const double* J, int src, int dst, int o0, int o1, int o2) {
    ora_bond& b = uc->bonds[uc->n_bonds++];
    b.src = src; b.dst = dst; b.off[0] = o0; b.off[1] = o1; b.off[2] = o2;
    std::memcpy(b.J, J, 9 * sizeof(double));
}

void uc_init(ora_unitcell* uc, int n_atoms) {
    std::memset(uc, 0, sizeof(*uc));
    uc->n_atoms = n_atoms;
    for (int a = 0; a < n_atoms; ++a) {            // unitcell.h:123-126 defaults
        double* F = uc->frames + 9 * a;
        F[0] = F[4] = F[8] = 1.0;
        uc->afm[a] = 1.0;
    }
}

// Pyrochlore primitive cell (unitcell.h:312-356).
void pyrochlore_cell(ora_unitcell* uc) {
    uc_init(uc, 4);
    const double p[12] = {0.125, 0.125, 0.125, 0.125, -0.125, -0.125,
                          -0.125, 0.125, -0.125, -0.125, -0.125, 0.125};
    std::memcpy(uc->pos, p, sizeof(p));
    const double lv[9] = {0, 0.5, 0.5, 0.5, 0, 0.5, 0.5, 0.5, 0};
    std::memcpy(uc->lattice_vectors, lv, sizeof(lv));
    const double s3 = 1 / std::sqrt(3.0), s2 = 1 / std::sqrt(2.0);
    const double s6a = 2 / std::sqrt(6.0), s6b = 1 / std::sqrt(6.0);
    const double z[4][3] = {{s3, s3, s3}, {s3, -s3, -s3}, {-s3, s3, -s3}, {-s3, -s3, s3}};
    const double y[4][3] = {{0, -s2, s2}, {0, s2, -s2}, {0, -s2, -s2}, {0, s2, s2}};
    const double x[4][3] = {{-s6a, s6b, s6b}, {-s6a, -s6b, -s6b}, {s6a, s6b, -s6b}, {s6a, -s6b, s6b}};
    for (int a = 0; a < 4; ++a) {
        double* F = uc->frames + 9 * a;
        for (int r = 0; r < 3; ++r) {     // frame.col(0)=x, col(1)=y, col(2)=z
            F[3 * r + 0] = x[a][r];
            F[3 * r + 1] = y[a][r];
            F[3 * r + 2] = z[a][r];
        }
    }
}

inline double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

inline void norm3(double* v, double s) { v[0] /= s; v[1] /= s; v[2] /= s; }

// Drive envelope (lattice_md.cpp:45-56).
inline void drive_factors(const ora_lattice* L, double t, double& f1, double& f2) {
    const double dt1 = t - L->t_pulse[0];
    const double dt2 = t - L->t_pulse[1];
    f1 = L->amp * std::exp(-std::pow(dt1 / (2.0 * L->width), 2)) * std::cos(L->freq * dt1);
    f2 = L->amp * std::exp(-std::pow(dt2 / (2.0 * L->width), 2)) * std::cos(L->freq * dt2);
}

// get_local_field_flat, no twist, no trilinear (lattice.h:1653-1711).
inline void local_field_site(const ora_lattice* L, const double* x, size_t i, double* H) {
    for (int d = 0; d < 3; ++d) H[d] = -L->field[3 * i + d];
    const double* S = x + 3 * i;
    const double* A = &L->onsite[9 * i];
    for (int d = 0; d < 3; ++d)
        for (int d2 = 0; d2 < 3; ++d2) H[d] += 2.0 * A[3 * d + d2] * S[d2];
    for (size_t k = L->off[i]; k < L->off[i + 1]; ++k) {
        const double* Sp = x + 3 * L->part[k];
        const double* Jk = &L->J[9 * k];
        for (int d = 0; d < 3; ++d) {
            double row = 0.0;
            for (int d2 = 0; d2 < 3; ++d2) row += Jk[3 * d + d2] * Sp[d2];
            H[d] += row;
        }
    }
}

// landau_lifshitz_flat SU(2) branch (lattice_md.cpp:39-103).
void rhs(const ora_lattice* L, const double* x, double* dx, double t) {
    const bool drive_active = (L->amp != 0.0);
    double f1 = 0.0, f2 = 0.0;
    if (drive_active) drive_factors(L, t, f1, f2);
    const long N = (long)L->N;
    const double alpha = L->alpha;
#pragma omp parallel for schedule(static) if (N >= 64)
    for (long i = 0; i < N; ++i) {
        double H[3];
        local_field_site(L, x, (size_t)i, H);
        if (drive_active) {                          // apply_drive_field_flat :178-191
            const size_t atom = (size_t)i % L->n_atoms;
            const double* fd0 = L->fd[0].data() + atom * 3;
            const double* fd1 = L->fd[1].data() + atom * 3;
            for (int d = 0; d < 3; ++d) H[d] -= fd0[d] * f1 + fd1[d] * f2;
        }
        const double Sx = x[3 * i], Sy = x[3 * i + 1], Sz = x[3 * i + 2];
        double dSx = H[1] * Sz - H[2] * Sy;
        double dSy = H[2] * Sx - H[0] * Sz;
        double dSz = H[0] * Sy - H[1] * Sx;
        if (alpha > 0.0) {
            const double ax = Sy * dSz - Sz * dSy;
            const double ay = Sz * dSx - Sx * dSz;
            const double az = Sx * dSy - Sy * dSx;
            const double inv_S = 1.0 / std::sqrt(Sx * Sx + Sy * Sy + Sz * Sz);
            dSx -= alpha * inv_S * ax;
            dSy -= alpha * inv_S * ay;
            dSz -= alpha * inv_S * az;
        }
        dx[3 * i] = dSx; dx[3 * i + 1] = dSy; dx[3 * i + 2] = dSz;
    }
}

// total_energy_flat without twist / trilinear (lattice.h:1485-1555).
double energy(const ora_lattice* L, const double* x) {
    double E = 0.0;
    for (size_t i = 0; i < L->N; ++i) {
        const double* Si = x + 3 * i;
        for (int d = 0; d < 3; ++d) E -= L->field[3 * i + d] * Si[d];
        const double* A = &L->onsite[9 * i];
        for (int d = 0; d < 3; ++d)
            for (int d2 = 0; d2 < 3; ++d2) E += Si[d] * A[3 * d + d2] * Si[d2];
        const size_t nb = L->partners[i].size();
        for (size_t n = 0; n < nb; ++n) {
            const size_t p = L->partners[i][n];
            if (p > i) {
                const double* Sj = x + 3 * p;
                const double* Jn = &L->Jlist[i][9 * n];
                for (int d = 0; d < 3; ++d)
                    for (int d2 = 0; d2 < 3; ++d2) E += Si[d] * Jn[3 * d + d2] * Sj[d2];
            }
        }
    }
    return E;
}

// Observer magnetisations (lattice.h:4461-4512, lattice_md.cpp:406-417).
void mags(const ora_lattice* L, const double* x, double* out) {
    double ml[3] = {0, 0, 0}, mg[3] = {0, 0, 0}, ma[3] = {0, 0, 0};
    for (size_t i = 0; i < L->N; ++i)
        for (int d = 0; d < 3; ++d) ml[d] += x[3 * i + d];
    for (size_t i = 0; i < L->N; ++i) {
        const size_t atom = i % L->n_atoms;
        const double* R = &L->frames[9 * atom];
        for (int mu = 0; mu < 3; ++mu)
            for (int nu = 0; nu < 3; ++nu) mg[mu] += R[3 * mu + nu] * x[3 * i + nu];
    }
    for (size_t i = 0; i < L->N; ++i) {
        const size_t atom = i % L->n_atoms;
        const double* R = &L->frames[9 * atom];
        const double sign = L->afm[atom];
        for (int mu = 0; mu < 3; ++mu)
            for (int nu = 0; nu < 3; ++nu) ma[mu] += sign * R[3 * mu + nu] * x[3 * i + nu];
    }
    const double n = double(L->N);
    for (int d = 0; d < 3; ++d) {
        out[d] = ma[d] / n;
        out[3 + d] = ml[d] / n;
        out[6 + d] = mg[d] / n;
    }
}

void write_row(const ora_lattice* L, const double* x, double t, double* row, bool with_E) {
    row[0] = t;
    mags(L, x, row + 1);
    if (with_E) row[10] = energy(L, x) / double(L->N);
}

struct Work {
    std::vector<double> k1, k2, k3, k4, k5, k6, k7, tmp, xnew, err;
    explicit Work(size_t n) : k1(n), k2(n), k3(n), k4(n), k5(n), k6(n), k7(n), tmp(n), xnew(n), err(n) {}
};

// odeint runge_kutta4 (explicit generic RK with the classic tableau).
void rk4_step(const ora_lattice* L, double* x, double t, double dt, Work& w) {
    const size_t n = 3 * L->N;
    rhs(L, x, w.k1.data(), t);
    const double a = 0.5 * dt;
    for (size_t i = 0; i < n; ++i) w.tmp[i] = 1.0 * x[i] + a * w.k1[i];
    rhs(L, w.tmp.data(), w.k2.data(), t + 0.5 * dt);
    for (size_t i = 0; i < n; ++i) w.tmp[i] = 1.0 * x[i] + a * w.k2[i];
    rhs(L, w.tmp.data(), w.k3.data(), t + 0.5 * dt);
    for (size_t i = 0; i < n; ++i) w.tmp[i] = 1.0 * x[i] + dt * w.k3[i];
    rhs(L, w.tmp.data(), w.k4.data(), t + dt);
    const double b1 = (1.0 / 6.0) * dt, b2 = (1.0 / 3.0) * dt;
    for (size_t i = 0; i < n; ++i)
        x[i] = 1.0 * x[i] + b1 * w.k1[i] + b2 * w.k2[i] + b2 * w.k3[i] + b1 * w.k4[i];
}

// Reference GPU stepper arithmetic (integrator.cuh:115-139, gpu_common_helpers.cu:9-52).
void rk4_step_gpu_form(const ora_lattice* L, double* x, double t, double dt, Work& w) {
    const size_t n = 3 * L->N;
    rhs(L, x, w.k1.data(), t);
    for (size_t i = 0; i < n; ++i) w.tmp[i] = 1.0 * x[i] + (0.5 * dt) * w.k1[i];
    rhs(L, w.tmp.data(), w.k2.data(), t + 0.5 * dt);
    for (size_t i = 0; i < n; ++i) w.tmp[i] = 1.0 * x[i] + (0.5 * dt) * w.k2[i];
    rhs(L, w.tmp.data(), w.k3.data(), t + 0.5 * dt);
    for (size_t i = 0; i < n; ++i) w.tmp[i] = 1.0 * x[i] + dt * w.k3[i];
    rhs(L, w.tmp.data(), w.k4.data(), t + dt);
    const double c = dt / 6.0;
    for (size_t i = 0; i < n; ++i) x[i] += c * (w.k1[i] + 2.0 * w.k2[i] + 2.0 * w.k3[i] + w.k4[i]);
}

// odeint less_with_sign / less_eq_with_sign for dt > 0.
inline bool less_with_sign(double t1, double t2) {
    return t2 - t1 > std::numeric_limits<double>::epsilon();
}
inline bool less_eq_with_sign(double t1, double t2) {
    return t1 - t2 <= std::numeric_limits<double>::epsilon();
}

// Dormand-Prince 5(4) controlled stepper in the odeint style (FSAL; default
// error checker a_x = a_dxdt = 1; default step adjuster).
struct Dopri5 {
    const ora_lattice* L;
    double eps_abs, eps_rel;
    Work w;
    std::vector<double> dxdt;   // FSAL derivative at the current point
    bool first = true;
    long n_acc = 0, n_rej = 0, n_rhs = 0;

    Dopri5(const ora_lattice* L_, double ea, double er)
        : L(L_), eps_abs(ea), eps_rel(er), w(3 * L_->N), dxdt(3 * L_->N) {}

    // Returns true on success (x, t, dt updated), false on rejection (dt shrunk).
    bool try_step(double* x, double& t, double& dt) {
        static const double a21 = 1.0 / 5.0;
        static const double a31 = 3.0 / 40.0, a32 = 9.0 / 40.0;
        static const double a41 = 44.0 / 45.0, a42 = -56.0 / 15.0, a43 = 32.0 / 9.0;
        static const double a51 = 19372.0 / 6561.0, a52 = -25360.0 / 2187.0,
                            a53 = 64448.0 / 6561.0, a54 = -212.0 / 729.0;
        static const double a61 = 9017.0 / 3168.0, a62 = -355.0 / 33.0, a63 = 46732.0 / 5247.0,
                            a64 = 49.0 / 176.0, a65 = -5103.0 / 18656.0;
        static const double c2 = 1.0 / 5.0, c3 = 3.0 / 10.0, c4 = 4.0 / 5.0, c5 = 8.0 / 9.0;
        static const double b1 = 35.0 / 384.0, b3 = 500.0 / 1113.0, b4 = 125.0 / 192.0,
                            b5 = -2187.0 / 6784.0, b6 = 11.0 / 84.0;
        static const double dc1 = b1 - 5179.0 / 57600.0, dc3 = b3 - 7571.0 / 16695.0,
                            dc4 = b4 - 393.0 / 640.0, dc5 = b5 - (-92097.0 / 339200.0),
                            dc6 = b6 - 187.0 / 2100.0, dc7 = -1.0 / 40.0;
        const size_t n = 3 * L->N;
        if (first) { rhs(L, x, dxdt.data(), t); ++n_rhs; first = false; }
        const double* k1 = dxdt.data();
        double *k2 = w.k2.data(), *k3 = w.k3.data(), *k4 = w.k4.data(), *k5 = w.k5.data(),
               *k6 = w.k6.data(), *k7 = w.k7.data(), *tmp = w.tmp.data(), *xn = w.xnew.data();
        for (size_t i = 0; i < n; ++i) tmp[i] = x[i] + dt * a21 * k1[i];
        rhs(L, tmp, k2, t + dt * c2);
        for (size_t i = 0; i < n; ++i) tmp[i] = x[i] + dt * a31 * k1[i] + dt * a32 * k2[i];
        rhs(L, tmp, k3, t + dt * c3);
        for (size_t i = 0; i < n; ++i)
            tmp[i] = x[i] + dt * a41 * k1[i] + dt * a42 * k2[i] + dt * a43 * k3[i];
        rhs(L, tmp, k4, t + dt * c4);
        for (size_t i = 0; i < n; ++i)
            tmp[i] = x[i] + dt * a51 * k1[i] + dt * a52 * k2[i] + dt * a53 * k3[i] + dt * a54 * k4[i];
        rhs(L, tmp, k5, t + dt * c5);
        for (size_t i = 0; i < n; ++i)
            tmp[i] = x[i] + dt * a61 * k1[i] + dt * a62 * k2[i] + dt * a63 * k3[i] +
                     dt * a64 * k4[i] + dt * a65 * k5[i];
        rhs(L, tmp, k6, t + dt);
        for (size_t i = 0; i < n; ++i)
            xn[i] = x[i] + dt * b1 * k1[i] + dt * b3 * k3[i] + dt * b4 * k4[i] + dt * b5 * k5[i] +
                    dt * b6 * k6[i];
        rhs(L, xn, k7, t + dt);
        n_rhs += 6;
        double err = 0.0;
        for (size_t i = 0; i < n; ++i) {
            const double e = dt * dc1 * k1[i] + dt * dc3 * k3[i] + dt * dc4 * k4[i] +
                             dt * dc5 * k5[i] + dt * dc6 * k6[i] + dt * dc7 * k7[i];
            const double r = std::abs(e) / (eps_abs + eps_rel * (1.0 * std::abs(x[i]) +
                                                                 1.0 * dt * std::abs(k1[i])));
            err = std::max(err, r);
        }
        if (err > 1.0) {            // decrease_step, error_order 4
            dt *= std::max(0.9 * std::pow(err, -1.0 / (4 - 1)), 1.0 / 5.0);
            ++n_rej;
            return false;
        }
        std::memcpy(x, xn, n * sizeof(double));
        std::memcpy(dxdt.data(), k7, n * sizeof(double));
        t += dt;
        if (err < 0.5) {            // increase_step, stepper_order 5
            err = std::max(std::pow(5.0, -5.0), err);
            dt *= 0.9 * std::pow(err, -1.0 / 5);
        }
        ++n_acc;
        return true;
    }
};

template <class Obs>
bool dopri5_adaptive(Dopri5& st, double* x, double& t, double t_end, double& dt, Obs obs,
                     long max_accepted) {
    while (less_with_sign(t, t_end)) {
        obs(x, t);
        if (less_with_sign(t_end, t + dt)) dt = t_end - t;
        int fails = 0;
        while (!st.try_step(x, t, dt)) {
            if (++fails >= 500) return false;
        }
        if (max_accepted > 0 && st.n_acc >= max_accepted) break;
    }
    obs(x, t);
    return true;
}

}  // namespace

extern "C" {

void ora_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

// build_kitaev_honeycomb (unitcell_builders.cpp:178-283) on HoneyComb(3) (unitcell.h:283-289).
void ora_uc_kitaev(const double* kp, double h, const double* dir, const double* g, ora_unitcell* uc) {
    const double K = kp[0], Gamma = kp[1], Gammap = kp[2], J = kp[3];
    const double J2_A = kp[4], J2_B = kp[5], J3 = kp[6], J_perp = kp[7];
    const double Ka = kp[8], Kb = kp[9], Kc = kp[10];
    uc_init(uc, 2);
    uc->pos[4] = 1 / std::sqrt(3.0);
    const double lv[9] = {1, 0, 0, 0.5, std::sqrt(3.0) / 2, 0, 0, 0, 1};
    std::memcpy(uc->lattice_vectors, lv, sizeof(lv));
    double Jx[9], Jy[9], Jz[9];
    set3x3(Jx, J + K, Gammap, Gammap, Gammap, J, Gamma, Gammap, Gamma, J);
    set3x3(Jy, J, Gammap, Gamma, Gammap, J + K, Gammap, Gamma, Gammap, J);
    set3x3(Jz, J, Gamma, Gammap, Gamma, J, Gammap, Gammap, Gammap, J + K);
    add_bond(uc, Jx, 0, 1, 0, -1, 0);
    add_bond(uc, Jy, 0, 1, 1, -1, 0);
    add_bond(uc, Jz, 0, 1, 0, 0, 0);
    if (std::abs(J2_A) > 1e-12 || std::abs(J2_B) > 1e-12) {
        double A[9] = {0}, B[9] = {0};
        A[0] = A[4] = A[8] = J2_A;
        B[0] = B[4] = B[8] = J2_B;
        add_bond(uc, A, 0, 0, 1, 0, 0);
        add_bond(uc, A, 0, 0, 0, 1, 0);
        add_bond(uc, A, 0, 0, 1, -1, 0);
        add_bond(uc, B, 1, 1, 1, 0, 0);
        add_bond(uc, B, 1, 1, 0, 1, 0);
        add_bond(uc, B, 1, 1, 1, -1, 0);
    }
    if (std::abs(J3) > 1e-12) {
        double M[9] = {0};
        M[0] = M[4] = M[8] = J3;
        add_bond(uc, M, 0, 1, 1, -2, 0);
        add_bond(uc, M, 0, 1, -1, 0, 0);
        add_bond(uc, M, 0, 1, 1, 0, 0);
    }
    if (std::abs(J_perp) > 1e-12) {
        double M[9] = {0};
        M[0] = M[4] = M[8] = J_perp;
        add_bond(uc, M, 0, 0, 0, 0, 1);
        add_bond(uc, M, 1, 1, 0, 0, 1);
    }
    if (std::abs(Ka) > 1e-12 || std::abs(Kb) > 1e-12 || std::abs(Kc) > 1e-12) {
        for (int a = 0; a < 2; ++a) {
            double* A = uc->onsite + 9 * a;
            A[0] = Ka; A[4] = Kb; A[8] = Kc;
        }
    }
    double F[9];
    set3x3(F, 1.0 / std::sqrt(6.0), -1.0 / std::sqrt(2.0), 1.0 / std::sqrt(3.0),
           1.0 / std::sqrt(6.0), 1.0 / std::sqrt(2.0), 1.0 / std::sqrt(3.0),
           -2.0 / std::sqrt(6.0), 0.0, 1.0 / std::sqrt(3.0));
    for (int a = 0; a < 2; ++a) {
        std::memcpy(uc->frames + 9 * a, F, sizeof(F));
        for (int d = 0; d < 3; ++d) uc->field[3 * a + d] = g[d] * h * dir[d];
    }
}

// build_pyrochlore_non_kramer (unitcell_builders.cpp:370-471).
void ora_uc_pyrochlore_nk(const double* pp, double h, const double* dir, ora_unitcell* uc) {
    const double Jpm = pp[0], Jzz = pp[1], Jpmpm = pp[2], J2 = pp[3];
    const double delta1 = pp[4], delta2 = pp[5];
    pyrochlore_cell(uc);
    double z[4][3] = {{1, 1, 1}, {1, -1, -1}, {-1, 1, -1}, {-1, -1, 1}};
    double y[4][3] = {{0, -1, 1}, {0, 1, -1}, {0, -1, -1}, {0, 1, 1}};
    double x[4][3] = {{-2, 1, 1}, {-2, -1, -1}, {2, 1, -1}, {2, -1, 1}};
    for (int i = 0; i < 4; ++i) {
        norm3(z[i], std::sqrt(3.0));
        norm3(y[i], std::sqrt(2.0));
        norm3(x[i], std::sqrt(6.0));
    }
    auto build_exchange = [&](double th, double* J) {
        set3x3(J, -2 * Jpm + 2 * Jpmpm * std::cos(th), -2 * Jpmpm * std::sin(th), 0,
               -2 * Jpmpm * std::sin(th), -2 * Jpm - 2 * Jpmpm * std::cos(th), 0, 0, 0, Jzz);
    };
    double Jx[9], Jy[9], Jz[9];
    build_exchange(2 * M_PI / 3, Jx);
    build_exchange(4 * M_PI / 3, Jy);
    build_exchange(0, Jz);
    add_bond(uc, Jz, 0, 1, 0, 0, 0);
    add_bond(uc, Jx, 0, 2, 0, 0, 0);
    add_bond(uc, Jy, 0, 3, 0, 0, 0);
    add_bond(uc, Jy, 1, 2, 0, 0, 0);
    add_bond(uc, Jx, 1, 3, 0, 0, 0);
    add_bond(uc, Jz, 2, 3, 0, 0, 0);
    add_bond(uc, Jz, 0, 1, 1, 0, 0);
    add_bond(uc, Jx, 0, 2, 0, 1, 0);
    add_bond(uc, Jy, 0, 3, 0, 0, 1);
    add_bond(uc, Jy, 1, 2, -1, 1, 0);
    add_bond(uc, Jx, 1, 3, -1, 0, 1);
    add_bond(uc, Jz, 2, 3, 0, 1, -1);
    double J2m[9] = {0};
    J2m[0] = J2m[4] = J2m[8] = J2;            // Identity * J2, added even when J2 == 0
    for (int s = 0; s < 4; ++s) {
        add_bond(uc, J2m, s, s, 1, 0, 0);
        add_bond(uc, J2m, s, s, 0, 1, 0);
        add_bond(uc, J2m, s, s, 0, 0, 1);
    }
    const double fg[3] = {dir[0] * h, dir[1] * h, dir[2] * h};
    for (int i = 0; i < 4; ++i) {
        const double hx = dot3(fg, x[i]), hy = dot3(fg, y[i]), hz = dot3(fg, z[i]);
        uc->field[3 * i + 0] = delta1 * hx * hz + delta2 * (hy * hy - hx * hx);
        uc->field[3 * i + 1] = delta1 * hy * hz + 2 * delta2 * hx * hy;
        uc->field[3 * i + 2] = hz;
    }
}

// 16-site conventional cubic cell: atom 4q+s sits at FCC translation t_q plus the
// primitive sublattice offset r_s; every primitive bond (s -> s', n) of the
// primitive cell is re-expressed from each (q, s) as (4q'+s', integer cube offset).
void ora_uc_pyrochlore_nk_cubic(const double* pp, double h, const double* dir, ora_unitcell* uc) {
    ora_unitcell prim;
    ora_uc_pyrochlore_nk(pp, h, dir, &prim);
    uc_init(uc, 16);
    const double tq[4][3] = {{0, 0, 0}, {0, 0.5, 0.5}, {0.5, 0, 0.5}, {0.5, 0.5, 0}};
    const double a[3][3] = {{0, 0.5, 0.5}, {0.5, 0, 0.5}, {0.5, 0.5, 0}};
    const double lv[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    std::memcpy(uc->lattice_vectors, lv, sizeof(lv));
    for (int q = 0; q < 4; ++q)
        for (int s = 0; s < 4; ++s) {
            const int at = 4 * q + s;
            for (int d = 0; d < 3; ++d) {
                uc->pos[3 * at + d] = tq[q][d] + prim.pos[3 * s + d];
                uc->field[3 * at + d] = prim.field[3 * s + d];
            }
            std::memcpy(uc->frames + 9 * at, prim.frames + 9 * s, 9 * sizeof(double));
            std::memcpy(uc->onsite + 9 * at, prim.onsite + 9 * s, 9 * sizeof(double));
            uc->afm[at] = prim.afm[s];
        }
    for (int q = 0; q < 4; ++q)
        for (int b = 0; b < prim.n_bonds; ++b) {
            const ora_bond& pb = prim.bonds[b];
            double T[3];
            for (int d = 0; d < 3; ++d)
                T[d] = tq[q][d] + pb.off[0] * a[0][d] + pb.off[1] * a[1][d] + pb.off[2] * a[2][d];
            int qq = -1, m[3] = {0, 0, 0};
            for (int c = 0; c < 4 && qq < 0; ++c) {
                double r[3];
                bool integral = true;
                for (int d = 0; d < 3; ++d) {
                    r[d] = T[d] - tq[c][d];
                    if (std::abs(r[d] - std::round(r[d])) > 1e-9) integral = false;
                }
                if (integral) {
                    qq = c;
                    for (int d = 0; d < 3; ++d) m[d] = (int)std::lround(r[d]);
                }
            }
            add_bond(uc, pb.J, 4 * q + pb.src, 4 * qq + pb.dst, m[0], m[1], m[2]);
        }
}

// Lattice constructor bond tables (lattice.h:601-855, 868-903).
ora_lattice* ora_lattice_create(const ora_unitcell* uc, int d1, int d2, int d3) {
    if (!uc || uc->n_atoms <= 0 || d1 <= 0 || d2 <= 0 || d3 <= 0) return nullptr;
    ora_lattice* L = new ora_lattice();
    L->n_atoms = uc->n_atoms; L->d1 = d1; L->d2 = d2; L->d3 = d3;
    const size_t NA = (size_t)uc->n_atoms;
    L->N = NA * d1 * d2 * d3;
    L->field.resize(3 * L->N);
    L->onsite.resize(9 * L->N);
    L->frames.assign(uc->frames, uc->frames + 9 * NA);
    L->afm.assign(uc->afm, uc->afm + NA);
    L->partners.assign(L->N, {});
    L->Jlist.assign(L->N, {});
    auto flatten = [&](long i, long j, long k, long atom) -> size_t {
        return (size_t)(((i * d2 + j) * d3 + k) * (long)NA + atom);
    };
    size_t site = 0;
    for (long i = 0; i < d1; ++i)
        for (long j = 0; j < d2; ++j)
            for (long k = 0; k < d3; ++k)
                for (long atom = 0; atom < (long)NA; ++atom) {
                    for (int d = 0; d < 3; ++d) L->field[3 * site + d] = uc->field[3 * atom + d];
                    for (int d = 0; d < 9; ++d) L->onsite[9 * site + d] = uc->onsite[9 * atom + d];
                    for (int b = 0; b < uc->n_bonds; ++b) {     // multimap equal_range(atom)
                        const ora_bond& bo = uc->bonds[b];
                        if (bo.src != atom) continue;
                        long pi = i + bo.off[0], pj = j + bo.off[1], pk = k + bo.off[2];
                        if (pi < 0) pi += d1; else if (pi >= d1) pi -= d1;
                        if (pj < 0) pj += d2; else if (pj >= d2) pj -= d2;
                        if (pk < 0) pk += d3; else if (pk >= d3) pk -= d3;
                        if (pi < 0 || pi >= d1 || pj < 0 || pj >= d2 || pk < 0 || pk >= d3) {
                            delete L;      // offset larger than the box: reference UB
                            return nullptr;
                        }
                        const size_t p = flatten(pi, pj, pk, bo.dst);
                        L->partners[site].push_back(p);
                        L->Jlist[site].insert(L->Jlist[site].end(), bo.J, bo.J + 9);
                        L->partners[p].push_back(site);
                        for (int r = 0; r < 3; ++r)           // J^T at the partner
                            for (int c = 0; c < 3; ++c) L->Jlist[p].push_back(bo.J[3 * c + r]);
                    }
                    ++site;
                }
    L->off.assign(L->N + 1, 0);
    for (size_t i = 0; i < L->N; ++i) {
        L->off[i + 1] = L->off[i] + L->partners[i].size();
        L->num_bi = std::max(L->num_bi, L->partners[i].size());
    }
    L->part.resize(L->off[L->N]);
    L->J.resize(9 * L->off[L->N]);
    for (size_t i = 0; i < L->N; ++i)
        for (size_t n = 0; n < L->partners[i].size(); ++n) {
            L->part[L->off[i] + n] = L->partners[i][n];
            std::memcpy(&L->J[9 * (L->off[i] + n)], &L->Jlist[i][9 * n], 9 * sizeof(double));
        }
    L->fd[0].assign(3 * NA, 0.0);
    L->fd[1].assign(3 * NA, 0.0);
    return L;
}

void ora_lattice_destroy(ora_lattice* L) { delete L; }
size_t ora_lattice_size(const ora_lattice* L) { return L->N; }
size_t ora_lattice_nnz(const ora_lattice* L) { return L->off[L->N]; }
int ora_lattice_max_bilinear(const ora_lattice* L) { return (int)L->num_bi; }

void ora_lattice_csr(const ora_lattice* L, int64_t* offsets, int64_t* partners, double* J) {
    for (size_t i = 0; i <= L->N; ++i) offsets[i] = (int64_t)L->off[i];
    for (size_t k = 0; k < L->part.size(); ++k) partners[k] = (int64_t)L->part[k];
    std::memcpy(J, L->J.data(), L->J.size() * sizeof(double));
}

// ensure_gpu_data_initialized flattening (lattice.h:5441-5487).
void ora_lattice_ell(const ora_lattice* L, double* field, double* onsite, double* bilinear,
                     int64_t* partners, int64_t* counts) {
    const size_t zmax = L->num_bi;
    std::memcpy(field, L->field.data(), 3 * L->N * sizeof(double));
    std::memcpy(onsite, L->onsite.data(), 9 * L->N * sizeof(double));
    for (size_t i = 0; i < L->N; ++i) {
        counts[i] = (int64_t)L->partners[i].size();
        for (size_t n = 0; n < zmax; ++n) {
            const size_t e = i * zmax + n;
            if (n < L->partners[i].size()) {
                partners[e] = (int64_t)L->partners[i][n];
                std::memcpy(bilinear + 9 * e, &L->Jlist[i][9 * n], 9 * sizeof(double));
            } else {
                partners[e] = 0;
                std::memset(bilinear + 9 * e, 0, 9 * sizeof(double));
            }
        }
    }
}

void ora_lattice_frames(const ora_lattice* L, double* frames, double* afm) {
    std::memcpy(frames, L->frames.data(), L->frames.size() * sizeof(double));
    std::memcpy(afm, L->afm.data(), L->afm.size() * sizeof(double));
}

// set_pulse (lattice_md.cpp:210-224): field_drive[p][atom] = R_atom * field_in_p[atom].
void ora_set_pulse(ora_lattice* L, const double* in1, double t1, const double* in2, double t2,
                   double amp, double width, double freq) {
    for (int a = 0; a < L->n_atoms; ++a) {
        const double* R = &L->frames[9 * a];
        for (int r = 0; r < 3; ++r) {
            L->fd[0][3 * a + r] = R[3 * r] * in1[3 * a] + R[3 * r + 1] * in1[3 * a + 1] + R[3 * r + 2] * in1[3 * a + 2];
            L->fd[1][3 * a + r] = R[3 * r] * in2[3 * a] + R[3 * r + 1] * in2[3 * a + 1] + R[3 * r + 2] * in2[3 * a + 2];
        }
    }
    L->t_pulse[0] = t1; L->t_pulse[1] = t2;
    L->amp = amp; L->width = width; L->freq = freq;
}

// Pulse reset at the end of single/double_pulse_drive (lattice_md.cpp:580-584).
void ora_clear_pulse(ora_lattice* L) {
    std::fill(L->fd[0].begin(), L->fd[0].end(), 0.0);
    std::fill(L->fd[1].begin(), L->fd[1].end(), 0.0);
    L->amp = 0.0;
}

void ora_set_gilbert(ora_lattice* L, double alpha) { L->alpha = alpha; }

void ora_rhs(const ora_lattice* L, const double* state, double t, double* dsdt) { rhs(L, state, dsdt, t); }

void ora_local_field(const ora_lattice* L, const double* state, double* H) {
    for (size_t i = 0; i < L->N; ++i) local_field_site(L, state, i, H + 3 * i);
}

double ora_energy(const ora_lattice* L, const double* state) { return energy(L, state); }

void ora_magnetizations(const ora_lattice* L, const double* state, double* out) { mags(L, state, out); }

// max_dSdt_norm_no_drive (lattice_md.cpp:236-280).
double ora_max_dsdt_no_drive(ora_lattice* L, const double* state) {
    std::vector<double> d(3 * L->N);
    const double saved = L->amp;
    L->amp = 0.0;
    rhs(L, state, d.data(), 0.0);
    L->amp = saved;
    double m = 0.0;
    for (double v : d) m = std::max(m, std::abs(v));
    return m;
}

void ora_rk4_step(const ora_lattice* L, double* state, double t, double dt) {
    Work w(3 * L->N);
    rk4_step(L, state, t, dt, w);
}

void ora_rk4_step_gpu_form(const ora_lattice* L, double* state, double t, double dt) {
    Work w(3 * L->N);
    rk4_step_gpu_form(L, state, t, dt, w);
}

// integrate_const(runge_kutta4) + the molecular_dynamics_cpu observer (lattice_md.cpp:383-436).
long ora_md_rk4_const(const ora_lattice* L, double* state, double T0, double T1, double dt,
                      long save_interval, double* rows, long max_rows) {
    Work w(3 * L->N);
    long n_rows = 0, calls = 0;
    auto obs = [&](double t) {
        if (calls % save_interval == 0 && n_rows < max_rows) write_row(L, state, t, rows + 11 * n_rows++, true);
        ++calls;
    };
    long step = 0;
    double time = T0;
    while (less_eq_with_sign(time + dt, T1)) {
        obs(time);
        rk4_step(L, state, time, dt, w);
        ++step;
        time = T0 + double(step) * dt;
    }
    obs(time);
    return n_rows;
}

// Reference GPU-API loop (integrator.cuh:470-488) with the GPU stepper arithmetic.
long ora_md_rk4_gpu_loop(const ora_lattice* L, double* state, double T0, double T1, double dt,
                         long save_interval, double* rows, long max_rows) {
    Work w(3 * L->N);
    long n_rows = 0, step = 0;
    double t = T0;
    while (t < T1) {
        if (step % save_interval == 0 && n_rows < max_rows) write_row(L, state, t, rows + 11 * n_rows++, true);
        rk4_step_gpu_form(L, state, t, dt, w);
        t += dt;
        ++step;
    }
    if (n_rows < max_rows) write_row(L, state, t, rows + 11 * n_rows++, true);
    return n_rows;
}

// integrate_adaptive(make_controlled<runge_kutta_dopri5>) + MD observer.
long ora_md_dopri5_adaptive(const ora_lattice* L, double* state, double T0, double T1, double dt0,
                            double abs_tol, double rel_tol, long max_accepted, double* rows,
                            long max_rows, long* stats) {
    Dopri5 st(L, abs_tol, rel_tol);
    long n_rows = 0;
    double t = T0, dt = dt0;
    auto obs = [&](const double* x, double tt) {
        if (n_rows < max_rows) write_row(L, x, tt, rows + 11 * n_rows++, true);
    };
    const bool ok = dopri5_adaptive(st, state, t, T1, dt, obs, max_accepted);
    if (stats) { stats[0] = st.n_acc; stats[1] = st.n_rej; stats[2] = st.n_rhs; }
    return ok ? n_rows : -1;
}

// integrate_const(controlled dopri5): adaptive sub-steps between observer points.
long ora_md_dopri5_const(const ora_lattice* L, double* state, double T0, double T1, double dt,
                         double abs_tol, double rel_tol, double* rows, long max_rows, long* stats) {
    Dopri5 st(L, abs_tol, rel_tol);
    long n_rows = 0;
    auto obs = [&](double tt) {
        if (n_rows < max_rows) write_row(L, state, tt, rows + 11 * n_rows++, true);
    };
    const double time_step = dt;
    double time = T0;
    long step = 0;
    bool ok = true;
    while (less_eq_with_sign(time + time_step, T1)) {
        obs(time);
        double tt = time;
        ok = dopri5_adaptive(st, state, tt, time + time_step, dt, [](const double*, double) {}, 0);
        if (!ok) break;
        ++step;
        time = T0 + double(step) * time_step;
    }
    if (ok) obs(time);
    if (stats) { stats[0] = st.n_acc; stats[1] = st.n_rej; stats[2] = st.n_rhs; }
    return ok ? n_rows : -1;
}

// build_pulse_segments (pulse_chunking.h:82-161).
int ora_pulse_segments(double T_start, double T_end, const double* centers, int n_centers,
                       double window, double T_step, double free_dt_factor, double* segs,
                       int max_segs) {
    int n = 0;
    auto push = [&](double a, double b, double c) {
        if (n < max_segs) { segs[3 * n] = a; segs[3 * n + 1] = b; segs[3 * n + 2] = c; }
        ++n;
    };
    if (T_end <= T_start || T_step <= 0.0) return 0;
    auto snap = [&](double t) { return T_start + std::round((t - T_start) / T_step) * T_step; };
    const double T_end_snapped = T_start + std::floor((T_end - T_start) / T_step + 1e-9) * T_step;
    if (T_end_snapped <= T_start) return 0;
    std::vector<std::pair<double, double>> win, merged;
    for (int c = 0; c < n_centers; ++c) {
        const double w0 = std::max(T_start, snap(centers[c] - window));
        const double w1 = std::min(T_end_snapped, snap(centers[c] + window));
        if (w0 < w1) win.emplace_back(w0, w1);
    }
    std::sort(win.begin(), win.end());
    for (const auto& w : win) {
        if (!merged.empty() && w.first <= merged.back().second)
            merged.back().second = std::max(merged.back().second, w.second);
        else
            merged.push_back(w);
    }
    const double free_dt = std::max(T_step, free_dt_factor * T_step);
    double cursor = T_start;
    for (const auto& w : merged) {
        if (cursor < w.first) push(cursor, w.first, std::min(free_dt, w.first - cursor));
        push(w.first, w.second, T_step);
        cursor = w.second;
    }
    if (cursor < T_end_snapped) push(cursor, T_end_snapped, std::min(free_dt, T_end_snapped - cursor));
    return n;
}

// single_pulse_drive / double_pulse_drive CPU path (lattice_md.cpp:493-680).
long ora_pulse_drive(ora_lattice* L, const double* state0, const double* in1, double t1,
                     const double* in2, double t2, int n_pulses, double amp, double width,
                     double freq, double T0, double T1, double step, int method, int chunking,
                     double abs_tol, double rel_tol, double* rows, long max_rows) {
    std::vector<double> zeros(3 * L->n_atoms, 0.0);
    if (n_pulses == 1) ora_set_pulse(L, in1, t1, zeros.data(), 0.0, amp, width, freq);
    else ora_set_pulse(L, in1, t1, in2, t2, amp, width, freq);
    std::vector<double> x(state0, state0 + 3 * L->N);
    long n_rows = 0;
    double last_save = T0;
    auto observer = [&](const double* s, double t) {
        if (t - last_save >= step - 1e-10 || t >= T1 - 1e-10) {
            if (n_rows < max_rows) {
                double* r = rows + 10 * n_rows;
                r[0] = t;
                mags(L, s, r + 1);
            }
            ++n_rows;
            last_save = t;
        }
    };
    auto integrate = [&](double a, double b) -> bool {
        if (method == 0) {      // integrate_const(runge_kutta4)
            Work w(3 * L->N);
            long k = 0;
            double time = a;
            while (less_eq_with_sign(time + step, b)) {
                observer(x.data(), time);
                rk4_step(L, x.data(), time, step, w);
                ++k;
                time = a + double(k) * step;
            }
            observer(x.data(), time);
            return true;
        }
        Dopri5 st(L, abs_tol, rel_tol);        // integrate_const(controlled dopri5)
        double dt = step, time = a;
        long k = 0;
        while (less_eq_with_sign(time + step, b)) {
            observer(x.data(), time);
            double tt = time;
            if (!dopri5_adaptive(st, x.data(), tt, time + step, dt, [](const double*, double) {}, 0))
                return false;
            ++k;
            time = a + double(k) * step;
        }
        observer(x.data(), time);
        return true;
    };
    bool ok = true;
    if (chunking) {
        double centers[2] = {t1, t2};
        std::vector<double> segs(3 * 64);
        const int ns = ora_pulse_segments(T0, T1, centers, n_pulses, 9.0 * width, step, 20.0,
                                          segs.data(), 64);
        for (int s = 0; s < ns && s < 64 && ok; ++s) ok = integrate(segs[3 * s], segs[3 * s + 1]);
    } else {
        ok = integrate(T0, T1);
    }
    ora_clear_pulse(L);
    return ok ? n_rows : -1;
}

// Trajectory-parallel RK4 batch (W2-style outer loop, lattice_md.cpp:809-904), used
// only to time the CPU baseline.  Each trajectory owns a private drive.
void ora_batch_rk4(const ora_lattice* L, double* states, int B, const double* t1,
                   const double* t2, const double* s1, const double* s2, double amp,
                   double width, double freq, const double* dir1, const double* dir2, double T0,
                   double dt, long nsteps, double* obs, int with_energy) {
#ifdef _OPENMP
    const int saved_levels = omp_get_max_active_levels();
    omp_set_max_active_levels(1);
#endif
#pragma omp parallel
    {
        ora_lattice local(*L);          // per-thread clone, like the W2 loop (lattice_md.cpp:867)
        Work w(3 * L->N);
#pragma omp for schedule(dynamic, 1)
        for (int b = 0; b < B; ++b) {
            ora_set_pulse(&local, dir1, t1[b], dir2, t2[b], 1.0, width, freq);
            // per-trajectory amplitude masks on the two pulses
            for (auto& v : local.fd[0]) v *= s1[b] * amp;
            for (auto& v : local.fd[1]) v *= s2[b] * amp;
            local.amp = (s1[b] != 0.0 || s2[b] != 0.0) ? 1.0 : 0.0;
            double* x = states + (size_t)b * 3 * L->N;
            double t = T0;
            for (long s = 0; s <= nsteps; ++s) {
                double* o = obs ? obs + ((size_t)b * (nsteps + 1) + s) * 10 : nullptr;
                if (o) {
                    mags(&local, x, o);
                    o[9] = with_energy ? energy(&local, x) / double(L->N) : 0.0;
                }
                if (s == nsteps) break;
                rk4_step_gpu_form(&local, x, t, dt, w);
                t += dt;
            }
        }
    }
#ifdef _OPENMP
    omp_set_max_active_levels(saved_levels);
#endif
}

}  // extern "C"

// ---- tangent-linear reference gradient --------------------------------------
namespace {

// dY = d(f)(Y)[Ydot] + (df/dtheta_q)(Y) for one parameter; reference RHS form:
// f_i = H_i x S_i, H_i = -B_i + 2 A_i S_i + sum_n J_n S_p(n) - drive(t).
void rhs_tangent(const ora_lattice* L, const ora_lattice* D, const double* Y, const double* Yd, double t,
                 double* out) {
    const bool drive_active = (L->amp != 0.0);
    double f1 = 0.0, f2 = 0.0;
    if (drive_active) drive_factors(L, t, f1, f2);
    for (size_t i = 0; i < L->N; ++i) {
        double H[3], Hd[3];
        local_field_site(L, Y, i, H);
        if (drive_active) {
            const size_t atom = i % L->n_atoms;
            for (int d = 0; d < 3; ++d) H[d] -= L->fd[0][3 * atom + d] * f1 + L->fd[1][3 * atom + d] * f2;
        }
        // linearised field: couplings of L on Yd, plus derivative couplings of D on Y
        for (int d = 0; d < 3; ++d) Hd[d] = -D->field[3 * i + d];
        for (int d = 0; d < 3; ++d)
            for (int d2 = 0; d2 < 3; ++d2)
                Hd[d] += 2.0 * L->onsite[9 * i + 3 * d + d2] * Yd[3 * i + d2] +
                         2.0 * D->onsite[9 * i + 3 * d + d2] * Y[3 * i + d2];
        for (size_t k = L->off[i]; k < L->off[i + 1]; ++k) {
            const double* J = &L->J[9 * k];
            const double* DJ = &D->J[9 * k];
            const double* P = Y + 3 * L->part[k];
            const double* Pd = Yd + 3 * L->part[k];
            for (int d = 0; d < 3; ++d)
                for (int d2 = 0; d2 < 3; ++d2) Hd[d] += J[3 * d + d2] * Pd[d2] + DJ[3 * d + d2] * P[d2];
        }
        const double* S = Y + 3 * i;
        const double* Sd = Yd + 3 * i;
        out[3 * i + 0] = Hd[1] * S[2] - Hd[2] * S[1] + H[1] * Sd[2] - H[2] * Sd[1];
        out[3 * i + 1] = Hd[2] * S[0] - Hd[0] * S[2] + H[2] * Sd[0] - H[0] * Sd[2];
        out[3 * i + 2] = Hd[0] * S[1] - Hd[1] * S[0] + H[0] * Sd[1] - H[1] * Sd[0];
    }
}

void mloc(const ora_lattice* L, const double* x, double* m) {
    m[0] = m[1] = m[2] = 0.0;
    for (size_t i = 0; i < L->N; ++i)
        for (int d = 0; d < 3; ++d) m[d] += x[3 * i + d];
    for (int d = 0; d < 3; ++d) m[d] /= double(L->N);
}

}  // namespace

extern "C" double ora_loss(const ora_lattice* L, const double* state0, double T0, double dt, long nsteps,
                           const double* target) {
    const size_t n = 3 * L->N;
    std::vector<double> y(state0, state0 + n);
    Work w(n);
    double loss = 0.0, m[3], t = T0;
    for (long s = 0; s <= nsteps; ++s) {
        mloc(L, y.data(), m);
        for (int d = 0; d < 3; ++d) loss += (m[d] - target[3 * s + d]) * (m[d] - target[3 * s + d]);
        if (s == nsteps) break;
        rk4_step_gpu_form(L, y.data(), t, dt, w);
        t += dt;
    }
    return loss;
}

extern "C" double ora_loss_grad_tlm(const ora_lattice* L, const ora_lattice* const* D, int nq,
                                    const double* state0, double T0, double dt, long nsteps,
                                    const double* target, double* grad) {
    const size_t n = 3 * L->N;
    std::vector<double> y(state0, state0 + n), tmp(n), k1(n), k2(n), k3(n), k4(n);
    std::vector<std::vector<double>> yd(nq, std::vector<double>(n, 0.0));
    std::vector<double> Yd(n), kd1(n), kd2(n), kd3(n), kd4(n);
    for (int q = 0; q < nq; ++q) grad[q] = 0.0;
    double loss = 0.0, m[3], t = T0;
    const double invN = 1.0 / double(L->N);
    for (long s = 0; s <= nsteps; ++s) {
        mloc(L, y.data(), m);
        double r[3];
        for (int d = 0; d < 3; ++d) {
            r[d] = m[d] - target[3 * s + d];
            loss += r[d] * r[d];
        }
        for (int q = 0; q < nq; ++q) {           // dL/dtheta += 2 r . dM/dtheta
            double dm[3] = {0, 0, 0};
            for (size_t i = 0; i < L->N; ++i)
                for (int d = 0; d < 3; ++d) dm[d] += yd[q][3 * i + d];
            for (int d = 0; d < 3; ++d) grad[q] += 2.0 * r[d] * dm[d] * invN;
        }
        if (s == nsteps) break;
        // stages of the GPU-form RK4 step (integrator.cuh:115-139) and their tangents
        rhs(L, y.data(), k1.data(), t);
        std::vector<double> Y2(n), Y3(n), Y4(n);
        for (size_t i = 0; i < n; ++i) Y2[i] = 1.0 * y[i] + (0.5 * dt) * k1[i];
        rhs(L, Y2.data(), k2.data(), t + 0.5 * dt);
        for (size_t i = 0; i < n; ++i) Y3[i] = 1.0 * y[i] + (0.5 * dt) * k2[i];
        rhs(L, Y3.data(), k3.data(), t + 0.5 * dt);
        for (size_t i = 0; i < n; ++i) Y4[i] = 1.0 * y[i] + dt * k3[i];
        rhs(L, Y4.data(), k4.data(), t + dt);
        for (int q = 0; q < nq; ++q) {
            std::vector<double>& v = yd[q];
            rhs_tangent(L, D[q], y.data(), v.data(), t, kd1.data());
            for (size_t i = 0; i < n; ++i) Yd[i] = v[i] + (0.5 * dt) * kd1[i];
            rhs_tangent(L, D[q], Y2.data(), Yd.data(), t + 0.5 * dt, kd2.data());
            for (size_t i = 0; i < n; ++i) Yd[i] = v[i] + (0.5 * dt) * kd2[i];
            rhs_tangent(L, D[q], Y3.data(), Yd.data(), t + 0.5 * dt, kd3.data());
            for (size_t i = 0; i < n; ++i) Yd[i] = v[i] + dt * kd3[i];
            rhs_tangent(L, D[q], Y4.data(), Yd.data(), t + dt, kd4.data());
            const double c = dt / 6.0;
            for (size_t i = 0; i < n; ++i) v[i] += c * (kd1[i] + 2.0 * kd2[i] + 2.0 * kd3[i] + kd4[i]);
        }
        const double c = dt / 6.0;
        for (size_t i = 0; i < n; ++i) y[i] += c * (k1[i] + 2.0 * k2[i] + 2.0 * k3[i] + k4[i]);
        t += dt;
    }
    return loss;
}
