// rk_fixed.cuh -- one step of each fixed-step method of the reference GPU
// integrator (integrator.cuh:91-452), generic over the right-hand side, the
// state elements a thread owns and the barrier, so the per-trajectory
// integrator (rk_global.cuh, CTA barrier) and the mixed SU(2)/SU(3) integrator
// (mixed.cuh, cluster barrier) share one copy of every tableau.
//
// fixed_step<XM>(mode, c, y, k, Ya, Yb, yn, t, dt) advances y by one step of dt.
// The caller has already evaluated k[0] = f(y, t) (that evaluation also feeds
// the observers).  The context c provides
//   c.rhs(Y, K, ts)   K = f(Y, ts) on the own elements (Y read anywhere),
//   c.each(f)         f(i) for every own element index i,
//   c.sync()          a barrier over every thread of the trajectory.
// Stage inputs use the reference's update arithmetic: the chains of
// update_arrays_kernel / update_arrays_three_kernel launches
// (gpu_common_helpers.cu:10-35) summed in the same order.  Buffers: y, seven
// stage derivatives k[0..6], three stage inputs Ya, Yb, yn; a barrier separates
// every write of a buffer from the last read of it by another thread.  Methods
// past RK4 / DOPRI5 / Cash-Karp are compiled only when XM is set.
#pragma once

namespace cmd {

enum {
    kModeRK45 = 0, kModeDopri5Fixed = 1, kModeRK4 = 2, kModeCashKarpFixed = 3,
    kModeEuler = 4, kModeMidpoint = 5, kModeSSPRK53 = 6, kModeRK78 = 7, kModeBulirschStoer = 8
};

// Z = 1.0 * X + s[0] K[0], then Z = 1.0 * Z + s[j] K[j] for j = 1..M-1: the rounding
// sequence of a chain of single-term update launches.  Z may alias X.
template <int M, class Ctx>
__device__ __forceinline__ void lin_chain(const Ctx& c, double* Z, const double* X, const double* const (&K)[M],
                                          const double (&s)[M]) {
    c.each([&](long long i) {
        double v = 1.0 * X[i] + s[0] * K[0][i];
#pragma unroll
        for (int j = 1; j < M; ++j) v = 1.0 * v + s[j] * K[j][i];
        Z[i] = v;
    });
}

// Z = a1 X1 + a2 X2 (+ a3 X3).  Z may alias an input.
template <class Ctx>
__device__ __forceinline__ void lin2(const Ctx& c, double* Z, double a1, const double* X1, double a2,
                                     const double* X2) {
    c.each([&](long long i) { Z[i] = a1 * X1[i] + a2 * X2[i]; });
}
template <class Ctx>
__device__ __forceinline__ void lin3(const Ctx& c, double* Z, double a1, const double* X1, double a2,
                                     const double* X2, double a3, const double* X3) {
    c.each([&](long long i) { Z[i] = a1 * X1[i] + a2 * X2[i] + a3 * X3[i]; });
}

template <bool XM, class Ctx>
__device__ void fixed_step(int mode, const Ctx& c, double* y, double* const* k, double* Ya, double* Yb, double* yn,
                           double t, double dt) {
    if (mode == kModeRK4) {                 // integrator.cuh:115-139 arithmetic
        c.sync();
        c.each([&](long long i) { Ya[i] = 1.0 * y[i] + (0.5 * dt) * k[0][i]; });
        c.sync();
        c.rhs(Ya, k[1], t + 0.5 * dt);
        c.each([&](long long i) { Yb[i] = 1.0 * y[i] + (0.5 * dt) * k[1][i]; });
        c.sync();
        c.rhs(Yb, k[2], t + 0.5 * dt);
        c.each([&](long long i) { Ya[i] = 1.0 * y[i] + dt * k[2][i]; });
        c.sync();
        c.rhs(Ya, k[3], t + dt);
        c.each([&](long long i) { y[i] += (dt / 6.0) * (k[0][i] + 2.0 * k[1][i] + 2.0 * k[2][i] + k[3][i]); });
        c.sync();
        return;
    }
    if (mode == kModeDopri5Fixed || mode == kModeCashKarpFixed) {
        // The six-stage tableaux: Dormand-Prince 5 (integrator.cuh:186-228) and
        // Cash-Karp 5 (integrator.cuh:141-185, "rk5"), whose final update the
        // reference forms with the dopri5 kernel, b5 = 0 and k6 in the k5 slot.
        const bool ck = mode == kModeCashKarpFixed;
        const double a21 = 1.0 / 5.0, a31 = 3.0 / 40.0, a32 = 9.0 / 40.0;
        const double a41 = ck ? 3.0 / 10.0 : 44.0 / 45.0, a42 = ck ? -9.0 / 10.0 : -56.0 / 15.0;
        const double a43 = ck ? 6.0 / 5.0 : 32.0 / 9.0;
        const double a51 = ck ? -11.0 / 54.0 : 19372.0 / 6561.0, a52 = ck ? 5.0 / 2.0 : -25360.0 / 2187.0;
        const double a53 = ck ? -70.0 / 27.0 : 64448.0 / 6561.0, a54 = ck ? 35.0 / 27.0 : -212.0 / 729.0;
        const double a61 = ck ? 1631.0 / 55296.0 : 9017.0 / 3168.0, a62 = ck ? 175.0 / 512.0 : -355.0 / 33.0;
        const double a63 = ck ? 575.0 / 13824.0 : 46732.0 / 5247.0, a64 = ck ? 44275.0 / 110592.0 : 49.0 / 176.0;
        const double a65 = ck ? 253.0 / 4096.0 : -5103.0 / 18656.0;
        const double c2 = 1.0 / 5.0, c3 = 3.0 / 10.0, c4 = ck ? 3.0 / 5.0 : 4.0 / 5.0, c5 = ck ? 1.0 : 8.0 / 9.0;
        const double c6 = ck ? 7.0 / 8.0 : 1.0;
        const double b1 = ck ? 37.0 / 378.0 : 35.0 / 384.0, b3 = ck ? 250.0 / 621.0 : 500.0 / 1113.0;
        const double b4 = ck ? 125.0 / 594.0 : 125.0 / 192.0, b5 = ck ? 0.0 : -2187.0 / 6784.0;
        const double b6 = ck ? 512.0 / 1771.0 : 11.0 / 84.0;
        double* const k5b = ck ? k[5] : k[4];       // the reference's k5 slot (k6 again for Cash-Karp)
        c.sync();
        c.each([&](long long i) { Ya[i] = 1.0 * y[i] + (a21 * dt) * k[0][i]; });
        c.sync();
        c.rhs(Ya, k[1], t + c2 * dt);
        c.each([&](long long i) { Yb[i] = y[i] + dt * (a31 * k[0][i] + a32 * k[1][i]); });
        c.sync();
        c.rhs(Yb, k[2], t + c3 * dt);
        c.each([&](long long i) { Ya[i] = y[i] + dt * (a41 * k[0][i] + a42 * k[1][i] + a43 * k[2][i]); });
        c.sync();
        c.rhs(Ya, k[3], t + c4 * dt);
        c.each([&](long long i) {
            Yb[i] = y[i] + dt * (a51 * k[0][i] + a52 * k[1][i] + a53 * k[2][i] + a54 * k[3][i]);
        });
        c.sync();
        c.rhs(Yb, k[4], t + c5 * dt);
        c.each([&](long long i) {
            Ya[i] = y[i] + dt * (a61 * k[0][i] + a62 * k[1][i] + a63 * k[2][i] + a64 * k[3][i] + a65 * k[4][i]);
        });
        c.sync();
        c.rhs(Ya, k[5], t + c6 * dt);
        c.each([&](long long i) {
            y[i] += dt * (b1 * k[0][i] + b3 * k[2][i] + b4 * k[3][i] + b5 * k5b[i] + b6 * k[5][i]);
        });
        c.sync();
        return;
    }
    if constexpr (XM) {
        if (mode == kModeEuler) {           // integrator.cuh:91-99
            c.sync();
            lin2(c, y, 1.0, y, dt, k[0]);
            c.sync();
        } else if (mode == kModeMidpoint) { // "rk2" / "midpoint", integrator.cuh:100-114
            c.sync();
            lin2(c, Ya, 1.0, y, 0.5 * dt, k[0]);
            c.sync();
            c.rhs(Ya, k[1], t + 0.5 * dt);
            lin2(c, y, 1.0, y, dt, k[1]);
            c.sync();
        } else if (mode == kModeSSPRK53) {  // integrator.cuh:406-448; tmp = Ya, u = Yb
            // Five-stage third-order strong-stability-preserving tableau, the
            // reference's 15-digit coefficients.
            const double a30 = 0.355909775063327, a32 = 0.644090224936674;
            const double a40 = 0.367933791638137, a43 = 0.632066208361863;
            const double a52 = 0.237593836598569, a54 = 0.762406163401431;
            const double b10 = 0.377268915331368, b21 = 0.377268915331368, b32 = 0.242995220537396;
            const double b43 = 0.238458932846290, b54 = 0.287632146308408;
            const double c1 = 0.377268915331368, c2 = 0.754537830662736, c3 = 0.728985661612188;
            const double c4 = 0.699226135931670;
            c.sync();
            lin2(c, Ya, 1.0, y, b10 * dt, k[0]);
            c.sync();
            c.rhs(Ya, k[0], t + c1 * dt);
            lin2(c, Yb, 1.0, Ya, b21 * dt, k[0]);
            c.sync();
            c.rhs(Yb, k[0], t + c2 * dt);
            lin3(c, Ya, a30, y, a32, Yb, b32 * dt, k[0]);
            c.sync();
            c.rhs(Ya, k[0], t + c3 * dt);
            lin3(c, yn, a40, y, a43, Ya, b43 * dt, k[0]);     // the reference updates tmp in place
            c.sync();
            c.rhs(yn, k[0], t + c4 * dt);
            lin3(c, y, a52, Yb, a54, yn, b54 * dt, k[0]);
            c.sync();
        } else if (mode == kModeRK78) {
            // The reference GPU "rk78" / "rkf78" (integrator.cuh:230-370): the first 11
            // stages of Fehlberg 7(8) and its 7th-order weights, every stage input a chain
            // of single-term updates.  Slots: k2 and k8 share k[1], k3 and k9 share k[2]
            // (k2 is dead after stage 3, k3 after stage 5), k10 = yn, k11 = Yb, tmp = Ya.
            double* const K1 = k[0];
            double* const K4 = k[3];
            double* const K5 = k[4];
            double* const K6 = k[5];
            double* const K7 = k[6];
            c.sync();
            { const double* const K[1] = {K1}; const double s[1] = {(2.0 / 27.0) * dt};
              lin_chain<1>(c, Ya, y, K, s); }
            c.sync();
            c.rhs(Ya, k[1], t + (2.0 / 27.0) * dt);                            // k2
            c.sync();
            { const double* const K[2] = {K1, k[1]}; const double s[2] = {(1.0 / 36.0) * dt, (1.0 / 12.0) * dt};
              lin_chain<2>(c, Ya, y, K, s); }
            c.sync();
            c.rhs(Ya, k[2], t + (1.0 / 9.0) * dt);                             // k3
            c.sync();
            { const double* const K[2] = {K1, k[2]}; const double s[2] = {(1.0 / 24.0) * dt, (1.0 / 8.0) * dt};
              lin_chain<2>(c, Ya, y, K, s); }
            c.sync();
            c.rhs(Ya, K4, t + (1.0 / 6.0) * dt);
            c.sync();
            { const double* const K[3] = {K1, K4, k[2]};
              const double s[3] = {(5.0 / 12.0) * dt, (-25.0 / 16.0) * dt, (25.0 / 16.0) * dt};
              lin_chain<3>(c, Ya, y, K, s); }
            c.sync();
            c.rhs(Ya, K5, t + (5.0 / 12.0) * dt);
            c.sync();
            { const double* const K[3] = {K1, K4, K5};
              const double s[3] = {(1.0 / 20.0) * dt, (1.0 / 4.0) * dt, (1.0 / 5.0) * dt};
              lin_chain<3>(c, Ya, y, K, s); }
            c.sync();
            c.rhs(Ya, K6, t + (1.0 / 2.0) * dt);
            c.sync();
            { const double* const K[4] = {K1, K4, K5, K6};
              const double s[4] = {(-25.0 / 108.0) * dt, (125.0 / 108.0) * dt, (-65.0 / 27.0) * dt,
                                   (125.0 / 54.0) * dt};
              lin_chain<4>(c, Ya, y, K, s); }
            c.sync();
            c.rhs(Ya, K7, t + (5.0 / 6.0) * dt);
            c.sync();
            { const double* const K[4] = {K1, K5, K6, K7};
              const double s[4] = {(31.0 / 300.0) * dt, (61.0 / 225.0) * dt, (-2.0 / 9.0) * dt, (13.0 / 900.0) * dt};
              lin_chain<4>(c, Ya, y, K, s); }
            c.sync();
            c.rhs(Ya, k[1], t + (1.0 / 6.0) * dt);                             // k8
            c.sync();
            { const double* const K[6] = {K1, K4, K5, K6, K7, k[1]};
              const double s[6] = {2.0 * dt, (-53.0 / 6.0) * dt, (704.0 / 45.0) * dt, (-107.0 / 9.0) * dt,
                                   (67.0 / 90.0) * dt, 3.0 * dt};
              lin_chain<6>(c, Ya, y, K, s); }
            c.sync();
            c.rhs(Ya, k[2], t + (2.0 / 3.0) * dt);                             // k9
            c.sync();
            { const double* const K[7] = {K1, K4, K5, K6, K7, k[1], k[2]};
              const double s[7] = {(-91.0 / 108.0) * dt, (23.0 / 108.0) * dt, (-976.0 / 135.0) * dt,
                                   (311.0 / 54.0) * dt, (-19.0 / 60.0) * dt, (17.0 / 6.0) * dt, (-1.0 / 12.0) * dt};
              lin_chain<7>(c, Ya, y, K, s); }
            c.sync();
            c.rhs(Ya, yn, t + (1.0 / 3.0) * dt);                               // k10
            c.sync();
            { const double* const K[8] = {K1, K4, K5, K6, K7, k[1], k[2], yn};
              const double s[8] = {(2383.0 / 4100.0) * dt, (-341.0 / 164.0) * dt, (4496.0 / 1025.0) * dt,
                                   (-301.0 / 82.0) * dt, (2133.0 / 4100.0) * dt, (45.0 / 82.0) * dt,
                                   (45.0 / 164.0) * dt, (18.0 / 41.0) * dt};
              lin_chain<8>(c, Ya, y, K, s); }
            c.sync();
            c.rhs(Ya, Yb, t + 1.0 * dt);                                       // k11
            { const double* const K[7] = {K1, K6, K7, k[1], k[2], yn, Yb};
              const double s[7] = {(41.0 / 840.0) * dt, (34.0 / 105.0) * dt, (9.0 / 35.0) * dt, (9.0 / 35.0) * dt,
                                   (9.0 / 280.0) * dt, (9.0 / 280.0) * dt, (41.0 / 840.0) * dt};
              lin_chain<7>(c, y, y, K, s); }
            c.sync();
        } else if (mode == kModeBulirschStoer) {
            // The reference GPU "bulirsch_stoer" / "bs" (integrator.cuh:371-405): modified
            // midpoint over four substeps with the final smoothing step, no extrapolation.
            // y_prev / y_mid / y_next rotate over Ya, Yb and yn instead of being copied.
            const double hs = dt / 4;
            double* prev = y;
            double* mid = Ya;
            c.sync();
            lin2(c, mid, 1.0, y, hs, k[0]);
            c.sync();
            for (int sub = 1; sub < 4; ++sub) {
                c.rhs(mid, k[0], t + sub * hs);
                double* next = (Ya != prev && Ya != mid) ? Ya : (Yb != prev && Yb != mid) ? Yb : yn;
                lin2(c, next, 1.0, prev, 2.0 * hs, k[0]);
                prev = mid;
                mid = next;
                c.sync();
            }
            c.rhs(mid, k[0], t + dt);
            double* next = (Ya != prev && Ya != mid) ? Ya : (Yb != prev && Yb != mid) ? Yb : yn;
            lin2(c, next, 0.5, mid, 0.5, prev);
            lin2(c, y, 1.0, next, 0.5 * hs, k[0]);
            c.sync();
        }
    }
}

}  // namespace cmd
