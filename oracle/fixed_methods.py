"""Test oracle: numpy restatement of the reference GPU integrator's fixed-step methods.

Test infrastructure only (imported by tests/).  Each step follows
include/classical_spin/gpu/ode/integrator.cuh of the reference: the stage
inputs are formed with the same single- and three-term updates
(update_arrays_kernel / update_arrays_three_kernel, src/gpu/gpu_common_helpers.cu:10-35),
in the same order, over the right-hand side ``f(y, t)`` the caller passes (for
a lattice, ``OracleLattice.rhs``).

    euler            integrator.cuh:91-99
    rk2 / midpoint   integrator.cuh:100-114
    rk4              integrator.cuh:115-139
    rk5 / rkck54     integrator.cuh:141-185 (Cash-Karp 5, fixed step)
    dopri5 / rk54    integrator.cuh:186-228, 450-452 (Dormand-Prince 5, fixed step)
    rk78 / rkf78     integrator.cuh:230-370 (11 Fehlberg stages, 7th-order weights)
    bs               integrator.cuh:371-405 (modified midpoint, 4 substeps, smoothing)
    ssprk53          integrator.cuh:406-448
"""
from __future__ import annotations

import numpy as np


def _chain(y, terms, dt):
    """y + (c_1 dt) k_1, then + (c_j dt) k_j in order (one update launch per term)."""
    v = y.copy()
    for c, k in terms:
        v = 1.0 * v + (c * dt) * k
    return v


def _rk78(f, y, t, dt):
    k1 = f(y, t)
    k2 = f(_chain(y, [(2.0 / 27.0, k1)], dt), t + (2.0 / 27.0) * dt)
    k3 = f(_chain(y, [(1.0 / 36.0, k1), (1.0 / 12.0, k2)], dt), t + (1.0 / 9.0) * dt)
    k4 = f(_chain(y, [(1.0 / 24.0, k1), (1.0 / 8.0, k3)], dt), t + (1.0 / 6.0) * dt)
    k5 = f(_chain(y, [(5.0 / 12.0, k1), (-25.0 / 16.0, k4), (25.0 / 16.0, k3)], dt), t + (5.0 / 12.0) * dt)
    k6 = f(_chain(y, [(1.0 / 20.0, k1), (1.0 / 4.0, k4), (1.0 / 5.0, k5)], dt), t + 0.5 * dt)
    k7 = f(_chain(y, [(-25.0 / 108.0, k1), (125.0 / 108.0, k4), (-65.0 / 27.0, k5), (125.0 / 54.0, k6)], dt),
           t + (5.0 / 6.0) * dt)
    k8 = f(_chain(y, [(31.0 / 300.0, k1), (61.0 / 225.0, k5), (-2.0 / 9.0, k6), (13.0 / 900.0, k7)], dt),
           t + (1.0 / 6.0) * dt)
    k9 = f(_chain(y, [(2.0, k1), (-53.0 / 6.0, k4), (704.0 / 45.0, k5), (-107.0 / 9.0, k6), (67.0 / 90.0, k7),
                      (3.0, k8)], dt), t + (2.0 / 3.0) * dt)
    k10 = f(_chain(y, [(-91.0 / 108.0, k1), (23.0 / 108.0, k4), (-976.0 / 135.0, k5), (311.0 / 54.0, k6),
                       (-19.0 / 60.0, k7), (17.0 / 6.0, k8), (-1.0 / 12.0, k9)], dt), t + (1.0 / 3.0) * dt)
    k11 = f(_chain(y, [(2383.0 / 4100.0, k1), (-341.0 / 164.0, k4), (4496.0 / 1025.0, k5), (-301.0 / 82.0, k6),
                       (2133.0 / 4100.0, k7), (45.0 / 82.0, k8), (45.0 / 164.0, k9), (18.0 / 41.0, k10)], dt),
            t + dt)
    return _chain(y, [(41.0 / 840.0, k1), (34.0 / 105.0, k6), (9.0 / 35.0, k7), (9.0 / 35.0, k8),
                      (9.0 / 280.0, k9), (9.0 / 280.0, k10), (41.0 / 840.0, k11)], dt)


def _bs(f, y, t, dt):
    h = dt / 4
    prev = y.copy()
    k = f(y, t)
    mid = 1.0 * y + h * k
    for i in range(1, 4):
        k = f(mid, t + i * h)
        nxt = 1.0 * prev + (2.0 * h) * k
        prev, mid = mid, nxt
    k = f(mid, t + dt)
    nxt = 0.5 * mid + 0.5 * prev
    return 1.0 * nxt + (0.5 * h) * k


# Five-stage third-order SSP tableau as the reference writes it (15 digits).
_SSP = dict(a30=0.355909775063327, a32=0.644090224936674, a40=0.367933791638137, a43=0.632066208361863,
            a52=0.237593836598569, a54=0.762406163401431, b10=0.377268915331368, b21=0.377268915331368,
            b32=0.242995220537396, b43=0.238458932846290, b54=0.287632146308408, c1=0.377268915331368,
            c2=0.754537830662736, c3=0.728985661612188, c4=0.699226135931670)


def _ssprk53(f, y, t, dt):
    s = _SSP
    tmp = 1.0 * y + (s["b10"] * dt) * f(y, t)
    u = 1.0 * tmp + (s["b21"] * dt) * f(tmp, t + s["c1"] * dt)
    tmp = s["a30"] * y + s["a32"] * u + (s["b32"] * dt) * f(u, t + s["c2"] * dt)
    tmp = s["a40"] * y + s["a43"] * tmp + (s["b43"] * dt) * f(tmp, t + s["c3"] * dt)
    return s["a52"] * u + s["a54"] * tmp + (s["b54"] * dt) * f(tmp, t + s["c4"] * dt)


def _rk_tableau(f, y, t, dt, A, c, b):
    ks = []
    for i in range(len(c)):
        yi = y + dt * sum(A[i][j] * ks[j] for j in range(i)) if i else y
        ks.append(f(yi, t + c[i] * dt))
    return y + dt * sum(bj * k for bj, k in zip(b, ks))


_CK = ([[], [1 / 5], [3 / 40, 9 / 40], [3 / 10, -9 / 10, 6 / 5], [-11 / 54, 5 / 2, -70 / 27, 35 / 27],
        [1631 / 55296, 175 / 512, 575 / 13824, 44275 / 110592, 253 / 4096]],
       [0, 1 / 5, 3 / 10, 3 / 5, 1, 7 / 8], [37 / 378, 0, 250 / 621, 125 / 594, 0, 512 / 1771])
_DP = ([[], [1 / 5], [3 / 40, 9 / 40], [44 / 45, -56 / 15, 32 / 9],
        [19372 / 6561, -25360 / 2187, 64448 / 6561, -212 / 729],
        [9017 / 3168, -355 / 33, 46732 / 5247, 49 / 176, -5103 / 18656]],
       [0, 1 / 5, 3 / 10, 4 / 5, 8 / 9, 1], [35 / 384, 0, 500 / 1113, 125 / 192, -2187 / 6784, 11 / 84])


def step(f, y, t, dt, method):
    """One fixed step of ``method`` (a reference GPU method name) of dy/dt = f(y, t)."""
    y = np.asarray(y, dtype=np.float64)
    if method == "euler":
        return 1.0 * y + dt * f(y, t)
    if method in ("rk2", "midpoint"):
        tmp = 1.0 * y + (0.5 * dt) * f(y, t)
        return 1.0 * y + dt * f(tmp, t + 0.5 * dt)
    if method == "rk4":
        k1 = f(y, t)
        k2 = f(y + (0.5 * dt) * k1, t + 0.5 * dt)
        k3 = f(y + (0.5 * dt) * k2, t + 0.5 * dt)
        k4 = f(y + dt * k3, t + dt)
        return y + (dt / 6.0) * (k1 + 2.0 * k2 + 2.0 * k3 + k4)
    if method in ("rk5", "rkck54"):
        return _rk_tableau(f, y, t, dt, *_CK)
    if method in ("dopri5", "rk54", "rkf54"):
        return _rk_tableau(f, y, t, dt, *_DP)
    if method in ("rk78", "rkf78"):
        return _rk78(f, y, t, dt)
    if method in ("bs", "bulirsch_stoer"):
        return _bs(f, y, t, dt)
    if method == "ssprk53":
        return _ssprk53(f, y, t, dt)
    raise ValueError(f"unknown method {method!r}")


def integrate(f, y, T0, T1, dt, save_interval, method):
    """The reference GPU loop (integrator.cuh:470-488): save every save_interval steps while t < T1
    with t += dt, and the final state.  Returns (times, states)."""
    y = np.asarray(y, dtype=np.float64).copy()
    t, k = T0, 0
    times, states = [], []
    while t < T1:
        if k % save_interval == 0:
            times.append(t)
            states.append(y.copy())
        y = step(f, y, t, dt, method)
        t += dt
        k += 1
    times.append(t)
    states.append(y.copy())
    return np.array(times), np.array(states)
