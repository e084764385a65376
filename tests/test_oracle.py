"""The CPU oracle against the reference's own code, golden vectors and known answers.

The reference ships no golden vectors for the LL path and its CPU integrator
cannot be built here (Eigen3 / Boost / HDF5 / MPI are absent), so the oracle is
pinned three ways: (1) the reference's pulse_chunking.h and its own test,
compiled in place into oracle/_ref; (2) fixtures produced by the reference's
own GPU integrator (src/gpu/lattice_gpu.cu, compiled in place) on a B200,
committed under tests/golden/; (3) analytic known answers.
"""
import ctypes as C
import subprocess
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"


def _spins(n, seed):
    from classical_mcmc_spin_b200.states import random_unit_spins
    return random_unit_spins(n, seed).ravel()


def test_reference_chunking_test_binary_passes(oracle):
    exe = oracle.REF_DIR / "test_pulse_chunking_alignment"
    if not exe.exists():
        pytest.skip("oracle/_ref not built (needs the reference tree)")
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0 and "PASS" in out.stdout


@pytest.mark.parametrize("case", range(40))
def test_pulse_segments_match_reference(oracle, case):
    if not oracle.ref_available("libref_chunking.so"):
        pytest.skip("oracle/_ref not built")
    rng = np.random.default_rng(case)
    T0 = float(rng.choice([0.0, -5.0, -1.3]))
    T_step = float(rng.choice([0.01, 0.02, 0.005, 0.013]))
    T1 = T0 + float(rng.uniform(1, 200))
    width = float(rng.uniform(0.1, 2.0))
    centers = rng.uniform(T0 - 10, T1 + 10, size=int(rng.integers(1, 3)))
    a = oracle.pulse_segments(T0, T1, centers, 9.0 * width, T_step)
    b = oracle.ref_pulse_segments(T0, T1, centers, 9.0 * width, T_step)
    assert a.shape == b.shape
    np.testing.assert_array_equal(a, b)


def test_lattice_tables_reverse_transpose(oracle):
    L = oracle.OracleLattice.kitaev(4, 5, 1)
    off, part, J = L.csr()
    N = L.N
    assert off[-1] == 3 * N and np.all(np.diff(off) == 3)
    # every entry i->p with J has a partner entry p->i with J^T
    for i in range(N):
        for k in range(off[i], off[i + 1]):
            p = part[k]
            back = [q for q in range(off[p], off[p + 1]) if part[q] == i and np.array_equal(J[q], J[k].T)]
            assert back, (i, p)


def test_single_spin_precession(oracle):
    """dS/dt = H x S with H = -B z: S_x(t) = cos(Bt) S_x0 + sin(Bt) S_y0 (known answer)."""
    uc = oracle.UnitCell()
    uc.n_atoms = 1
    for r in range(3):
        uc.frames[4 * r] = 1.0
    uc.afm[0] = 1.0
    B = 0.7
    uc.field[2] = B
    uc.n_bonds = 0
    L = oracle.OracleLattice(uc, 1, 1, 1)
    s0 = np.array([0.6, 0.0, 0.8])
    rows, s = L.md_rk4(s0, 0.0, 10.0, 0.001)
    t = 10.0
    expect = np.array([np.cos(B * t) * 0.6, -np.sin(B * t) * 0.6, 0.8])
    np.testing.assert_allclose(s, expect, atol=1e-10)


def test_ferromagnet_ground_state_is_stationary(oracle):
    L = oracle.OracleLattice.kitaev(6, 6, 1, K=0.0, Gamma=0.0, Gammap=0.0, J=-1.0)
    s = np.tile([0.0, 0.0, 1.0], L.N)
    assert L.rhs(s).max() == 0.0 and L.rhs(s).min() == 0.0


def test_energy_conservation_and_norm(oracle):
    L = oracle.OracleLattice.kitaev(6, 6, 1)
    s = _spins(L.N, 3)
    rows, fin = L.md_rk4(s, 0.0, 5.0, 0.01)
    E = rows[:, 10]
    assert np.abs(E - E[0]).max() < 1e-7 * abs(E[0]) + 1e-9
    assert np.abs(np.linalg.norm(fin.reshape(-1, 3), axis=1) - 1).max() < 1e-8


def test_energy_identity_used_by_the_kernel(oracle):
    """total_energy_flat == 1/2 sum_i S_i.(H_i - B_i) (H = static local field)."""
    L = oracle.OracleLattice.kitaev(5, 4, 1, h=0.3, direction=(0.2, 0.9, 0.1), Ka=0.1, Kb=0.05, Kc=-0.2)
    s = _spins(L.N, 4)
    H = L.local_field(s).reshape(-1, 3)
    Bf = L.ell()["field"].reshape(-1, 3)
    e = 0.5 * np.sum(s.reshape(-1, 3) * (H - Bf))
    assert abs(e - L.energy(s)) < 1e-12 * L.N


def test_dopri5_converges_to_rk4(oracle):
    L = oracle.OracleLattice.kitaev(4, 4, 1)
    s = _spins(L.N, 5)
    r1, f1 = L.md_rk4(s, 0.0, 2.0, 0.0005)
    r2, f2, st = L.md_dopri5(s, 0.0, 2.0, 0.01, 1e-12, 1e-12)
    assert np.abs(f1 - f2).max() < 1e-9
    assert st[0] > 0


def test_pulse_drive_cpu_semantics(oracle):
    """single_pulse_drive: observer skips t = T_start and records every step after."""
    L = oracle.OracleLattice.kitaev(3, 3, 1)
    s = _spins(L.N, 6)
    d = np.tile(np.ones(3) / np.sqrt(3), 2)
    rows = L.pulse_drive(s, d, 0.0, None, 0.0, 1, 0.5, 0.5, 0.0, -1.0, 1.0, 0.01)
    assert rows.shape[0] == 200
    np.testing.assert_allclose(rows[0, 0], -0.99, atol=1e-12)


def _golden(name):
    p = GOLDEN / name
    if not p.exists():
        pytest.skip(f"{name} not generated yet (tests/golden/make_golden.py on a GPU)")
    return np.load(p)


@pytest.mark.parametrize("name", ["ref_gpu_rk4_kitaev.npz", "ref_gpu_rk4_kitaev24.npz", "ref_gpu_rk4_pyrochlore.npz"])
def test_oracle_matches_reference_gpu_rk4_golden(oracle, name):
    """The reference's own GPU integrator (integrate_gpu, 'rk4') vs the oracle, saved states."""
    g = _golden(name)
    if "pyrochlore" in name:
        R111 = np.ones(3) / np.sqrt(3.0)
        L = oracle.OracleLattice.pyrochlore_nk(*[int(x) for x in g["dims"]], h=float(g["h"]), direction=R111,
                                               Jzz=1.0, Jpm=0.05, Jpmpm=0.02)
    else:
        L = oracle.OracleLattice.kitaev(int(g["d1"]), int(g["d2"]), 1)
    s = g["init"].copy()
    save = int(g["save_interval"])
    dt = float(g["dt"])
    t = 0.0
    steps = 0
    for r, t_ref in enumerate(g["times"]):
        assert abs(t - t_ref) <= 1e-12
        assert np.abs(s - g["states"][r]).max() < 1e-12, r
        if r + 1 < len(g["times"]):
            n = save if r + 2 < len(g["times"]) else int(round((g["times"][r + 1] - t_ref) / dt))
            for k in range(n):
                s = L.rk4_step(s, t, dt, gpu_form=True)
                t += dt
                steps += 1
    assert steps > 0


def test_oracle_matches_reference_gpu_driven_golden(oracle):
    """Driven run (two Gaussian pulses) of the reference GPU integrator vs the oracle."""
    g = _golden("ref_gpu_rk4_kitaev_driven.npz")
    L = oracle.OracleLattice.kitaev(int(g["d1"]), int(g["d2"]), 1)
    L.set_pulse(g["field_in1"], float(g["t1"]), g["field_in2"], float(g["t2"]), float(g["amp"]),
                float(g["width"]), float(g["freq"]))
    rows, fin = L.md_rk4(g["init"], float(g["T0"]), float(g["T1"]), float(g["dt"]), 1, gpu_loop=True)
    assert len(rows) == len(g["times"])
    np.testing.assert_allclose(rows[:, 0], g["times"], rtol=0, atol=0)
    assert np.abs(fin - g["final"]).max() < 1e-11
    assert np.abs(rows[:, 1:10] - g["mags"]).max() < 1e-12


def test_oracle_matches_reference_gpu_batched_golden(oracle):
    """integrate_gpu_batched of the reference (M0 + M01(tau) replicas) vs the oracle."""
    g = _golden("ref_gpu_batched_kitaev.npz")
    L = oracle.OracleLattice.kitaev(int(g["d1"]), int(g["d2"]), 1)
    for b, tau in enumerate(g["tau2"]):
        L.set_pulse(g["field_in"], 0.0, g["field_in"], float(tau), float(g["amp"]), float(g["width"]),
                    float(g["freq"]))
        s = g["init"].copy()
        t = float(g["T0"])
        dt = float(g["dt"])
        for r in range(len(g["times"])):
            assert t == g["times"][r]
            m = L.magnetizations(s)
            assert np.abs(m - g["mags"][r, b]).max() < 1e-12, (b, r)
            if r + 1 < len(g["times"]):
                s = L.rk4_step(s, t, dt, gpu_form=True)
                t += dt
