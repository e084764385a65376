"""The mixed SU(2)/SU(3) path on the GPU (cmd_mixed.h through mixed_gpu_api) against the oracle's numpy
restatement and against the reference's own mixed GPU code (oracle/_ref/libref_mixed.so).

Tolerances: states <= 1e-12 after 20 steps (the two sides sum the same terms in another order);
magnetisations <= 1e-14.  Lattices: seeded TmFeO3-shaped synthetic lattices of 8 sites per cell with a
two-pulse drive on both kinds of site: 2x2x2 cells (one CTA), 3^3, 4^3, 5^3 and 6^3 cells (clusters of
2, 4, 8 and 16 CTAs) and 12^3 (13824 sites on 16 CTAs of 512 threads: two sites per thread)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

METHODS = ["ssprk53", "rk4", "dopri5", "rk5", "rk78", "bs", "euler", "rk2"]


@pytest.fixture(scope="module")
def mg(native):
    from classical_mcmc_spin_b200 import mixed_gpu_api
    return mixed_gpu_api


@pytest.fixture(scope="module")
def mo(oracle):
    import mixed_oracle
    return mixed_oracle


def _pulses(arr):
    rng = np.random.default_rng(9)
    return {2: (rng.normal(size=(2, arr["na2"], 3)), 0.6, 0.3, 1.2, 0.05, 0.25),
            3: (rng.normal(size=(2, arr["na3"], 8)), 0.4, 0.2, 0.8, 0.1, 0.3)}


def _setup(mg, mo, L, seed, driven=True):
    arr = mg.synthetic_mixed_lattice(L, seed=seed)
    h = mg.create_from(arr)
    o = mo.MixedOracle(arr)
    if driven:
        for sub, (fd, *p) in _pulses(arr).items():
            (mg.set_gpu_pulse_SU2 if sub == 2 else mg.set_gpu_pulse_SU3)(h, fd.ravel(), *p)
            o.set_pulse(sub, fd, *p)
    return arr, h, o


@pytest.mark.parametrize("method", METHODS)
def test_mixed_matches_oracle(mg, mo, method):
    import fixed_methods as fm
    arr, h, o = _setup(mg, mo, (2, 2, 2), 11)
    y0 = mg.random_mixed_state(arr, 12)
    mg.set_gpu_mixed_spins(h, y0)
    traj, times = mg.integrate_mixed_gpu(h, 0.0, 0.4, 0.02, 5, method)
    rt, rs = fm.integrate(lambda y, t: o.rhs(y, t), y0, 0.0, 0.4, 0.02, 5, method)
    np.testing.assert_array_equal(times, rt)
    assert np.abs(np.stack([s for _, s in traj]) - rs).max() <= 1e-12
    np.testing.assert_array_equal(mg.get_gpu_mixed_spins(h), traj[-1][1])


@pytest.mark.parametrize("method", ["ssprk53", "rk4", "dopri5", "rk78", "bs"])
def test_mixed_matches_reference_gpu(mg, mo, oracle, method):
    if not (mo.REF_DIR / "libref_mixed.so").exists():
        pytest.skip("oracle/_ref/libref_mixed.so not built")
    arr, h, _ = _setup(mg, mo, (2, 2, 2), 13)
    y0 = mg.random_mixed_state(arr, 14)
    ref = mo.RefMixedGPU(arr)
    for sub, (fd, *p) in _pulses(arr).items():
        ref.set_pulse(sub, fd, *p)
    ref.set_spins(y0)
    rt, rs = ref.integrate(0.0, 0.4, 0.02, 5, method)
    ref.set_spins(y0)
    ref.step(0.1, 0.02, method)
    r1 = ref.get_spins()
    ref.set_spins(rs[-1])
    rm = ref.magnetization()
    ref.normalize(1.5, 0.7)
    rn = ref.get_spins()
    ref.close()
    mg.set_gpu_mixed_spins(h, y0)
    traj, times = mg.integrate_mixed_gpu(h, 0.0, 0.4, 0.02, 5, method)
    np.testing.assert_array_equal(times, rt)
    assert np.abs(np.stack([s for _, s in traj]) - rs).max() <= 1e-12
    mg.set_gpu_mixed_spins(h, y0)
    mg.step_mixed_gpu(h, 0.1, 0.02, method)
    assert np.abs(mg.get_gpu_mixed_spins(h) - r1).max() <= 1e-14
    mg.set_gpu_mixed_spins(h, rs[-1])
    for a, b in zip(mg.compute_magnetization_mixed_gpu(h), rm):
        assert np.abs(a - b).max() <= 1e-14
    mg.normalize_spins_mixed_gpu(h, 1.5, 0.7)
    assert np.abs(mg.get_gpu_mixed_spins(h) - rn).max() <= 1e-14


@pytest.mark.parametrize("L", [(3, 3, 3), (4, 4, 4), (5, 5, 5), (6, 6, 6), (12, 12, 12)])
def test_mixed_cluster_sizes_match_oracle(mg, mo, L):
    import fixed_methods as fm
    arr, h, o = _setup(mg, mo, L, 15)
    y0 = mg.random_mixed_state(arr, 16)
    mg.set_gpu_mixed_spins(h, y0)
    traj, times = mg.integrate_mixed_gpu(h, 0.0, 0.1, 0.02, 5, "rk4")
    rt, rs = fm.integrate(lambda y, t: o.rhs(y, t), y0, 0.0, 0.1, 0.02, 5, "rk4")
    np.testing.assert_array_equal(times, rt)
    assert np.abs(np.stack([s for _, s in traj]) - rs).max() <= 1e-12
    for a, b in zip(mg.compute_magnetization_mixed_gpu(h), o.magnetizations(traj[-1][1])):
        assert np.abs(a - b).max() <= 1e-14


def test_mixed_long_run_conserves(mg, mo):
    """No drive: energy and lengths over 2000 RK4 steps, on the GPU (drift of the method only)."""
    arr, h, o = _setup(mg, mo, (6, 6, 6), 17, driven=False)
    y0 = mg.random_mixed_state(arr, 18)
    mg.set_gpu_mixed_spins(h, y0)
    mg.integrate_mixed_gpu(h, 0.0, 10.0, 0.005, 2000, "rk4")
    y = mg.get_gpu_mixed_spins(h)
    n2 = arr["n2"]
    assert abs(o.energy(y) - o.energy(y0)) <= 1e-8 * abs(o.energy(y0))
    assert np.abs(np.linalg.norm(y[:3 * n2].reshape(-1, 3), axis=1) - 1).max() <= 1e-9
    assert np.abs(np.linalg.norm(y[3 * n2:].reshape(-1, 8), axis=1) - 1).max() <= 1e-9


def test_mixed_api_behaviour(mg, native):
    from classical_mcmc_spin_b200._native import CmdError
    arr = mg.synthetic_mixed_lattice((2, 2, 2), seed=19)
    h = mg.create_from(arr)
    assert mg.get_mixed_lattice_dims(h) == (arr["n2"], 3, arr["na2"], arr["n3"], 8, arr["na3"])
    with pytest.raises(CmdError) as e:
        mg.step_mixed_gpu(h, 0.0, 0.01)
    assert e.value.code == native.CMD_ERR_STATE
    y0 = mg.random_mixed_state(arr, 20)
    bad = y0.copy()
    bad[7] = np.inf
    with pytest.raises(CmdError) as e:
        mg.set_gpu_mixed_spins(h, bad)
    assert e.value.code == native.CMD_ERR_NONFINITE
    mg.set_gpu_mixed_spins(h, y0)
    with pytest.raises(CmdError) as e:
        mg.step_mixed_gpu(h, 0.0, 0.01, native.CMD_RK45)
    assert e.value.code == native.CMD_ERR_INVALID_ARG
    mg.step_mixed_gpu(h, 0.0, 0.01)                     # the reference default, ssprk53
    a = mg.get_gpu_mixed_spins(h)
    mg.set_gpu_mixed_spins(h, y0)
    mg.step_mixed_gpu(h, 0.0, 0.01, "ssprk53")
    np.testing.assert_array_equal(a, mg.get_gpu_mixed_spins(h))
    h.close()


def test_mixed_faster_than_reference_gpu(mg, mo, capsys):
    """The 1728-site TmFeO3-shaped lattice (6x6x6 cells), 400 RK4 steps: the B200 path against the reference's
    own mixed GPU code on the same GPU (wall clock around each integrate call, after a warm-up).  The
    reference launches two RHS kernels and an update kernel per stage with a device synchronisation after
    each; this path runs one persistent cluster launch.  Asserts a conservative 3x margin and prints both."""
    import time
    if not (mo.REF_DIR / "libref_mixed.so").exists():
        pytest.skip("oracle/_ref/libref_mixed.so not built")
    arr = mg.synthetic_mixed_lattice((6, 6, 6), seed=30)
    y0 = mg.random_mixed_state(arr, 32)
    S, dt = 400, 0.005
    ref = mo.RefMixedGPU(arr)
    ref.set_spins(y0)
    ref.integrate(0.0, 0.05, dt, 10, "rk4")
    ref.set_spins(y0)
    t0 = time.perf_counter()
    _, rs = ref.integrate(0.0, S * dt, dt, S, "rk4")
    t_ref = time.perf_counter() - t0
    ref.close()
    h = mg.create_from(arr)
    mg.set_gpu_mixed_spins(h, y0)
    mg.integrate_mixed_gpu(h, 0.0, 0.05, dt, 10, "rk4")
    mg.set_gpu_mixed_spins(h, y0)
    t0 = time.perf_counter()
    traj, _ = mg.integrate_mixed_gpu(h, 0.0, S * dt, dt, S, "rk4")
    t_b200 = time.perf_counter() - t0
    assert np.abs(traj[-1][1] - rs[-1]).max() <= 1e-10
    with capsys.disabled():
        print(f"\nmixed 6x6x6 RK4: reference {t_ref / (4 * S) * 1e6:.1f} us/stage, "
              f"B200 {t_b200 / (4 * S) * 1e6:.1f} us/stage, {t_ref / t_b200:.1f}x")
    assert t_ref >= 3.0 * t_b200


def test_mixed_ragged_tables_match_reference_gpu(mg, mo):
    """Ragged ELL tables: per-site counts below the width and partners outside the lattice (the reference
    skips them, mixed_lattice_gpu.cu:92-118, 157-185); the unused slots hold garbage matrices, which must not
    enter.  Against the reference's own code and the oracle."""
    import fixed_methods as fm
    if not (mo.REF_DIR / "libref_mixed.so").exists():
        pytest.skip("oracle/_ref/libref_mixed.so not built")
    arr = mg.synthetic_mixed_lattice((2, 2, 2), seed=40)
    rng = np.random.default_rng(41)
    for kp, kc, kv, z, n, limit, w in (("part2", "cnt2", "bil2", arr["z2"], arr["n2"], arr["n2"], 9),
                                       ("part3", "cnt3", "bil3", arr["z3"], arr["n3"], arr["n3"], 64),
                                       ("mpart2", "mcnt2", "mix2", arr["zm2"], arr["n2"], arr["n3"], 24),
                                       ("mpart3", "mcnt3", "mix3", arr["zm3"], arr["n3"], arr["n2"], 24)):
        cnt = rng.integers(0, z + 1, size=n)
        part = arr[kp].reshape(n, z).copy()
        part[rng.random((n, z)) < 0.2] = limit + rng.integers(0, 5)     # outside the lattice
        val = arr[kv].reshape(n, z, w).copy()
        for s in range(n):
            val[s, cnt[s]:] = rng.normal(size=(z - cnt[s], w)) * 100     # never read
        arr[kc], arr[kp], arr[kv] = cnt.astype(np.int64), part.ravel(), val.ravel()
    y0 = mg.random_mixed_state(arr, 42)
    h = mg.create_from(arr)
    mg.set_gpu_mixed_spins(h, y0)
    traj, times = mg.integrate_mixed_gpu(h, 0.0, 0.2, 0.02, 5, "rk4")
    ref = mo.RefMixedGPU(arr)
    ref.set_spins(y0)
    rt, rs = ref.integrate(0.0, 0.2, 0.02, 5, "rk4")
    ref.close()
    np.testing.assert_array_equal(times, rt)
    assert np.abs(np.stack([s for _, s in traj]) - rs).max() <= 1e-12
    o = mo.MixedOracle(arr)
    _, os_ = fm.integrate(lambda y, t: o.rhs(y, t), y0, 0.0, 0.2, 0.02, 5, "rk4")
    assert np.abs(np.stack([s for _, s in traj]) - os_).max() <= 1e-12
