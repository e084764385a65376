"""The reference GPU integrator's other fixed-step methods (integrator.cuh:91-452: euler, rk2 /
midpoint, ssprk53 -- the API's default --, rk78 / rkf78, bulirsch_stoer / bs, rk54 / rkf54) through
the C ABI, against the reference's own GPU code built from its sources (oracle/_ref/libref_gpu.so),
with a two-pulse drive on so every stage time t + c dt enters.

Tolerance: states <= 1e-12 after 50 steps (the two sides differ only in the FMA contraction of
the same update expressions); observables of each saved row <= 1e-13 of the oracle's
magnetisations of the reference's state.  The same methods are also checked against the oracle's
numpy restatement (oracle/fixed_methods.py), whose convergence orders the CPU suite pins.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

R111 = np.ones(3) / np.sqrt(3.0)
NAMES = ["ssprk53", "euler", "rk2", "midpoint", "rk78", "rkf78", "bs", "bulirsch_stoer", "rk54", "rkf54"]


@pytest.fixture(scope="module")
def api(native):
    from classical_mcmc_spin_b200 import gpu_api
    return gpu_api


def _spins(n, seed):
    from classical_mcmc_spin_b200.states import random_unit_spins
    return random_unit_spins(n, seed).ravel()


def _pair(oracle, kind):
    from classical_mcmc_spin_b200.lattice import Lattice
    if kind == "kitaev":
        return (Lattice.kitaev(6, 6, 1, h=0.3, field_direction=(0.0, 1.0, 0.0)),
                oracle.OracleLattice.kitaev(6, 6, 1, h=0.3, direction=(0.0, 1.0, 0.0)))
    kw = dict(Jzz=1.0, Jpm=0.05, Jpmpm=0.02)
    return (Lattice.pyrochlore_non_kramer(2, 2, 2, h=0.2, field_direction=R111, **kw),
            oracle.OracleLattice.pyrochlore_nk(2, 2, 2, h=0.2, direction=R111, **kw))


@pytest.mark.parametrize("kind", ["kitaev", "pyro"])
@pytest.mark.parametrize("method", NAMES)
def test_method_matches_reference_gpu(api, oracle, method, kind):
    if not oracle.ref_available("libref_gpu.so"):
        pytest.skip("oracle/_ref/libref_gpu.so not built")
    lat, o = _pair(oracle, kind)
    s0 = _spins(lat.lattice_size, 61)
    fin = np.tile(R111, lat.N_atoms)
    fd = lat.rotate_pulse(fin, fin)
    pulse = (0.5, 0.4, 0.9, 0.2, 0.6)                      # amp, width, freq, t1, t2
    ref = oracle.RefGPU(o.ell(), o.n_atoms)
    ref.set_pulse(fd, *pulse)
    ref.set_spins(s0)
    rt, rs = ref.integrate(0.0, 1.0, 0.02, save_interval=5, method=method)
    ref.set_spins(s0)
    ref.step(0.1, 0.02, method=method)
    r1 = ref.get_spins()
    ref.close()
    h = lat.to_gpu()
    api.set_gpu_pulse(h, fd, *pulse)
    api.set_gpu_spins(h, s0)
    traj, obs, times = api.integrate_gpu(h, 0.0, 1.0, 0.02, 5, method)
    np.testing.assert_array_equal(times, rt)
    assert np.abs(np.stack([s for _, s in traj]) - rs).max() <= 1e-12
    for r in range(len(rt)):
        assert np.abs(obs[r, :9] - o.magnetizations(rs[r])).max() <= 1e-13
    api.set_gpu_spins(h, s0)
    api.step_gpu(h, 0.1, 0.02, method)
    assert np.abs(api.get_gpu_spins(h) - r1).max() <= 1e-14


def test_default_method_is_ssprk53(api, oracle):
    lat, _ = _pair(oracle, "kitaev")
    s0 = _spins(lat.lattice_size, 62)
    h = lat.to_gpu()
    api.set_gpu_spins(h, s0)
    api.step_gpu(h, 0.0, 0.05)
    a = api.get_gpu_spins(h)
    api.set_gpu_spins(h, s0)
    api.step_gpu(h, 0.0, 0.05, "ssprk53")
    np.testing.assert_array_equal(a, api.get_gpu_spins(h))


@pytest.mark.parametrize("method", ["ssprk53", "euler", "rk2", "rk78", "bs", "rk5", "dopri5", "rk4"])
def test_method_matches_oracle_restatement(api, oracle, method):
    """The same methods against oracle/fixed_methods.py over the oracle's RHS (64 steps, drive on)."""
    import fixed_methods as fm
    lat, o = _pair(oracle, "pyro")
    s0 = _spins(lat.lattice_size, 64)
    fin = np.tile(R111, lat.N_atoms)
    api_h = lat.to_gpu()
    api.set_gpu_pulse(api_h, lat.rotate_pulse(fin, fin), 0.5, 0.4, 0.9, 0.2, 0.6)
    o.set_pulse(fin, 0.2, fin, 0.6, 0.5, 0.4, 0.9)
    api.set_gpu_spins(api_h, s0)
    traj, _, times = api.integrate_gpu(api_h, 0.0, 1.0, 1.0 / 64, 16, method)
    rt, rs = fm.integrate(lambda y, t: o.rhs(y, t), s0, 0.0, 1.0, 1.0 / 64, 16, method)
    np.testing.assert_array_equal(times, rt)
    assert np.abs(np.stack([s for _, s in traj]) - rs).max() <= 1e-12
