"""The reference's call sequence through the header-only drop-in (tests/cpp/shim_calls.cpp over
include/classical_spin/gpu/lattice_gpu_api.h) on the GPU: identical results to the Python mirror
(same library, so bit-exact) and to the reference's own GPU code (oracle/_ref) within the parity
tolerances (states 1e-12, magnetisations 1e-12); the reference's no-op and fall-back behaviour."""
import subprocess

import numpy as np
import pytest

from shim_build import build_shim_program

pytestmark = pytest.mark.gpu

R111 = np.ones(3) / np.sqrt(3.0)


def _spins(n, seed):
    from classical_mcmc_spin_b200.states import random_unit_spins
    return random_unit_spins(n, seed).ravel()


def _load(d, name):
    return np.fromfile(d / f"out_{name}.bin", dtype=np.float64)


def test_shim_call_sequence(native, oracle, tmp_path):
    from classical_mcmc_spin_b200 import gpu_api as api
    from classical_mcmc_spin_b200.lattice import Lattice
    exe = build_shim_program(tmp_path / "shim_calls")
    lat = Lattice.kitaev(6, 6, 1, h=0.3, field_direction=(0.0, 1.0, 0.0))
    o = oracle.OracleLattice.kitaev(6, 6, 1, h=0.3, direction=(0.0, 1.0, 0.0))
    ell = o.ell()
    N = lat.lattice_size
    s0 = _spins(N, 71)
    fd = lat.rotate_pulse(np.tile(R111, 2), np.tile(R111, 2))
    fr, afm = o.frames()
    tau2 = np.array([0.1, 0.5, 0.9])
    d = tmp_path / "io"
    d.mkdir()
    (d / "meta.txt").write_text(f"{N} {o.n_atoms} {ell['max_bilinear']}\n")
    for name, arr, dt in (("field", ell["field"], np.float64), ("onsite", ell["onsite"], np.float64),
                          ("bilinear", ell["bilinear"], np.float64), ("partners", ell["partners"], np.uint64),
                          ("counts", ell["counts"], np.uint64), ("spins", s0, np.float64),
                          ("drive", fd, np.float64), ("afm", afm, np.float64), ("frames", fr, np.float64),
                          ("tau2", tau2, np.float64)):
        np.ascontiguousarray(arr, dtype=dt).tofile(d / f"{name}.bin")
    r = subprocess.run([str(exe), str(d)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "Unknown GPU integration method 'no_such_method', using ssprk53" in r.stderr
    assert "method='dopri5' is not supported in batched mode; using rk4" in r.stderr

    np.testing.assert_array_equal(_load(d, "noop"), [1.0, 0.0, 0.0, 0.0])

    # Python mirror, same calls
    h = lat.to_gpu()
    api.set_gpu_pulse(h, fd, 0.5, 0.4, 0.9, 0.2, 0.6)
    api.set_gpu_spins(h, s0)
    traj, _, times = api.integrate_gpu(h, 0.0, 1.0, 0.02, 5)
    np.testing.assert_array_equal(_load(d, "traj_times"), times)
    np.testing.assert_array_equal(_load(d, "traj_states").reshape(len(times), -1), np.stack([s for _, s in traj]))
    api.step_gpu(h, 1.0, 0.02, "rk4")
    np.testing.assert_array_equal(_load(d, "step_rk4"), api.get_gpu_spins(h))
    api.step_gpu(h, 1.02, 0.02, "ssprk53")
    s_fb = api.get_gpu_spins(h)
    np.testing.assert_array_equal(_load(d, "step_fallback"), s_fb)
    ml, ms = api.compute_magnetization_gpu(h)
    sc = _load(d, "scalars")
    assert sc[0] == api.compute_energy_gpu(h)
    np.testing.assert_array_equal(sc[1:4], ml)
    np.testing.assert_array_equal(sc[4:7], ms)
    np.testing.assert_allclose(sc[7:10], np.array([1.0, 2.0, 3.0]) / N + ml, rtol=0, atol=1e-15)
    ref_m = s_fb.reshape(N, 3)
    np.testing.assert_allclose(ml, ref_m.mean(0), atol=1e-15)
    np.testing.assert_allclose(ms, (ref_m * np.where(np.arange(N) % 2 == 0, 1.0, -1.0)[:, None]).mean(0), atol=1e-15)
    assert abs(sc[0] - o.energy(s_fb)) <= 1e-12 * N
    normed = _load(d, "normalized").reshape(N, 3)
    np.testing.assert_allclose(np.linalg.norm(normed, axis=1), 2.0, atol=1e-14)
    res = api.integrate_gpu_batched(h, s0, tau2, afm, fr, -0.5, 1.0, 0.01, 2)
    np.testing.assert_array_equal(_load(d, "batched_times"), res.times)
    np.testing.assert_array_equal(_load(d, "batched_mags"), res.mag_data.ravel())
    np.testing.assert_array_equal(_load(d, "batched_shape"), [3, 3, res.n_time_points])
    np.testing.assert_array_equal(_load(d, "batched_empty"), [0, 0])

    # The reference's own GPU code, same calls
    if not oracle.ref_available("libref_gpu.so"):
        pytest.skip("oracle/_ref/libref_gpu.so not built")
    ref = oracle.RefGPU(ell, o.n_atoms)
    ref.set_pulse(fd, 0.5, 0.4, 0.9, 0.2, 0.6)
    ref.set_spins(s0)
    rt, rs = ref.integrate(0.0, 1.0, 0.02, save_interval=5, method="ssprk53")
    np.testing.assert_array_equal(_load(d, "traj_times"), rt)
    assert np.abs(_load(d, "traj_states").reshape(len(rt), -1) - rs).max() <= 1e-12
    ref.step(1.0, 0.02, method="rk4")
    ref.step(1.02, 0.02, method="no_such_method")
    assert np.abs(_load(d, "step_fallback") - ref.get_spins()).max() <= 1e-12
    bt, bm = ref.batched(s0, tau2, afm, fr, -0.5, 1.0, 0.01, save_interval=2)
    ref.close()
    np.testing.assert_array_equal(_load(d, "batched_times"), bt)
    assert np.abs(_load(d, "batched_mags").reshape(bm.shape) - bm).max() <= 1e-12
