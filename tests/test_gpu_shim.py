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


def test_mixed_shim_call_sequence(native, oracle, tmp_path):
    """The mixed_gpu:: call sequence through include/classical_spin/gpu/mixed_lattice_gpu_api.h: bit-identical
    to the Python mirror (same library); no-ops, dims and the unknown-method fall-back as in the reference."""
    from classical_mcmc_spin_b200 import mixed_gpu_api as mg
    exe = build_shim_program(tmp_path / "mixed_shim_calls", "mixed_shim_calls.cpp")
    arr = mg.synthetic_mixed_lattice((2, 2, 3), seed=21)
    y0 = mg.random_mixed_state(arr, 22)
    rng = np.random.default_rng(23)
    d2, d3 = rng.normal(size=2 * arr["na2"] * 3), rng.normal(size=2 * arr["na3"] * 8)
    d = tmp_path / "io"
    d.mkdir()
    (d / "meta.txt").write_text(" ".join(str(arr[k]) for k in ("n2", "na2", "n3", "na3", "z2", "z3", "zm2", "zm3")))
    for k in ("field2", "onsite2", "bil2", "field3", "onsite3", "bil3", "mix2", "mix3"):
        np.ascontiguousarray(arr[k], dtype=np.float64).tofile(d / f"{k}.bin")
    for k in ("part2", "cnt2", "part3", "cnt3", "mpart2", "mcnt2", "mpart3", "mcnt3"):
        np.ascontiguousarray(arr[k], dtype=np.uint64).tofile(d / f"{k}.bin")
    for k, v in (("spins", y0), ("drive2", d2), ("drive3", d3)):
        np.ascontiguousarray(v, dtype=np.float64).tofile(d / f"{k}.bin")
    r = subprocess.run([str(exe), str(d)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "Unknown GPU integration method 'no_such_method', using ssprk53" in r.stderr
    np.testing.assert_array_equal(_load(d, "noop"), [1.0, 0.0, 0.0, arr["n2"], 3, arr["na2"], arr["n3"], 8,
                                                     arr["na3"]])
    h = mg.create_from(arr)
    mg.set_gpu_pulse_SU2(h, d2, 0.6, 0.3, 1.2, 0.05, 0.25)
    mg.set_gpu_pulse_SU3(h, d3, 0.4, 0.2, 0.8, 0.1, 0.3)
    mg.set_gpu_mixed_spins(h, y0)
    traj, times = mg.integrate_mixed_gpu(h, 0.0, 0.4, 0.02, 5)
    np.testing.assert_array_equal(_load(d, "traj_times"), times)
    np.testing.assert_array_equal(_load(d, "traj_states").reshape(len(times), -1), np.stack([s for _, s in traj]))
    mg.step_mixed_gpu(h, 0.4, 0.02, "rk4")
    np.testing.assert_array_equal(_load(d, "step_rk4"), mg.get_gpu_mixed_spins(h))
    mg.step_mixed_gpu(h, 0.42, 0.02, "ssprk53")
    np.testing.assert_array_equal(_load(d, "step_fallback"), mg.get_gpu_mixed_spins(h))
    np.testing.assert_array_equal(_load(d, "mags"), np.concatenate(mg.compute_magnetization_mixed_gpu(h)))
    mg.normalize_spins_mixed_gpu(h, 1.5, 0.7)
    np.testing.assert_array_equal(_load(d, "normalized"), mg.get_gpu_mixed_spins(h))
