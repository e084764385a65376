"""The command-line driver end to end on the GPU: molecular_dynamics, pump_probe and 2dcs param
files run through `cmd_spin_solver`, outputs compared with the oracle (rows <= 1e-12, states
<= 1e-10 as in the parity tests) and the 2DCS spectrum with the oracle's restatement of the
reference reader (<= 1e-12 of its maximum)."""
import json
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_S = 1e-10
TOL_M = 1e-12


@pytest.fixture(scope="module")
def driver(native):
    from classical_mcmc_spin_b200 import build
    return build.build_driver()


def _run(driver, tmp_path, text):
    p = tmp_path / "run.param"
    p.write_text(text)
    r = subprocess.run([str(driver), str(p)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    return r


def _state_file(tmp_path, n, seed):
    from classical_mcmc_spin_b200.states import random_unit_spins
    s = random_unit_spins(n, seed)
    path = tmp_path / "init.txt"
    np.savetxt(path, s, fmt="%.17e")
    return s.ravel(), path


def test_driver_molecular_dynamics(driver, tmp_path, oracle):
    s0, init = _state_file(tmp_path, 32, 3)
    out = tmp_path / "md"
    _run(driver, tmp_path, f"""system = honeycomb_kitaev
simulation_mode = molecular_dynamics
lattice_size = 4,4,1
K = -1.0
Gamma = 0.25
Gammap = -0.02
field_strength = 0.3
field_direction = 0,1,0
md_time_start = 0.0
md_time_end = 1.995
md_timestep = 0.01
md_save_interval = 10
md_integrator = rk4
initial_spin_config = {init}
output_dir = {out}
""")
    d = out / "sample_0"
    o = oracle.OracleLattice.kitaev(4, 4, 1, h=0.3, direction=(0, 1, 0))
    rows, fin = o.md_rk4(s0, 0.0, 1.995, 0.01, 10, gpu_loop=True)
    t = np.load(d / "trajectory_times.npy")
    np.testing.assert_array_equal(t, rows[:, 0])
    for name, cols in (("antiferro", slice(1, 4)), ("local", slice(4, 7)), ("global", slice(7, 10))):
        m = np.load(d / f"trajectory_magnetization_{name}.npy")
        assert np.abs(m - rows[:, cols]).max() <= TOL_M
    assert np.abs(np.load(d / "trajectory_energy_per_site.npy") - rows[:, 10]).max() <= TOL_M
    spins = np.load(d / "trajectory_spins.npy")
    np.testing.assert_array_equal(spins[0].ravel(), s0)
    assert np.abs(spins[-1].ravel() - fin).max() <= TOL_S
    assert np.abs(np.loadtxt(d / "initial_spins.txt").ravel() - s0).max() == 0.0
    meta = json.loads((d / "metadata.json").read_text())
    assert meta["rows"] == len(t) and meta["integration_method"] == "rk4"
    # the reference's trajectory.h5 layout from this run (hdf5_export)
    from classical_mcmc_spin_b200 import hdf5_export
    plan = {e.path: e for e in hdf5_export.plan_trajectory(d)}
    np.testing.assert_array_equal(plan["/trajectory/times"].data, t)
    assert plan["/trajectory/spins"].data.shape == spins.shape
    assert list(plan["/metadata/dimensions"].data) == [int(meta["dim1"]), int(meta["dim2"]), int(meta["dim3"])]


def test_driver_pump_probe(driver, tmp_path, oracle):
    s0, init = _state_file(tmp_path, 32, 4)
    out = tmp_path / "pp"
    _run(driver, tmp_path, f"""system = honeycomb_kitaev
simulation_mode = pump_probe
lattice_size = 4,4,1
pump_direction = 0,0,1
pump_amplitude = 0.5
pump_width = 0.4
pump_frequency = 0.3
pump_time = 0.5
md_time_start = 0.0
md_time_end = 1.5
md_timestep = 0.01
md_integrator = rk4
initial_spin_config = {init}
output_dir = {out}
""")
    traj = np.loadtxt(out / "sample_0" / "pump_probe_trajectory.txt")
    o = oracle.OracleLattice.kitaev(4, 4, 1)
    o.set_pulse(np.tile([0.0, 0.0, 1.0], 2), 0.5, np.zeros(6), 0.0, 0.5, 0.4, 0.3)
    rows, _ = o.md_rk4(s0, 0.0, 1.5, 0.01, 1, gpu_loop=True)
    assert traj.shape == (len(rows), 10)
    np.testing.assert_array_equal(traj[:, 0], rows[:, 0])
    assert np.abs(traj[:, 1:10] - rows[:, 1:10]).max() <= TOL_M


def test_driver_2dcs(driver, tmp_path, oracle):
    import spectra_oracle as so
    s0, init = _state_file(tmp_path, 32, 5)
    out = tmp_path / "2dcs"
    _run(driver, tmp_path, f"""system = honeycomb_kitaev
simulation_mode = 2dcs
lattice_size = 4,4,1
pump_direction = 0,0,1
pump_amplitude = 0.4
pump_width = 0.2
pump_frequency = 0.5
tau_start = -0.5
tau_end = 0.5
tau_step = 0.25
md_time_start = -1.0
md_time_end = 2.0
md_timestep = 0.01
md_integrator = rk4
initial_spin_config = {init}
output_dir = {out}
""")
    d = out / "sample_0"
    tau = np.load(d / "tau_scan_tau_values.npy")
    np.testing.assert_allclose(tau, [-0.5, -0.25, 0.0, 0.25, 0.5])
    times = np.load(d / "reference_times.npy")
    n_t = len(times)
    o = oracle.OracleLattice.kitaev(4, 4, 1)
    z = np.tile([0.0, 0.0, 1.0], 2)
    B = 1 + 2 * len(tau)
    t1, t2, s1, s2 = np.zeros(B), np.zeros(B), np.zeros(B), np.zeros(B)
    s1[0] = 1.0
    for k, tv in enumerate(tau):
        t2[1 + 2 * k] = tv
        s2[1 + 2 * k] = 1.0
        t2[2 + 2 * k] = tv
        s1[2 + 2 * k] = s2[2 + 2 * k] = 1.0
    _, obs = o.batch_rk4(np.tile(s0, (B, 1)), t1, t2, s1, s2, 0.4, 0.2, 0.5, z, z, -1.0, 0.01, n_t - 1)
    M = {}
    for q, name in enumerate(("antiferro", "local", "global")):
        m0 = np.load(d / f"reference_M_{name}.npy")
        m1 = np.load(d / f"tau_scan_M1_{name}.npy")
        m01 = np.load(d / f"tau_scan_M01_{name}.npy")
        assert np.abs(m0 - obs[0, :, 3 * q:3 * q + 3]).max() <= TOL_M
        assert np.abs(m1 - obs[1::2, :, 3 * q:3 * q + 3]).max() <= TOL_M
        assert np.abs(m01 - obs[2::2, :, 3 * q:3 * q + 3]).max() <= TOL_M
        M[name] = (m0, m1, m01)
    nl = np.load(d / "M_NL_local.npy")
    sp = np.load(d / "spectrum_local.npy")
    for c in range(3):
        np.testing.assert_array_equal(nl[c], so.nonlinear_signal(*M["local"], c))
        ref = so.compute_2d_fft(so.nonlinear_signal(*M["local"], c))
        assert np.abs(sp[c] - ref).max() <= 1e-12 * max(1.0, ref.max())
    meta = json.loads((d / "metadata.json").read_text())
    assert meta["tau_steps"] == 5 and meta["pulse_amp"] == 0.4
    assert meta["m1_synthesized"] == 0 and meta["max_dsdt_no_drive"] > 1e-3     # random state: M1 integrated
    # the reference's pump_probe_spectroscopy.h5 layout from this run (hdf5_export)
    from classical_mcmc_spin_b200 import hdf5_export
    plan = {e.path: e for e in hdf5_export.plan_pump_probe(d)}
    np.testing.assert_array_equal(plan["/tau_scan/tau_3/M01_local"].data, M["local"][2][3])
    assert plan["/metadata"].attrs["tau_steps"] == 5 and plan["/metadata"].attrs["dim1"] == 4


@pytest.mark.parametrize("integrator", ["rk5", "ssprk53", "rk78", "bs"])
def test_driver_md_with_the_reference_gpu_integrators(driver, tmp_path, integrator):
    """md_integrator = rk5 (the reference's example configs: fixed-step Cash-Karp) and the reference
    GPU's other fixed-step methods run as integrate_gpu with that method."""
    from classical_mcmc_spin_b200 import gpu_api
    from classical_mcmc_spin_b200.lattice import Lattice
    s0, init = _state_file(tmp_path, 72, 6)
    out = tmp_path / "rk5"
    _run(driver, tmp_path, f"""system = honeycomb_kitaev
simulation_mode = molecular_dynamics
lattice_size = 6,6,1
field_strength = 0.7
field_direction = 0.577,0.577,0.577
md_time_start = 0.0
md_time_end = 5.0
md_timestep = 0.25
md_save_interval = 1
md_integrator = {integrator}
initial_spin_config = {init}
output_dir = {out}
""")
    d = out / "sample_0"
    lat = Lattice.kitaev(6, 6, 1, h=0.7, field_direction=(0.577, 0.577, 0.577))
    h = lat.to_gpu()
    gpu_api.set_gpu_spins(h, s0)
    traj, obs, times = gpu_api.integrate_gpu(h, 0.0, 5.0, 0.25, 1, integrator)
    np.testing.assert_array_equal(np.load(d / "trajectory_times.npy"), times)
    np.testing.assert_array_equal(np.load(d / "trajectory_magnetization_local.npy"), obs[:, 3:6])
    np.testing.assert_array_equal(np.load(d / "trajectory_spins.npy").reshape(len(times), -1),
                                  np.stack([s for _, s in traj]))


def test_driver_2dcs_stationary_ground_state_reuses_m0(driver, tmp_path, oracle):
    """A stationary state (all spins along the [111] field of the Kitaev-Gamma model) passes the W1 guard:
    the batch holds M0 and M01 only and M1(tau) is M0 shifted in time (synthesize_M1_from_M0)."""
    R = np.ones(3) / np.sqrt(3.0)
    s0 = np.tile(R, 32)
    init = tmp_path / "fm.txt"
    np.savetxt(init, s0.reshape(-1, 3), fmt="%.17e")
    out = tmp_path / "2dcs_fm"
    _run(driver, tmp_path, f"""system = honeycomb_kitaev
simulation_mode = 2dcs
lattice_size = 4,4,1
field_strength = 0.5
field_direction = 1,1,1
pump_direction = 0,0,1
pump_amplitude = 0.4
pump_width = 0.2
pump_frequency = 0.5
tau_start = 0.0
tau_end = 0.6
tau_step = 0.3
md_time_start = -0.5
md_time_end = 1.5
md_timestep = 0.01
initial_spin_config = {init}
output_dir = {out}
""")
    d = out / "sample_0"
    meta = json.loads((d / "metadata.json").read_text())
    o = oracle.OracleLattice.kitaev(4, 4, 1, h=0.5, direction=R)
    assert meta["m1_synthesized"] == 1
    assert meta["max_dsdt_no_drive"] == pytest.approx(o.max_dsdt_no_drive(s0), abs=1e-15)
    assert meta["max_dsdt_no_drive"] <= 1e-12
    tau = np.load(d / "tau_scan_tau_values.npy")
    times = np.load(d / "reference_times.npy")
    n_t = len(times)
    z = np.tile([0.0, 0.0, 1.0], 2)
    B = 1 + len(tau)
    t2 = np.concatenate([[0.0], tau])
    s1 = np.ones(B)
    s2 = np.concatenate([[0.0], np.ones(len(tau))])
    _, obs = o.batch_rk4(np.tile(s0, (B, 1)), np.zeros(B), t2, s1, s2, 0.4, 0.2, 0.5, z, z, -0.5, 0.01, n_t - 1)
    ground = {"antiferro": np.zeros(3), "local": R, "global": o.magnetizations(s0)[6:9]}
    for q, name in enumerate(("antiferro", "local", "global")):
        m0 = np.load(d / f"reference_M_{name}.npy")
        m1 = np.load(d / f"tau_scan_M1_{name}.npy")
        m01 = np.load(d / f"tau_scan_M01_{name}.npy")
        assert np.abs(m0 - obs[0, :, 3 * q:3 * q + 3]).max() <= TOL_M
        assert np.abs(m01 - obs[1:, :, 3 * q:3 * q + 3]).max() <= TOL_M
        for k, tv in enumerate(tau):                 # lattice_md.cpp:283-317, restated
            for i, t in enumerate(times):
                if t < tv + times[0]:
                    np.testing.assert_allclose(m1[k, i], ground[name], atol=1e-15)
                else:
                    idx = int(np.clip(np.round((t - tv - times[0]) / 0.01), 0, n_t - 1))
                    np.testing.assert_array_equal(m1[k, i], m0[idx])
