"""The command-line driver's param-file handling (no GPU): the reference's `key = value` format,
comment and vector syntax, defaults of the builders, rejection of modes and systems off this path."""
import json
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def driver(native):
    from classical_mcmc_spin_b200 import build
    return build.build_driver()


def _parse(driver, tmp_path, text):
    p = tmp_path / "cfg.param"
    p.write_text(text)
    r = subprocess.run([str(driver), str(p), "--parse-only"], capture_output=True, text=True)
    return r, (json.loads(r.stdout) if r.returncode == 0 else None)


MD_KITAEV = """
# Kitaev honeycomb MD
system = honeycomb_kitaev
simulation_mode = molecular_dynamics
lattice_size = 24,24,1
K = -1.0        # Kitaev
Gamma = 0.25
Gammap = -0.02
J = 0.0
field_strength = 0.7
field_direction = [0.577, 0.577, 0.577]
h = 0.7
T_start = 5.0
use_twist_boundary = false
md_time_start = 0.0
md_time_end = 600.0
md_timestep = 0.25
md_save_interval = 1
md_integrator = rk4
output_dir = KITAEV_md
"""


def test_parse_md_config(driver, tmp_path):
    r, c = _parse(driver, tmp_path, MD_KITAEV)
    assert r.returncode == 0, r.stderr
    assert c["system"] == "honeycomb_kitaev" and c["simulation_mode"] == "molecular_dynamics"
    assert (c["L0"], c["L1"], c["L2"]) == (24, 24, 1)
    assert c["param:K"] == -1.0 and c["param:Gamma"] == 0.25 and c["param:Gammap"] == -0.02
    assert c["param:T_start"] == 5.0                    # numeric keys of other modes are kept, unused
    assert c["field_strength"] == 0.7 and c["md_timestep"] == 0.25 and c["md_time_end"] == 600.0
    assert "use_twist_boundary" in c["ignored"].split(",")


def test_parse_2dcs_and_pump_directions(driver, tmp_path):
    text = """system = pyrochlore_non_kramer
simulation_mode = 2DCS
lattice_size = (2, 2, 2)
Jzz = 1.0
Jpm = 0.05
pump_direction = 0,0,1, 1,0,0, 0,1,0, 1,1,1
pump_amplitude = 0.1
pump_width = 0.4
tau_start = -3
tau_end = 3
tau_step = 0.25
cubic_cell = true
seed = 12
"""
    r, c = _parse(driver, tmp_path, text)
    assert r.returncode == 0, r.stderr
    assert c["simulation_mode"] == "2dcs" and c["system"] == "pyrochlore_non_kramer"
    assert c["n_pump_directions"] == 4 and c["cubic_cell"] == 1 and c["seed"] == 12
    assert c["tau_start"] == -3 and c["tau_step"] == 0.25


@pytest.mark.parametrize("text,msg", [
    ("system = honeycomb_kitaev\nsimulation_mode = simulated_annealing\n", "simulation_mode"),
    ("system = tmfeo3\nsimulation_mode = md\n", "not on this path"),
    ("system = honeycomb_kitaev\n", "simulation_mode is missing"),
    ("system = honeycomb_kitaev\nsimulation_mode = MD\npump_direction = 1,0\n", "multiple of 3"),
    ("system = honeycomb_kitaev\nsimulation_mode = MD\nmd_timestep = -1\n", "md_timestep"),
    ("system = honeycomb_kitaev\nsimulation_mode = MD\nthis line has no equals sign\n", "key = value"),
    ("system = honeycomb_kitaev\nsimulation_mode = MD\nmd_integrator = rk99\n", "md_integrator"),
])
def test_config_errors(driver, tmp_path, text, msg):
    r, _ = _parse(driver, tmp_path, text)
    assert r.returncode == 1 and msg in r.stderr, r.stderr


def test_random_spins_are_seeded_unit_vectors(native):
    import numpy as np
    L = native.lib()
    a, b, c = (np.zeros(3 * 1000) for _ in range(3))
    for out, seed in ((a, 5), (b, 5), (c, 6)):
        native.check(L.cmd_lattice_random_spins(1000, seed, 1.0, native.dptr(out)), "random")
    np.testing.assert_array_equal(a, b)
    assert not np.array_equal(a, c)
    assert np.abs(np.linalg.norm(a.reshape(-1, 3), axis=1) - 1.0).max() < 1e-15
