"""The .npy -> HDF5 converter (classical_mcmc_spin_b200/hdf5_export.py) against the reference's layouts.

Group, dataset and attribute names are those of include/classical_spin/io/hdf5_io.h: HDF5MDWriter
(hdf5_io.h:53-170) for trajectory.h5, HDF5PumpProbeWriter (hdf5_io.h:720-900) for
pump_probe_spectroscopy.h5, whose /reference/{times,M_local}, /tau_scan/tau_values and
/tau_scan/tau_k/{M1,M01}_local the reader util/readers_new/reader_honeycomb.py:475-530 reads.
The plans are checked without HDF5; the written file only when h5py is importable.
"""
import json

import numpy as np
import pytest

from classical_mcmc_spin_b200 import hdf5_export as H

MD_DATASETS = {"/trajectory/times", "/trajectory/magnetization_antiferro", "/trajectory/magnetization_local",
               "/trajectory/magnetization_global", "/trajectory/spins", "/metadata/dimensions"}
MD_ATTRS = {"lattice_size", "spin_dim", "n_atoms", "integration_method", "dt_initial", "T_start", "T_end",
            "save_interval", "spin_length", "creation_time", "code_version", "file_format"}
PP_ATTRS = {"creation_time", "experiment_type", "code_version", "file_format", "lattice_size", "spin_dim", "n_atoms",
            "dim1", "dim2", "dim3", "spin_length", "pulse_amp", "pulse_width", "pulse_freq", "T_start", "T_end",
            "T_step", "integration_method", "tau_start", "tau_end", "tau_step", "tau_steps", "ground_state_energy"}


def _md_dir(tmp_path, n=5, N=8):
    d = tmp_path / "md"
    d.mkdir()
    rng = np.random.default_rng(0)
    np.save(d / "trajectory_times.npy", np.arange(n) * 0.1)
    for q in H.MAGS:
        np.save(d / f"trajectory_magnetization_{q}.npy", rng.normal(size=(n, 3)))
    np.save(d / "trajectory_spins.npy", rng.normal(size=(n, N, 3)))
    (d / "metadata.json").write_text(json.dumps(dict(lattice_size=N, spin_dim=3, N_atoms=2, dim1=2, dim2=2, dim3=1,
                                                     T_start=0.0, T_end=0.4, T_step=0.1, save_interval=1,
                                                     integration_method="rk4")))
    return d


def _pp_dir(tmp_path, n_t=7, n_tau=3):
    d = tmp_path / "pp"
    d.mkdir()
    rng = np.random.default_rng(1)
    np.save(d / "reference_times.npy", np.arange(n_t) * 0.1)
    np.save(d / "tau_scan_tau_values.npy", np.arange(n_tau) * 0.5)
    for q in H.MAGS:
        np.save(d / f"reference_M_{q}.npy", rng.normal(size=(n_t, 3)))
        np.save(d / f"tau_scan_M1_{q}.npy", rng.normal(size=(n_tau, n_t, 3)))
        np.save(d / f"tau_scan_M01_{q}.npy", rng.normal(size=(n_tau, n_t, 3)))
    (d / "metadata.json").write_text(json.dumps(dict(lattice_size=8, spin_dim=3, N_atoms=2, dim1=2, dim2=2, dim3=1,
                                                     pulse_amp=0.5, pulse_width=0.4, pulse_freq=0.0, T_start=0.0,
                                                     T_end=0.6, T_step=0.1, tau_start=0.0, tau_end=1.0,
                                                     tau_step=0.5, tau_steps=n_tau, ground_state_energy=-1.0,
                                                     integration_method="rk4")))
    return d


def test_trajectory_plan_follows_the_md_writer_layout(tmp_path):
    d = _md_dir(tmp_path)
    plan = H.plan_trajectory(d)
    groups = {e.path for e in plan if e.data is None}
    data = {e.path: e for e in plan if e.data is not None}
    assert groups == {"/trajectory", "/metadata"}
    assert set(data) == MD_DATASETS
    assert set(next(e for e in plan if e.path == "/metadata").attrs) == MD_ATTRS
    assert data["/trajectory/spins"].data.shape == (5, 8, 3)
    assert data["/trajectory/magnetization_local"].data.shape == (5, 3)
    np.testing.assert_array_equal(data["/metadata/dimensions"].data, [2, 2, 1])
    np.testing.assert_array_equal(data["/trajectory/magnetization_global"].data,
                                  np.load(d / "trajectory_magnetization_global.npy"))


def test_pump_probe_plan_follows_the_pump_probe_writer_layout(tmp_path):
    d = _pp_dir(tmp_path)
    plan = H.plan_pump_probe(d)
    paths = {e.path for e in plan}
    expect = {"/metadata", "/reference", "/tau_scan", "/reference/times", "/tau_scan/tau_values"}
    expect |= {f"/reference/M_{q}" for q in H.MAGS}
    for k in range(3):
        expect.add(f"/tau_scan/tau_{k}")
        expect |= {f"/tau_scan/tau_{k}/{w}_{q}" for w in ("M1", "M01") for q in H.MAGS}
    assert paths == expect
    assert set(next(e for e in plan if e.path == "/metadata").attrs) == PP_ATTRS
    by = {e.path: e for e in plan}
    assert by["/tau_scan/tau_2"].attrs == {"tau_value": 1.0}
    np.testing.assert_array_equal(by["/tau_scan/tau_1/M01_local"].data, np.load(d / "tau_scan_M01_local.npy")[1])
    # what the reference reader opens
    for p in ("/reference/times", "/reference/M_local", "/tau_scan/tau_values", "/tau_scan/tau_0/M1_local",
              "/tau_scan/tau_0/M01_local"):
        assert p in by


def test_written_files_round_trip(tmp_path):
    h5py = pytest.importorskip("h5py")
    md, pp = _md_dir(tmp_path), _pp_dir(tmp_path)
    files = H.export(md) + H.export(pp)
    assert [f.name for f in files] == ["trajectory.h5", "pump_probe_spectroscopy.h5"]
    with h5py.File(files[1], "r") as f:
        np.testing.assert_array_equal(f["/reference/M_local"][:], np.load(pp / "reference_M_local.npy"))
        assert f["/tau_scan/tau_1"].attrs["tau_value"] == 0.5
