"""Converter from the command-line driver's output (.npy per dataset + metadata.json) to the
reference's HDF5 files, so the reference's readers consume a run unchanged.

Layouts (include/classical_spin/io/hdf5_io.h):
  * trajectory.h5 (HDF5MDWriter, hdf5_io.h:53-170):
      /trajectory/times [n], spins [n][N][3] (when saved), magnetization_antiferro / _local / _global [n][3]
      /metadata attributes lattice_size, spin_dim, n_atoms, integration_method, dt_initial, T_start, T_end,
      save_interval, spin_length, creation_time, code_version, file_format; dataset /metadata/dimensions [3]
  * pump_probe_spectroscopy.h5 (HDF5PumpProbeWriter, hdf5_io.h:720-900, written by
    lattice.h:5749-5851):
      /reference/times [n_t], M_antiferro / M_local / M_global [n_t][3]
      /tau_scan/tau_values [n_tau]; /tau_scan/tau_k/{M1,M01}_{antiferro,local,global} [n_t][3], attribute
      tau_value
      /metadata attributes (experiment_type, file_format, lattice_size, spin_dim, n_atoms, dim1..dim3,
      spin_length, pulse_*, T_*, integration_method, tau_*, ground_state_energy)

plan_trajectory / plan_pump_probe build the file's content as a list of entries without touching HDF5;
write() creates the file with h5py, imported only there (h5py is not a dependency of the library).
``python -m classical_mcmc_spin_b200.hdf5_export DIR`` converts every run directory under DIR.
"""
from __future__ import annotations

import json
import sys
import time
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

MAGS = ("antiferro", "local", "global")


@dataclass
class Entry:
    """One group (data None) or dataset of the file, with its attributes."""
    path: str
    data: np.ndarray | None = None
    attrs: dict = field(default_factory=dict)


def _meta(d: Path) -> dict:
    p = d / "metadata.json"
    return json.loads(p.read_text()) if p.exists() else {}


def _load(d: Path, name: str) -> np.ndarray:
    return np.load(d / name)


def _stamp() -> str:
    return time.strftime("%Y-%m-%dT%H:%M:%S", time.localtime())


def plan_trajectory(d) -> list:
    """trajectory.h5 of a molecular_dynamics / pump_probe run directory."""
    d = Path(d)
    m = _meta(d)
    times = _load(d, "trajectory_times.npy")
    n = len(times)
    meta_attrs = {
        "lattice_size": int(m.get("lattice_size", 0)),
        "spin_dim": int(m.get("spin_dim", 3)),
        "n_atoms": int(m.get("N_atoms", 0)),
        "integration_method": str(m.get("integration_method", "")),
        "dt_initial": float(m.get("T_step", 0.0)),
        "T_start": float(m.get("T_start", 0.0)),
        "T_end": float(m.get("T_end", 0.0)),
        "save_interval": int(m.get("save_interval", 1)),
        "spin_length": float(m.get("spin_length", 1.0)),
        "creation_time": _stamp(),
        "code_version": "ClassicalSpin_Cpp v1.0",
        "file_format": "HDF5_MD_v1.0",
    }
    out = [Entry("/trajectory"), Entry("/metadata", attrs=meta_attrs),
           Entry("/metadata/dimensions", np.array([int(m.get(k, 0)) for k in ("dim1", "dim2", "dim3")],
                                                  dtype=np.uint64)),
           Entry("/trajectory/times", np.asarray(times, dtype=np.float64))]
    for q in MAGS:
        a = _load(d, f"trajectory_magnetization_{q}.npy")
        assert a.shape == (n, 3), (q, a.shape)
        out.append(Entry(f"/trajectory/magnetization_{q}", a))
    if (d / "trajectory_spins.npy").exists():
        s = _load(d, "trajectory_spins.npy")
        assert s.shape[0] == n and s.shape[2] == 3
        out.append(Entry("/trajectory/spins", s))
    return out


def plan_pump_probe(d) -> list:
    """pump_probe_spectroscopy.h5 of a 2dcs run directory."""
    d = Path(d)
    m = _meta(d)
    times = _load(d, "reference_times.npy")
    taus = _load(d, "tau_scan_tau_values.npy")
    n_t, n_tau = len(times), len(taus)
    meta_attrs = {
        "creation_time": _stamp(),
        "experiment_type": "pump_probe_spectroscopy",
        "code_version": "ClassicalSpin_Cpp v1.0",
        "file_format": "HDF5_PumpProbe_v1.0",
        "lattice_size": int(m.get("lattice_size", 0)),
        "spin_dim": int(m.get("spin_dim", 3)),
        "n_atoms": int(m.get("N_atoms", 0)),
        "dim1": int(m.get("dim1", 0)), "dim2": int(m.get("dim2", 0)), "dim3": int(m.get("dim3", 0)),
        "spin_length": float(m.get("spin_length", 1.0)),
        "pulse_amp": float(m.get("pulse_amp", 0.0)),
        "pulse_width": float(m.get("pulse_width", 0.0)),
        "pulse_freq": float(m.get("pulse_freq", 0.0)),
        "T_start": float(m.get("T_start", 0.0)),
        "T_end": float(m.get("T_end", 0.0)),
        "T_step": float(m.get("T_step", 0.0)),
        "integration_method": str(m.get("integration_method", "")),
        "tau_start": float(m.get("tau_start", 0.0)),
        "tau_end": float(m.get("tau_end", 0.0)),
        "tau_step": float(m.get("tau_step", 0.0)),
        "tau_steps": int(m.get("tau_steps", n_tau)),
        "ground_state_energy": float(m.get("ground_state_energy", 0.0)),
    }
    out = [Entry("/metadata", attrs=meta_attrs), Entry("/reference"), Entry("/tau_scan"),
           Entry("/reference/times", np.asarray(times, dtype=np.float64))]
    for q in MAGS:
        a = _load(d, f"reference_M_{q}.npy")
        assert a.shape == (n_t, 3), (q, a.shape)
        out.append(Entry(f"/reference/M_{q}", a))
    out.append(Entry("/tau_scan/tau_values", np.asarray(taus, dtype=np.float64)))
    m1 = {q: _load(d, f"tau_scan_M1_{q}.npy") for q in MAGS}
    m01 = {q: _load(d, f"tau_scan_M01_{q}.npy") for q in MAGS}
    for k in range(n_tau):
        g = f"/tau_scan/tau_{k}"
        out.append(Entry(g, attrs={"tau_value": float(taus[k])}))
        for q in MAGS:
            out.append(Entry(f"{g}/M1_{q}", np.ascontiguousarray(m1[q][k])))
            out.append(Entry(f"{g}/M01_{q}", np.ascontiguousarray(m01[q][k])))
    return out


def write(entries, filename) -> None:
    """Writes a plan to an HDF5 file (h5py)."""
    import h5py
    with h5py.File(filename, "w") as f:
        for e in entries:
            if e.data is None:
                obj = f.require_group(e.path)
            else:
                obj = f.create_dataset(e.path, data=e.data)
            for k, v in e.attrs.items():
                obj.attrs[k] = v


def export(d) -> list:
    """Converts one run directory; returns the files written."""
    d = Path(d)
    written = []
    if (d / "trajectory_times.npy").exists():
        write(plan_trajectory(d), d / "trajectory.h5")
        written.append(d / "trajectory.h5")
    if (d / "reference_times.npy").exists():
        write(plan_pump_probe(d), d / "pump_probe_spectroscopy.h5")
        written.append(d / "pump_probe_spectroscopy.h5")
    return written


if __name__ == "__main__":
    root = Path(sys.argv[1] if len(sys.argv) > 1 else ".")
    dirs = sorted({p.parent for p in root.rglob("metadata.json")})
    for d in dirs:
        for f in export(d):
            print(f)
