"""Generate the golden fixtures of this directory from the REFERENCE's own code.

Runs the reference's GPU LL integrator (src/gpu/lattice_gpu.cu +
gpu_common_helpers.cu of ze-bang/Classical_MCMC_Spin, compiled in place into
oracle/_ref/libref_gpu.so by `make -C oracle ref`) through its gpu:: API on
inputs built by the oracle's restatement of the reference Lattice (same bond
tables the reference's Lattice::ensure_gpu_data_initialized would upload).
Needs a CUDA GPU.  Usage:  python tests/golden/make_golden.py [outdir]

Fixtures (all FP64, small):
  ref_gpu_rk4_kitaev.npz         integrate_gpu("rk4"), Kitaev 4x4, saved states
  ref_gpu_rk4_kitaev_driven.npz  same with two Gaussian pulses (freq != 0)
  ref_gpu_batched_kitaev.npz     integrate_gpu_batched, M0 + 4 delays
  ref_gpu_rk4_pyrochlore.npz     integrate_gpu("rk4"), non-Kramers pyrochlore with field
  ref_gpu_rk4_kitaev24.npz       integrate_gpu("rk4"), Kitaev 24x24 (1152 spins), 200 steps
"""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))

import ll_oracle as O  # noqa: E402
from classical_mcmc_spin_b200.states import random_unit_spins  # noqa: E402

R111 = np.ones(3) / np.sqrt(3.0)


def rotated(L, fin):
    fr, _ = L.frames()
    R = fr.reshape(L.n_atoms, 3, 3)
    f = np.asarray(fin).reshape(L.n_atoms, 3)
    return np.concatenate([R[a] @ f[a] for a in range(L.n_atoms)])


def main(out: Path):
    out.mkdir(parents=True, exist_ok=True)
    # 1. plain rk4
    L = O.OracleLattice.kitaev(4, 4, 1)
    init = random_unit_spins(L.N, 11).ravel()
    g = O.RefGPU(L.ell(), L.n_atoms)
    g.set_spins(init)
    times, states = g.integrate(0.0, 2.0, 0.01, save_interval=10, method="rk4")
    np.savez_compressed(out / "ref_gpu_rk4_kitaev.npz", d1=4, d2=4, init=init, dt=0.01, save_interval=10,
                        times=times, states=states)
    g.close()
    # 2. driven rk4, two pulses
    L = O.OracleLattice.kitaev(4, 4, 1)
    init = random_unit_spins(L.N, 12).ravel()
    fin1 = np.tile(R111, 2)
    fin2 = np.tile(np.array([0.0, 1.0, 0.0]), 2)
    fd = np.concatenate([rotated(L, fin1), rotated(L, fin2)])
    g = O.RefGPU(L.ell(), L.n_atoms)
    g.set_spins(init)
    g.set_pulse(fd, 0.5, 0.5, 1.3, 0.3, 1.1)
    times, states = g.integrate(-0.5, 2.0, 0.01, save_interval=1, method="rk4")
    mags = np.stack([L.magnetizations(s) for s in states])
    np.savez_compressed(out / "ref_gpu_rk4_kitaev_driven.npz", d1=4, d2=4, init=init, T0=-0.5, T1=2.0, dt=0.01,
                        field_in1=fin1, field_in2=fin2, t1=0.3, t2=1.1, amp=0.5, width=0.5, freq=1.3,
                        times=times, final=states[-1], mags=mags)
    g.close()
    # 3. batched (reference 2DCS layout: replica 0 = M0 with pulse 2 pushed past T_end)
    L = O.OracleLattice.kitaev(4, 4, 1)
    init = random_unit_spins(L.N, 13).ravel()
    fin = np.tile(R111, 2)
    fd = np.concatenate([rotated(L, fin), rotated(L, fin)])
    T0, T1, dt = -1.0, 2.0, 0.01
    tau2 = np.array([T1 + 100.0, 0.0, 0.5, 1.0, 1.5])
    g = O.RefGPU(L.ell(), L.n_atoms)
    g.set_pulse(fd, 0.5, 0.5, 0.0, 0.0, 0.0)
    fr, afm = L.frames()
    times, mags = g.batched(init, tau2, afm, fr, T0, T1, dt, save_interval=1)
    np.savez_compressed(out / "ref_gpu_batched_kitaev.npz", d1=4, d2=4, init=init, field_in=fin, amp=0.5,
                        width=0.5, freq=0.0, T0=T0, T1=T1, dt=dt, tau2=tau2, times=times, mags=mags)
    g.close()
    # 4. pyrochlore with field, rk4
    L = O.OracleLattice.pyrochlore_nk(2, 2, 2, h=0.2, direction=R111, Jzz=1.0, Jpm=0.05, Jpmpm=0.02)
    init = random_unit_spins(L.N, 14).ravel()
    g = O.RefGPU(L.ell(), L.n_atoms)
    g.set_spins(init)
    times, states = g.integrate(0.0, 1.0, 0.005, save_interval=20, method="rk4")
    np.savez_compressed(out / "ref_gpu_rk4_pyrochlore.npz", dims=(2, 2, 2), h=0.2, init=init, dt=0.005,
                        save_interval=20, times=times, states=states)
    g.close()
    # 5. the plain-MD lattice (1152 spins), 200 steps
    L = O.OracleLattice.kitaev(24, 24, 1)
    init = random_unit_spins(L.N, 1).ravel()
    g = O.RefGPU(L.ell(), L.n_atoms)
    g.set_spins(init)
    times, states = g.integrate(0.0, 1.995, 0.01, save_interval=100, method="rk4")
    np.savez_compressed(out / "ref_gpu_rk4_kitaev24.npz", d1=24, d2=24, init=init, dt=0.01, save_interval=100,
                        T1=1.995, times=times, states=states)
    g.close()
    for p in sorted(out.glob("*.npz")):
        print(p.name, p.stat().st_size)


if __name__ == "__main__":
    main(Path(sys.argv[1]) if len(sys.argv) > 1 else Path(__file__).resolve().parent)
