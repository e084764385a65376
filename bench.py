#!/usr/bin/env python
"""Benchmark of the B200 Landau-Lifshitz MD path.

Headline workload (one bench step): the batched 2DCS delay scan on the
1152-spin Kitaev honeycomb (24x24x1, K=-1, Gamma=0.25, Gamma'=-0.02, no static
field), FP64 RK4 dt=0.01 for 2x10^4 steps from T_start=-5, 256 delays
tau_k = 100 k/255, each a pump-only, probe-only and pump+probe trajectory
(768 trajectories) in ONE launch; Gaussian pulses amp 0.5, width 0.5,
freq 0, direction (1,1,1)/sqrt3 on both sublattices (rotated by the
sublattice frame like Lattice::set_pulse); initial state zigzag +
Gaussian tilt sigma=0.05 (seed 2), renormalised; M_af/M_local/M_global and
E/N reduced every step.

Metric: spin*RK4-steps/s = B * N * steps / time (whole job, all GPUs).
  value      device-resident inputs, CUDA events on the launching stream;
  e2e        the public C-ABI call cmd_run_batch with pinned host buffers
             (initial state + pulses H2D, every step's observables D2H);
  plain_path the plain per-trajectory path (one trajectory per launch,
             random unit spins seed 1, 10^4 steps, observables every step);
  cpu_baseline the oracle (CPU restatement of the reference integrator) on
             a bounded sample of the same scan, all host threads.
`--impl reference` times only the reference CPU path (the oracle port; the
reference's own CPU build needs Eigen3/Boost/HDF5/MPI, absent here).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "batched LL spin\u00b7RK-steps/s on 1 B200 vs plain path; adjoint/forward cost"
UNIT = "spin\u00b7RK-steps/s"
FLOPS_PER_SPIN_STEP = 339.0        # 4*(18z + 9 + 12) + 39 with z = 3, drive on, no static field
N_DELAYS = 256
L_SIDE = 24


# --------------------------------------------------------------------------- workload
def zigzag_tilted(d1: int, d2: int, sigma: float, seed: int) -> np.ndarray:
    """The scan's initial state in numpy alone (the reference arm never imports the package): site
    (i, j, atom) of the 2-atom honeycomb gets (-1)^i (1,1,1)/sqrt3, tilted by i.i.d. Gaussian components of
    width sigma (seed) and renormalised.  Equal to classical_mcmc_spin_b200.states.zigzag_honeycomb
    (tests/test_bench_inputs.py checks it)."""
    axis = np.ones(3) / np.sqrt(3.0)
    i = np.arange(d1).repeat(d2 * 2)
    s = np.where(i % 2 == 0, 1.0, -1.0)[:, None] * axis[None, :]
    s = s + sigma * np.random.default_rng(seed).standard_normal(s.shape)
    return s / np.linalg.norm(s, axis=1, keepdims=True)


def scan_inputs(n_steps: int, rank: int = 0, world: int = 1) -> dict:
    """Inputs of the 2DCS scan (numpy only).  Weak scaling: rank r scans its interleaved share of a
    world x 256 delay scan, tau = 100 (k + r / world) / 255."""
    s0 = zigzag_tilted(L_SIDE, L_SIDE, 0.05, 2).ravel()
    fin = np.tile(np.ones(3) / np.sqrt(3.0), 2)
    taus = 100.0 * (np.arange(N_DELAYS) + rank / world) / (N_DELAYS - 1)
    pulses = []
    for tau in taus:
        for a1, a2 in ((0.5, 0.0), (0.0, 0.5), (0.5, 0.5)):
            pulses.append((0.0, tau, a1, a2))
    return dict(s0=s0, fin=fin, pulses=np.array(pulses), T0=-5.0, dt=0.01, n_steps=n_steps, width=0.5, freq=0.0)


def scan_workload(n_steps: int, rank: int = 0, world: int = 1):
    from classical_mcmc_spin_b200.lattice import Lattice

    wl = scan_inputs(n_steps, rank, world)
    lat = Lattice.kitaev(L_SIDE, L_SIDE, 1, K=-1.0, Gamma=0.25, Gammap=-0.02)
    fd = lat.rotate_pulse(wl["fin"], wl["fin"])
    wl.update(lat=lat, d1=fd[:6].copy(), d2=fd[6:].copy())
    return wl


def scan_config(n_steps: int, world: int) -> dict:
    """`config` of the headline line, identical in both arms."""
    return {"workload": "2dcs_scan_kitaev24x24_768traj_rk4", "spins": 2 * L_SIDE * L_SIDE,
            "trajectories": 3 * N_DELAYS, "rk4_steps": n_steps, "dt": 0.01, "T_start": -5.0, "delays": N_DELAYS,
            "observables_every_step": True, "energy_every_step": True,
            "l2": "flushed between timed iterations (256 MB write)",
            "parallelism": f"replicas: {world} GPU(s), trajectories sharded, no collective"}


# --------------------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.lines = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.gpu)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------------------- peaks
def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        return json.loads(p.read_text())
    except Exception:
        return {}


def fp64_peak_tflops(torch) -> float:
    """Dense FP64 peak measured here with cuBLAS DGEMM (best of 5, 8192^3)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    best = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = max(best, 2.0 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    del a, b
    return best


def profile_traffic():
    """DRAM bytes per launch from the committed ncu summary, if present."""
    p = ROOT / "profiles" / "rk4_lean_2dcs_kitaev1152.md"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


# --------------------------------------------------------------------------- further workloads
R111 = np.ones(3) / np.sqrt(3.0)
STREAM_BYTES_PER_SPIN_STEP = 408.0   # stages 72 + 120 + 120 + 96 B (input, y, RK4 sum, next input)


def leg_uneven(torch, dev, max_steps=10000, T1=100.0, B=512):
    """Uneven batch: 512 trajectories, honeycomb L in {8..32} and pyrochlore 16L^3, L in {4, 6, 8}, drawn from
    seed 3; controlled RK45 at tol 1e-10, T_end = 100, cap 1e4 accepted steps.  Each lattice class runs on the
    on-chip Dormand-Prince kernel with the tiling its autotuner picked (short runs before the timed call); the
    classes' launches run concurrently on the owner handle's streams."""
    from classical_mcmc_spin_b200 import gpu_api
    from classical_mcmc_spin_b200.lattice import Lattice
    from classical_mcmc_spin_b200.states import random_unit_spins
    opts = [("honeycomb", L) for L in (8, 12, 16, 24, 32)] + [("pyrochlore", L) for L in (4, 6, 8)]
    pick = np.random.default_rng(3).integers(0, len(opts), size=B)
    handles = {}
    for k in sorted(set(pick.tolist())):
        kind, L = opts[k]
        lat = (Lattice.kitaev(L, L, 1) if kind == "honeycomb" else
               Lattice.pyrochlore_non_kramer(L, L, L, cubic=True, Jzz=1.0, Jpm=0.05, Jpmpm=0.02))
        handles[k] = (lat, lat.to_gpu())
    specs = []
    for b in range(B):
        lat, h = handles[int(pick[b])]
        specs.append(dict(handle=h, state=random_unit_spins(lat.lattice_size, 3000 + b).ravel(), T0=0.0, T1=T1,
                          dt=0.01, max_rows=max_steps + 2))
    # tiling of each lattice class (CTAs per trajectory x threads x sites per thread) by the autotuner
    tilings = {}
    t_tune = time.perf_counter()
    for k, (lat, h) in handles.items():
        gpu_api.set_tolerances(h, 1e-10, 1e-10)
        gpu_api.set_gpu_spins(h, random_unit_spins(lat.lattice_size, 2999).ravel())
        best, _ = h.autotune_rk45(int((pick == k).sum()), 200)     # the class's own batch size: its occupancy
        tilings[f"{opts[k][0]}_L{opts[k][1]}"] = next(n for i, n, _ in h.rk45_variants() if i == best)
    t_tune = time.perf_counter() - t_tune
    walls = []
    for _ in range(2):                       # best of two calls; the first also allocates and builds its graph
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        out = gpu_api.run_uneven(specs, "rk45", 1e-10, 1e-10, max_steps=max_steps)
        torch.cuda.synchronize(dev)
        walls.append(time.perf_counter() - t0)
    wall = min(walls)
    acc = sum(o[2][1] for o in out)
    rej = sum(o[2][2] for o in out)
    work = sum(specs[b]["handle"].N * out[b][2][1] for b in range(B))
    for _, h in handles.values():
        h.close()
    return {"value": work / wall, "unit": "accepted spin·RK45-steps/s", "wall_s": wall, "trajectories": B,
            "accepted_steps": acc, "rejected_steps": rej, "spin_steps": work, "tol": 1e-10, "T_end": T1,
            "types": {f"{opts[k][0]}_L{opts[k][1]}": int((pick == k).sum()) for k in handles},
            "tilings": tilings, "autotune_s": t_tune, "wall_s_calls": walls,
            "timing": "wall clock around the public call (host buffers in and out), best of two calls; tilings "
                      "tuned before"}


def _adjoint_leg(torch, dev, build, theta, theta_target, n_params, B, S, dt, seed, ckpt, reps=2):
    """Forward-only and forward + adjoint calls of the public API, each timed `reps` times in turn (wall clock,
    host buffers in and out); the best of each is reported, the first call of each also allocating its buffers."""
    from classical_mcmc_spin_b200 import adjoint as A
    from classical_mcmc_spin_b200.states import random_unit_spins
    lat = build(theta)
    N = lat.lattice_size
    h, ht = lat.to_gpu(), build(theta_target).to_gpu()
    states = np.stack([random_unit_spins(N, seed * 1000 + b).ravel() for b in range(B)])
    _, _, target = A.adjoint_rk4(ht, [], states, 0.0, dt, S, np.zeros((B, S + 1, 3)), forward_only=True)
    dps = A.basis_lattices(build, n_params)
    tfs, tas = [], []
    for _ in range(max(1, reps)):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        loss_f, _, _ = A.adjoint_rk4(h, [], states, 0.0, dt, S, target, forward_only=True)
        torch.cuda.synchronize(dev)
        tfs.append(time.perf_counter() - t0)
        t0 = time.perf_counter()
        loss, grad, _ = A.adjoint_rk4(h, dps, states, 0.0, dt, S, target, checkpoint_every=ckpt)
        torch.cuda.synchronize(dev)
        tas.append(time.perf_counter() - t0)
    h.close()
    ht.close()
    tf, ta = min(tfs), min(tas)
    return {"spins": N, "trajectories": B, "rk4_steps": S, "dt": dt, "checkpoint_every": ckpt,
            "forward_s": tf, "forward_plus_adjoint_s": ta, "ratio": ta / tf,
            "forward_s_calls": tfs, "forward_plus_adjoint_s_calls": tas,
            "forward_value": B * N * S / tf, "unit": UNIT, "loss_mean": float(np.mean(loss)),
            "loss_forward_only_equal": bool(np.array_equal(loss, loss_f)),
            "grad_mean": np.mean(grad, axis=0).tolist(),
            "timing": f"wall clock around the public call (host buffers in and out), best of {max(1, reps)} calls "
                      "each, the first of which also allocates"}


def leg_adjoint_kitaev(torch, dev, S=20000, B=64):
    """Adjoint: honeycomb 48x48 (4608 spins), B states (64 in the configuration; seed 4), RK4 dt 0.01, M_local
    loss against targets at
    (K, G, G', J, h) = (-1, 0.3, -0.03, 0, 0.1); gradient at (-1, 0.25, -0.02, 0, 0) w.r.t. all five,
    checkpoint every 141 steps."""
    from classical_mcmc_spin_b200 import adjoint as A
    build = lambda th: A.kitaev_lattice(th, 48, 48)
    out = _adjoint_leg(torch, dev, build, np.array([-1.0, 0.25, -0.02, 0.0, 0.0]),
                       np.array([-1.0, 0.3, -0.03, 0.0, 0.1]), 5, B, S, 0.01, 4, 141)
    out["workload"] = f"adjoint_kitaev48x48_{B}traj_rk4"
    return out


def _forward_device(torch, dev, h, states, S, dt, streamed):
    """B trajectories from `states` for S RK4 steps through cmd_run_batch_device (device buffers, no drive,
    M and E every step), timed with CUDA events on the launching stream."""
    from classical_mcmc_spin_b200 import _native as nat
    B, N3 = states.shape
    N = N3 // 3
    d_states = torch.from_numpy(states).to(dev).contiguous()
    rows = int(nat.lib().cmd_batch_rows(S, 1))
    d_obs = torch.empty((B, rows, 10), dtype=torch.float64, device=dev)
    d_fin = torch.empty_like(d_states)
    desc = nat.BatchDesc()
    desc.B = B
    desc.states = d_states.data_ptr()
    desc.shared_initial = 0
    desc.method = nat.CMD_RK4
    desc.width, desc.freq, desc.T0, desc.dt = 1.0, 0.0, 0.0, dt
    desc.save_interval = 1
    desc.obs = d_obs.data_ptr()
    desc.final_states = d_fin.data_ptr()
    launches = C.c_int32()
    stream = torch.cuda.current_stream(dev)
    if stream.cuda_stream == 0:
        # stream 0 makes the library use the handle's own stream, which these events would not see
        stream = torch.cuda.Stream(device=dev)
    torch.cuda.synchronize(dev)

    def run(n):
        desc.n_steps = n
        nat.check(nat.lib().cmd_run_batch_device(h.ptr, C.byref(desc), C.c_void_p(stream.cuda_stream),
                                                 C.byref(launches)), "cmd_run_batch_device")

    run(8)                                   # warm
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    run(S)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1)
    value = B * N * S / (ms * 1e-3)
    out = {"value": value, "unit": UNIT, "ms": ms, "rk4_steps": S, "launches": launches.value,
           "final_norm_dev_max": float((d_fin.view(B, N, 3).norm(dim=2) - 1).abs().max().item()),
           "observables_finite": bool(torch.isfinite(d_obs).all().item())}
    if streamed:
        out["hbm_bytes_per_spin_step"] = STREAM_BYTES_PER_SPIN_STEP
        out["achieved_gbs"] = STREAM_BYTES_PER_SPIN_STEP * value / 1e9
    return out


def leg_kitaev48_forward(torch, dev, S=20000):
    """Forward of the adjoint workload: honeycomb 48x48 (4608 spins), 64 states (seed 4), RK4 dt 0.01, one
    trajectory per 4-CTA cluster (the lattice does not fit one CTA)."""
    from classical_mcmc_spin_b200 import adjoint as A
    from classical_mcmc_spin_b200.states import random_unit_spins
    lat = A.kitaev_lattice(np.array([-1.0, 0.25, -0.02, 0.0, 0.0]), 48, 48)
    h = lat.to_gpu()
    states = np.stack([random_unit_spins(lat.lattice_size, 4000 + b).ravel() for b in range(64)])
    out = _forward_device(torch, dev, h, states, S, 0.01, streamed=False)
    out["variant"] = next(n for i, n, _ in h.variants() if i == h.get_variant())
    out["workload"] = "kitaev48x48_64traj_rk4_forward"
    h.close()
    return out


def leg_mixed(torch, dev, S=20000):
    """Mixed SU(2)/SU(3) lattice shaped like TmFeO3: 6x6x6 cells of 4 SU(2) + 4 SU(3) atoms (864 + 864 sites;
    seeded synthetic couplings, fields and on-site terms), one trajectory through the reference API's
    integrate_mixed_gpu (mixed_gpu_api), dt 0.005, S steps, a two-pulse drive on both kinds of site; RK4 and the
    reference default SSPRK53.  Wall clock around the call (one persistent launch; two saved rows)."""
    from classical_mcmc_spin_b200 import mixed_gpu_api as mg
    arr = mg.synthetic_mixed_lattice((6, 6, 6), seed=30)
    h = mg.create_from(arr)
    rng = np.random.default_rng(31)
    mg.set_gpu_pulse_SU2(h, rng.normal(size=2 * arr["na2"] * 3), 0.5, 0.5, 1.0, 1.0, 2.0)
    mg.set_gpu_pulse_SU3(h, rng.normal(size=2 * arr["na3"] * 8), 0.5, 0.5, 1.0, 1.0, 2.0)
    y0 = mg.random_mixed_state(arr, 32)
    sites = arr["n2"] + arr["n3"]
    out = {"workload": "mixed_tmfeo3_shape_6x6x6_1728sites", "sites_su2": arr["n2"], "sites_su3": arr["n3"],
           "steps": S, "dt": 0.005, "unit": "site·steps/s"}
    for method, stages in (("rk4", 4), ("ssprk53", 5)):
        mg.set_gpu_mixed_spins(h, y0)
        mg.integrate_mixed_gpu(h, 0.0, 0.05, 0.005, 10, method)          # warm
        mg.set_gpu_mixed_spins(h, y0)
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        traj, _ = mg.integrate_mixed_gpu(h, 0.0, S * 0.005, 0.005, S, method)
        s = time.perf_counter() - t0
        y = traj[-1][1]
        out[method] = {"s": s, "value": sites * S / s, "us_per_stage": s / (S * stages) * 1e6,
                       "su2_norm_dev_max": float(np.abs(np.linalg.norm(y[:3 * arr["n2"]].reshape(-1, 3), axis=1)
                                                        - 1).max())}
    h.close()
    return out


def leg_pyrochlore(torch, dev, S=20000, S_adj=20000):
    """Large pyrochlore: 16^3 conventional cells (65536 spins), Jzz=1, J+-=0.05, J+-+-=0.02, h=0.2 along [111],
    32 states (seed 5), RK4 dt 0.005.  Forward through cmd_run_batch_device (device buffers, CUDA events, M and E
    every step); adjoint w.r.t. (Jzz, J+-, J+-+-, h) against targets at (1, 0.06, 0.03, 0.25)."""
    from classical_mcmc_spin_b200 import adjoint as A
    from classical_mcmc_spin_b200.states import random_unit_spins
    theta = np.array([1.0, 0.05, 0.02, 0.2])
    build = lambda th: A.pyrochlore_lattice(th, 16, 16, 16, cubic=True)
    lat = build(theta)
    N, B, dt = lat.lattice_size, 32, 0.005
    h = lat.to_gpu()
    states = np.stack([random_unit_spins(N, 5000 + b).ravel() for b in range(B)])
    clk = ClockSampler(dev.index if dev.index is not None else 0)
    clk.start()
    fwd = _forward_device(torch, dev, h, states, S, dt, streamed=True)
    fwd["clocks"] = clk.stop()
    # the same run with every stage launched directly (no CUDA graph)
    h.set_graphs(False)
    direct = _forward_device(torch, dev, h, states, S, dt, streamed=True)
    h.set_graphs(True)
    fwd["direct_launches"] = {"value": direct["value"], "ms": direct["ms"], "launches": direct["launches"],
                              "achieved_gbs": direct["achieved_gbs"]}
    fwd["graph_over_direct"] = fwd["value"] / direct["value"]
    h.close()
    adj = _adjoint_leg(torch, dev, build, theta, np.array([1.0, 0.06, 0.03, 0.25]), 4, B, S_adj, dt, 5,
                       int(np.ceil(np.sqrt(S_adj))))
    return {"workload": "pyrochlore16cubic_65536spins_32traj_rk4", "spins": N, "trajectories": B, "dt": dt,
            "forward": fwd, "adjoint": adj}


# --------------------------------------------------------------------------- CPU baseline
def _oracle():
    sys.path.insert(0, str(ROOT / "oracle"))
    import ll_oracle as O
    return O


def cpu_baseline(wl, target_s: float = 8.0, threads: int = 0):
    """The oracle (CPU restatement of the reference's landau_lifshitz_flat + RK4, OpenMP) on a bounded sample
    of the scan: max(threads, 8) trajectories spread over the delays, one per thread (the reference's W2 delay
    loop, lattice_md.cpp:809-904), observables and energy every step as on the GPU."""
    O = _oracle()
    threads = threads or (os.cpu_count() or 1)
    O.set_threads(threads)
    lat = O.OracleLattice.kitaev(L_SIDE, L_SIDE, 1, K=-1.0, Gamma=0.25, Gammap=-0.02)
    N = lat.N
    P = wl["pulses"]
    pick = np.linspace(0, len(P) - 1, max(threads, 8) if threads > 1 else 1).astype(int)
    B = len(pick)
    s = np.tile(wl["s0"], (B, 1))
    sub = P[pick]
    s1 = sub[:, 2] / 0.5
    s2 = sub[:, 3] / 0.5

    def run(steps):
        t0 = time.perf_counter()
        lat.batch_rk4(s, sub[:, 0], sub[:, 1], s1, s2, 0.5, wl["width"], wl["freq"], wl["fin"], wl["fin"], wl["T0"],
                      wl["dt"], steps, with_obs=True, with_energy=True)
        return time.perf_counter() - t0

    probe = 20
    tp = run(probe)
    steps = int(max(20, min(20000, probe * target_s / max(tp, 1e-6))))
    wall = run(steps)
    return dict(value=B * N * steps / wall, unit=UNIT, cores=threads, kind="port",
                sample=f"{B} of the 768 scan trajectories x {steps} RK4 steps (1152 spins, M and E every step), "
                       f"oracle restatement of the reference CPU RHS + RK4, "
                       f"{'trajectory-parallel OpenMP' if threads > 1 else 'one thread'}, {wall:.2f} s wall"), \
        (B, steps, wall)


def cpu_calibration(threads: int, n_rhs: int = 4000, repeats: int = 3) -> dict:
    """bench_md-style row (src/apps/bench_md.cpp:214-231, 365-385): RHS calls/s of the oracle's
    landau_lifshitz_flat restatement (site-parallel OpenMP) on the Kitaev honeycomb L = 32 (2048 spins, K=-1,
    Gamma=0.25, Gamma'=-0.02, no field), warm-up max(500, n/4) calls, best of `repeats`; for comparison with
    the reference's published 1.64e4 rhs/s (1 thread) ... 1.04e5 (16 threads) on its own host."""
    O = _oracle()
    O.set_threads(threads)
    lat = O.OracleLattice.kitaev(32, 32, 1, K=-1.0, Gamma=0.25, Gammap=-0.02)
    rng = np.random.default_rng(7)
    x = rng.standard_normal((lat.N, 3))
    x = (x / np.linalg.norm(x, axis=1, keepdims=True)).ravel()
    out = np.zeros_like(x)
    f = O.lib().ora_rhs
    xp, op = O._p(x), O._p(out)

    def run(n):
        t = 0.0
        for _ in range(n):
            f(lat.h, xp, t, op)
            t += 1e-3

    run(max(500, n_rhs // 4))
    best = 0.0
    for _ in range(repeats):
        t0 = time.perf_counter()
        run(n_rhs)
        best = max(best, n_rhs / (time.perf_counter() - t0))
    return {"rhs_per_s": best, "threads": threads, "spins": lat.N,
            "spin_rk4_steps_per_s": best * lat.N / 4.0,
            "workload": "bench_md lattice row: kitaev-honeycomb-su2 L=32, oracle landau_lifshitz_flat restatement"}


def cpu_rows(wl, target_s: float) -> dict:
    """The CPU figures printed beside the baseline: the scan sample on one thread and the bench_md-style
    calibration rows on one thread and on every host thread."""
    n = os.cpu_count() or 1
    one, _ = cpu_baseline(wl, target_s=max(2.0, target_s / 2), threads=1)
    return {"one_thread": one, "calibration": [cpu_calibration(1), cpu_calibration(n)]}


# --------------------------------------------------------------------------- reference arm
def run_reference(args):
    """The reference's CPU path on the host cores: the oracle port (the reference's own CPU build needs
    Eigen3 / Boost / HDF5 / MPI, absent here).  Inputs come from numpy alone; this arm never imports the
    package or loads its library."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    wl = scan_inputs(args.md_steps)
    results = []
    for i in range(args.warmup + args.steps):
        base, (B, steps, wall) = cpu_baseline(wl, target_s=args.cpu_seconds)
        if i >= args.warmup:
            results.append((base["value"], wall, B, steps))
    vals = [r[0] for r in results]
    v = statistics.median(vals)
    B, steps = results[-1][2], results[-1][3]
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * statistics.median([r[1] for r in results]), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": scan_config(args.md_steps, args.gpus),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                             "sample": f"{B} scan trajectories x {steps} RK4 steps per bench step, M and E every "
                                       "step; the reference's own CPU build needs Eigen3/Boost/HDF5/MPI (absent), "
                                       "so the oracle restatement of its CPU integrator is timed"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if not args.no_cpu_rows:
        line["cpu_rows"] = cpu_rows(wl, args.cpu_seconds)
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------------------- B200 arm
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--md-steps", type=int, default=20000, help="RK4 steps per trajectory (config: 2e4)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=8.0)
    ap.add_argument("--no-cpu-rows", action="store_true", help="skip the 1-thread and calibration CPU rows")
    ap.add_argument("--no-peak", action="store_true", help="skip the DGEMM peak probe (profiling runs)")
    ap.add_argument("--legs", default="uneven,adjoint,kitaev48,pyrochlore,mixed",
                    help="further workloads to time on rank 0 (comma list; empty for none)")
    ap.add_argument("--adjoint-steps", type=int, default=20000, help="RK4 steps of the 48x48 adjoint leg")
    ap.add_argument("--adjoint-traj", type=int, default=64, help="trajectories of the 48x48 adjoint leg (config: 64)")
    ap.add_argument("--mixed-steps", type=int, default=20000, help="steps of the mixed SU(2)/SU(3) leg")
    ap.add_argument("--pyro-steps", type=int, default=20000, help="RK4 steps of the 65536-spin forward leg")
    ap.add_argument("--pyro-adjoint-steps", type=int, default=20000, help="RK4 steps of the 65536-spin adjoint")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)

    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))

    from classical_mcmc_spin_b200 import _native as nat
    from classical_mcmc_spin_b200 import gpu_api
    from classical_mcmc_spin_b200.sharding import max_over_ranks

    wl = scan_workload(args.md_steps, rank, world)
    lat = wl["lat"]
    N = lat.lattice_size
    P = wl["pulses"]
    B = len(P)
    S = wl["n_steps"]
    h = lat.to_gpu()
    rows = int(nat.lib().cmd_batch_rows(S, 1))
    dev = torch.device("cuda", local)
    d_states = torch.from_numpy(wl["s0"]).to(dev).contiguous()
    d_pulse = torch.from_numpy(P.astype(np.float64)).to(dev).contiguous()
    d_obs = torch.empty((B, rows, 10), dtype=torch.float64, device=dev)
    d_fin = torch.empty((B, 3 * N), dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)   # > 126 MB L2
    keep = dict(d1=wl["d1"], d2=wl["d2"])
    desc = nat.BatchDesc()
    desc.B = B
    desc.states = d_states.data_ptr()
    desc.shared_initial = 1
    desc.method = nat.CMD_RK4
    desc.d1 = keep["d1"].ctypes.data
    desc.d2 = keep["d2"].ctypes.data
    desc.width = wl["width"]
    desc.freq = wl["freq"]
    desc.T0 = wl["T0"]
    desc.dt = wl["dt"]
    desc.n_steps = S
    desc.save_interval = 1
    desc.obs = d_obs.data_ptr()
    desc.final_states = d_fin.data_ptr()
    desc.pulse4 = d_pulse.data_ptr()
    launches = C.c_int32()
    # A dedicated stream: the kernel, the L2 flush and every CUDA event below go
    # to this one stream, so the events bracket exactly the launched work.
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)

    def launch():
        st = torch.cuda.current_stream(dev).cuda_stream
        assert st != 0
        nat.check(nat.lib().cmd_run_batch_device(h.ptr, C.byref(desc), C.c_void_p(st), C.byref(launches)),
                  "cmd_run_batch_device")

    for _ in range(args.warmup):
        flush.zero_()
        launch()
    torch.cuda.synchronize(dev)

    sampler = ClockSampler(local)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize(dev)
    sampler.start()
    time.sleep(0.3)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    n_launch = 0
    t_start.record()
    for k in range(args.steps):
        flush.zero_()                       # L2 flush between timed iterations
        ev[k][0].record()
        launch()
        ev[k][1].record()
        n_launch += launches.value
    t_end.record()
    torch.cuda.synchronize(dev)
    clocks = sampler.stop()
    total_ms = t_start.elapsed_time(t_end)
    kern_ms = [a.elapsed_time(b) for a, b in ev]
    if dist is not None:
        total_ms = max_over_ranks(total_ms, dist, dev)
        dist.barrier()
    ms_per_step = total_ms / args.steps
    value = world * B * N * S / (ms_per_step * 1e-3)
    kernel_ms = statistics.mean(kern_ms)

    # ---- parity spot check of the benched run against itself: finite, unit norm
    obs_last = d_obs[:, -1, :].cpu().numpy()
    fin = d_fin.view(B, N, 3)
    norm_dev = float((fin.norm(dim=2) - 1).abs().max().item())
    finite = bool(np.isfinite(obs_last).all())

    # ---- end to end through the public C ABI (pinned host buffers)
    e2e = None
    if not args.no_e2e:
        h_init = torch.from_numpy(wl["s0"]).pin_memory()
        h_obs = torch.empty((B, rows, 10), dtype=torch.float64).pin_memory()
        t1 = np.ascontiguousarray(P[:, 0]); t2 = np.ascontiguousarray(P[:, 1])
        a1 = np.ascontiguousarray(P[:, 2]); a2 = np.ascontiguousarray(P[:, 3])
        hd = nat.BatchDesc()
        hd.B = B
        hd.states = h_init.data_ptr()
        hd.shared_initial = 1
        hd.method = nat.CMD_RK4
        hd.t1, hd.t2, hd.a1, hd.a2 = t1.ctypes.data, t2.ctypes.data, a1.ctypes.data, a2.ctypes.data
        hd.d1 = keep["d1"].ctypes.data
        hd.d2 = keep["d2"].ctypes.data
        hd.width, hd.freq, hd.T0, hd.dt = wl["width"], wl["freq"], wl["T0"], wl["dt"]
        hd.n_steps, hd.save_interval = S, 1
        hd.obs = h_obs.data_ptr()
        hd.final_states = None
        nat.check(nat.lib().cmd_run_batch(h.ptr, C.byref(hd)), "cmd_run_batch")   # warm
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        n_e2e = max(1, min(args.steps, 3))
        for _ in range(n_e2e):
            nat.check(nat.lib().cmd_run_batch(h.ptr, C.byref(hd)), "cmd_run_batch")
        torch.cuda.synchronize(dev)
        e2e_s = (time.perf_counter() - t0) / n_e2e
        if dist is not None:
            e2e_s = max_over_ranks(e2e_s, dist, dev)
        e2e = {"value": world * B * N * S / e2e_s, "unit": UNIT,
               "h2d_bytes_per_step": int(h_init.numel() * 8 + P.size * 8),
               "d2h_bytes_per_step": int(h_obs.numel() * 8)}
        del h_obs

    # ---- plain path: one trajectory per launch (drop-in integrate_gpu)
    plain = None
    if not args.no_plain and rank == 0:
        from classical_mcmc_spin_b200.states import random_unit_spins
        s1 = random_unit_spins(N, 1).ravel()
        gpu_api.set_gpu_spins(h, s1)
        gpu_api.integrate_gpu(h, 0.0, 1.0, 0.01, 1, "rk4", with_states=False)     # warm
        gpu_api.set_gpu_spins(h, s1)
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        _, pobs, ptimes = gpu_api.integrate_gpu(h, 0.0, 99.995, 0.01, 1, "rk4", with_states=False)
        dtp = time.perf_counter() - t0
        nsteps = len(ptimes) - 1
        plain = {"value": N * nsteps / dtp, "unit": UNIT, "steps": nsteps,
                 "workload": "plain MD Kitaev 24x24 (1152 spins), random spins seed 1, RK4 dt=0.01, "
                             "M and E every step, via integrate_gpu (host buffers)"}

    peaks = measured_peaks()
    fp64 = fp64_peak_tflops(torch) if (rank == 0 and not args.no_peak) else None
    achieved_tflops = FLOPS_PER_SPIN_STEP * B * N * S / (kernel_ms * 1e-3) / 1e12
    traffic = profile_traffic()
    roofline = {"bound": "fp64", "achieved": achieved_tflops, "peak": fp64, "unit": "TFLOP/s",
                "frac": (achieved_tflops / fp64) if fp64 else None, "traffic": traffic,
                "peak_source": "measured in this run: cuBLAS DGEMM 8192^3 best of 5 (MEASURED_PEAKS.json "
                               "has no FP64 figure; the kernel is FP64-pipe bound, not HBM or tensor)",
                "flops_per_spin_step": FLOPS_PER_SPIN_STEP,
                "kernel_ms_per_launch": kernel_ms,
                "hbm_peak_gbs_measured": peaks.get("hbm_gbs")}
    legs = {}
    if rank == 0:
        want = [x for x in args.legs.split(",") if x]
        if "uneven" in want:
            legs["uneven_rk45"] = leg_uneven(torch, dev)
        if "adjoint" in want:
            legs["adjoint_kitaev48"] = leg_adjoint_kitaev(torch, dev, S=args.adjoint_steps, B=args.adjoint_traj)
        if "kitaev48" in want:
            legs["kitaev48_forward"] = leg_kitaev48_forward(torch, dev)
        if "mixed" in want:
            legs["mixed_tmfeo3_shape"] = leg_mixed(torch, dev, S=args.mixed_steps)
        if "pyrochlore" in want:
            legs["pyrochlore65536"] = leg_pyrochlore(torch, dev, S=args.pyro_steps, S_adj=args.pyro_adjoint_steps)
    # host-core measurements last, so the GPU legs' host work shares the cores with nothing
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu, _ = cpu_baseline(wl, target_s=args.cpu_seconds)
    cpu_extra = cpu_rows(wl, args.cpu_seconds) if (rank == 0 and not args.no_cpu_baseline
                                                   and not args.no_cpu_rows) else None

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": scan_config(S, world),
                "roofline": roofline, "cpu_baseline": cpu, "cpu_rows": cpu_extra, "e2e": e2e, "clocks": clocks,
                "gpu_launches": n_launch, "plain_path": plain,
                "batched_over_plain": (value / world) / plain["value"] if plain else None,
                "adjoint_over_forward": legs["adjoint_kitaev48"]["ratio"] if "adjoint_kitaev48" in legs else None,
                "legs": legs,
                "checks": {"final_norm_dev_max": norm_dev, "observables_finite": finite}}
        print(json.dumps(line), flush=True)
    h.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
