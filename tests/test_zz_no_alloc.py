"""cmd_run_batch_device_noalloc against cmd_run_batch_device, through the C ABI.

Both entry points run the same resident RK4 kernels on the same device
buffers; the allocation-free one keeps its scratch (step-time grid, pulse
envelope table, and for 4-atom cells the raw observable rows) in one static
device array.  Two calls in a row, with different pulses and initial states,
must each match the allocating entry point within the parity tests' absolute
tolerance on M / E rows and final spins (1e-12).  The file is collected last
so that it also runs after every other GPU test; it must pass alone too.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _lattice(kind):
    from classical_mcmc_spin_b200.lattice import Lattice
    if kind == "kitaev":       # 2-atom cells: raw rows are written into obs in place
        return Lattice.kitaev(6, 6, 1, h=0.1, field_direction=(0.0, 1.0, 0.0))
    # 4-atom cells: raw rows (13 per row) go to the scratch array
    d = np.ones(3) / np.sqrt(3.0)
    return Lattice.pyrochlore_non_kramer(2, 2, 2, h=0.2, field_direction=d, cubic=True)


def _run(native, fn_name, h, lat, states, pulse4, n_steps, save, stream):
    import torch
    B = states.shape[0]
    rows = native.lib().cmd_batch_rows(n_steps, save)
    obs = torch.full((B, rows, 10), float("nan"), dtype=torch.float64, device="cuda")
    fin = torch.full_like(states, float("nan"))
    d1 = np.tile([0.0, 0.0, 1.0], lat.N_atoms)
    d2 = np.tile([1.0, 0.0, 0.0], lat.N_atoms)
    desc = native.BatchDesc()
    desc.B = B
    desc.states = states.data_ptr()
    desc.shared_initial = 0
    desc.method = native.CMD_RK4
    desc.d1 = d1.ctypes.data
    desc.d2 = d2.ctypes.data
    desc.width, desc.freq = 0.4, 2.0
    desc.T0, desc.dt = 0.0, 0.01
    desc.n_steps, desc.save_interval = n_steps, save
    desc.obs = obs.data_ptr()
    desc.final_states = fin.data_ptr()
    desc.pulse4 = pulse4.data_ptr()
    launches = C.c_int32()
    fn = getattr(native.lib(), fn_name)
    torch.cuda.synchronize()           # inputs and output fills written on torch's stream are complete
    native.check(fn(h.ptr, C.byref(desc), C.c_void_p(stream.cuda_stream), C.byref(launches)), fn_name)
    stream.synchronize()
    return obs.cpu().numpy(), fin.cpu().numpy(), launches.value


def _inputs(lat, B, seed):
    import torch
    from classical_mcmc_spin_b200.states import random_unit_spins
    rng = np.random.default_rng(seed)
    st = np.stack([random_unit_spins(lat.lattice_size, seed * 100 + b).ravel() for b in range(B)])
    p = np.stack([rng.uniform(0.5, 1.5, B), rng.uniform(1.0, 2.0, B), rng.uniform(0.2, 1.0, B),
                  rng.uniform(0.2, 1.0, B)], axis=1)
    return (torch.tensor(st, dtype=torch.float64, device="cuda"),
            torch.tensor(p, dtype=torch.float64, device="cuda").contiguous())


@pytest.mark.parametrize("kind", ["kitaev", "pyrochlore"])
def test_noalloc_matches_allocating_entry_point_twice(native, kind):
    import torch
    lat = _lattice(kind)
    h = lat.to_gpu()
    stream = torch.cuda.Stream()
    n_steps, save = 300, 7
    try:
        for call, seed in enumerate((11, 12)):       # two calls in a row share the scratch array
            states, pulse4 = _inputs(lat, 5 + call, seed)
            o_ref, f_ref, _ = _run(native, "cmd_run_batch_device", h, lat, states, pulse4, n_steps, save, stream)
            o_na, f_na, nl = _run(native, "cmd_run_batch_device_noalloc", h, lat, states, pulse4, n_steps, save,
                                  stream)
            assert nl >= 3
            assert np.isfinite(o_na).all() and np.isfinite(f_na).all()
            np.testing.assert_allclose(o_na, o_ref, rtol=0, atol=TOL)
            np.testing.assert_allclose(f_na, f_ref, rtol=0, atol=TOL)
    finally:
        h.close()


def test_noalloc_rejects_batches_beyond_the_static_scratch(native):
    import torch
    lat = _lattice("kitaev")
    h = lat.to_gpu()
    stream = torch.cuda.Stream()
    try:
        B, n_steps = 100, 7000           # 100 * 7000 * 6 doubles > 2^22
        states = torch.zeros((B, 3 * lat.lattice_size), dtype=torch.float64, device="cuda")
        states[:, 2::3] = 1.0
        pulse4 = torch.ones((B, 4), dtype=torch.float64, device="cuda")
        with pytest.raises(native.CmdError) as e:
            _run(native, "cmd_run_batch_device_noalloc", h, lat, states, pulse4, n_steps, 1000, stream)
        assert e.value.code == native.CMD_ERR_INVALID_ARG
        assert "split the batch" in str(e.value)
    finally:
        h.close()
