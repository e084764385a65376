"""cmd_run_batch_device_noalloc against cmd_run_batch_device, through the C ABI.

Both entry points run the same resident RK4 kernels on the same device
buffers; the allocation-free one keeps its scratch (step-time grid, pulse
envelope table, and for 4-atom cells the raw observable rows) in one static
device array.  Two calls in a row, with different pulses and initial states,
must each match the allocating entry point within the parity tests' absolute
tolerance on M / E rows and final spins (1e-12), driven and undriven, with
per-trajectory and shared initial states, and for zero steps.  A warmed call
must leave the device's free memory (cudaMemGetInfo) unchanged.  The file is
collected last so that it also runs after every other GPU test; it must pass
alone too.
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


class _Call:
    """Device buffers and a cmd_batch_desc for one batch, allocated up front."""

    def __init__(self, native, lat, states, pulse4, n_steps, save, driven=True, shared=False):
        import torch
        B = pulse4.shape[0]
        rows = native.lib().cmd_batch_rows(n_steps, save)
        self.obs = torch.full((B, rows, 10), float("nan"), dtype=torch.float64, device="cuda")
        self.fin = torch.full((B, states.shape[1]), float("nan"), dtype=torch.float64, device="cuda")
        self.d1 = np.tile([0.0, 0.0, 1.0], lat.N_atoms)
        self.d2 = np.tile([1.0, 0.0, 0.0], lat.N_atoms)
        self.states, self.pulse4 = states, pulse4
        d = native.BatchDesc()
        d.B = B
        d.states = states.data_ptr()
        d.shared_initial = 1 if shared else 0
        d.method = native.CMD_RK4
        d.d1 = self.d1.ctypes.data if driven else None
        d.d2 = self.d2.ctypes.data if driven else None
        d.width, d.freq = 0.4, 2.0
        d.T0, d.dt = 0.0, 0.01
        d.n_steps, d.save_interval = n_steps, save
        d.obs = self.obs.data_ptr()
        d.final_states = self.fin.data_ptr()
        d.pulse4 = pulse4.data_ptr() if driven else None
        self.desc = d
        self.native = native

    def run(self, fn_name, h, stream):
        import torch
        launches = C.c_int32()
        fn = getattr(self.native.lib(), fn_name)
        torch.cuda.synchronize()       # inputs and output fills written on torch's stream are complete
        self.native.check(fn(h.ptr, C.byref(self.desc), C.c_void_p(stream.cuda_stream), C.byref(launches)),
                          fn_name)
        stream.synchronize()
        return self.obs.cpu().numpy(), self.fin.cpu().numpy(), launches.value


def _inputs(lat, B, seed, shared=False):
    import torch
    from classical_mcmc_spin_b200.states import random_unit_spins
    rng = np.random.default_rng(seed)
    st = np.stack([random_unit_spins(lat.lattice_size, seed * 100 + b).ravel() for b in range(1 if shared else B)])
    p = np.stack([rng.uniform(0.5, 1.5, B), rng.uniform(1.0, 2.0, B), rng.uniform(0.2, 1.0, B),
                  rng.uniform(0.2, 1.0, B)], axis=1)
    return (torch.tensor(st, dtype=torch.float64, device="cuda"),
            torch.tensor(p, dtype=torch.float64, device="cuda").contiguous())


def _compare(native, h, lat, stream, B, seed, n_steps, save, driven, shared):
    states, pulse4 = _inputs(lat, B, seed, shared)
    ref = _Call(native, lat, states, pulse4, n_steps, save, driven, shared)
    o_ref, f_ref, _ = ref.run("cmd_run_batch_device", h, stream)
    na = _Call(native, lat, states, pulse4, n_steps, save, driven, shared)
    o_na, f_na, nl = na.run("cmd_run_batch_device_noalloc", h, stream)
    assert nl >= 2
    assert np.isfinite(o_na).all() and np.isfinite(f_na).all()
    np.testing.assert_allclose(o_na, o_ref, rtol=0, atol=TOL)
    np.testing.assert_allclose(f_na, f_ref, rtol=0, atol=TOL)


@pytest.mark.parametrize("kind", ["kitaev", "pyrochlore"])
@pytest.mark.parametrize("driven,shared,n_steps", [(True, False, 300), (False, False, 300), (True, True, 300),
                                                   (False, True, 0), (True, False, 0)])
def test_noalloc_matches_allocating_entry_point_twice(native, kind, driven, shared, n_steps):
    import torch
    lat = _lattice(kind)
    h = lat.to_gpu()
    stream = torch.cuda.Stream()
    try:
        for call, seed in enumerate((11, 12)):       # two calls in a row share the scratch array
            _compare(native, h, lat, stream, 5 + call, seed, n_steps, 7, driven, shared)
    finally:
        h.close()


@pytest.mark.parametrize("kind", ["kitaev", "pyrochlore"])
def test_noalloc_call_leaves_free_device_memory_unchanged(native, kind):
    """The property the entry point exists for: on a warmed handle, the call takes no device memory."""
    import torch
    lat = _lattice(kind)
    h = lat.to_gpu()
    stream = torch.cuda.Stream()
    try:
        states, pulse4 = _inputs(lat, 9, 21)
        call = _Call(native, lat, states, pulse4, 500, 3)
        call.run("cmd_run_batch_device_noalloc", h, stream)        # warm: first launches, lazy kernel loads
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info()
        for _ in range(3):
            call.run("cmd_run_batch_device_noalloc", h, stream)
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info()
        assert free1 == free0, (free0, free1)
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
        call = _Call(native, lat, states, pulse4, n_steps, 1000)
        with pytest.raises(native.CmdError) as e:
            call.run("cmd_run_batch_device_noalloc", h, stream)
        assert e.value.code == native.CMD_ERR_INVALID_ARG
        assert "split the batch" in str(e.value)
    finally:
        h.close()


def test_noalloc_rejects_streamed_lattices_with_a_pointer_to_the_allocating_call(native):
    import torch
    from classical_mcmc_spin_b200.lattice import Lattice
    lat = Lattice.kitaev(64, 64, 1)      # 4096 cells: beyond every resident variant (streamed kernels)
    h = lat.to_gpu()
    stream = torch.cuda.Stream()
    try:
        states, pulse4 = _inputs(lat, 2, 31)
        call = _Call(native, lat, states, pulse4, 10, 5)
        with pytest.raises(native.CmdError) as e:
            call.run("cmd_run_batch_device_noalloc", h, stream)
        assert e.value.code == native.CMD_ERR_UNSUPPORTED
        assert "cmd_run_batch_device" in str(e.value) and "resident lattices only" in str(e.value)
        o, f, _ = call.run("cmd_run_batch_device", h, stream)   # the allocating entry point runs it
        assert np.isfinite(o).all() and np.isfinite(f).all()
    finally:
        h.close()
