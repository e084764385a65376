"""cmd_run_batch on long runs (>= 4096 steps) computes in time chunks and copies each chunk's rows
back while the next one runs.  Every row and final state must equal one cmd_run_batch_device
launch bit for bit (same steps, same accumulated times, same arithmetic)."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

R111 = np.ones(3) / np.sqrt(3.0)


def _single_launch(native, h, s0, B, P, d1, d2, S, save, T0, dt, width, freq):
    import torch
    rows = int(native.lib().cmd_batch_rows(S, save))
    d_states = torch.tensor(s0, dtype=torch.float64, device="cuda")
    d_pulse = torch.tensor(P, dtype=torch.float64, device="cuda").contiguous()
    d_obs = torch.empty((B, rows, 10), dtype=torch.float64, device="cuda")
    d_fin = torch.empty((B, s0.size), dtype=torch.float64, device="cuda")
    desc = native.BatchDesc()
    desc.B, desc.states, desc.shared_initial, desc.method = B, d_states.data_ptr(), 1, native.CMD_RK4
    desc.d1, desc.d2 = d1.ctypes.data, d2.ctypes.data
    desc.width, desc.freq, desc.T0, desc.dt = width, freq, T0, dt
    desc.n_steps, desc.save_interval = S, save
    desc.obs, desc.final_states, desc.pulse4 = d_obs.data_ptr(), d_fin.data_ptr(), d_pulse.data_ptr()
    st = torch.cuda.Stream()
    torch.cuda.synchronize()
    native.check(native.lib().cmd_run_batch_device(h.ptr, C.byref(desc), C.c_void_p(st.cuda_stream), None), "dev")
    torch.cuda.synchronize()
    return d_obs.cpu().numpy(), d_fin.cpu().numpy()


@pytest.mark.parametrize("S,save", [(5000, 1), (6001, 7), (4096, 5000)])
def test_chunked_host_batch_equals_single_launch(native, S, save):
    from classical_mcmc_spin_b200 import gpu_api
    from classical_mcmc_spin_b200.lattice import Lattice
    from classical_mcmc_spin_b200.states import random_unit_spins
    lat = Lattice.kitaev(6, 6, 1, h=0.1, field_direction=(0.0, 1.0, 0.0))
    h = lat.to_gpu()
    s0 = random_unit_spins(lat.lattice_size, 31).ravel()
    fd = lat.rotate_pulse(np.tile(R111, 2), np.tile(R111, 2))
    d1, d2 = np.ascontiguousarray(fd[:6]), np.ascontiguousarray(fd[6:])
    t1 = [0.0, 0.0, 0.0, 1.0, 3.0]
    t2 = [0.0, 2.0, 2.0, 5.0, 3.5]
    a1 = [0.5, 0.0, 0.5, 0.3, 0.2]
    a2 = [0.0, 0.5, 0.5, 0.3, 0.6]
    B = len(t1)
    T0, dt, width, freq = -2.0, 0.01, 0.5, 0.2
    obs, fin = gpu_api.run_batch(h, s0, S, dt, T0=T0, save_interval=save, t1=t1, t2=t2, a1=a1, a2=a2, d1=d1, d2=d2,
                                 width=width, freq=freq, shared_initial=True)
    P = np.stack([t1, t2, a1, a2], axis=1)
    o1, f1 = _single_launch(native, h, s0, B, P, d1, d2, S, save, T0, dt, width, freq)
    assert obs.shape == o1.shape
    np.testing.assert_array_equal(obs, o1)
    np.testing.assert_array_equal(fin, f1)
