"""Handles on two devices in one process.

Function attributes (the dynamic shared-memory limit above 48 KB that the resident kernels need) belong to
each device's context, so a process that drives two GPUs must see every launch configured on both.  The
1152-spin scan uses 55 KB of shared memory per CTA.  Skipped when fewer than two devices are visible.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_handles_on_two_devices_in_one_process(native):
    import torch
    if torch.cuda.device_count() < 2:
        pytest.skip("needs two visible CUDA devices")
    from classical_mcmc_spin_b200 import gpu_api
    from classical_mcmc_spin_b200.lattice import Lattice
    from classical_mcmc_spin_b200.states import zigzag_honeycomb
    lat = Lattice.kitaev(24, 24, 1)
    s0 = zigzag_honeycomb(24, 24, 1, tilt_sigma=0.05, seed=2).ravel()
    fin = np.tile(np.ones(3) / np.sqrt(3.0), 2)
    fd = lat.rotate_pulse(fin, fin)
    kw = dict(T0=-1.0, t1=[0.0, 0.0], t2=[0.3, 0.6], a1=[0.5, 0.5], a2=[0.5, 0.5], d1=fd[:6], d2=fd[6:],
              width=0.5, freq=0.0, shared_initial=True)
    out = []
    for dev in (0, 1):
        torch.cuda.set_device(dev)
        h = lat.to_gpu()
        out.append(gpu_api.run_batch(h, s0, 200, 0.01, **kw))
        h.close()
    torch.cuda.set_device(0)
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_array_equal(out[0][1], out[1][1])
