"""The 2DCS analysis step: the oracle's restatement of the reference reader on known answers (CPU)
and the device implementation cmd_nonlinear_spectrum against it (GPU).

Tolerance: the device FFT and numpy's differ only in summation order, so the spectra agree to
1e-12 of their maximum; M_NL is formed identically (bit for bit).
"""
import ctypes as C

import numpy as np
import pytest


def _oracle():
    import spectra_oracle
    return spectra_oracle


def test_oracle_known_answer_single_tone():
    so = _oracle()
    n_tau, n_t, dt, dtau = 64, 128, 0.25, 0.5
    w_tau, w_t = so.omega_axes(n_tau, dtau, n_t, dt)
    k0, j0 = 5, 12                      # bins of the tone
    tau = dtau * np.arange(n_tau)[:, None]
    t = dt * np.arange(n_t)[None, :]
    wt_true = 2 * np.pi * j0 / (n_t * dt)
    wtau_true = 2 * np.pi * k0 / (n_tau * dtau)
    data = np.cos(wtau_true * tau + wt_true * t) + 3.0         # the constant part is removed
    S = so.compute_2d_fft(data)
    kk, jj = np.unravel_index(np.argmax(S), S.shape)
    # the flip of the omega_t axis maps frequency w to column where flipped axis meets it
    w_t_flipped = w_t[::-1]
    assert np.isclose(abs(w_tau[kk]), wtau_true) and np.isclose(abs(w_t_flipped[jj]), wt_true)
    assert np.isclose(S.max(), n_tau * n_t / 2)
    assert S.sum() / S.max() < 2.0 + 1e-9                      # two delta peaks only


def test_oracle_nonlinear_signal_definition():
    so = _oracle()
    rng = np.random.default_rng(0)
    M0 = rng.normal(size=(10, 3))
    M1 = rng.normal(size=(4, 10, 3))
    M01 = rng.normal(size=(4, 10, 3))
    nl = so.nonlinear_signal(M0, M1, M01, 2)
    assert nl.shape == (4, 10)
    assert nl[3, 7] == M01[3, 7, 2] - M0[7, 2] - M1[3, 7, 2]


@pytest.mark.gpu
@pytest.mark.parametrize("n_tau,n_t", [(1, 1), (7, 33), (64, 100), (241, 401)])
def test_device_spectrum_matches_oracle(native, n_tau, n_t):
    so = _oracle()
    rng = np.random.default_rng(n_tau * 1000 + n_t)
    M0 = rng.normal(size=(n_t, 3))
    M1 = rng.normal(size=(n_tau, n_t, 3))
    M01 = M1 + M0[None] + 0.1 * rng.normal(size=(n_tau, n_t, 3))
    for c in range(3):
        nl = np.zeros((n_tau, n_t))
        sp = np.zeros((n_tau, n_t))
        D = native.dptr
        native.check(native.lib().cmd_nonlinear_spectrum(D(M0), D(M1), D(M01), n_tau, n_t, c, D(nl), D(sp)),
                     "cmd_nonlinear_spectrum")
        np.testing.assert_array_equal(nl, so.nonlinear_signal(M0, M1, M01, c))
        ref = so.compute_2d_fft(so.nonlinear_signal(M0, M1, M01, c))
        assert np.abs(sp - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max())


def test_spectrum_rejects_bad_arguments(native):
    L = native.lib()
    z = np.zeros(3)
    assert L.cmd_nonlinear_spectrum(None, None, None, 1, 1, 0, None, None) == native.CMD_ERR_INVALID_ARG
    assert L.cmd_nonlinear_spectrum(native.dptr(z), native.dptr(z), native.dptr(z), 1, 1, 3, None, None) \
        == native.CMD_ERR_INVALID_ARG
