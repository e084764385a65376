"""Oracle for the 2DCS analysis step (test infrastructure only).

Restates the reference's offline analysis in util/readers_new/reader_honeycomb.py:
  * :521-531  M_NL[c][k][t] = M01_k[t][c] - M0[t][c] - M1_k[t][c] on M_local;
  * :536-541  omega_tau = fftshift(fftfreq(n_tau, dtau)) 2 pi, omega_t likewise with dt;
  * :545-553  compute_2d_fft: subtract the global mean, fft2, fftshift, abs, flip axis 1.
"""
import numpy as np


def nonlinear_signal(M0, M1, M01, component):
    """M0 [n_t][3], M1 / M01 [n_tau][n_t][3] -> M_NL [n_tau][n_t] of one component."""
    M0 = np.asarray(M0, dtype=np.float64)
    return (np.asarray(M01, dtype=np.float64)[:, :, component] - M0[None, :, component]
            - np.asarray(M1, dtype=np.float64)[:, :, component])


def compute_2d_fft(data):
    data = np.asarray(data, dtype=np.float64)
    ff = np.fft.fft2(data - np.mean(data))
    ff = np.abs(np.fft.fftshift(ff))
    return np.flip(ff, axis=1)


def omega_axes(n_tau, dtau, n_t, dt):
    w_tau = np.fft.fftshift(np.fft.fftfreq(int(n_tau), dtau) * 2 * np.pi)
    w_t = np.fft.fftshift(np.fft.fftfreq(int(n_t), dt) * 2 * np.pi)
    return w_tau, w_t
