"""Discrete-adjoint gradients of M(t) losses and a thin torch.autograd.Function.

The loss of trajectory b is  L_b = sum_{n=0..S} |M_local(t_n) - target_b[n]|^2
over the RK4 trajectory of the C-ABI integrator; the gradient with respect to
the coupling parameters comes from the hand-written discrete adjoint of the
RK4 step (cmd_adjoint_rk4, csrc/rk_adjoint.cuh) with sqrt(S)-step
checkpointing and recomputation.  The parameters must enter the couplings
linearly (Kitaev K, Gamma, Gamma', J and the field strength h; non-Kramers
pyrochlore Jzz, J+-, J+-+- and h); parameter q is described by the lattice
built at theta = e_q.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as nat
from ._native import check, f64
from .lattice import Lattice

KITAEV_PARAMS = ("K", "Gamma", "Gammap", "J", "h")
PYRO_PARAMS = ("Jzz", "Jpm", "Jpmpm", "h")


class AdjointDesc(C.Structure):
    _fields_ = [("B", C.c_int64), ("states", C.c_void_p), ("T0", C.c_double), ("dt", C.c_double),
                ("n_steps", C.c_int64), ("target", C.c_void_p), ("checkpoint_every", C.c_int64),
                ("n_params", C.c_int32), ("forward_only", C.c_int32), ("dparams", C.c_void_p),
                ("loss", C.c_void_p), ("grad", C.c_void_p), ("m_local", C.c_void_p), ("path", C.c_int32),
                ("reserved", C.c_int32)]


def _call(handle, desc):
    return nat.lib().cmd_adjoint_rk4(handle.ptr, C.cast(C.pointer(desc), C.c_void_p))


def kitaev_lattice(theta, d1, d2, d3=1, field_direction=(0.0, 1.0, 0.0), g_factor=(1.0, 1.0, 1.0)) -> Lattice:
    K, G, Gp, J, h = (float(x) for x in theta)
    return Lattice.kitaev(d1, d2, d3, h=h, field_direction=field_direction, g_factor=g_factor, K=K, Gamma=G,
                          Gammap=Gp, J=J)


def pyrochlore_lattice(theta, d1, d2, d3, field_direction=(1.0, 1.0, 1.0), cubic=True) -> Lattice:
    Jzz, Jpm, Jpmpm, h = (float(x) for x in theta)
    d = np.asarray(field_direction, dtype=np.float64)
    d = d / np.linalg.norm(d)
    return Lattice.pyrochlore_non_kramer(d1, d2, d3, h=h, field_direction=d, cubic=cubic, Jzz=Jzz, Jpm=Jpm,
                                         Jpmpm=Jpmpm)


def basis_lattices(build, n_params: int) -> list:
    """Lattices built at theta = e_q: their couplings are dJ/dtheta_q (linear models)."""
    return [build(np.eye(n_params)[q]) for q in range(n_params)]


PATHS = {"auto": 0, "resident": 1, "streamed": 2, "global": 3}


def adjoint_rk4(handle, dparams, states, T0, dt, n_steps, targets, checkpoint_every=0, forward_only=False,
                path="auto"):
    """(loss[B], grad[B][n_params], m_local[B][n_steps+1][3]) through cmd_adjoint_rk4.

    ``path``: "auto" (resident when a CTA or cluster holds the lattice), or force "resident",
    "streamed" or "global" (one CTA per trajectory, state in global memory)."""
    st = f64(states).reshape(-1, 3 * handle.N)
    B = st.shape[0]
    tg = f64(targets).reshape(B, n_steps + 1, 3)
    nq = len(dparams)
    descs = (nat.LatticeDesc * max(nq, 1))()
    for q, lat in enumerate(dparams):
        check(nat.lib().cmd_lattice_desc_of(lat._ptr, C.byref(descs[q])), "cmd_lattice_desc_of")
    loss = np.zeros(B)
    grad = np.zeros((B, max(nq, 1)))
    mloc = np.zeros((B, n_steps + 1, 3))
    d = AdjointDesc()
    d.B = B
    d.states = st.ctypes.data
    d.T0 = float(T0)
    d.dt = float(dt)
    d.n_steps = int(n_steps)
    d.target = tg.ctypes.data
    d.checkpoint_every = int(checkpoint_every)
    d.n_params = nq
    d.forward_only = int(bool(forward_only))
    d.dparams = C.cast(descs, C.c_void_p)
    d.loss = loss.ctypes.data
    d.grad = grad.ctypes.data
    d.m_local = mloc.ctypes.data
    d.path = PATHS[path]
    check(_call(handle, d), "cmd_adjoint_rk4")
    return loss, grad[:, :nq], mloc


try:
    import torch

    class LLTrajectoryLoss(torch.autograd.Function):
        """L(theta) = sum_b sum_n |M_local_b(t_n; theta) - target_b[n]|^2.

        forward(theta, build, states, targets, T0, dt, n_steps, checkpoint_every)
        with ``build(theta_numpy) -> Lattice`` building the lattice for the
        parameters (linear models only).  backward uses the discrete adjoint.
        """

        @staticmethod
        def forward(ctx, theta, build, states, targets, T0, dt, n_steps, checkpoint_every=0):
            th = theta.detach().cpu().numpy().astype(np.float64)
            lat = build(th)
            h = lat.to_gpu()
            try:
                dps = basis_lattices(build, th.size)
                loss, grad, _ = adjoint_rk4(h, dps, states, T0, dt, n_steps, targets, checkpoint_every)
            finally:
                h.close()
            ctx.save_for_backward(torch.as_tensor(grad.sum(axis=0), dtype=theta.dtype, device=theta.device))
            return torch.as_tensor(loss.sum(), dtype=theta.dtype, device=theta.device)

        @staticmethod
        def backward(ctx, grad_out):
            (g,) = ctx.saved_tensors
            return grad_out * g, None, None, None, None, None, None, None

except ImportError:     # torch is optional for the C-ABI path
    LLTrajectoryLoss = None
