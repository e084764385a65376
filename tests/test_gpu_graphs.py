"""CUDA graphs on the batched resident path, the uneven batch and the streamed adjoint.

With graphs on (the default) a batched resident run (drive table, resident
kernel, row finisher) and an uneven batch (its concurrent per-lattice launches
and their fork / join) are captured and replayed as one graph per call, the
handle's executable graph updated in place when only launch arguments change
and rebuilt when the launch topology changes; the streamed adjoint replays
128-step chunks of its forward and whole checkpoint segments of its reverse
sweep.  The kernels and their arguments are the same either way, so every
result here must equal the direct launches' bit for bit, across calls that
change pulses, batch size, step count, kernel variant and the set of lattices.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

R111 = np.ones(3) / np.sqrt(3.0)


@pytest.fixture(scope="module")
def api(native):
    from classical_mcmc_spin_b200 import gpu_api
    return gpu_api


def _spins(n, seed):
    from classical_mcmc_spin_b200.states import random_unit_spins
    return random_unit_spins(n, seed).ravel()


def _both(h, fn):
    h.set_graphs(True)
    g = fn()
    h.set_graphs(False)
    d = fn()
    h.set_graphs(True)
    return g, d


@pytest.mark.parametrize("L", [6, 48])
def test_batched_resident_graph_equals_direct_launches(api, oracle, L):
    """Kitaev 6x6 (one CTA per trajectory) and 48x48 (4-CTA clusters): a sequence of calls with graphs on --
    new pulses, a larger batch, another step count -- each equal to the same call launched directly; the 6x6
    case also against the oracle."""
    from classical_mcmc_spin_b200.lattice import Lattice
    lat = Lattice.kitaev(L, L, 1)
    h = lat.to_gpu()
    fin = np.tile(R111, 2)
    fd = lat.rotate_pulse(fin, fin)
    s0 = _spins(lat.lattice_size, 11)
    calls = [(2, [0.0, 0.2], [0.5, 0.9], 120), (2, [0.1, 0.3], [0.7, 1.0], 120), (3, [0.0, 0.2, 0.4], [0.6, 0.8, 1.1], 90)]
    for B, t1, t2, nsteps in calls:
        kw = dict(T0=-0.5, t1=t1, t2=t2, a1=[0.5] * B, a2=[0.4] * B, d1=fd[:6], d2=fd[6:], width=0.5, freq=0.0,
                  shared_initial=True)
        (og, fg), (od, fdir) = _both(h, lambda: api.run_batch(h, s0, nsteps, 0.01, **kw))
        np.testing.assert_array_equal(og, od)
        np.testing.assert_array_equal(fg, fdir)
        if L == 6:
            st, oobs = oracle.OracleLattice.kitaev(L, L, 1).batch_rk4(
                np.tile(s0, (B, 1)), t1, t2, np.full(B, 1.0), np.full(B, 0.8), 0.5, 0.5, 0.0, fin, fin, -0.5, 0.01,
                nsteps)
            assert np.abs(fg - st).max() <= 1e-10
            assert np.abs(og - oobs).max() <= 1e-12
    h.close()


def test_graph_follows_variant_changes(api):
    """Pinning other resident variants between calls changes the kernel in the captured graph."""
    from classical_mcmc_spin_b200.lattice import Lattice
    lat = Lattice.kitaev(8, 8, 1)
    h = lat.to_gpu()
    s0 = _spins(lat.lattice_size, 12)
    fits = [i for i, _, ok in h.variants() if ok][:4]
    assert len(fits) >= 2
    ref = None
    for v in fits:
        h.set_variant(v)
        (og, fg), (od, fdir) = _both(h, lambda: api.run_batch(h, np.tile(s0, (2, 1)), 80, 0.01))
        np.testing.assert_array_equal(og, od)
        np.testing.assert_array_equal(fg, fdir)
        if ref is None:
            ref = fg
        assert np.abs(fg - ref).max() <= 1e-12
    h.close()


def test_uneven_batch_graph_equals_direct_launches(api):
    """Controlled RK45 over honeycomb 4x4 / 8x8 and pyrochlore 1 / 2 (concurrent on-chip launches, one per
    lattice), then a batch without the pyrochlore lattices (another launch topology): graphs on equal to direct
    launches in rows, final states and step statistics."""
    from classical_mcmc_spin_b200.lattice import Lattice
    kw = dict(Jzz=1.0, Jpm=0.05, Jpmpm=0.02)
    lats = [Lattice.kitaev(4, 4, 1), Lattice.kitaev(8, 8, 1),
            Lattice.pyrochlore_non_kramer(1, 1, 1, h=0.2, field_direction=R111, **kw),
            Lattice.pyrochlore_non_kramer(2, 2, 2, h=0.2, field_direction=R111, **kw)]
    hs = [lat.to_gpu() for lat in lats]
    specs = [dict(handle=h, state=_spins(lat.lattice_size, 60 + i), T0=0.0, T1=1.0, dt=0.01, max_rows=4000)
             for i, (lat, h) in enumerate(zip(lats, hs))]
    for sub in (specs, specs[:2], specs):
        g, d = _both(hs[0], lambda: api.run_uneven(sub, "rk45", 1e-10, 1e-10))
        for (rg, fg, sg), (rd, fd, sd) in zip(g, d):
            np.testing.assert_array_equal(rg, rd)
            np.testing.assert_array_equal(fg, fd)
            assert list(sg) == list(sd)
    for h in hs:
        h.close()


@pytest.mark.parametrize("ckpt", [20, 17])
def test_streamed_adjoint_graph_equals_direct_launches(ckpt):
    """Streamed adjoint (honeycomb 64x64, no resident kernel holds it), 300 steps: the forward replays two
    128-step chunks, the reverse sweep replays its full checkpoint segments (even and odd segment lengths, so
    both orders of the cotangent buffers); loss and gradient equal to direct launches bit for bit."""
    from classical_mcmc_spin_b200 import adjoint as A
    theta = np.array([-1.0, 0.25, -0.02, 0.05, 0.1])
    build = lambda th: A.kitaev_lattice(th, 64, 64)
    lat = build(theta)
    h = lat.to_gpu()
    B, S, dt = 2, 300, 0.01
    states = np.stack([_spins(lat.lattice_size, 70 + b) for b in range(B)])
    targets = np.random.default_rng(11).normal(scale=0.05, size=(B, S + 1, 3))
    dps = A.basis_lattices(build, 5)
    (lg, gg, mg), (ld, gd, md) = _both(h, lambda: A.adjoint_rk4(h, dps, states, 0.0, dt, S, targets,
                                                                   checkpoint_every=ckpt, path="streamed"))
    np.testing.assert_array_equal(lg, ld)
    np.testing.assert_array_equal(gg, gd)
    np.testing.assert_array_equal(mg, md)
    # and again with graphs on: the kept graphs replay
    l2, g2, _ = A.adjoint_rk4(h, dps, states, 0.0, dt, S, targets, checkpoint_every=ckpt, path="streamed")
    np.testing.assert_array_equal(l2, ld)
    np.testing.assert_array_equal(g2, gd)
    h.close()
