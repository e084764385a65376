"""Host-side logic of the product: bond tables, layout planning, states, spin I/O (no GPU)."""
import ctypes as C

import numpy as np
import pytest

from classical_mcmc_spin_b200 import _native as nat
from classical_mcmc_spin_b200.lattice import Lattice
from classical_mcmc_spin_b200.states import random_unit_spins, zigzag_honeycomb

R111 = np.ones(3) / np.sqrt(3.0)


def _same_tables(prod, orc):
    e, oe = prod.export(), orc.ell()
    for k in ("partners", "counts"):
        np.testing.assert_array_equal(e[k], oe[k])
    for k in ("field", "onsite", "bilinear"):
        np.testing.assert_allclose(e[k], oe[k], rtol=0, atol=1e-15)
    fr, afm = orc.frames()
    np.testing.assert_allclose(e["frames"], fr, rtol=0, atol=1e-15)
    np.testing.assert_array_equal(e["afm"], afm)


@pytest.mark.parametrize("dims", [(1, 1, 1), (2, 3, 1), (4, 4, 1), (24, 24, 1), (5, 4, 2)])
@pytest.mark.parametrize("extra", [{}, dict(J2_A=0.1, J2_B=-0.05), dict(J3=0.2, J_perp=0.1, Ka=0.1, Kc=-0.3)])
def test_kitaev_tables_match_oracle(native, oracle, dims, extra):
    if extra.get("J3") and min(dims[:2]) < 2:
        pytest.skip("J3 offset -2 needs d2 >= 2")
    p = Lattice.kitaev(*dims, h=0.3, field_direction=(0.1, 0.8, 0.2), g_factor=(1.0, 2.0, 0.5), **extra)
    o = oracle.OracleLattice.kitaev(*dims, h=0.3, direction=(0.1, 0.8, 0.2), g=(1.0, 2.0, 0.5), **extra)
    _same_tables(p, o)


@pytest.mark.parametrize("dims", [(1, 1, 1), (2, 2, 2), (3, 2, 4)])
@pytest.mark.parametrize("cubic", [False, True])
def test_pyrochlore_tables_match_oracle(native, oracle, dims, cubic):
    kw = dict(Jzz=1.0, Jpm=0.05, Jpmpm=0.02, delta1=0.1, delta2=0.05)
    p = Lattice.pyrochlore_non_kramer(*dims, h=0.2, field_direction=R111, cubic=cubic, **kw)
    o = oracle.OracleLattice.pyrochlore_nk(*dims, h=0.2, direction=R111, cubic=cubic, **kw)
    _same_tables(p, o)


def test_cubic_cell_reproduces_primitive_local_fields(oracle):
    """For a 4-sublattice-periodic state the conventional cubic cell and the
    reference's primitive cell give identical per-sublattice fields and energy per site."""
    kw = dict(Jzz=1.0, Jpm=0.05, Jpmpm=0.02)
    prim = oracle.OracleLattice.pyrochlore_nk(2, 2, 2, h=0.2, direction=R111, **kw)
    cub = oracle.OracleLattice.pyrochlore_nk(2, 2, 2, h=0.2, direction=R111, cubic=True, **kw)
    sub = random_unit_spins(4, 9)
    sp = np.tile(sub, (prim.N // 4, 1)).ravel()
    sc = np.tile(sub, (cub.N // 4, 1)).ravel()
    Hp = prim.local_field(sp).reshape(-1, 4, 3)
    Hc = cub.local_field(sc).reshape(-1, 4, 3)
    np.testing.assert_allclose(Hp[0], Hc[0], atol=1e-14)
    np.testing.assert_allclose(Hc, np.broadcast_to(Hc[0], Hc.shape), atol=1e-14)
    assert abs(prim.energy(sp) / prim.N - cub.energy(sc) / cub.N) < 1e-14


def _plan(lat):
    d = nat.LatticeDesc()
    nat.check(nat.lib().cmd_lattice_desc_of(lat._ptr, C.byref(d)), "desc")
    info = np.zeros(7, np.int64)
    rc = nat.lib().cmd_plan_layout(C.byref(d), nat.iptr(info))
    return rc, info, nat.lib().cmd_last_error().decode()


def test_layout_plan_honeycomb_configs(native):
    rc, info, _ = _plan(Lattice.kitaev(24, 24, 1))
    assert rc == nat.CMD_OK
    assert list(info[[0, 1, 2, 6]]) == [2, 576, 3, 1]        # 2 atoms/cell, 576 cells, 3 bonds, 1 in-cell
    assert info[3] == 576 and info[4] == 1
    # the lean variant: two stage buffers with the component stride of its 640-thread bound
    assert info[5] == 2 * 2 * 3 * 640 * 8 + (32 * 16 + 12) * 8
    rc, info, _ = _plan(Lattice.kitaev(32, 32, 1))
    assert rc == nat.CMD_OK and info[4] == 2 and info[3] == 512


def test_layout_plan_pyrochlore_drops_zero_j2(native):
    lat = Lattice.pyrochlore_non_kramer(4, 4, 4, h=0.2, field_direction=R111, Jzz=1.0, Jpm=0.05, Jpmpm=0.02)
    assert lat.num_bi == 12                        # reference keeps the J2 = 0 bonds
    rc, info, _ = _plan(lat)
    assert rc == nat.CMD_OK and list(info[[0, 2, 6]]) == [4, 6, 3]


def test_layout_plan_rejects_with_reason(native):
    rc, info, msg = _plan(Lattice.kitaev(8, 8, 1, J2_A=0.1, J2_B=0.1))
    assert rc == nat.CMD_ERR_UNSUPPORTED and "9 bonds/site" in msg
    rc, info, msg = _plan(Lattice.kitaev(64, 64, 1))         # no CTA or 4-CTA cluster holds 4096 cells
    assert rc == nat.CMD_ERR_UNSUPPORTED and "4096 cells" in msg
    rc, info, _ = _plan(Lattice.kitaev(48, 48, 1))           # 4 CTAs of 576 cells
    assert rc == nat.CMD_OK and info[3] == 576 and info[5] == (2 * 576 * 2 * 3 + 32 * 16 + 12 + 16) * 8


def test_layout_plan_rejects_non_uniform_couplings(native):
    lat = Lattice.kitaev(4, 4, 1)
    e = lat.export()
    e["bilinear"][9 * 5] += 1e-3                  # one bond of one site differs
    d = nat.LatticeDesc()
    d.lattice_size, d.spin_dim, d.n_atoms, d.max_bilinear = lat.lattice_size, 3, 2, e["max_bilinear"]
    d.field, d.onsite, d.bilinear = nat.dptr(e["field"]), nat.dptr(e["onsite"]), nat.dptr(e["bilinear"])
    d.partners, d.counts = nat.iptr(e["partners"]), nat.iptr(e["counts"])
    info = np.zeros(7, np.int64)
    assert nat.lib().cmd_plan_layout(C.byref(d), nat.iptr(info)) == nat.CMD_ERR_UNSUPPORTED
    assert b"not identical" in nat.lib().cmd_last_error()


def test_bad_unit_cell_is_rejected(native):
    out = C.c_void_p()
    bonds = np.array([[0, 1, 0, -3, 0]], np.int32)   # offset larger than the box
    J = np.eye(3).ravel()
    rc = nat.lib().cmd_lattice_generic(2, bonds.ctypes.data_as(C.POINTER(C.c_int32)), nat.dptr(J), 1, None,
                                       None, None, None, 2, 2, 1, C.byref(out))
    assert rc == nat.CMD_ERR_INVALID_ARG and not out.value


def test_random_spins_seeded_unit():
    a = random_unit_spins(5000, 7)
    b = random_unit_spins(5000, 7)
    np.testing.assert_array_equal(a, b)
    np.testing.assert_allclose(np.linalg.norm(a, axis=1), 1.0, atol=1e-15)
    assert np.abs(a.mean(axis=0)).max() < 0.05
    assert not np.array_equal(a, random_unit_spins(5000, 8))


def test_zigzag_state():
    s = zigzag_honeycomb(4, 4, 1)
    assert s.shape == (32, 3)
    np.testing.assert_allclose(s.sum(axis=0), 0.0, atol=1e-14)
    t = zigzag_honeycomb(4, 4, 1, tilt_sigma=0.05, seed=2)
    np.testing.assert_allclose(np.linalg.norm(t, axis=1), 1.0, atol=1e-15)
    assert 0.0 < np.abs(t - s).max() < 0.5


def test_spin_config_round_trip(tmp_path):
    lat = Lattice.kitaev(3, 3, 1)
    lat.spins = random_unit_spins(lat.lattice_size, 1)
    f = tmp_path / "initial_spins.txt"
    lat.save_spin_config(str(f))
    other = Lattice.kitaev(3, 3, 1)
    other.load_spin_config(str(f))
    np.testing.assert_array_equal(other.spins, lat.spins)


def test_rotate_pulse_is_frame_times_field(native):
    lat = Lattice.kitaev(2, 2, 1)
    fin = np.tile(R111, 2)
    fd = lat.rotate_pulse(fin, 2 * fin)
    R = lat.sublattice_frames
    np.testing.assert_allclose(fd[:3], R[0] @ R111, atol=1e-15)
    np.testing.assert_allclose(fd[6:9], R[0] @ (2 * R111), atol=1e-15)


def test_layout_plan_groups_the_cubic_pyrochlore_cell(native):
    """The 16-site cubic cell is 4 FCC translations of the 4-site group: it maps onto
    the 4-atom kernels (same couplings, fields and frames per sublattice class)."""
    lat = Lattice.pyrochlore_non_kramer(2, 2, 2, cubic=True, h=0.2, field_direction=R111, Jzz=1.0, Jpm=0.05,
                                        Jpmpm=0.02)
    assert lat.N_atoms == 16
    rc, info, msg = _plan(lat)
    assert rc == nat.CMD_OK, msg
    assert list(info[[0, 1, 2, 6]]) == [4, lat.lattice_size // 4, 6, 3]
