"""The numpy restatement of the mixed SU(2)/SU(3) dynamics (oracle/mixed_oracle.py) and the seeded
synthetic lattices (mixed_gpu_api.synthetic_mixed_lattice), on the CPU.

Pins: the su(3) structure constants derived from the Gell-Mann matrices are totally antisymmetric,
take the textbook values and satisfy the Jacobi identity; the local fields are the gradient of the
energy (central differences, 1e-7 relative); every bond is stored at both ends with transposed
couplings; under RK4 the energy, every SU(2) spin length and every SU(3) vector length are conserved
to the method's truncation error (<= 5e-9 over t = 1 at dt = 0.01, falling 16x when dt halves)."""
import numpy as np
import pytest

from classical_mcmc_spin_b200.mixed_gpu_api import random_mixed_state, synthetic_mixed_lattice


@pytest.fixture(scope="module")
def mo(oracle):
    import mixed_oracle
    return mixed_oracle


def test_structure_constants(mo):
    f = mo.F_SU3
    assert np.abs(f + f.transpose(1, 0, 2)).max() < 1e-15
    assert np.abs(f + f.transpose(0, 2, 1)).max() < 1e-15
    h, q = 0.5, np.sqrt(3) / 2
    for (a, b, c), v in {(1, 2, 3): 1, (1, 4, 7): h, (1, 5, 6): -h, (2, 4, 6): h, (2, 5, 7): h, (3, 4, 5): h,
                         (3, 6, 7): -h, (4, 5, 8): q, (6, 7, 8): q}.items():
        assert abs(f[a - 1, b - 1, c - 1] - v) < 1e-15
    assert np.count_nonzero(np.abs(f) > 1e-12) == 54
    jac = (np.einsum("abd,dce->abce", f, f) + np.einsum("bcd,dae->abce", f, f) + np.einsum("cad,dbe->abce", f, f))
    assert np.abs(jac).max() < 1e-14


def test_fields_are_the_energy_gradient(mo):
    arr = synthetic_mixed_lattice((2, 2, 2), seed=1)
    o = mo.MixedOracle(arr)
    Y = random_mixed_state(arr, 2)
    H2, H3 = o.fields(Y, 0.0)
    H = np.concatenate([H2.ravel(), H3.ravel()])
    rng = np.random.default_rng(3)
    for i in rng.choice(Y.size, 40, replace=False):
        e = np.zeros_like(Y)
        e[i] = 1e-6
        g = (o.energy(Y + e) - o.energy(Y - e)) / 2e-6
        assert abs(g - H[i]) <= 1e-7 * max(1.0, abs(H[i])), (i, g, H[i])


def test_bonds_stored_at_both_ends():
    arr = synthetic_mixed_lattice((3, 2, 2), seed=4)
    n2, n3, z2, zm2, zm3 = arr["n2"], arr["n3"], arr["z2"], arr["zm2"], arr["zm3"]
    p2 = arr["part2"].reshape(n2, z2)
    J2 = arr["bil2"].reshape(n2, z2, 3, 3)
    for i in range(n2):
        for k in range(z2):
            j = p2[i, k]
            back = [m for m in range(z2) if p2[j, m] == i and np.allclose(J2[j, m], J2[i, k].T)]
            assert back, (i, k)
    mp2, mp3 = arr["mpart2"].reshape(n2, zm2), arr["mpart3"].reshape(n3, zm3)
    M2, M3 = arr["mix2"].reshape(n2, zm2, 3, 8), arr["mix3"].reshape(n3, zm3, 8, 3)
    for s in range(n3):
        for k in range(zm3):
            p = mp3[s, k]
            assert any(mp2[p, m] == s and np.allclose(M2[p, m], M3[s, k].T) for m in range(zm2))


def test_rk4_conserves_energy_and_lengths(mo):
    """The drifts are RK4 truncation: below 5e-9 at dt = 0.01 and 16x smaller (order 4) at dt = 0.005."""
    import fixed_methods as fm
    arr = synthetic_mixed_lattice((2, 2, 2), seed=5)
    o = mo.MixedOracle(arr)
    Y0 = random_mixed_state(arr, 6)
    n2 = arr["n2"]
    drifts = []
    for dt in (0.01, 0.005):
        n = int(round(1.0 / dt))
        _, st = fm.integrate(lambda y, t: o.rhs(y, t), Y0, 0.0, 1.0, dt, n, "rk4")
        Y = st[-1]
        assert np.abs(Y - Y0).max() > 1e-3          # it moved
        drifts.append((abs(o.energy(Y) - o.energy(Y0)) / abs(o.energy(Y0)),
                       np.abs(np.linalg.norm(Y[:3 * n2].reshape(-1, 3), axis=1) - 1).max(),
                       np.abs(np.linalg.norm(Y[3 * n2:].reshape(-1, 8), axis=1) - 1).max()))
    for coarse, fine in zip(*drifts):
        assert coarse <= 5e-9 and fine <= coarse / 10, drifts


def test_mixed_api_rejects_bad_input_without_a_gpu():
    from classical_mcmc_spin_b200 import mixed_gpu_api as mg
    arr = synthetic_mixed_lattice((2, 2, 2), seed=7)
    with pytest.raises(ValueError):
        mg.create_gpu_mixed_lattice_data(arr["n2"], 4, arr["na2"], arr["n3"], 8, arr["na3"], 6, 2, 8, 8,
                                         *([np.zeros(1)] * 17))
    with pytest.raises(ValueError):
        mg._method("rk45")
    with pytest.raises(ValueError):
        mg._method("no_such_method")
    assert mg._method("ssprk53") == mg.nat.CMD_SSPRK53
