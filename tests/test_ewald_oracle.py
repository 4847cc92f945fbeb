"""Pins of the FP64 Ewald oracle (oracle/ewald.py), CPU only.

The reference has no Ewald sum, so the oracle of the library's Ewald mode is
pinned by properties instead of golden vectors:
  * independence of the splitting parameter alpha (real space converged),
  * forces equal to minus the central-difference gradient of the energy
    (dipoles re-solved at every displaced geometry, torque mapping included),
  * stationarity of the energy in the induced dipoles,
  * the large-box limit: fields and induced dipoles of the compiled
    reference's NoCutoff code, and the vacuum energy of the same sums,
  * the neutralising-plasma test of the reference
    (TestReferenceTholeDipoleForce.cpp:761-801) under a true Ewald sum,
  * the smooth-PME restatement converging to the explicit reciprocal sum.
"""
import math

import numpy as np
import pytest

from oracle import ewald as EW
from oracle import oracle as O
from tholedipoleplugin_b200 import systems as S


def rel(x, y):
    return float(np.sqrt(((x - y) ** 2).sum() / (y ** 2).sum()))


@pytest.fixture(scope="module")
def tiny_box():
    # 8 waters in a 0.7 nm box: cutoff 0.34 nm.
    return S.water_box(2, 0.7, seed=3, cutoff=0.34)


def test_bspline_partition_of_unity():
    w = np.linspace(0.0, 0.999, 37)
    th, d1, d2 = EW.bspline(w)
    assert np.allclose(th.sum(-1), 1.0, atol=1e-14)
    assert np.allclose(d1.sum(-1), 0.0, atol=1e-14)
    assert np.allclose(d2.sum(-1), 0.0, atol=1e-13)
    # M_5 at the integers: 1/24, 11/24, 11/24, 1/24.
    th0 = EW.bspline(np.array([0.0]))[0][0]
    assert np.allclose(th0[1:], [1 / 24, 11 / 24, 11 / 24, 1 / 24], atol=1e-15)
    assert EW.smooth_size(29) == 30 and EW.smooth_size(143) == 144 and EW.smooth_size(11) == 12


def test_alpha_independence(tiny_box):
    # erfc(alpha * cutoff) < 1e-14 for both alphas; reciprocal sums to exp(-42).
    a = EW.Ewald(tiny_box, 18.0, recip="direct").evaluate()
    b = EW.Ewald(tiny_box, 21.0, recip="direct").evaluate()
    assert abs(a.energy - b.energy) <= 1e-12 * abs(a.energy)
    assert rel(a.fixed_field, b.fixed_field) < 1e-12
    assert rel(a.induced, b.induced) < 1e-12
    assert rel(a.forces, b.forces) < 1e-12


def test_forces_are_minus_energy_gradient(tiny_box):
    alpha = 9.0
    r0 = EW.Ewald(tiny_box, alpha, recip="direct").evaluate()
    h = 2e-5
    scale = np.abs(r0.forces).max()
    # O (frame centre), both H (frame axis atoms) and atoms of another water.
    for i, c in [(0, 0), (0, 2), (1, 0), (2, 1), (4, 2), (9, 0)]:
        e = []
        for sg in (1.0, -1.0):
            s2 = tiny_box.copy()
            s2.positions[i, c] += sg * h
            e.append(EW.Ewald(s2, alpha, recip="direct").evaluate().energy)
        fd = -(e[0] - e[1]) / (2 * h)
        assert abs(fd - r0.forces[i, c]) < 2e-8 * scale, (i, c, fd, r0.forces[i, c])


def _cluster_in_big_box():
    rng = np.random.default_rng(5)
    c = S.water_cluster(4, rng, target_eps=1e-12, max_iter=5000)
    L = 30.0
    c.positions = c.positions - c.positions.mean(0) + L / 2
    return c, c.copy(method=S.PME, box=np.array([L, L, L]), cutoff=14.9)


def test_large_box_limit_matches_reference_nocutoff():
    cluster, boxed = _cluster_in_big_box()
    backend = "reference" if O.reference_available() else "port"
    ew = EW.Ewald(boxed, 0.4, recip="direct")
    r = ew.evaluate()
    # Tin-foil periodic images of a neutral 12-atom cluster in a 30 nm box perturb the
    # field by ~4 pi M / (3 V): relative 1e-5 here.
    assert rel(r.fixed_field, O.fixed_field(cluster, backend)) < 2e-5
    assert rel(r.induced, O.induced_dipoles(cluster, backend)[0]) < 2e-5
    # Charges only: the reference's pair energy is the plain Coulomb sum.
    q_only = boxed.copy(dipoles=np.zeros((boxed.n, 3)), polarizabilities=np.zeros(boxed.n))
    e_q = EW.Ewald(q_only, 0.4, recip="direct").evaluate().energy
    e_ref = O.compute(cluster.copy(dipoles=np.zeros((boxed.n, 3)), polarizabilities=np.zeros(boxed.n)),
                      backend).energy
    assert abs(e_q - e_ref) < 1e-4 * abs(e_ref)
    # Dipole terms: the vacuum sum of the same bare pair energies (the reference's
    # own pair energy follows its quasi-internal-frame convention, not this one).
    z = np.zeros(boxed.n)
    e_vac, _, _ = EW.pair_energy_force(ew.d, tuple(ew.M * k for k in ew.bare), ew.q, ew.lab, ew.q, ew.lab)
    perm = EW.Ewald(boxed.copy(polarizabilities=np.zeros(boxed.n)), 0.4, recip="direct").evaluate().energy
    assert abs(perm - 0.5 * e_vac) < 2e-4 * abs(perm)
    # Polarization energy -1/2 mu.E_M with the reference's own fields and dipoles.
    mu_ref = O.induced_dipoles(cluster, backend)[0]
    E_ref = O.fixed_field(cluster, backend)
    assert abs((r.energy - perm) - (-0.5 * (mu_ref * E_ref).sum())) < 1e-4 * abs(r.energy - perm)


def test_energy_stationary_in_induced_dipoles():
    _, boxed = _cluster_in_big_box()
    ew = EW.Ewald(boxed, 0.4, recip="direct")
    mu, E = ew.solve()
    u0 = ew.evaluate(mu, E).energy
    d = np.random.default_rng(1).standard_normal(mu.shape) * 1e-4 * np.abs(mu).max()
    d1 = ew.evaluate(mu + d, E).energy - u0
    d2 = ew.evaluate(mu + 0.5 * d, E).energy - u0
    assert d1 > 0 and abs(d1 / d2 - 4.0) < 1e-3


def _plasma_system(q0):
    # TestReferenceTholeDipoleForce.cpp:761-801: two NoAxisType particles, net charge,
    # default 2 nm box.
    pos = np.array([[0.0, 0.0, 0.0], [0.3, 0.4, 0.0]])
    n = 2
    return S.TholeSystem(positions=pos, charges=np.array([q0, 1.0]), dipoles=np.zeros((n, 3)),
                         polarizabilities=np.full(n, 0.001), tholes=np.full(n, 0.39),
                         axis=np.array([[S.NOAXISTYPE, 0, 0, 0]] * n, dtype=np.int32),
                         cov12=[[], []], cov13=[[], []], method=S.PME, box=np.array([2.0, 2.0, 2.0]),
                         cutoff=1.0, target_eps=1e-10, max_iter=500)


@pytest.mark.parametrize("q0", [1.0, 2.0])
def test_neutralizing_plasma(q0):
    s = _plasma_system(q0)
    e = []
    for cutoff in (1.0, 0.7):
        sc = s.copy(cutoff=cutoff)
        alpha, _ = EW.pme_parameters(cutoff, 1e-4, sc.box)
        e.append(EW.Ewald(sc, alpha, recip="direct").evaluate().energy)
    assert abs(e[0] - e[1]) < 1e-4 * abs(e[0])
    # Without the plasma term the two differ by pi Q^2/(2V) (1/alpha_2^2 - 1/alpha_1^2).
    a1 = EW.pme_parameters(1.0, 1e-4, s.box)[0]
    a2 = EW.pme_parameters(0.7, 1e-4, s.box)[0]
    Q = q0 + 1.0
    assert math.pi * Q * Q / (2 * 8.0) * abs(1 / a2 ** 2 - 1 / a1 ** 2) > 100 * abs(e[0] - e[1])


def test_pme_restatement_converges_to_direct_sum():
    s = S.config_small()
    alpha, grid = EW.pme_parameters(s.cutoff, s.ewald_tolerance, s.box)
    assert grid == (30, 30, 30)
    direct = EW.Ewald(s, alpha, recip="direct")
    pme = EW.Ewald(s, alpha, recip="pme", grid=grid)
    fine = EW.Ewald(s, alpha, recip="pme", grid=tuple(2 * g for g in grid))
    E_d = direct.fixed_field()
    e1 = rel(pme.fixed_field(), E_d)
    e2 = rel(fine.fixed_field(), E_d)
    # Order-5 B-splines: the grid error falls by ~2^5 when the spacing halves.
    assert e1 < 1e-4 and e2 < e1 / 16.0


def test_variational_nocutoff_oracle():
    # recip="none", alpha = 0: the fields and induced dipoles are exactly the
    # reference's NoCutoff ones, and the forces are the energy's gradient.
    from tests.fixtures import reference_test_systems
    backend = "reference" if O.reference_available() else "port"
    s = dict(reference_test_systems())["ammonia_mutual"].copy(target_eps=1e-13, max_iter=5000)
    r = EW.variational_nocutoff(s)
    assert rel(r.fixed_field, O.fixed_field(s, backend)) < 1e-13
    assert rel(r.induced, O.induced_dipoles(s, backend)[0]) < 1e-9
    h = 1e-6
    scale = np.abs(r.forces).max()
    for i in range(s.n):
        for c in range(3):
            e = []
            for sg in (1.0, -1.0):
                s2 = s.copy()
                s2.positions[i, c] += sg * h
                e.append(EW.variational_nocutoff(s2).energy)
            assert abs(-(e[0] - e[1]) / (2 * h) - r.forces[i, c]) < 1e-8 * scale


def test_direct_forces_are_minus_energy_gradient(tiny_box):
    # Direct polarization: mu = alpha E_M at every position, energy U_perm - 1/2 mu.E_M.
    s = tiny_box.copy(polarization=S.DIRECT)
    alpha = 9.0
    r0 = EW.Ewald(s, alpha, recip="direct").evaluate()
    assert rel(r0.induced, r0.fixed_field * s.polarizabilities[:, None]) < 1e-15
    # The functional at its stationary point is U_perm - 1/2 mu.E_M.
    perm = EW.Ewald(s.copy(polarizabilities=np.zeros(s.n)), alpha, recip="direct").evaluate().energy
    assert abs((r0.energy - perm) - (-0.5 * (r0.induced * r0.fixed_field).sum())) < 1e-12 * abs(r0.energy)
    h = 2e-5
    scale = np.abs(r0.forces).max()
    for i, c in [(0, 0), (0, 2), (1, 0), (2, 1), (4, 2), (9, 0)]:
        e = []
        for sg in (1.0, -1.0):
            s2 = s.copy()
            s2.positions[i, c] += sg * h
            e.append(EW.Ewald(s2, alpha, recip="direct").evaluate().energy)
        fd = -(e[0] - e[1]) / (2 * h)
        assert abs(fd - r0.forces[i, c]) < 2e-8 * scale, (i, c, fd, r0.forces[i, c])


def test_direct_energy_stationary_and_alpha_independent(tiny_box):
    s = tiny_box.copy(polarization=S.DIRECT)
    a = EW.Ewald(s, 18.0, recip="direct")
    b = EW.Ewald(s, 21.0, recip="direct").evaluate()
    ra = a.evaluate()
    assert abs(ra.energy - b.energy) <= 1e-12 * abs(ra.energy)
    assert rel(ra.forces, b.forces) < 1e-12
    u0 = ra.energy
    d = np.random.default_rng(2).standard_normal(ra.induced.shape) * 1e-4 * np.abs(ra.induced).max()
    d1 = a.evaluate(ra.induced + d, ra.fixed_field).energy - u0
    d2 = a.evaluate(ra.induced + 0.5 * d, ra.fixed_field).energy - u0
    assert d1 > 0 and abs(d1 / d2 - 4.0) < 1e-3
