"""Ewald mode (TDP_FLAG_EWALD) on the GPU, through the C ABI, against the FP64
Ewald oracle (oracle/ewald.py; its pins are in tests/test_ewald_oracle.py).

The oracle's smooth-PME restatement uses the same alpha, grid, order-5
B-splines and influence function as the CUDA kernels, so the comparison
isolates the kernels' arithmetic from the PME discretisation.

Tolerances (written per test):
  * plain (FP64) form: energy relative 1e-9, forces, induced dipoles and the
    permanent field RMS relative 1e-8 (the solve runs to 1e-11);
  * mixed form (FP32 real space, FP32 B-splines and FFT, 64-bit fixed-point
    spreading, FP64 CG): energy relative 1e-6, forces RMS relative 2e-5,
    induced dipoles RMS relative 2e-5 -- the north-star accuracy targets.
"""
import math

import numpy as np
import pytest

from oracle import ewald as EW
from tholedipoleplugin_b200 import systems as S
from tholedipoleplugin_b200.kernel import CudaCalcTholeDipoleForceKernel

from .gpu_util import rel_err, rel_rms

pytestmark = pytest.mark.gpu

_CACHE = {}


def water216():
    return S.config_small(target_eps=1e-12, max_iter=500)


def oracle_pme(name, make):
    if name not in _CACHE:
        s = make()
        alpha, grid = EW.pme_parameters(s.cutoff, s.ewald_tolerance, s.box)
        ew = EW.Ewald(s, alpha, recip="pme", grid=grid)
        _CACHE[name] = (ew, ew.evaluate(), alpha, grid)
    return _CACHE[name]


def run(s, precision, eps, **kw):
    with CudaCalcTholeDipoleForceKernel(s.copy(target_eps=eps, max_iter=2000), precision=precision, ewald=True,
                                        **kw) as k:
        e, f = k.execute(s.positions)
        mu = k.getInducedDipoles()
        params = k.getPMEParameters()
        stats = k.solverStats()
    return e, f, mu, params, stats


def test_pme_parameters_match_oracle():
    _, _, alpha, grid = oracle_pme("w216", water216)
    _, _, _, params, _ = run(water216(), "double", 1e-11)
    assert abs(params[0] - alpha) < 1e-14 * alpha
    assert tuple(params[1:]) == tuple(grid) == (30, 30, 30)


@pytest.mark.parametrize("precision,eps,e_tol,f_tol,mu_tol", [
    ("double", 1e-11, 1e-9, 1e-8, 1e-8),
    ("mixed", 1e-9, 1e-6, 2e-5, 2e-5),
])
def test_water216_matches_oracle(precision, eps, e_tol, f_tol, mu_tol):
    _, ref, _, _ = oracle_pme("w216", water216)
    e, f, mu, _, stats = run(water216(), precision, eps)
    assert stats["converged"]
    assert rel_err(e, ref.energy) < e_tol, (e, ref.energy)
    assert rel_rms(f, ref.forces) < f_tol
    assert rel_rms(mu, ref.induced) < mu_tol


@pytest.mark.parametrize("precision,tol", [("double", 1e-8), ("mixed", 2e-5)])
def test_permanent_field(precision, tol):
    # A Mutual solve capped at zero iterations returns its starting point
    # mu = alpha E_M, which exposes the permanent field (real space + PME +
    # self) atom by atom.
    ew, _, _, _ = oracle_pme("w216", water216)
    s = water216().copy(max_iter=0)
    with CudaCalcTholeDipoleForceKernel(s, precision=precision, ewald=True) as k:
        mu = k.getInducedDipoles(s.positions)
    E = ew.fixed_field()
    assert rel_rms(mu, E * s.polarizabilities[:, None]) < tol


def test_extrapolated_rejected():
    from tholedipoleplugin_b200._capi import TdpError
    with pytest.raises(TdpError, match="Mutual or Direct polarization"):
        CudaCalcTholeDipoleForceKernel(water216().copy(polarization=S.EXTRAPOLATED), ewald=True)


@pytest.mark.parametrize("precision,e_tol,f_tol", [("double", 1e-9, 1e-8), ("mixed", 1e-6, 2e-5)])
def test_direct_water216_matches_oracle(precision, e_tol, f_tol):
    # Direct polarization: mu = alpha E_M, energy U_perm - 1/2 mu.E_M (the
    # Mutual functional without the induced-induced term), forces its gradient.
    _, ref, _, _ = oracle_pme("w216_direct", lambda: water216().copy(polarization=S.DIRECT))
    e, f, mu, _, stats = run(water216().copy(polarization=S.DIRECT), precision, 1e-11)
    assert stats["iterations"] == 0
    assert rel_rms(mu, ref.induced) < f_tol
    assert rel_err(e, ref.energy) < e_tol, (e, ref.energy)
    assert rel_rms(f, ref.forces) < f_tol


def test_direct_forces_are_gradient_of_gpu_energy():
    s = S.water_box(5, 1.5525, seed=9, cutoff=0.7, polarization=S.DIRECT)
    with CudaCalcTholeDipoleForceKernel(s, precision="double", ewald=True) as k:
        _, f0 = k.execute(s.positions)
        h = 1e-5
        scale = np.abs(f0).max()
        for i, c in [(0, 0), (0, 2), (1, 1), (2, 0), (100, 2), (374, 1)]:
            e = []
            for sg in (1.0, -1.0):
                p = s.positions.copy()
                p[i, c] += sg * h
                e.append(k.execute(p)[0])
            fd = -(e[0] - e[1]) / (2 * h)
            assert abs(fd - f0[i, c]) < 1e-7 * scale, (i, c, fd, f0[i, c])


def test_forces_are_gradient_of_gpu_energy():
    # 125 waters in a 1.553 nm box (the smallest water box whose cutoff, 0.7 nm,
    # keeps the Thole damping below 1e-12 at the cutoff).
    s = S.water_box(5, 1.5525, seed=9, cutoff=0.7, target_eps=1e-13, max_iter=1000)
    with CudaCalcTholeDipoleForceKernel(s, precision="double", ewald=True) as k:
        _, f0 = k.execute(s.positions)
        h = 1e-5
        scale = np.abs(f0).max()
        for i, c in [(0, 0), (0, 2), (1, 1), (2, 0), (100, 2), (374, 1)]:
            e = []
            for sg in (1.0, -1.0):
                p = s.positions.copy()
                p[i, c] += sg * h
                e.append(k.execute(p)[0])
            fd = -(e[0] - e[1]) / (2 * h)
            assert abs(fd - f0[i, c]) < 1e-7 * scale, (i, c, fd, f0[i, c])


def _plasma(q0, cutoff):
    pos = np.array([[0.0, 0.0, 0.0], [0.3, 0.4, 0.0]])
    n = 2
    return S.TholeSystem(positions=pos, charges=np.array([q0, 1.0]), dipoles=np.zeros((n, 3)),
                         polarizabilities=np.full(n, 0.001), tholes=np.full(n, 0.39),
                         axis=np.array([[S.NOAXISTYPE, 0, 0, 0]] * n, dtype=np.int32),
                         cov12=[[], []], cov13=[[], []], method=S.PME, box=np.array([2.0, 2.0, 2.0]),
                         cutoff=cutoff, target_eps=1e-10, max_iter=500)


@pytest.mark.parametrize("precision", ["double", "mixed"])
@pytest.mark.parametrize("q0", [1.0, 2.0])
def test_neutralizing_plasma(precision, q0):
    # TestReferenceTholeDipoleForce.cpp:761-801 under a true Ewald sum: the
    # energy of a net-charged pair does not depend on alpha (cutoff 1.0 vs 0.7).
    e = []
    for cutoff in (1.0, 0.7):
        s = _plasma(q0, cutoff)
        with CudaCalcTholeDipoleForceKernel(s, precision=precision, ewald=True) as k:
            e.append(k.execute(s.positions)[0])
    assert abs(e[0] - e[1]) < 1e-4 * abs(e[0])
    ref = EW.ewald(_plasma(q0, 1.0), recip="direct")
    assert rel_err(e[0], ref.energy) < 1e-4


def test_mixed_matches_plain_at_12k():
    # 4,096 waters: many folded tile pairs and the full neighbour-list path.
    s = S.config_medium(target_eps=1e-10, max_iter=500)
    ep, fp, mup, _, _ = run(s, "double", 1e-11)
    em, fm, mum, _, _ = run(s, "mixed", 1e-9)
    assert rel_err(em, ep) < 1e-6
    assert rel_rms(fm, fp) < 2e-5
    assert rel_rms(mum, mup) < 2e-5


def test_translation_invariance():
    # Shifting every atom by a lattice-incommensurate vector moves atoms across
    # the box faces and the PME grid; energies agree to the PME interpolation
    # error of the tolerance-1e-4 grid.
    s = water216()
    e0 = run(s, "double", 1e-11)[0]
    s2 = s.copy(positions=s.positions + np.array([0.37, -1.21, 2.9]))
    e1 = run(s2, "double", 1e-11)[0]
    assert rel_err(e1, e0) < 1e-4


def test_mixed_matches_plain_at_tight_tolerance():
    # Ewald tolerance 1e-6: alpha * cutoff = 3.6, deeper into the tail of the
    # FP32 erfc approximation of the mixed real-space kernels.
    s = water216().copy(ewald_tolerance=1e-6)
    ep, fp, mup, params, _ = run(s, "double", 1e-11)
    em, fm, mum, _, _ = run(s, "mixed", 1e-9)
    assert params[1] > 30  # finer grid than at 1e-4
    assert rel_err(em, ep) < 1e-6
    assert rel_rms(fm, fp) < 2e-5
    assert rel_rms(mum, mup) < 2e-5


@pytest.mark.parametrize("precision,te,tf", [("double", 1e-9, 1e-8), ("mixed", 5e-6, 2e-5)])
def test_fused_start_matches_separate_walks(precision, te, tf, monkeypatch):
    # A warm-started Ewald solve starts with one permanent-field pass over the
    # dipole records m + mu0 (real space with the partners' M/I split,
    # reciprocal space and self term of the sum), giving E + T mu0; along a
    # trajectory it must match the separate permanent-field pass and matvec.
    s = water216().copy(target_eps=1e-11 if precision == "double" else 1e-9, max_iter=2000)
    v = np.random.default_rng(12).normal(size=s.positions.shape) * 3e-4
    traj = [s.positions + k * v for k in range(5)]
    out = {}
    for fused in ("1", "0"):
        monkeypatch.setenv("TDP_FUSED_START", fused)
        with CudaCalcTholeDipoleForceKernel(s, precision=precision, warm_start=True, ewald=True) as k:
            k.enableTiming(True)
            res = []
            for p in traj:
                res.append(k.execute(p))
                assert k.solverStats()["converged"]
            out[fused] = (res, int(k.stageTimes()[10]))
    assert out["1"][1] == 1 and out["0"][1] == 0
    for (e1, f1), (e0, f0) in zip(out["1"][0], out["0"][0]):
        assert rel_err(e1, e0) < te and rel_rms(f1, f0) < tf
    ref = EW.ewald(s.copy(positions=traj[-1]))
    assert rel_err(out["1"][0][-1][0], ref.energy) < (1e-9 if precision == "double" else 1e-6)
