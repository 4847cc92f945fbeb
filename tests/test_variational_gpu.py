"""Variational NoCutoff mode (TDP_FLAG_VARIATIONAL) on the GPU against the FP64
oracle (oracle/ewald.py, recip="none", alpha = 0).

The mode keeps the reference's fields and induced dipoles exactly (checked
against the default mode on the same inputs) and replaces its energy and
forces by the variational energy U_perm - 1/2 mu.E_M and its exact gradient.
Tolerances: plain form energy 1e-9, forces and dipoles 1e-8 (RMS relative);
mixed form energy 1e-6 |E| + 3e-7 sqrt(sum (q_i q_j / r_ij)^2) (the FP32
rounding of the pair terms adds in quadrature; a cluster's total energy is a
small residual of them), forces and dipoles 2e-5.
"""
import numpy as np
import pytest

from oracle import ewald as EW
from tholedipoleplugin_b200 import systems as S
from tholedipoleplugin_b200.kernel import CudaCalcTholeDipoleForceKernel

from .fixtures import reference_test_systems
from .gpu_util import energy_rms_scale, rel_err, rel_rms

pytestmark = pytest.mark.gpu


def cluster():
    return S.water_cluster(40, np.random.default_rng(4), target_eps=1e-12, max_iter=1000)


def run(s, precision, eps, variational=True):
    with CudaCalcTholeDipoleForceKernel(s.copy(target_eps=eps, max_iter=2000), precision=precision,
                                        variational=variational) as k:
        e, f = k.execute(s.positions)
        mu = k.getInducedDipoles()
    return e, f, mu


@pytest.mark.parametrize("polarization", [S.MUTUAL, S.DIRECT])
@pytest.mark.parametrize("precision,eps,e_tol,f_tol", [("double", 1e-11, 1e-9, 1e-8), ("mixed", 1e-9, 1e-6, 2e-5)])
def test_water_cluster_matches_oracle(precision, eps, e_tol, f_tol, polarization):
    s = cluster().copy(polarization=polarization)
    ref = EW.variational_nocutoff(s)
    e, f, mu = run(s, precision, eps)
    bound = e_tol * abs(ref.energy) + (3e-7 * energy_rms_scale(s) if precision == "mixed" else 0.0)
    assert abs(e - ref.energy) < bound, (e, ref.energy, bound)
    assert rel_rms(f, ref.forces) < f_tol
    assert rel_rms(mu, ref.induced) < f_tol


def test_same_dipoles_as_reference_semantics():
    s = cluster()
    _, _, mu_v = run(s, "double", 1e-11)
    _, _, mu_r = run(s, "double", 1e-11, variational=False)
    assert rel_rms(mu_v, mu_r) < 1e-9


@pytest.mark.parametrize("name", ["ammonia_mutual", "ammonia_scaled"])
def test_reference_test_systems(name):
    # The reference's NoCutoff ammonia systems (three-fold and Z-then-X frames).
    s = dict(reference_test_systems())[name].copy(target_eps=1e-12, max_iter=2000)
    ref = EW.variational_nocutoff(s)
    e, f, mu = run(s, "double", 1e-11)
    assert rel_err(e, ref.energy) < 1e-9
    assert rel_rms(f, ref.forces) < 1e-8
    assert rel_rms(mu, ref.induced) < 1e-8


def test_forces_are_gradient_of_gpu_energy():
    s = S.water_cluster(12, np.random.default_rng(2), target_eps=1e-13, max_iter=1000)
    with CudaCalcTholeDipoleForceKernel(s, precision="double", variational=True) as k:
        _, f0 = k.execute(s.positions)
        h = 1e-5
        scale = np.abs(f0).max()
        for i, c in [(0, 0), (0, 2), (1, 1), (2, 0), (20, 2), (35, 1)]:
            e = []
            for sg in (1.0, -1.0):
                p = s.positions.copy()
                p[i, c] += sg * h
                e.append(k.execute(p)[0])
            fd = -(e[0] - e[1]) / (2 * h)
            assert abs(fd - f0[i, c]) < 1e-7 * scale, (i, c, fd, f0[i, c])
