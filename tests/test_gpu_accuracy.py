"""The error bounds at the solver tolerances the timed workloads use
(tholedipoleplugin_b200/systems.py: BOX_SOLVER_EPS, CLUSTER_SOLVER_EPS):
energy within 1e-6 relative and forces within 2e-5 RMS relative of the
converged FP64 answer, for both precision forms -- on the 216-water box
against the oracle solved to 1e-12, on the 4,096-water box against the
compiled reference's golden, and per cluster on 48 seeded clusters of the
1024-cluster workload against the oracle."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from tholedipoleplugin_b200 import systems as S
from tholedipoleplugin_b200.batch import ClusterBatch
from tholedipoleplugin_b200.kernel import CudaCalcTholeDipoleForceKernel

from .gpu_util import rel_err, rel_rms

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("precision", ["mixed", "double"])
def test_water216_at_timed_tolerance(precision):
    s = S.config_small(target_eps=S.BOX_SOLVER_EPS)
    ref = O.compute(s.copy(target_eps=1e-12, max_iter=5000), "port")
    with CudaCalcTholeDipoleForceKernel(s, precision=precision) as k:
        e, f = k.execute(s.positions)
        mu = k.getInducedDipoles()
    assert rel_err(e, ref.energy) < 1e-6
    assert rel_rms(f, ref.forces) < 2e-5
    assert rel_rms(mu, ref.induced) < 2e-5


@pytest.mark.parametrize("precision", ["mixed", "double"])
def test_water12288_at_timed_tolerance(precision):
    g = np.load(os.path.join(GOLDEN, "water12288.npz"))
    s = S.config_medium(seed=1, target_eps=S.BOX_SOLVER_EPS)
    with CudaCalcTholeDipoleForceKernel(s, precision=precision) as k:
        e, f = k.execute(s.positions)
    assert rel_err(e, float(g["energy"])) < 1e-6
    assert rel_rms(f, g["forces"]) < 2e-5


@pytest.mark.parametrize("precision", ["mixed", "double"])
def test_clusters_at_timed_tolerance(precision):
    cl = S.cluster_batch(1024, 4, 64, seed=3, target_eps=S.CLUSTER_SOLVER_EPS, max_iter=500)
    sample = sorted(np.random.default_rng(0).choice(1024, 48, replace=False))
    clusters = [cl[k] for k in sample]
    with ClusterBatch(clusters, precision=precision) as b:
        e, f = b.compute()
        offs = b.offsets
    for c, cs in enumerate(clusters):
        ref = O.compute(cs.copy(target_eps=1e-12, max_iter=5000), "port")
        sl = slice(int(offs[c]), int(offs[c + 1]))
        assert rel_err(e[c], ref.energy) < 1e-6, (c, e[c], ref.energy)
        assert rel_rms(f[sl], ref.forces) < 2e-5
