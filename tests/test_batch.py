"""Cluster batches (tdp_batch_*) against the FP64 oracle, cluster by cluster.

Every cluster of a batch must give what the oracle gives for that cluster as
a system of its own.  Tolerances are those of the single-system parity tests:
  * plain (FP64) form: energy within 1e-9 |E| + 1e-11 sum |q_i q_j|/r_ij (the
    second term covers clusters whose total nearly cancels), forces and
    induced dipoles RMS relative 1e-8 (solve to 1e-11);
  * mixed form: energy within 1e-6 |E| + 3e-7 sqrt(sum (q_i q_j/r_ij)^2),
    forces and induced dipoles RMS relative 2e-5 (solve to 1e-9).
The oracle solves Mutual polarization to 1e-12."""
import numpy as np
import pytest

from oracle import oracle as O
from tholedipoleplugin_b200 import systems as S
from tholedipoleplugin_b200.batch import ClusterBatch

from .fixtures import ammonia, small_random_system, water4, zbisect, zonly
from .gpu_util import energy_rms_scale, energy_scale, rel_err, rel_rms

pytestmark = pytest.mark.gpu


def _mixed_clusters(polarization, seed=5):
    """Waters of ragged sizes (1 to 64 molecules) plus clusters with every
    axis type, ragged covalent lists and non-neutral charges."""
    rng = np.random.default_rng(seed)
    out = []
    for nw in (1, 2, 5, 13, 64, 9, 31):
        out.append(S.water_cluster(nw, rng))
    out.append(ammonia(polarization, S.NO_CUTOFF))
    out.append(ammonia(polarization, S.NO_CUTOFF, scaled=True))
    out.append(water4(polarization))
    out.append(zbisect())
    out.append(zonly())
    out.append(small_random_system(40, seed=31, method=S.NO_CUTOFF))
    out.append(small_random_system(23, seed=32, method=S.NO_CUTOFF))
    out.append(small_random_system(77, seed=33, method=S.NO_CUTOFF))
    return [c.copy(method=S.NO_CUTOFF, polarization=polarization) for c in out]


def _oracle(c, **kw):
    return O.compute(c.copy(target_eps=1e-12, max_iter=5000), "port", **kw)


def _check(batch, clusters, energies, forces, induced, precision, refs):
    for k, c in enumerate(clusters):
        sl = batch.cluster_slice(k)
        ref = refs[k]
        e, f, mu = energies[k], forces[sl], induced[sl]
        if precision == "double":
            c1 = energy_scale(c) if c.n > 1 else 0.0
            assert abs(e - ref.energy) < 1e-9 * abs(ref.energy) + 1e-11 * c1 + 1e-14, (k, e, ref.energy, c1)
            assert rel_rms(f, ref.forces) < 1e-8, k
            if np.any(ref.induced):
                assert rel_rms(mu, ref.induced) < 1e-8, k
        else:
            c2 = energy_rms_scale(c) if c.n > 1 else 0.0
            assert abs(e - ref.energy) < 1e-6 * abs(ref.energy) + 3e-7 * c2 + 1e-12, (k, e, ref.energy, c2)
            assert rel_rms(f, ref.forces) < 2e-5, (k, rel_rms(f, ref.forces))
            if np.any(ref.induced):
                assert rel_rms(mu, ref.induced) < 2e-5, k


@pytest.mark.parametrize("precision", ["double", "mixed"])
@pytest.mark.parametrize("polarization", [S.MUTUAL, S.DIRECT, S.EXTRAPOLATED])
def test_batch_matches_oracle(precision, polarization):
    clusters = _mixed_clusters(polarization)
    eps = 1e-11 if precision == "double" else 1e-9
    clusters = [c.copy(target_eps=eps, max_iter=2000) for c in clusters]
    refs = [_oracle(c) for c in clusters]
    with ClusterBatch(clusters, precision=precision) as b:
        e, f = b.compute()
        mu = b.inducedDipoles()
        it, ep = b.solverStats()
        tile = b.tile()
    _check(b, clusters, e, f, mu, precision, refs)
    assert tile["threads"] > 0 and tile["ctas"] > 0
    if polarization == S.MUTUAL:
        assert np.all(ep <= eps), ep


@pytest.mark.parametrize("precision", ["double", "mixed"])
def test_batch_dd_force_r4(precision):
    clusters = [c.copy(target_eps=1e-11, max_iter=2000) for c in _mixed_clusters(S.MUTUAL, seed=6)]
    refs = [_oracle(c, rinv4_mode=1) for c in clusters]
    with ClusterBatch(clusters, precision=precision, dd_force_r4=True) as b:
        e, f = b.compute()
        mu = b.inducedDipoles()
    _check(b, clusters, e, f, mu, precision, refs)


def test_batch_is_deterministic_and_reusable():
    """Replays of the captured launch give bitwise-identical results, and new
    positions are picked up on every call."""
    rng = np.random.default_rng(8)
    clusters = [S.water_cluster(int(s), rng, target_eps=1e-9, max_iter=500) for s in rng.integers(4, 65, 40)]
    with ClusterBatch(clusters, precision="mixed") as b:
        e1, f1 = b.compute()
        e2, f2 = b.compute()
        assert np.array_equal(e1, e2) and np.array_equal(f1, f2)
        moved = b.positions + rng.normal(scale=0.002, size=b.positions.shape)
        e3, f3 = b.compute(moved)
        ref = _oracle(clusters[3].copy(positions=moved[b.cluster_slice(3)]))
        assert rel_rms(f3[b.cluster_slice(3)], ref.forces) < 2e-5
        assert abs(e3[3] - ref.energy) < 1e-6 * abs(ref.energy) + 3e-7 * energy_rms_scale(clusters[3])


def test_batch_matches_single_system_path():
    """The batch and the single-system kernel agree on the same cluster (FP64 form)."""
    from tholedipoleplugin_b200.kernel import CudaCalcTholeDipoleForceKernel
    rng = np.random.default_rng(9)
    clusters = [S.water_cluster(nw, rng, target_eps=1e-11, max_iter=2000) for nw in (3, 17, 48)]
    with ClusterBatch(clusters, precision="double") as b:
        e, f = b.compute()
    for k, c in enumerate(clusters):
        with CudaCalcTholeDipoleForceKernel(c, precision="double") as kk:
            ek, fk = kk.execute(c.positions)
        assert rel_err(e[k], ek) < 1e-10
        assert rel_rms(f[b.cluster_slice(k)], fk) < 1e-9


def test_cluster_workload_sample_matches_oracle():
    """1024 clusters of 4-64 waters (the measured cluster workload) in one
    launch.  At the workload's 1e-6 target every cluster converges; solved to
    1e-9, a seeded sample of 48 clusters matches the oracle."""
    clusters = S.cluster_batch(1024, 4, 64, seed=3, target_eps=1e-6, max_iter=500)
    with ClusterBatch(clusters, precision="mixed") as b:
        e, f = b.compute()
        it, ep = b.solverStats()
    assert np.all(ep <= 1e-6) and np.all(it >= 1)
    assert np.all(np.isfinite(e)) and np.all(np.isfinite(f))
    tight = [c.copy(target_eps=1e-9) for c in clusters]
    with ClusterBatch(tight, precision="mixed") as b:
        e, f = b.compute()
        mu = b.inducedDipoles()
    sample = np.random.default_rng(0).choice(1024, 48, replace=False)
    for k in sample:
        c = clusters[k]
        ref = _oracle(c)
        sl = b.cluster_slice(k)
        assert abs(e[k] - ref.energy) < 1e-6 * abs(ref.energy) + 3e-7 * energy_rms_scale(c), k
        assert rel_rms(f[sl], ref.forces) < 2e-5, (k, rel_rms(f[sl], ref.forces))
        assert rel_rms(mu[sl], ref.induced) < 2e-5, k
