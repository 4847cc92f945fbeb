"""GPU kernels (through the C ABI) against the FP64 oracle on the same inputs.

Tolerances:
  * plain (FP64) form: energy relative 1e-9, forces and induced dipoles RMS
    relative 1e-8 (rounding-level agreement; the solve runs to 1e-11);
  * mixed form: energy within 1e-6 |E| + 3e-7 sqrt(sum (q_i q_j/r_ij)^2) (the
    second term is the FP32 rounding of the pair terms, adding in quadrature;
    it only matters where the total nearly cancels) and RMS relative
    force error 2e-5 (the accuracy targets for the FP32 path), induced
    dipoles RMS relative 2e-5;
  * Jacobi solver: the same iteration count as the reference loop.
The oracle solves Mutual polarization to 1e-12 so that its own convergence
error is far below these tolerances."""
import numpy as np
import pytest

from oracle import oracle as O
from tholedipoleplugin_b200 import systems as S
from tholedipoleplugin_b200.kernel import CudaCalcTholeDipoleForceKernel

from .fixtures import reference_test_systems, small_random_system, sparse_clumps
from .gpu_util import energy_rms_scale, rel_err, rel_rms

pytestmark = pytest.mark.gpu


def _systems():
    out = dict(reference_test_systems())
    out["random_nocutoff"] = small_random_system(70, seed=11, method=S.NO_CUTOFF)
    out["random_pme"] = small_random_system(97, seed=12, method=S.PME)
    out["random_zonly_no_x"] = small_random_system(50, seed=13, method=S.NO_CUTOFF, zonly_without_x=True)
    out["random_direct"] = small_random_system(65, seed=14, method=S.PME, polarization=S.DIRECT)
    out["random_extrap"] = small_random_system(66, seed=15, method=S.PME, polarization=S.EXTRAPOLATED)
    out["water216"] = S.config_small()
    out["water_cluster"] = S.water_cluster(40, np.random.default_rng(4))
    out["sparse_clumps"] = sparse_clumps()
    return out


SYSTEMS = _systems()
_ORACLE = {}


def tight(s):
    return s.copy(target_eps=1e-12, max_iter=5000)


def oracle_result(name):
    if name not in _ORACLE:
        _ORACLE[name] = O.compute(tight(SYSTEMS[name]), "port")
    return _ORACLE[name]


@pytest.mark.parametrize("name", sorted(SYSTEMS))
def test_plain_matches_oracle(name):
    s = SYSTEMS[name]
    ref = oracle_result(name)
    with CudaCalcTholeDipoleForceKernel(s.copy(target_eps=1e-11, max_iter=2000), precision="double") as k:
        e, f = k.execute(s.positions)
        mu = k.getInducedDipoles()
        lab = k.getLabFramePermanentDipoles()
    assert rel_err(e, ref.energy) < 1e-9, (e, ref.energy)
    assert rel_rms(f, ref.forces) < 1e-8
    assert rel_rms(mu, ref.induced) < 1e-8
    assert rel_rms(lab, ref.lab) < 1e-12


@pytest.mark.parametrize("name", sorted(SYSTEMS))
def test_mixed_matches_oracle(name):
    s = SYSTEMS[name]
    ref = oracle_result(name)
    with CudaCalcTholeDipoleForceKernel(s.copy(target_eps=1e-9, max_iter=2000), precision="mixed") as k:
        e, f = k.execute(s.positions)
        mu = k.getInducedDipoles()
    # Energy: 1e-6 of |E| plus the FP32 rounding of the pair terms, which adds
    # in quadrature (~6e-8 per term relative): 3e-7 * sqrt(sum (q_i q_j/r_ij)^2).
    # The second term matters only where the total nearly cancels (randomly
    # oriented clusters, sparse boxes, random non-neutral charges).
    c2 = energy_rms_scale(s)
    assert abs(e - ref.energy) < 1e-6 * abs(ref.energy) + 3e-7 * c2, (e, ref.energy, c2)
    assert rel_rms(f, ref.forces) < 2e-5
    if s.polarization != S.DIRECT or np.abs(ref.induced).max() > 0:
        assert rel_rms(mu, ref.induced) < 2e-5


@pytest.mark.parametrize("name", ["ammonia_mutual", "water4_pme", "triclinic8", "water216", "random_pme"])
def test_jacobi_matches_reference_loop(name):
    s = SYSTEMS[name]
    ref = O.compute(s, "port")
    with CudaCalcTholeDipoleForceKernel(s, precision="double", solver="jacobi") as k:
        e, f = k.execute(s.positions)
        st = k.solverStats()
    assert st["iterations"] == ref.iterations
    assert st["converged"] == ref.converged
    assert rel_err(st["epsilon"], ref.epsilon) < 1e-6
    assert rel_err(e, ref.energy) < 1e-10
    assert rel_rms(f, ref.forces) < 1e-9


@pytest.mark.parametrize("precision", ["double", "mixed"])
def test_forces_are_added(precision):
    s = SYSTEMS["water4_pme"]
    with CudaCalcTholeDipoleForceKernel(s, precision=precision) as k:
        base = np.full((s.n, 3), 3.25)
        e, f = k.execute(s.positions, forces=base.copy())
        e2, f2 = k.execute(s.positions)
    assert np.allclose(f - 3.25, f2, rtol=0, atol=1e-12)
    assert e == e2


@pytest.mark.parametrize("name", ["ammonia_mutual", "water216", "random_pme", "random_extrap", "water_cluster"])
@pytest.mark.parametrize("precision", ["double", "mixed"])
def test_queries_match_oracle(precision, name):
    # Potential on a grid spanning the system (minimum image for PME), the 13
    # multipole moments and the total dipoles (RTDF.cpp:1157-1372).
    s = SYSTEMS[name]
    lo, hi = s.positions.min(0) - 0.3, s.positions.max(0) + 0.3
    grid = np.random.default_rng(3).uniform(lo, hi, size=(33, 3))
    ts = tight(s)
    with CudaCalcTholeDipoleForceKernel(s.copy(target_eps=1e-11 if precision == "double" else 1e-9,
                                                max_iter=2000), precision=precision) as k:
        pot = k.getElectrostaticPotential(grid, s.positions)
        mom = k.getSystemMultipoleMoments(s.masses, s.positions)
        tot = k.getTotalDipoles(s.positions)
    # Dipoles as in the induced-dipole parity checks (the solve stops at 1e-11,
    # which leaves ~1e-9 relative in a cluster's dipoles); potential and
    # moments sum over many sites and carry less of it.
    tol = 1e-9 if precision == "double" else 2e-5
    assert rel_rms(pot, O.potential(ts, grid, "port")) < tol
    assert rel_rms(mom, O.moments(ts, "port")) < tol
    assert rel_rms(tot, O.total_dipoles(ts, "port")) < (1e-8 if precision == "double" else 2e-5)


def test_rinv4_power_flag():
    s = SYSTEMS["water4_pme"]
    ref = O.compute(tight(s), "port", rinv4_mode=O.RINV4_POWER)
    with CudaCalcTholeDipoleForceKernel(s.copy(target_eps=1e-11), precision="double", dd_force_r4=True) as k:
        e, f = k.execute(s.positions)
    assert rel_err(e, ref.energy) < 1e-9
    assert rel_rms(f, ref.forces) < 1e-8


@pytest.mark.parametrize("precision", ["double", "mixed"])
def test_warm_start_predictor(precision):
    # A smooth trajectory (every atom moving at a constant velocity): with
    # TDP_FLAG_WARM_START the solve starts from mu(n-1) on the second call and
    # from the polynomial through the last (up to 4) solutions after that.
    # The converged dipoles are the
    # cold-start ones to the solver tolerance, in fewer iterations.  A NoCutoff
    # cluster keeps the dipoles smooth in the positions (in a minimum-image box
    # a pair crossing half a box edge switches images discontinuously).
    s = S.water_cluster(40, np.random.default_rng(4)).copy(target_eps=1e-8, max_iter=500)
    v = np.random.default_rng(21).standard_normal(s.positions.shape) * 1e-3   # nm per call
    warm_it, cold_it = [], []
    with CudaCalcTholeDipoleForceKernel(s, precision=precision, warm_start=True) as kw, \
            CudaCalcTholeDipoleForceKernel(s, precision=precision) as kc:
        for step in range(6):
            p = s.positions + step * v
            ew, fw = kw.execute(p)
            ec, fc = kc.execute(p)
            warm_it.append(kw.solverStats()["iterations"])
            cold_it.append(kc.solverStats()["iterations"])
            assert kw.solverStats()["converged"]
            # (No dipole query on kw here: a query at the same positions is a
            # call of its own and would become the predictor's last point.)
            assert rel_rms(fw, fc) < 1e-5
            # The pair energy is first order in the dipoles, and the two solves
            # stop at different points inside the 1e-8 tolerance; the mixed
            # form adds the FP32 rounding of its pair sums on a small total
            # (about 1.04 in the reference's Coulomb-prefactor-1 units).
            assert rel_err(ew, ec) < (1e-6 if precision == "double" else 1e-5)
    # Calls 3.. start from the extrapolated guess: fewer iterations than from
    # the constant guess of call 2, which needs fewer than a cold start.
    assert warm_it[1] < cold_it[1], (warm_it, cold_it)
    assert max(warm_it[2:]) < warm_it[1], (warm_it, cold_it)


@pytest.mark.parametrize("precision", ["double", "mixed"])
def test_predictor_orders(precision, monkeypatch):
    # Along a smooth trajectory (a cluster on a curved path), predictors
    # through 1, 2, 3 and 4 past solutions all converge to the cold-start
    # dipoles; from the fifth call on, the extrapolating ones need no more CG
    # iterations than the constant guess, the quadratic and cubic fewer.
    s = S.water_cluster(40, np.random.default_rng(4)).copy(target_eps=1e-9, max_iter=500)
    rng = np.random.default_rng(8)
    v = rng.standard_normal(s.positions.shape) * 1e-3
    a = rng.standard_normal(s.positions.shape) * 2e-4
    traj = [s.positions + k * v + 0.5 * k * k * a for k in range(8)]
    with CudaCalcTholeDipoleForceKernel(s, precision=precision) as kc:
        cold = []
        for p in traj:
            kc.execute(p)
            cold.append(kc.getInducedDipoles())
    its = {}
    for order in (1, 2, 3, 4):
        monkeypatch.setenv("TDP_PREDICTOR", str(order))
        with CudaCalcTholeDipoleForceKernel(s, precision=precision, warm_start=True) as kw:
            its[order] = []
            for k, p in enumerate(traj):
                kw.execute(p)
                st = kw.solverStats()
                assert st["converged"]
                its[order].append(st["iterations"])
                if k == len(traj) - 1:
                    # Two solves that each stop inside the tolerance.
                    assert rel_rms(kw.getInducedDipoles(), cold[k]) < 1e-5
    late = {o: sum(its[o][4:]) for o in its}
    assert late[3] < late[1] and late[4] < late[1], its
    assert late[2] <= late[1], its


@pytest.mark.parametrize("precision", ["double", "mixed"])
@pytest.mark.parametrize("method", [S.PME, S.NO_CUTOFF])
def test_fused_warm_start_matches_separate_walks(precision, method, monkeypatch):
    """A warm-started solve starts with one walk over the operand m + mu0
    (E + T mu0 in one pass; covalent partners split into their M and I
    scales).  Along a short trajectory it must give the results of the
    separate permanent-field walk and starting matvec (TDP_FUSED_START=0) to
    the solver tolerance, and the adjoint after such a solve must match a
    cold one."""
    base = S.water_box(5, 1.6 if method == S.PME else 1.55, seed=77, cutoff=0.7, method=method)
    s = base.copy(target_eps=1e-11 if precision == "double" else 1e-9, max_iter=2000)
    rng = np.random.default_rng(3)
    traj = [s.positions + 0.002 * k * rng.normal(size=s.positions.shape) for k in range(4)]
    out = {}
    for fused in ("1", "0"):
        monkeypatch.setenv("TDP_FUSED_START", fused)
        with CudaCalcTholeDipoleForceKernel(s, precision=precision, warm_start=True) as k:
            res = [k.execute(p) for p in traj]
            out[fused] = (res, k.getInducedDipoles(), k.adjoint(np.ones((s.n, 3)), 0.5))
    # Mixed form: two FP32 evaluations whose solves start from differently
    # rounded fields, on a small total (4.4 in Coulomb-prefactor-1 units).
    te, tf = (1e-9, 1e-8) if precision == "double" else (5e-6, 2e-5)
    for (e1, f1), (e0, f0) in zip(out["1"][0], out["0"][0]):
        assert rel_err(e1, e0) < te and rel_rms(f1, f0) < tf
    assert rel_rms(out["1"][1], out["0"][1]) < tf
    g1, g0 = out["1"][2], out["0"][2]
    for c in range(6):
        assert np.abs(g1[:, c] - g0[:, c]).max() <= (1e-7 if precision == "double" else 1e-4) * np.abs(g0[:, c]).max()
    ref = O.compute(s.copy(positions=traj[-1], target_eps=1e-12, max_iter=5000), "port")
    # Against the oracle the mixed form adds the FP32 rounding of its pair
    # sums, here on a small total (4.9 in Coulomb-prefactor-1 units).
    assert rel_err(out["1"][0][-1][0], ref.energy) < (te if precision == "double" else 2e-5)


@pytest.mark.parametrize("precision", ["double", "mixed"])
def test_true_residual_check_skipped_under_drift_bound(precision, monkeypatch):
    """Warm-started solves skip the final true-residual matvec when the drift
    bound (a multiple of the recursive residuals' sum) is below the margin to
    the target.  The check only confirms (it does not change the dipoles), so
    the results equal those of solves that always take it."""
    s = S.water_box(6, 1.8643, seed=5, cutoff=0.8, target_eps=1e-7, max_iter=2000)
    v = np.random.default_rng(7).normal(size=s.positions.shape) * 2e-4   # nm per call
    traj = [s.positions + k * v for k in range(6)]
    out, mv = {}, {}
    for flag in ("0", "1"):
        monkeypatch.setenv("TDP_TRUE_RESIDUAL", flag)
        with CudaCalcTholeDipoleForceKernel(s, precision=precision, warm_start=True) as k:
            k.enableTiming(True)
            res = []
            mv[flag] = []
            for p in traj:
                res.append(k.execute(p))
                st = k.solverStats()
                assert st["converged"] and st["epsilon"] <= s.target_eps
                mv[flag].append(int(k.stageTimes()[6]) - st["iterations"])
            out[flag] = res
    # Matvecs beyond the CG iterations: with the check forced, one per warm
    # solve; by default none once the warm start is close.
    assert all(m == 1 for m in mv["1"][1:]), mv
    assert all(m == 0 for m in mv["0"][2:]), mv
    for (e0, f0), (e1, f1) in zip(out["0"], out["1"]):
        assert rel_err(e0, e1) < 1e-12 and rel_rms(f0, f1) < 1e-12
