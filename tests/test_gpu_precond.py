"""The Ewald-operator preconditioner of the minimum-image CG solve.

The reference's PME flag means the minimum image over all pairs
(ReferenceTholeDipoleForce.cpp:1414-1423); its Mutual solve converges the
induced dipoles to the fixed point mu = alpha (E + T mu) (:820-851).  The
preconditioner only changes the path to that fixed point: it applies a few CG
iterations on the Ewald operator of the same box (plus the minimum-image
cube's uniform depolarising field) to every residual.  So:
  * the converged results equal the unpreconditioned solve's and the FP64
    oracle's, within the parity tolerances (plain form: energy 1e-9, forces
    and induced dipoles 1e-8; mixed form: 2e-5 against the plain one);
  * the outer iteration count (all-pairs matvecs) drops;
  * a box below twice the preconditioner's cutoff falls back to plain CG;
  * warm-started trajectories, covalent partners with their scales and every
    axis type go through the same code."""
import numpy as np
import pytest

from oracle import oracle as O
from tholedipoleplugin_b200 import systems as S
from tholedipoleplugin_b200.kernel import CudaCalcTholeDipoleForceKernel

from .fixtures import small_random_system
from .gpu_util import energy_rms_scale, rel_err, rel_rms

pytestmark = pytest.mark.gpu


def _run(s, precision, monkeypatch, pre, warm=False, traj=None):
    monkeypatch.setenv("TDP_PRECOND", "1" if pre else "0")
    out = []
    with CudaCalcTholeDipoleForceKernel(s, precision=precision, warm_start=warm) as k:
        k.enableTiming(True)
        for p in (traj if traj is not None else [s.positions]):
            e, f = k.execute(p)
            st = k.solverStats()
            t = k.stageTimes()
            out.append(dict(e=e, f=f, mu=k.getInducedDipoles(), its=st["iterations"], conv=st["converged"],
                            eps=st["epsilon"], applications=int(t[12]), matvecs=int(t[6])))
    return out


@pytest.mark.parametrize("precision", ["double", "mixed"])
@pytest.mark.parametrize("name", ["water216", "water512", "random_pme"])
def test_preconditioned_solve_matches_plain_cg_and_oracle(name, precision, monkeypatch):
    base = {"water216": lambda: S.config_small(),
            "water512": lambda: S.water_box(8, 2.4843, seed=21, cutoff=0.9),
            "random_pme": lambda: small_random_system(97, seed=12, method=S.PME)}[name]()
    eps = 1e-11 if precision == "double" else 1e-9
    s = base.copy(target_eps=eps, max_iter=2000)
    (pc,) = _run(s, precision, monkeypatch, True)
    (cg,) = _run(s, precision, monkeypatch, False)
    assert pc["conv"] and cg["conv"] and pc["eps"] <= eps
    # One application per outer iteration, plus the cold start y = M(sqrt(alpha) E).
    assert pc["applications"] == pc["its"] + 1 and pc["its"] > 0 and cg["applications"] == 0
    assert pc["its"] < cg["its"], (pc["its"], cg["its"])
    te, tf = (1e-9, 1e-8) if precision == "double" else (2e-6, 2e-5)
    assert rel_err(pc["e"], cg["e"]) < te
    assert rel_rms(pc["f"], cg["f"]) < tf
    assert rel_rms(pc["mu"], cg["mu"]) < tf
    if precision == "double":
        ref = O.compute(base.copy(target_eps=1e-12, max_iter=5000), "port")
        assert rel_err(pc["e"], ref.energy) < 1e-9
        assert rel_rms(pc["f"], ref.forces) < 1e-8
        assert rel_rms(pc["mu"], ref.induced) < 1e-8


@pytest.mark.parametrize("precision", ["double", "mixed"])
def test_preconditioned_warm_trajectory(precision, monkeypatch):
    """Warm-started solves along a short trajectory (the MD drivers' path,
    fused start included): each converges to the cold plain-CG dipoles, with
    fewer all-pairs matvecs per solve."""
    s = S.water_box(7, 2.1738, seed=9, cutoff=0.9, target_eps=1e-7, max_iter=2000)
    rng = np.random.default_rng(5)
    v = rng.normal(size=s.positions.shape) * 3e-4
    traj = [s.positions + k * v for k in range(6)]
    pc = _run(s, precision, monkeypatch, True, warm=True, traj=traj)
    cg = _run(s, precision, monkeypatch, False, warm=True, traj=traj)
    tight = _run(s.copy(target_eps=1e-11), "double", monkeypatch, False, traj=traj)
    # The mixed form's energy also carries the FP32 rounding of its pair terms,
    # 3e-7 sqrt(sum (q_i q_j / r_ij)^2), which matters here: this box's total
    # (11 in Coulomb-prefactor-1 units) is a small difference of large terms.
    c2 = energy_rms_scale(s) if precision == "mixed" else 0.0
    for a, b in zip(pc, tight):
        assert a["conv"] and a["eps"] <= 1e-7
        assert rel_rms(a["mu"], b["mu"]) < 2e-5
        assert abs(a["e"] - b["e"]) < 1e-6 * abs(b["e"]) + 3e-7 * c2
        assert rel_rms(a["f"], b["f"]) < 2e-5
    assert sum(a["matvecs"] for a in pc[2:]) < sum(b["matvecs"] for b in cg[2:]), \
        ([a["matvecs"] for a in pc], [b["matvecs"] for b in cg])


def test_small_box_falls_back_to_plain_cg(monkeypatch):
    """A box edge below twice the preconditioner's real-space cutoff (0.63 nm
    for these Thole factors): the solve runs unpreconditioned."""
    s = S.water_box(3, 0.9321, seed=4, cutoff=0.45, target_eps=1e-11, max_iter=2000)
    (pc,) = _run(s, "double", monkeypatch, True)
    assert pc["applications"] == 0 and pc["conv"]
    ref = O.compute(s.copy(target_eps=1e-12, max_iter=5000), "port")
    assert rel_err(pc["e"], ref.energy) < 1e-9
    assert rel_rms(pc["mu"], ref.induced) < 1e-8


@pytest.mark.parametrize("precision", ["double", "mixed"])
def test_preconditioned_adjoint_matches_plain_cg(precision, monkeypatch):
    """The adjoint's solve of the same system goes through the same
    preconditioned CG; its gradients equal the unpreconditioned ones."""
    s = S.water_box(6, 1.8643, seed=3, cutoff=0.8, target_eps=1e-11 if precision == "double" else 1e-9,
                    max_iter=2000)
    g = np.random.default_rng(2).normal(size=(s.n, 3))
    out = {}
    for pre in (True, False):
        monkeypatch.setenv("TDP_PRECOND", "1" if pre else "0")
        with CudaCalcTholeDipoleForceKernel(s, precision=precision) as k:
            k.execute(s.positions)
            out[pre] = k.adjoint(g, 0.3)
    tol = 1e-7 if precision == "double" else 1e-4
    for c in range(out[True].shape[1]):
        scale = np.abs(out[False][:, c]).max()
        assert np.abs(out[True][:, c] - out[False][:, c]).max() <= tol * scale


@pytest.mark.parametrize("pre", [True, False])
def test_solver_history(pre, monkeypatch):
    """tdp_solver_history: the stopping quantity at the start, after every
    iteration and after a true-residual check, oldest first; its last entry is
    the epsilon tdp_solver_stats reports, and below the target."""
    monkeypatch.setenv("TDP_PRECOND", "1" if pre else "0")
    s = S.config_small().copy(target_eps=1e-9, max_iter=2000)
    with CudaCalcTholeDipoleForceKernel(s, precision="double") as k:
        k.execute(s.positions)
        st = k.solverStats()
        h = k.solverHistory()
    assert st["converged"]
    assert len(h) in (st["iterations"] + 1, st["iterations"] + 2)   # + the true-residual check
    assert h[-1] == st["epsilon"] and h[-1] <= 1e-9 < h[0]
    assert np.all(np.isfinite(h))
