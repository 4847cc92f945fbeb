"""Batched reverse pass (tdp_batch_adjoint) and the device-resident autograd
paths.

* Every cluster's gradients from the one persistent reverse launch equal those
  of a single-system handle's tdp_adjoint on that cluster alone (FP64 form:
  1e-9 relative to the largest gradient of the kind), for Mutual and Direct
  polarization and for energy and force cotangents together.
* The mixed form's batched gradients agree with the FP64 form's to 1e-4
  relative (the north star's gradient tolerance).
* TholeDipoleFunction and ClusterBatchFunction on CUDA tensors give the same
  gradients as on CPU tensors (device pointers into tdp_update_particle_params,
  tdp_adjoint_device, tdp_batch_update_params and tdp_batch_adjoint).
* The mixed form's adjoint on a water box against central differences of the
  FP64 oracle, 1e-4 relative.

The reverse pass differentiates the reference's evaluation
(ReferenceTholeDipoleForce.cpp:100-127 with the solve of :820-851)."""
import numpy as np
import pytest

from oracle import oracle as O
from tholedipoleplugin_b200 import systems as S
from tholedipoleplugin_b200.batch import ClusterBatch
from tholedipoleplugin_b200.kernel import CudaCalcTholeDipoleForceKernel

pytestmark = pytest.mark.gpu


def _clusters(pol, count=48, eps=1e-12):
    cl = S.cluster_batch(1024, 4, 64, seed=3, target_eps=eps, max_iter=2000)
    pick = np.random.default_rng(4).choice(1024, count, replace=False)
    return [cl[k].copy(polarization=pol) for k in sorted(pick)]


def _close_per_kind(a, b, tol):
    for c in range(6):
        scale = max(np.abs(b[:, c]).max(), 1e-300)
        assert np.abs(a[:, c] - b[:, c]).max() <= tol * scale, (c, np.abs(a[:, c] - b[:, c]).max(), scale)


@pytest.mark.parametrize("pol", [S.MUTUAL, S.DIRECT])
def test_batch_adjoint_matches_single_handles(pol):
    clusters = _clusters(pol)
    rng = np.random.default_rng(5)
    with ClusterBatch(clusters, precision="double") as b:
        b.compute()
        gF = rng.normal(size=(b.n, 3))
        gE = rng.normal(size=b.num_clusters)
        got = b.adjoint(gF, gE)
        offs = b.offsets
        it, _ = b.adjointStats()
        if pol == S.MUTUAL:
            assert it.min() > 0
    want = np.zeros_like(got)
    for c, cl in enumerate(clusters):
        sl = slice(int(offs[c]), int(offs[c + 1]))
        with CudaCalcTholeDipoleForceKernel(cl, precision="double") as k:
            k.execute(cl.positions)
            want[sl] = k.adjoint(gF[sl], float(gE[c]))
    _close_per_kind(got, want, 1e-9)


def test_batch_adjoint_mixed_matches_double():
    clusters = _clusters(S.MUTUAL, count=64, eps=1e-10)
    rng = np.random.default_rng(6)
    out = {}
    for prec in ("double", "mixed"):
        with ClusterBatch(clusters, precision=prec) as b:
            b.compute()
            gF = rng.normal(size=(b.n, 3)) if prec == "double" else out["gF"]
            gE = np.full(b.num_clusters, 0.3)
            out["gF"] = gF
            out[prec] = b.adjoint(gF, gE)
    _close_per_kind(out["mixed"], out["double"], 1e-4)


def test_batch_update_params_and_empty_cotangents():
    clusters = _clusters(S.MUTUAL, count=16)
    with ClusterBatch(clusters, precision="double") as b:
        s = b.system
        b.updateParams(s.charges * 1.05, s.dipoles * 0.9, s.polarizabilities * 1.1, s.tholes * 1.02)
        e, f = b.compute()
        g0 = b.adjoint(None, None)
        assert np.all(g0 == 0.0)
        gE = np.ones(b.num_clusters)
        g = b.adjoint(None, gE)
        offs = b.offsets
    for c, cl in enumerate(clusters):
        sl = slice(int(offs[c]), int(offs[c + 1]))
        cs = cl.copy(charges=cl.charges * 1.05, dipoles=cl.dipoles * 0.9, polarizabilities=cl.polarizabilities * 1.1,
                     tholes=cl.tholes * 1.02)
        ref = O.compute(cs, "port")
        assert abs(e[c] - ref.energy) <= 1e-9 * abs(ref.energy) + 1e-12
        with CudaCalcTholeDipoleForceKernel(cs, precision="double") as k:
            k.execute(cs.positions)
            _close_per_kind(g[sl], k.adjoint(None, 1.0), 1e-9)


def test_autograd_device_path_matches_host_path():
    import torch
    from tholedipoleplugin_b200.autograd import thole_dipole

    s = S.config_small(target_eps=1e-11, max_iter=2000)
    rng = np.random.default_rng(7)
    w = rng.normal(size=(s.n, 3))
    grads = {}
    for dev in ("cpu", "cuda"):
        params = [torch.tensor(a, dtype=torch.float64, device=dev, requires_grad=True)
                  for a in (s.charges, s.polarizabilities, s.tholes, s.dipoles)]
        with CudaCalcTholeDipoleForceKernel(s, precision="double") as k:
            energy, forces = thole_dipole(*params, k, s)
            loss = 0.3 * energy + (forces * torch.tensor(w, device=dev)).sum()
            loss.backward()
        grads[dev] = [p.grad.detach().cpu().numpy() for p in params]
        assert forces.device.type == dev
    for a, b in zip(grads["cuda"], grads["cpu"]):
        assert np.abs(a - b).max() <= 1e-10 * max(np.abs(b).max(), 1e-300)


def test_cluster_autograd_device_path_matches_host_path():
    import torch
    from tholedipoleplugin_b200.autograd import ClusterGradients, thole_dipole_clusters

    clusters = _clusters(S.MUTUAL, count=32, eps=1e-11)
    grads = {}
    with ClusterGradients(clusters, precision="double") as cg:
        s = cg.system
        rng = np.random.default_rng(8)
        w = rng.normal(size=(s.n, 3))
        for dev in ("cpu", "cuda"):
            params = [torch.tensor(a, dtype=torch.float64, device=dev, requires_grad=True)
                      for a in (s.charges, s.polarizabilities, s.tholes, s.dipoles)]
            energies, forces = thole_dipole_clusters(*params, cg)
            loss = energies.sum() + (forces * torch.tensor(w, device=dev)).sum()
            loss.backward()
            grads[dev] = [p.grad.detach().cpu().numpy() for p in params]
    for a, b in zip(grads["cuda"], grads["cpu"]):
        assert np.abs(a - b).max() <= 1e-10 * max(np.abs(b).max(), 1e-300)


def test_mixed_adjoint_matches_oracle_finite_differences():
    # Mixed form (FP32 pair arithmetic in the forward and the adjoint solve's
    # matvec, FP64 VJPs and refinement) on 64 waters against central
    # differences of the FP64 oracle at relative step 1e-4.
    s = S.water_box(4, 1.25, seed=41, cutoff=0.6, target_eps=1e-12, max_iter=5000)
    rng = np.random.default_rng(9)
    s = s.copy(tholes=s.tholes * (1 + 0.05 * rng.uniform(-1, 1, s.n)))
    g = rng.normal(size=(s.n, 3))
    gE = 0.7
    with CudaCalcTholeDipoleForceKernel(s.copy(target_eps=1e-10), precision="mixed") as k:
        k.execute(s.positions)
        grad = k.adjoint(g, gE)

    def loss(t):
        r = O.compute(t, "port")
        return gE * r.energy + float(np.sum(g * r.forces))

    for c, kind in enumerate(["q", "alpha", "thole", "mx", "my", "mz"]):
        scale = np.abs(grad[:, c]).max()
        for i in (0, 1, 2, s.n // 2, s.n - 1):
            sp, sm = s.copy(), s.copy()
            if kind == "q":
                v, arr = s.charges[i], "charges"
            elif kind == "alpha":
                v, arr = s.polarizabilities[i], "polarizabilities"
            elif kind == "thole":
                v, arr = s.tholes[i], "tholes"
            else:
                v, arr = s.dipoles[i]["xyz".index(kind[1])], "dipoles"
            h = 1e-4 * abs(v) if v != 0 else 1e-6
            if arr == "dipoles":
                sp.dipoles[i]["xyz".index(kind[1])] += h
                sm.dipoles[i]["xyz".index(kind[1])] -= h
            else:
                getattr(sp, arr)[i] += h
                getattr(sm, arr)[i] -= h
            fd = (loss(sp) - loss(sm)) / (2 * h)
            assert abs(grad[i, c] - fd) <= 1e-4 * max(scale, 1e-12), (kind, i, grad[i, c], fd)
