"""Hand-written adjoint (tdp_adjoint / TholeDipoleFunction) against central
finite differences of the FP64 oracle.

Per-particle gradients of L = gE*E + g.F (random g, gE) with respect to
charge, polarizability, Thole factor and the three molecular-dipole
components are checked on systems that exercise every axis type and both
solver paths (Mutual: one adjoint solve; Direct: none; Extrapolated: the
perturbation recursion run backwards), with a relative step
of 1e-4 and the oracle converged to 1e-12.  Tolerance: 1e-5 relative to the
largest gradient of the same kind (FD truncation is ~1e-8 relative here).
Where two Thole factors tie, min(t_i, t_j) has a kink; the adjoint gives each
side half of the derivative there (the symmetric subgradient).

The force-matching loss of the differentiation workload (mean squared force
difference against targets made with alpha_O x1.1, alpha_H x0.9, a = 0.42)
is differentiated with respect to alpha_O, alpha_H, a, q_O (q_H = -q_O/2)
and the permanent-dipole magnitude, through torch.autograd, and compared
with finite differences (relative step 1e-4) to 1e-4 relative."""
import numpy as np
import pytest

from oracle import oracle as O
from tholedipoleplugin_b200 import systems as S

from .fixtures import ammonia, small_random_system, water4

pytestmark = pytest.mark.gpu

KINDS = ["q", "alpha", "thole", "mx", "my", "mz"]


def _loss(s, g, gE):
    r = O.compute(s, "port")
    return gE * r.energy + float(np.sum(g * r.forces))


def _perturb(s, kind, i, h):
    s = s.copy()
    if kind == "q":
        s.charges[i] += h
    elif kind == "alpha":
        s.polarizabilities[i] += h
    elif kind == "thole":
        s.tholes[i] += h
    else:
        s.dipoles[i]["xyz".index(kind[1])] += h
    return s


def _value(s, kind, i):
    return {"q": s.charges[i], "alpha": s.polarizabilities[i], "thole": s.tholes[i]}.get(
        kind, s.dipoles[i]["xyz".index(kind[1])] if kind[0] == "m" else None)


@pytest.mark.parametrize("name", ["ammonia_mutual", "ammonia_direct", "ammonia_extrapolated", "water4_pme",
                                  "random_mutual", "random_extrapolated"])
def test_particle_gradients_match_finite_differences(name):
    from tholedipoleplugin_b200.kernel import CudaCalcTholeDipoleForceKernel

    s = {"ammonia_mutual": ammonia(S.MUTUAL), "ammonia_direct": ammonia(S.DIRECT),
         "ammonia_extrapolated": ammonia(S.EXTRAPOLATED), "water4_pme": water4(S.MUTUAL),
         "random_mutual": small_random_system(24, seed=31, method=S.PME),
         "random_extrapolated": small_random_system(24, seed=32, method=S.PME, polarization=S.EXTRAPOLATED)}[name]
    # Ties t_i == t_j put every pair on the kink of min(t_i, t_j), where a
    # central difference is only first-order accurate; a 5% jitter of the
    # Thole factors moves the evaluation point well off it (gaps >> the
    # 1e-5 relative step used for t).  The tied case is covered by the
    # global-parameter test below, where both factors move together.
    rng = np.random.default_rng(9)
    s = s.copy(target_eps=1e-12, max_iter=5000, tholes=s.tholes * (1 + 0.05 * rng.uniform(-1, 1, s.n)))
    g = rng.normal(size=(s.n, 3))
    gE = 0.7
    with CudaCalcTholeDipoleForceKernel(s, precision="double") as k:
        k.execute(s.positions)
        grad = k.adjoint(g, gE)
    atoms = sorted(set([0, 1, s.n // 2, s.n - 1]))
    for c, kind in enumerate(KINDS):
        scale = np.abs(grad[:, c]).max()
        for i in atoms:
            v = _value(s, kind, i)
            h = (1e-5 if kind == "thole" else 1e-4) * abs(v) if v != 0 else 1e-6
            fd = (_loss(_perturb(s, kind, i, h), g, gE) - _loss(_perturb(s, kind, i, -h), g, gE)) / (2 * h)
            assert abs(grad[i, c] - fd) <= 1e-5 * max(scale, 1e-12) + 1e-9, (kind, i, grad[i, c], fd)


def _global_system(base, p):
    aO, aH, a, qO, m = p
    s = base.copy()
    o = np.arange(0, s.n, 3)
    hh = np.setdiff1d(np.arange(s.n), o)
    s.polarizabilities[o], s.polarizabilities[hh] = aO, aH
    s.tholes[:] = a
    s.charges[o], s.charges[hh] = qO, -qO / 2
    s.dipoles[o, 2] = m
    return s


def test_force_matching_gradients_through_autograd():
    import torch
    from tholedipoleplugin_b200.autograd import thole_dipole
    from tholedipoleplugin_b200.kernel import CudaCalcTholeDipoleForceKernel

    base = S.config_small(target_eps=1e-12, max_iter=5000)
    p0 = np.array([S.ALPHA_O, S.ALPHA_H, S.THOLE, S.Q_O, S.DIPOLE_O])
    target = O.compute(_global_system(base, [S.ALPHA_O * 1.1, S.ALPHA_H * 0.9, 0.42, S.Q_O, S.DIPOLE_O]),
                       "port").forces
    n = base.n

    def loss_np(p):
        f = O.compute(_global_system(base, p), "port").forces
        return float(np.mean((f - target) ** 2))

    params = torch.tensor(p0, dtype=torch.float64, requires_grad=True)
    o = torch.zeros(n, dtype=torch.bool)
    o[0::3] = True
    q = torch.where(o, params[3], -params[3] / 2)
    alpha = torch.where(o, params[0], params[1])
    thole = params[2].expand(n)
    dip = torch.zeros(n, 3, dtype=torch.float64)
    dip = dip.index_put((torch.arange(0, n, 3), torch.full((n // 3,), 2)), params[4].expand(n // 3))
    with CudaCalcTholeDipoleForceKernel(base, precision="double") as k:
        energy, forces = thole_dipole(q, alpha, thole, dip, k, base)
        loss = torch.mean((forces - torch.tensor(target)) ** 2)
        loss.backward()
    grad = params.grad.numpy()
    assert abs(loss.item() - loss_np(p0)) < 1e-9 * abs(loss.item())
    for k in range(5):
        h = 1e-4 * abs(p0[k])
        pp, pm = p0.copy(), p0.copy()
        pp[k] += h
        pm[k] -= h
        fd = (loss_np(pp) - loss_np(pm)) / (2 * h)
        assert abs(grad[k] - fd) <= 1e-4 * abs(fd), (k, grad[k], fd)


def _global_params_tensors(base, params, torch):
    """Per-particle tensors of the five global water parameters (alpha_O, alpha_H,
    Thole a, q_O with q_H = -q_O/2, dipole magnitude) for a system of waters."""
    n = base.n
    o = torch.zeros(n, dtype=torch.bool)
    o[0::3] = True
    q = torch.where(o, params[3], -params[3] / 2)
    alpha = torch.where(o, params[0], params[1])
    thole = params[2].expand(n)
    dip = torch.zeros(n, 3, dtype=torch.float64)
    dip = dip.index_put((torch.arange(0, n, 3), torch.full((n // 3,), 2)), params[4].expand(n // 3))
    return q, alpha, thole, dip


P0 = np.array([S.ALPHA_O, S.ALPHA_H, S.THOLE, S.Q_O, S.DIPOLE_O])
P_TARGET = [S.ALPHA_O * 1.1, S.ALPHA_H * 0.9, 0.42, S.Q_O, S.DIPOLE_O]


def test_force_matching_gradients_4096_water_box():
    # The differentiation workload on the 4,096-water box: targets from the FP64
    # form with alpha_O x1.1, alpha_H x0.9, a = 0.42; loss = mean (F - F_target)^2;
    # gradients of the five global parameters through the adjoint, against
    # central differences (relative step 1e-4) of the same FP64 forward, which
    # the parity tests pin to the reference at 1e-10.
    import torch
    from tholedipoleplugin_b200.autograd import thole_dipole
    from tholedipoleplugin_b200.kernel import CudaCalcTholeDipoleForceKernel

    base = S.config_medium(target_eps=1e-12, max_iter=2000)
    with CudaCalcTholeDipoleForceKernel(base, precision="double") as k:
        def forces_at(p):
            s = _global_system(base, p)
            k.copyParametersToContext(s)
            return k.execute(s.positions)[1]

        target = forces_at(P_TARGET)

        def loss_np(p):
            return float(np.mean((forces_at(p) - target) ** 2))

        params = torch.tensor(P0, dtype=torch.float64, requires_grad=True)
        q, alpha, thole, dip = _global_params_tensors(base, params, torch)
        _, forces = thole_dipole(q, alpha, thole, dip, k, base)
        loss = torch.mean((forces - torch.tensor(target)) ** 2)
        loss.backward()
        grad = params.grad.numpy()
        for j in range(5):
            h = 1e-4 * abs(P0[j])
            pp, pm = P0.copy(), P0.copy()
            pp[j] += h
            pm[j] -= h
            fd = (loss_np(pp) - loss_np(pm)) / (2 * h)
            assert abs(grad[j] - fd) <= 1e-4 * abs(fd), (j, grad[j], fd)


def test_force_matching_gradients_256_clusters():
    # The same gradients over 256 clusters of the cluster workload (4-64 waters,
    # seeded), against central differences of the FP64 oracle.
    import torch
    from tholedipoleplugin_b200.autograd import ClusterGradients, thole_dipole_clusters

    clusters = S.cluster_batch(1024, 4, 64, seed=3, target_eps=1e-12, max_iter=5000)[:256]
    allw, _ = S.concat_clusters(clusters)

    def oracle_forces(p):
        return np.concatenate([O.compute(_global_system(c, p), "port").forces for c in clusters])

    target = oracle_forces(P_TARGET)

    def loss_np(p):
        return float(np.mean((oracle_forces(p) - target) ** 2))

    with ClusterGradients(clusters, precision="double") as batch:
        params = torch.tensor(P0, dtype=torch.float64, requires_grad=True)
        q, alpha, thole, dip = _global_params_tensors(allw, params, torch)
        _, forces = thole_dipole_clusters(q, alpha, thole, dip, batch)
        loss = torch.mean((forces - torch.tensor(target)) ** 2)
        loss.backward()
    grad = params.grad.numpy()
    assert abs(loss.item() - loss_np(P0)) < 1e-9 * abs(loss.item())
    for j in range(5):
        h = 1e-4 * abs(P0[j])
        pp, pm = P0.copy(), P0.copy()
        pp[j] += h
        pm[j] -= h
        fd = (loss_np(pp) - loss_np(pm)) / (2 * h)
        assert abs(grad[j] - fd) <= 1e-4 * abs(fd), (j, grad[j], fd)


@pytest.mark.parametrize("name", ["random220_nocutoff", "water216_pme"])
def test_wide_damping_overflows_damped_lists(name):
    """Thole factors near 0.8 (damping width t_i t_j ~ 0.64) put every pair of
    the system within the damping range, so every atom has more damped
    partners than a row of the adjoint's damped-partner list holds: the
    overflowing pairs are evaluated in place and the list passes of the
    fixed-field and matvec Thole terms fall back to scanning all partners.
    The FP64 adjoint must still match central finite differences of the oracle
    along one direction of all six per-particle parameters (relative step 1e-5
    of each parameter), to 1e-6 relative, and the mixed form the FP64 form to
    1e-4 of the largest gradient of each kind."""
    from tholedipoleplugin_b200.kernel import CudaCalcTholeDipoleForceKernel

    base = (small_random_system(220, seed=41, method=S.NO_CUTOFF, box=1.6) if name == "random220_nocutoff"
            else S.config_small())
    rng = np.random.default_rng(12)
    s = base.copy(target_eps=1e-12, max_iter=5000, tholes=0.8 * (1 + 0.05 * rng.uniform(-1, 1, base.n)))
    g = rng.normal(size=(s.n, 3))
    gE = 0.4
    grads = {}
    for prec in ("double", "mixed"):
        with CudaCalcTholeDipoleForceKernel(s.copy(target_eps=1e-12 if prec == "double" else 1e-9),
                                            precision=prec) as k:
            k.execute(s.positions)
            grads[prec] = k.adjoint(g, gE)
    # Direction: every particle's (q, alpha, dipole) scaled by its own
    # magnitude; the Thole factors all scaled by one common factor, which
    # keeps their order (so no pair crosses the kink of min(t_i, t_j)).
    v = rng.uniform(-1, 1, size=(s.n, 6))
    v[:, 0] *= np.abs(s.charges)
    v[:, 1] *= s.polarizabilities
    v[:, 2] = 0.7 * s.tholes
    v[:, 3:] *= np.abs(np.asarray(s.dipoles)).max()
    h = 1e-5

    def moved(sign):
        return s.copy(charges=s.charges + sign * h * v[:, 0], polarizabilities=s.polarizabilities + sign * h * v[:, 1],
                      tholes=s.tholes + sign * h * v[:, 2], dipoles=np.asarray(s.dipoles) + sign * h * v[:, 3:])

    fd = (_loss(moved(1), g, gE) - _loss(moved(-1), g, gE)) / (2 * h)
    dd = float(np.sum(grads["double"] * v))
    assert abs(dd - fd) <= 1e-6 * max(abs(fd), 1e-12), (dd, fd)
    for c in range(6):
        scale = np.abs(grads["double"][:, c]).max()
        assert np.abs(grads["mixed"][:, c] - grads["double"][:, c]).max() <= 1e-4 * scale
