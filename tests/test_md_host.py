"""Host-side rigid-water constraints of the e2e MD loop (tholedipoleplugin_b200/md.py):
matrix SHAKE (Newton on each water's three constraints) and RATTLE (one 3x3
solve per water), CPU only."""
import numpy as np

from tholedipoleplugin_b200 import md as M
from tholedipoleplugin_b200 import systems as S


def _iterative_shake(x0, x, v, dt, iters=2000, tol=1e-14):
    """Classic SHAKE, one constraint at a time, as the check."""
    x0w, xw, vw = x0.reshape(-1, 3, 3), x.reshape(-1, 3, 3), v.reshape(-1, 3, 3)
    for _ in range(iters):
        worst = 0.0
        for k, (a, b) in enumerate(M._PAIRS):
            d = M._D[k]
            s = xw[:, a] - xw[:, b]
            r0 = x0w[:, a] - x0w[:, b]
            diff = d * d - np.einsum("ij,ij->i", s, s)
            g = diff / (2.0 * np.einsum("ij,ij->i", s, r0) * (M._INV_M[a] + M._INV_M[b]))
            xw[:, a] += (g * M._INV_M[a])[:, None] * r0
            xw[:, b] -= (g * M._INV_M[b])[:, None] * r0
            vw[:, a] += (g * M._INV_M[a] / dt)[:, None] * r0
            vw[:, b] -= (g * M._INV_M[b] / dt)[:, None] * r0
            worst = max(worst, float(np.max(np.abs(diff))) / (d * d))
        if worst < tol:
            return


def _step(seed=0):
    s = S.water_box(4, 1.242, seed=seed)
    nw = s.n // 3
    x = s.positions.copy()
    v = M.maxwell_boltzmann(nw, 300.0, seed)
    M._rattle_host(x, v)
    f = np.random.default_rng(seed).standard_normal((s.n, 3)) * 100.0
    inv_m = 1.0 / np.tile([M.MASS_O, M.MASS_H, M.MASS_H], nw)[:, None]
    dt = 0.002
    v = v + 0.5 * dt * f * inv_m
    x0 = x.copy()
    x = x + dt * v
    return x0, x, v, dt


def test_shake_restores_bonds_and_matches_iterative_shake():
    x0, x, v, dt = _step()
    xa, va = x.copy(), v.copy()
    M._shake_host(x0, xa, va, dt)
    L = np.sqrt((M._bonds(xa.reshape(-1, 3, 3)) ** 2).sum(-1))
    assert np.abs(L - M._D[None, :]).max() < 1e-13
    xb, vb = x.copy(), v.copy()
    _iterative_shake(x0, xb, vb, dt)
    assert np.abs(xa - xb).max() < 1e-12
    assert np.abs(va - vb).max() < 1e-9


def test_constraint_forces_conserve_momentum():
    x0, x, v, dt = _step(1)
    m = np.tile([M.MASS_O, M.MASS_H, M.MASS_H], x.shape[0] // 3)[:, None]
    p0 = (m * v).sum(0)
    M._shake_host(x0, x, v, dt)
    M._rattle_host(x, v)
    assert np.abs((m * v).sum(0) - p0).max() < 1e-10
    w = M._bonds(v.reshape(-1, 3, 3))
    s = M._bonds(x.reshape(-1, 3, 3))
    assert np.abs(np.einsum("nkc,nkc->nk", s, w)).max() < 1e-12
