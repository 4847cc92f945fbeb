"""Host-side rigid-water half steps of the e2e MD loop (tdp_md_host_kick_drift /
tdp_md_host_kick through tholedipoleplugin_b200/md.py), CPU only: the library's
per-water SHAKE/RATTLE on host threads against a numpy restatement of classic
SHAKE, constraint satisfaction and momentum conservation."""
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


def _state(n_side=4, box=1.242, seed=0):
    s = S.water_box(n_side, box, seed=seed)
    nw = s.n // 3
    x = np.ascontiguousarray(s.positions.copy())
    v = M.maxwell_boltzmann(nw, 300.0, seed)
    M.host_kick(x, v, None, 0.0)
    f = np.random.default_rng(seed).standard_normal((s.n, 3)) * 100.0
    return x, v, f, 0.002


def test_kick_drift_matches_classic_shake():
    x, v, f, dt = _state()
    inv_m = 1.0 / np.tile([M.MASS_O, M.MASS_H, M.MASS_H], x.shape[0] // 3)[:, None]
    xa, va = x.copy(), v.copy()
    M.host_kick_drift(xa, va, f, dt)
    L = np.sqrt((M._bonds(xa.reshape(-1, 3, 3)) ** 2).sum(-1))
    assert np.abs(L - M._D[None, :]).max() < 1e-11
    vb = v + 0.5 * dt * f * inv_m
    xb = x + dt * vb
    _iterative_shake(x, xb, vb, dt)
    assert np.abs(xa - xb).max() < 1e-11
    assert np.abs(va - vb).max() < 1e-8


def test_constraint_forces_conserve_momentum():
    x, v, f, dt = _state(seed=1)
    f -= f.mean(0)   # no net external force
    m = np.tile([M.MASS_O, M.MASS_H, M.MASS_H], x.shape[0] // 3)[:, None]
    p0 = (m * v).sum(0)
    M.host_kick_drift(x, v, f, dt)
    M.host_kick(x, v, f, dt)
    assert np.abs((m * v).sum(0) - p0).max() < 1e-9
    w = M._bonds(v.reshape(-1, 3, 3))
    s = M._bonds(x.reshape(-1, 3, 3))
    assert np.abs(np.einsum("nkc,nkc->nk", s, w)).max() < 1e-10


def test_threaded_equals_single_range():
    # 4,000 waters split across host threads give the same result as the same
    # waters stepped in small calls (one thread each).
    x, v, f, dt = _state(16, 4.968, seed=2)
    xa, va = x.copy(), v.copy()
    M.host_kick_drift(xa, va, f, dt)
    M.host_kick(xa, va, f, dt)
    xb, vb = x.copy(), v.copy()
    for r in range(0, x.shape[0], 300):
        sl = slice(r, r + 300)
        xs, vs, fs = xb[sl].copy(), vb[sl].copy(), f[sl].copy()
        M.host_kick_drift(xs, vs, fs, dt)
        M.host_kick(xs, vs, fs, dt)
        xb[sl], vb[sl] = xs, vs
    assert np.array_equal(xa, xb) and np.array_equal(va, vb)
