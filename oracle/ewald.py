"""FP64 Ewald restatement of the Thole-dipole electrostatics.  TEST
INFRASTRUCTURE ONLY: tests/ and bench.py's CPU leg use it as the checker of the
library's Ewald mode; the library never loads it.

The reference plugin (aehogan/tholedipoleplugin) has no Ewald sum.  Its "PME"
method is the orthorhombic minimum image over all pairs
(platforms/reference/src/ReferenceTholeDipoleForce.cpp:1414-1423, "RTDF.cpp"),
and the Ewald parameters are only reported (ReferenceTholeDipoleKernels.cpp:
143-152).  The library's Ewald mode (TDP_FLAG_EWALD) is therefore a mode of
its own whose parity the reference cannot pin.  This module defines it and is
pinned instead by properties: independence of the splitting parameter alpha,
forces equal to minus the finite-difference gradient of the energy, the
neutralising-plasma test of TestReferenceTholeDipoleForce.cpp:761-801, and the
large-box limit, in which its fields, induced dipoles and energy approach the
compiled reference's NoCutoff values.

Physics (Coulomb prefactor 1, RTDF.cpp:20-21; nm, e, e*nm, nm^3):
* Permanent multipoles P_i = (q_i, p_i), p_i the lab-frame dipole (the
  reference's rotation, RTDF.cpp:454-571, via the C oracle); induced dipoles
  U_i = (0, mu_i); total T_i = (q_i, p_i + mu_i).
* Pair energy of two charge+dipole sites for a radial kernel set
  B = (B0, B1, B2, B3), r = r_j - r_i:
      E = q_i q_j B0 + [q_j (d_i.r) - q_i (d_j.r) + d_i.d_j] B1 - (d_i.r)(d_j.r) B2,
  bare kernels b = (1/r, 1/r^3, 3/r^5, 15/r^7), Ewald real-space kernels from
  erfc(alpha r) (B_n recursion), Thole-damped kernels (., l3 b1, l5 b2, l7 b3)
  with the reference's damping width t_i t_j, a = min(t_i, t_j) and cut at
  a u^3 >= 50 (getAndScaleInverseRs, RTDF.cpp:646-676); l7 continues the
  family (d/dr of l5 b2 = -r l7 b3).
* Energy functional at fixed positions (minimised by the induced dipoles):
      U(mu) = sum_{i<j} [ m E_bare(P_i,P_j) + m (E_damp(P_i,U_j) + E_damp(U_i,P_j))
                          + s E_damp(U_i,U_j) ]   over all periodic images
              + 1/2 sum |mu_i|^2 / alpha_i,
  m, s the reference's M and I scales (RTDF.cpp:37-47, 609-644).  Its
  stationary point is the reference's fixed point mu = alpha (E_M + T mu)
  (RTDF.cpp:735-851) with the fields made periodic; the energy there is
  U_perm - 1/2 mu.E_M.
* Ewald split: all images of every bare term are summed in reciprocal space
  (tin-foil boundary) plus the erfc real space within the cutoff; the
  nearest-image pair then gets -(1 - m) E_bare(P,P) - (1 - m l) E_bare(...)
  corrections for scaled and damped terms, at any distance; self terms
  -alpha/sqrt(pi) sum q^2 - 2 alpha^3/(3 sqrt(pi)) sum |p + mu|^2 and the
  neutralising plasma -pi Q^2 / (2 V alpha^2).
* Direct polarization (mu = alpha E_M): the functional without the s E_damp(U_i,U_j)
  term, whose stationary point is mu = alpha E_M; written as U(mu) minus the
  Ewald energy of the induced dipoles alone, U(0, mu) = -1/2 mu.T mu, so its
  forces are those of U minus those of that induced-only energy.
* Forces are -dU/dr at the converged dipoles (the energy is stationary in
  mu); the torques p_i x (-dU/dp_i) go through the reference's torque map
  (RTDF.cpp:915-1115, via the C oracle).  Unlike the reference's own forces
  (which follow its quasi-internal frame quirks), these are the gradient.

Reciprocal space comes in two forms: ``direct`` (an explicit sum over
reciprocal vectors, the truth) and ``pme`` (smooth particle-mesh Ewald of
order 5 with the same grid and B-spline conventions as the library's CUDA
kernels, for tight parity).
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Optional

import numpy as np
from scipy.special import erfc as _erfc

from . import oracle as O

SQRT_PI = math.sqrt(math.pi)
PME_ORDER = 5
_M_TABLE = (0.0, 0.0, 0.0, 0.5, 1.0)   # RTDF.cpp:37-47
_I_TABLE = (0.0, 1.0, 1.0, 1.0, 1.0)


# ---------------------------------------------------------------------------
# Parameters
# ---------------------------------------------------------------------------
def smooth_size(n: int) -> int:
    """Smallest m >= n whose prime factors are all 2, 3, 5 or 7."""
    m = max(int(n), 1)
    while True:
        k = m
        for p in (2, 3, 5, 7):
            while k % p == 0:
                k //= p
        if k == 1:
            return m
        m += 1


def pme_parameters(cutoff: float, tolerance: float, box) -> tuple:
    """alpha = sqrt(-ln(2 tol))/cutoff and grid n_k = ceil(2 alpha L_k / (3 tol^(1/5))),
    at least 6 -- the formula behind ReferenceTholeDipoleKernels.cpp:143-152 --
    each rounded up to a 2,3,5,7-smooth size for the FFT."""
    a = math.sqrt(-math.log(2.0 * tolerance)) / cutoff
    g = tuple(smooth_size(max(6, int(math.ceil(2.0 * a * float(L) / (3.0 * tolerance ** 0.2))))) for L in box)
    return a, g


# ---------------------------------------------------------------------------
# Pair tables
# ---------------------------------------------------------------------------
def scale_matrices(sys):
    """Dense M and I scales: pair (i<j) from atom i's Covalent12 / Covalent13
    lists by list position, a later duplicate overwriting an earlier one
    (RTDF.cpp:609-644, :382-385, :806-808)."""
    n = sys.n
    M = np.ones((n, n))
    S = np.ones((n, n))
    for table, lists, out in ((_M_TABLE, sys.cov12, M), (_I_TABLE, sys.cov13, S)):
        for i in range(n):
            for pos, j in enumerate(lists[i]):
                if j > i:
                    out[i, j] = out[j, i] = table[pos]
    np.fill_diagonal(M, 0.0)
    np.fill_diagonal(S, 0.0)
    return M, S


def _displacements(pos, box):
    d = pos[None, :, :] - pos[:, None, :]        # d[i, j] = r_j - r_i
    L = np.asarray(box, dtype=np.float64)
    d = d - L * np.floor(d / L + 0.5)
    return d


def thole_factors(r, ti, tj):
    """l3, l5, l7 of every pair: getAndScaleInverseRs's damping (RTDF.cpp:646-676),
    width t_i t_j, a = min(t_i, t_j), undamped where t_i t_j = 0 or a u^3 >= 50."""
    w = ti[:, None] * tj[None, :]
    a = np.minimum(ti[:, None], tj[None, :])
    l3 = np.ones_like(r)
    l5 = np.ones_like(r)
    l7 = np.ones_like(r)
    with np.errstate(divide="ignore", invalid="ignore"):
        au3 = np.where(w != 0.0, a * (r / np.where(w != 0.0, w, 1.0)) ** 3, np.inf)
    m = au3 < 50.0
    e = np.exp(-au3[m])
    x = au3[m]
    l3[m] = 1.0 - e
    l5[m] = 1.0 - (1.0 + x) * e
    l7[m] = 1.0 - (1.0 + x + 0.6 * x * x) * e
    return l3, l5, l7


def bare_kernels(r):
    with np.errstate(divide="ignore"):
        ri = np.where(r > 0, 1.0 / np.where(r > 0, r, 1.0), 0.0)
    r2 = ri * ri
    return ri, ri * r2, 3.0 * ri * r2 * r2, 15.0 * ri * r2 * r2 * r2


def erfc_kernels(r, alpha, cutoff):
    """B0..B3 of erfc(alpha r)/r (B_{n+1} = ((2n+1) B_n + (2 alpha^2)^(n+1)/(alpha sqrt(pi)) e^(-alpha^2 r^2)) / r^2),
    zero beyond the cutoff and on the diagonal; alpha = 0 gives the bare kernels."""
    inside = (r > 0) & (r < cutoff)
    if alpha == 0.0:
        z = np.zeros_like(r)
        return tuple(np.where(inside, b, z) for b in bare_kernels(r))
    rs = np.where(inside, r, 1.0)
    e = np.exp(-(alpha * rs) ** 2) / (alpha * SQRT_PI)
    r2 = rs * rs
    a2 = 2.0 * alpha * alpha
    B0 = _erfc(alpha * rs) / rs
    B1 = (B0 + a2 * e) / r2
    B2 = (3.0 * B1 + a2 * a2 * e) / r2
    B3 = (5.0 * B2 + a2 * a2 * a2 * e) / r2
    z = np.zeros_like(r)
    return tuple(np.where(inside, b, z) for b in (B0, B1, B2, B3))


# ---------------------------------------------------------------------------
# Generic bilinear pair terms (dense over i, j with d[i, j] = r_j - r_i)
# ---------------------------------------------------------------------------
def pair_field(d, K1, K2, qj, dj):
    """Field at i from the charges and dipoles of j: -K1 (q_j r + d_j) + K2 (d_j.r) r,
    summed over j (K1, K2 already hold scales and masks)."""
    dr = np.einsum("ijc,jc->ij", d, dj)
    f = -(K1 * qj[None, :])[:, :, None] * d - K1[:, :, None] * dj[None, :, :] + (K2 * dr)[:, :, None] * d
    return f.sum(axis=1)


def pair_energy_force(d, K, qi, di, qj, dj):
    """Energy (sum over ordered i, j -- halve for unordered), force on i, and the
    field -dE/dd_i at i, for kernel set K = (K0, K1, K2, K3)."""
    K0, K1, K2, K3 = K
    di_r = np.einsum("ic,ijc->ij", di, d)
    dj_r = np.einsum("ijc,jc->ij", d, dj)
    didj = di @ dj.T
    G0 = qi[:, None] * qj[None, :]
    G1 = qj[None, :] * di_r - qi[:, None] * dj_r + didj
    G2 = -di_r * dj_r
    E = (G0 * K0 + G1 * K1 + G2 * K2).sum()
    # F_j = r (G0 K1 + G1 K2 + G2 K3) - K1 (q_j d_i - q_i d_j) + K2 ((d_j.r) d_i + (d_i.r) d_j);  F_i = -F_j
    c = G0 * K1 + G1 * K2 + G2 * K3
    Fj = (c[:, :, None] * d
          - K1[:, :, None] * (qj[None, :, None] * di[:, None, :] - qi[:, None, None] * dj[None, :, :])
          + K2[:, :, None] * (dj_r[:, :, None] * di[:, None, :] + di_r[:, :, None] * dj[None, :, :]))
    Fi = -Fj.sum(axis=1)
    field_i = (-K1[:, :, None] * (qj[None, :, None] * d + dj[None, :, :]) + (K2 * dj_r)[:, :, None] * d).sum(axis=1)
    return E, Fi, field_i


# ---------------------------------------------------------------------------
# Reciprocal space
# ---------------------------------------------------------------------------
def _kvectors(box, kmax):
    r = np.arange(-kmax, kmax + 1)
    n = np.stack(np.meshgrid(r, r, r, indexing="ij"), axis=-1).reshape(-1, 3)
    n = n[np.any(n != 0, axis=1)]
    return n / np.asarray(box, dtype=np.float64)


class DirectRecip:
    """Explicit sum over reciprocal vectors m = n/L, |n_k| <= kmax:
    S(m) = sum_j (q_j + 2 pi i m.d_j) exp(2 pi i m.r_j), G(m) = exp(-pi^2 m^2/alpha^2) / (pi V m^2),
    E = 1/2 sum_m G |S|^2."""

    def __init__(self, pos, box, alpha, kmax, chunk=4096):
        self.pos = pos
        self.box = np.asarray(box, dtype=np.float64)
        self.V = float(np.prod(self.box))
        m = _kvectors(box, kmax)
        m2 = (m * m).sum(1)
        self.m = m
        self.G = np.exp(-(math.pi ** 2) * m2 / alpha ** 2) / (math.pi * self.V * m2)
        self.chunk = chunk

    def _chunks(self):
        for a in range(0, self.m.shape[0], self.chunk):
            m = self.m[a:a + self.chunk]
            ph = 2.0 * math.pi * (self.pos @ m.T)                 # (n, k)
            yield m, self.G[a:a + self.chunk], np.cos(ph), np.sin(ph)

    def energy_field(self, q, dip):
        """(E_rec, field at every atom) of the density (q, dip); the field includes self terms."""
        E = 0.0
        field = np.zeros_like(self.pos)
        for m, G, c, s in self._chunks():
            md = 2.0 * math.pi * (dip @ m.T)                      # (n, k)
            # S = sum_j (q_j + i md_j)(c_j + i s_j)
            Sr = (q[:, None] * c - md * s).sum(0)
            Si = (q[:, None] * s + md * c).sum(0)
            E += 0.5 * (G * (Sr * Sr + Si * Si)).sum()
            # field_i = -2 pi sum_m G m Im[S exp(-i th_i)];  Im[S e^{-i th}] = Si c - Sr s
            im = Si[None, :] * c - Sr[None, :] * s
            field += -2.0 * math.pi * (im * G[None, :]) @ m
        return E, field

    def field_tensor(self):
        """Dense 3n x 3n field-of-dipole tensor (including i = j): -4 pi^2 sum_m G m m^T cos(2 pi m.(r_j - r_i))."""
        n = self.pos.shape[0]
        T = np.zeros((n, 3, n, 3))
        for m, G, c, s in self._chunks():
            for a in range(3):
                for b in range(3):
                    w = G * m[:, a] * m[:, b]
                    T[:, a, :, b] += -4.0 * math.pi ** 2 * ((c * w) @ c.T + (s * w) @ s.T)
        return T.reshape(3 * n, 3 * n)

    def forces(self, q, dip):
        """-dE_rec/dr_i of the density (q, dip)."""
        F = np.zeros_like(self.pos)
        for m, G, c, s in self._chunks():
            md = 2.0 * math.pi * (dip @ m.T)
            Sr = (q[:, None] * c - md * s).sum(0)
            Si = (q[:, None] * s + md * c).sum(0)
            # dS/dr_i = (q_i + i md_i)(2 pi i m) e^{i th_i};  F_i = -sum G Re[conj(S) dS/dr_i]
            # (q + i md)(i)(c + i s) = i q c - q s - md c - i md s  -> re = -(q s + md c), im = q c - md s
            re = -(q[:, None] * s + md * c)
            im = q[:, None] * c - md * s
            val = Sr[None, :] * re + Si[None, :] * im            # Re[conj(S) * (re + i im)]
            F += -2.0 * math.pi * (val * G[None, :]) @ m
        return F


def bspline(w, order=PME_ORDER):
    """theta[k] = M_n(w + k), k = 0..n-1 (grid point floor(u) - k), with first and
    second derivatives, for w in [0, 1) (cardinal B-splines by the recursion
    M_k(x) = (x M_{k-1}(x) + (k - x) M_{k-1}(x - 1)) / (k - 1))."""
    w = np.asarray(w, dtype=np.float64)

    def level(k):
        m = np.zeros(w.shape + (order,))
        m[..., 0] = w
        m[..., 1] = 1.0 - w
        for kk in range(3, k + 1):
            new = np.zeros_like(m)
            for j in range(kk):
                x = w + j
                a = m[..., j] if j < kk - 1 else 0.0
                b = m[..., j - 1] if j >= 1 else 0.0
                new[..., j] = (x * a + (kk - x) * b) / (kk - 1)
            m = new
        return m

    mn, m1, m2 = level(order), level(order - 1), level(order - 2)
    d1 = np.zeros_like(mn)
    d2 = np.zeros_like(mn)
    for j in range(order):
        d1[..., j] = m1[..., j] - (m1[..., j - 1] if j >= 1 else 0.0)
        d2[..., j] = m2[..., j] - 2.0 * (m2[..., j - 1] if j >= 1 else 0.0) + (m2[..., j - 2] if j >= 2 else 0.0)
    return mn, d1, d2


def bspline_moduli(K, order=PME_ORDER):
    """|b(m)|^2 = 1 / |sum_{j=0}^{n-2} M_n(j+1) exp(2 pi i m j / K)|^2; a (near) zero
    denominator -- at m = K/2 for odd orders -- takes the mean of its neighbours' moduli."""
    mj = np.array([bspline(np.array(0.0), order)[0][j] for j in range(order)])  # M_n(j) for j = 0..n-1
    vals = np.array([mj[j] for j in range(1, order)])                           # M_n(1..n-1)
    m = np.arange(K)
    ph = 2.0 * math.pi * np.outer(m, np.arange(order - 1)) / K
    den = (vals[None, :] * np.cos(ph)).sum(1) ** 2 + (vals[None, :] * np.sin(ph)).sum(1) ** 2
    mod = den.copy()
    for i in range(K):
        if mod[i] < 1e-7:
            mod[i] = 0.5 * (mod[(i - 1) % K] + mod[(i + 1) % K])
    return 1.0 / mod


class PmeRecip:
    """Smooth PME of order 5 on a (K1, K2, K3) grid: u_k = K_k frac(x_k/L_k),
    Q(g) = sum_i [q_i Th_i(g) + d_i . grad_{r_i} Th_i(g)], Th_i = prod_k M_n(u_ik - g_k),
    phi = IDFT(C . DFT(Q)) with C(m) = G(m) |b(m)|^2, E = 1/2 sum_g Q phi,
    atom fields and field gradients from the derivatives of Th_i."""

    def __init__(self, pos, box, alpha, grid, order=PME_ORDER):
        self.box = np.asarray(box, dtype=np.float64)
        self.K = np.asarray(grid, dtype=np.int64)
        self.V = float(np.prod(self.box))
        self.order = order
        n = pos.shape[0]
        f = pos / self.box
        f = f - np.floor(f)
        u = f * self.K
        base = np.floor(u).astype(np.int64)
        w = u - base
        th, d1, d2 = bspline(w, order)                             # (n, 3, order)
        self.th, self.d1, self.d2 = th, d1, d2
        self.idx = [(base[:, k:k + 1] - np.arange(order)[None, :]) % self.K[k] for k in range(3)]  # (n, order)
        self.scale = self.K / self.box                            # du/dx
        mods = [bspline_moduli(int(K), order) for K in self.K]
        ms = [np.where(np.arange(K) <= K // 2, np.arange(K), np.arange(K) - K) / L for K, L in zip(self.K, self.box)]
        mx, my, mz = np.meshgrid(*ms, indexing="ij")
        m2 = mx ** 2 + my ** 2 + mz ** 2
        with np.errstate(divide="ignore", invalid="ignore"):
            G = np.exp(-(math.pi ** 2) * m2 / alpha ** 2) / (math.pi * self.V * m2)
        G[0, 0, 0] = 0.0
        B = mods[0][:, None, None] * mods[1][None, :, None] * mods[2][None, None, :]
        self.C = G * B
        self.n = n

    def _weights(self, i):
        """(5,5,5) value and first/second derivative (w.r.t. x, y, z) weight tensors of atom i."""
        th, d1, d2, s = self.th[i], self.d1[i], self.d2[i], self.scale
        t = [th[k] for k in range(3)]
        g = [d1[k] * s[k] for k in range(3)]
        h = [d2[k] * s[k] * s[k] for k in range(3)]
        W = np.einsum("a,b,c->abc", t[0], t[1], t[2])
        D = [np.einsum("a,b,c->abc", g[0], t[1], t[2]), np.einsum("a,b,c->abc", t[0], g[1], t[2]),
             np.einsum("a,b,c->abc", t[0], t[1], g[2])]
        H = np.zeros((3, 3) + W.shape)
        fac = [t, g, h]
        for a in range(3):
            for b in range(3):
                cnt = [0, 0, 0]
                cnt[a] += 1
                cnt[b] += 1
                H[a, b] = np.einsum("a,b,c->abc", fac[cnt[0]][0], fac[cnt[1]][1], fac[cnt[2]][2])
        return W, D, H

    def _ix(self, i):
        return np.ix_(self.idx[0][i], self.idx[1][i], self.idx[2][i])

    def spread(self, q, dip):
        Q = np.zeros(tuple(self.K))
        for i in range(self.n):
            W, D, _ = self._weights(i)
            val = q[i] * W + dip[i, 0] * D[0] + dip[i, 1] * D[1] + dip[i, 2] * D[2]
            np.add.at(Q, self._ix(i), val)
        return Q

    def potential_grid(self, Q):
        return np.real(np.fft.ifftn(self.C * np.fft.fftn(Q))) * float(np.prod(self.K))

    def energy_field(self, q, dip, gradient=False):
        Q = self.spread(q, dip)
        phi = self.potential_grid(Q)
        E = 0.5 * float((Q * phi).sum())
        field = np.zeros((self.n, 3))
        grad = np.zeros((self.n, 3, 3))
        for i in range(self.n):
            W, D, H = self._weights(i)
            loc = phi[self._ix(i)]
            for a in range(3):
                field[i, a] = -(D[a] * loc).sum()
                if gradient:
                    for b in range(3):
                        grad[i, a, b] = -(H[a, b] * loc).sum()   # d field_b / d x_a
        return (E, field, grad) if gradient else (E, field)

    def forces(self, q, dip):
        _, field, grad = self.energy_field(q, dip, gradient=True)
        # F_i,a = q_i E_i,a + sum_b d_i,b dE_i,b/dx_a
        return q[:, None] * field + np.einsum("iab,ib->ia", grad, dip)


# ---------------------------------------------------------------------------
# The Ewald evaluation
# ---------------------------------------------------------------------------
@dataclass
class EwaldResult:
    energy: float
    forces: np.ndarray
    induced: np.ndarray
    lab: np.ndarray
    fixed_field: np.ndarray
    alpha: float
    grid: Optional[tuple] = None


class NoRecip:
    """No reciprocal space (the variational NoCutoff model: bare pairs, no images)."""

    def __init__(self, n):
        self.n = n

    def energy_field(self, q, dip):
        return 0.0, np.zeros((self.n, 3))

    def forces(self, q, dip):
        return np.zeros((self.n, 3))


class Ewald:
    """Dense FP64 Ewald model of one system at its positions (orthorhombic box
    sys.box).  recip="none" with alpha = 0 is the variational model without
    periodicity (all pairs, bare kernels): the NoCutoff counterpart."""

    def __init__(self, sys, alpha: float, cutoff: Optional[float] = None, recip: str = "direct",
                 kmax: Optional[int] = None, grid=None):
        self.sys = sys
        self.alpha = float(alpha)
        vacuum = recip == "none"
        self.cutoff = float("inf") if vacuum else float(sys.cutoff if cutoff is None else cutoff)
        self.box = np.zeros(3) if vacuum else np.asarray(sys.box, dtype=np.float64)
        if vacuum and self.alpha != 0.0:
            raise ValueError("recip='none' needs alpha = 0")
        if not vacuum and np.any(self.box < 2.0 * self.cutoff * 0.999999):
            raise ValueError("box smaller than twice the cutoff")
        self.pos = np.asarray(sys.positions, dtype=np.float64).reshape(-1, 3)
        self.q = np.asarray(sys.charges, dtype=np.float64)
        self.pol = np.asarray(sys.polarizabilities, dtype=np.float64)
        n = self.pos.shape[0]
        self.n = n
        self.lab = O.lab_dipoles(sys)
        self.M, self.S = scale_matrices(sys)
        if vacuum:
            self.d = self.pos[None, :, :] - self.pos[:, None, :]
        else:
            self.d = _displacements(self.pos, self.box)
        r = np.sqrt((self.d ** 2).sum(-1))
        np.fill_diagonal(r, 0.0)
        self.r = r
        th = np.asarray(sys.tholes, dtype=np.float64)
        l3, l5, l7 = thole_factors(r, th, th)
        b0, b1, b2, b3 = bare_kernels(r)
        e0, e1, e2, e3 = erfc_kernels(r, self.alpha, self.cutoff)
        self.bare = (b0, b1, b2, b3)
        self.erfc = (e0, e1, e2, e3)
        self.damp = (np.zeros_like(r), l3 * b1, l5 * b2, l7 * b3)
        if recip == "direct":
            if kmax is None:
                kmax = int(math.ceil(6.5 * self.alpha * float(self.box.max()) / math.pi))
            self.rec = DirectRecip(self.pos, self.box, self.alpha, kmax)
        elif recip == "pme":
            if grid is None:
                grid = pme_parameters(self.cutoff, sys.ewald_tolerance, self.box)[1]
            self.rec = PmeRecip(self.pos, self.box, self.alpha, grid)
        elif recip == "none":
            self.rec = NoRecip(n)
        else:
            raise ValueError(recip)
        self.grid = grid
        self.selfc = 4.0 * self.alpha ** 3 / (3.0 * SQRT_PI)

    # Fields ---------------------------------------------------------------
    def fixed_field(self):
        """E_M: real space (erfc - bare + m damped) + reciprocal + self."""
        Kr1 = self.erfc[1] - self.bare[1] + self.M * self.damp[1]
        Kr2 = self.erfc[2] - self.bare[2] + self.M * self.damp[2]
        f = pair_field(self.d, Kr1, Kr2, self.q, self.lab)
        _, fr = self.rec.energy_field(self.q, self.lab)
        return f + fr + self.selfc * self.lab

    def induced_field(self, v):
        """T v: the periodic, I-scaled, damped field of dipoles v at every atom."""
        Kr1 = self.erfc[1] - self.bare[1] + self.S * self.damp[1]
        Kr2 = self.erfc[2] - self.bare[2] + self.S * self.damp[2]
        f = pair_field(self.d, Kr1, Kr2, np.zeros(self.n), v)
        _, fr = self.rec.energy_field(np.zeros(self.n), v)
        return f + fr + self.selfc * v

    def solve(self, E=None, tol=1e-13, max_iter=10000):
        """Converged induced dipoles: CG on (I - S T S) y = S E, S = diag(sqrt(alpha)), mu = S y."""
        if E is None:
            E = self.fixed_field()
        s = np.sqrt(np.maximum(self.pol, 0.0))[:, None]
        b = s * E
        y = b.copy()
        r = b - (y - s * self.induced_field(s * y))
        p = r.copy()
        rr = float((r * r).sum())
        bb = max(float((b * b).sum()), 1e-300)
        for _ in range(max_iter):
            if rr <= tol * tol * bb:
                break
            Ap = p - s * self.induced_field(s * p)
            a = rr / float((p * Ap).sum())
            y += a * p
            r -= a * Ap
            rr_new = float((r * r).sum())
            p = r + (rr_new / rr) * p
            rr = rr_new
        return s * y, E

    # Energy and forces ------------------------------------------------------
    def direct(self) -> bool:
        return int(self.sys.polarization) == 0

    def evaluate(self, mu=None, E=None) -> EwaldResult:
        """Energy functional and forces at mu (the converged dipoles when None:
        the CG solution for Mutual, alpha E_M for Direct polarization)."""
        if mu is None:
            if self.direct():
                E = self.fixed_field()
                mu = self.pol[:, None] * E
            else:
                mu, E = self.solve()
        elif E is None:
            E = self.fixed_field()
        energy, forces, torque = self._energy_forces(self.q, self.lab, mu, induction=True)
        if self.direct():
            z = np.zeros(self.n)
            e_uu, f_uu, _ = self._energy_forces(z, np.zeros((self.n, 3)), mu, induction=False)
            energy -= e_uu
            forces = forces - f_uu
        forces = forces + map_torque(self.sys, torque)
        return EwaldResult(energy, forces, mu, self.lab.copy(), E, self.alpha, self.grid)

    def _energy_forces(self, q, p, mu, induction):
        """Energy, pair forces and the torques on p of multipoles (q, p) with
        induced dipoles mu (induction adds 1/2 mu.alpha^-1 mu)."""
        z = np.zeros(self.n)
        tot = p + mu
        M, S = self.M, self.S
        # Real space: erfc(T,T) - bare(T,T) + m bare(P,P) + m [damp(P,U) + damp(U,P)] + s damp(U,U),
        # as sums over ordered pairs (each unordered pair twice).
        terms = [
            (self.erfc, 1.0, (q, tot, q, tot), (tot, "T")),
            (self.bare, -1.0, (q, tot, q, tot), (tot, "T")),
            (tuple(M * k for k in self.bare), 1.0, (q, p, q, p), (p, "P")),
            (tuple(M * k for k in self.damp), 1.0, (q, p, z, mu), (mu, "U")),
            (tuple(M * k for k in self.damp), 1.0, (z, mu, q, p), (p, "P")),
            (tuple(S * k for k in self.damp), 1.0, (z, mu, z, mu), (mu, "U")),
        ]
        e_real = 0.0
        f_real = np.zeros((self.n, 3))
        eff = np.zeros((self.n, 3))     # -dU/dp_i
        for K, sign, (qi, di, qj, dj), _ in terms:
            e, fi, fld = pair_energy_force(self.d, K, qi, di, qj, dj)
            e_real += sign * 0.5 * e
            # Forces: each ordered pair gives the force on i; the unordered pair energy is
            # half the ordered sum, and the (j, i) term supplies the force on j.
            f_real += sign * fi
        # -dU/dp_i: fields at i acting on the permanent dipole of i.
        eff += pair_field(self.d, self.erfc[1] - self.bare[1] + M * self.bare[1],
                          self.erfc[2] - self.bare[2] + M * self.bare[2], q, p)
        eff += pair_field(self.d, self.erfc[1] - self.bare[1] + M * self.damp[1],
                          self.erfc[2] - self.bare[2] + M * self.damp[2], z, mu)
        e_rec, f_rec_field = self.rec.energy_field(q, tot)
        f_rec = self.rec.forces(q, tot)
        eff += f_rec_field + self.selfc * tot
        Q = float(q.sum())
        V = float(np.prod(self.box))
        e_self = -self.alpha / SQRT_PI * float((q * q).sum()) - 2.0 * self.alpha ** 3 / (3.0 * SQRT_PI) * float(
            (tot * tot).sum())
        e_plasma = -math.pi * Q * Q / (2.0 * V * self.alpha ** 2) if self.alpha > 0.0 else 0.0
        pos_mask = self.pol > 0
        e_ind = 0.5 * float((mu[pos_mask] ** 2 / self.pol[pos_mask, None]).sum()) if induction else 0.0
        energy = e_real + e_rec + e_self + e_plasma + e_ind
        return energy, f_real + f_rec, np.cross(p, eff)

    def energy_at(self, mu=None):
        return self.evaluate(mu).energy


def map_torque(sys, torque) -> np.ndarray:
    """Forces from per-atom torques through the reference's torque map (C oracle)."""
    return O.map_torque(sys, torque)


def variational_nocutoff(sys) -> EwaldResult:
    """The variational NoCutoff model (TDP_FLAG_VARIATIONAL): all pairs, bare kernels."""
    return Ewald(sys, 0.0, recip="none").evaluate()


def ewald(sys, alpha: Optional[float] = None, recip: str = "pme", **kw) -> EwaldResult:
    """Converged Ewald-mode evaluation of sys (alpha and grid from its cutoff and
    tolerance unless given)."""
    a, g = pme_parameters(sys.cutoff, sys.ewald_tolerance, sys.box)
    if alpha is None:
        alpha = a
    if recip == "pme" and kw.get("grid") is None:
        kw["grid"] = g
    return Ewald(sys, alpha, recip=recip, **kw).evaluate()
