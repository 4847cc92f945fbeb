"""Rigid-water molecular dynamics driven by the TholeDipoleForce kernels.

Velocity Verlet with 1 fs steps; each water (O, H1, H2 consecutive) is held
rigid by three distance constraints (SHAKE on positions, RATTLE on
velocities).  Forces are used as the force returns them: the reference's
energy unit is e^2/nm (Coulomb prefactor 1), and an OpenMM context would read
it as kJ/mol, so this integrator does the same.

* :class:`DeviceRigidWaterMD` keeps positions, velocities and forces in HBM and
  runs the whole step on the GPU (tdp_compute on device buffers plus the
  kernels of include/tholedipole_b200_md.h).
* :class:`HostRigidWaterMD` is the user-level loop through the public C ABI
  with host buffers: every step copies positions in and forces out, and the
  integration runs on the host in numpy.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _capi as A
from .kernel import CudaCalcTholeDipoleForceKernel
from .systems import HOH_ANGLE, MASS_H, MASS_O, OH_BOND, TholeSystem

KB = 0.0083144626  # kJ/(mol K)
D_OH = OH_BOND
D_HH = 2.0 * OH_BOND * np.sin(0.5 * HOH_ANGLE)
NS_PER_DAY_PER_STEP_PER_S = 1e-6 * 86400.0  # 1 fs steps


def maxwell_boltzmann(n_waters: int, temperature: float, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    m = np.tile([MASS_O, MASS_H, MASS_H], n_waters)
    v = rng.standard_normal((3 * n_waters, 3)) * np.sqrt(KB * temperature / m)[:, None]
    vcom = (m[:, None] * v).sum(0) / m.sum()
    return v - vcom


# Constraints of a rigid water (atoms O, H1, H2): k = 0 (O,H1), 1 (O,H2), 2 (H1,H2).
_PAIRS = ((0, 1), (0, 2), (1, 2))
_D = np.array([D_OH, D_OH, D_HH])
_INV_M = np.array([1.0 / MASS_O, 1.0 / MASS_H, 1.0 / MASS_H])


def _coupling() -> np.ndarray:
    """K[k, l]: how a multiplier of constraint l moves the bond vector of constraint k
    (x_a += g_l c_{a,l} r_l / m_a with c = +1 for the first atom of l, -1 for the second)."""
    c = np.zeros((3, 3))
    for l, (a, b) in enumerate(_PAIRS):
        c[a, l] = 1.0
        c[b, l] = -1.0
    K = np.zeros((3, 3))
    for k, (a, b) in enumerate(_PAIRS):
        K[k] = c[a] * _INV_M[a] - c[b] * _INV_M[b]
    return K


_K = _coupling()


def _bonds(xw: np.ndarray) -> np.ndarray:
    """(nw, 3 constraints, 3) bond vectors x_a - x_b."""
    return np.stack([xw[:, a] - xw[:, b] for a, b in _PAIRS], axis=1)


def _apply(xw: np.ndarray, g: np.ndarray, r: np.ndarray, scale: float = 1.0) -> None:
    """x_a += scale g_l c_{a,l} r_l / m_a for the three constraints of every water."""
    for l, (a, b) in enumerate(_PAIRS):
        d = (scale * g[:, l])[:, None] * r[:, l]
        xw[:, a] += _INV_M[a] * d
        xw[:, b] -= _INV_M[b] * d


def _rattle_host(x: np.ndarray, v: np.ndarray, iters: int = 200, tol: float = 1e-12) -> None:
    """Project water velocities onto the rigid constraints (numpy, in place): the
    three conditions s_k.(v_a - v_b) = 0 are linear in the multipliers, one 3x3
    solve per water."""
    xw = x.reshape(-1, 3, 3)
    vw = v.reshape(-1, 3, 3)
    s = _bonds(xw)
    w = _bonds(vw)
    A = _K[None, :, :] * np.einsum("nkc,nlc->nkl", s, s)
    rhs = -np.einsum("nkc,nkc->nk", s, w)
    h = np.linalg.solve(A, rhs[..., None])[..., 0]
    _apply(vw, h, s)


def _shake_host(x0: np.ndarray, x: np.ndarray, v: np.ndarray, dt: float, iters: int = 50, tol: float = 1e-12):
    """Positions onto the rigid constraints (SHAKE with the old bond vectors r0),
    solving each water's three constraints together by Newton's method, with the
    matching velocity correction (numpy, in place)."""
    x0w = x0.reshape(-1, 3, 3)
    xw = x.reshape(-1, 3, 3)
    vw = v.reshape(-1, 3, 3)
    r0 = _bonds(x0w)
    s_free = _bonds(xw)
    g = np.zeros((xw.shape[0], 3))
    for _ in range(iters):
        s = s_free + np.einsum("kl,nl,nlc->nkc", _K, g, r0)
        sig = np.einsum("nkc,nkc->nk", s, s) - _D[None, :] ** 2
        if not sig.size or float(np.max(np.abs(sig) / _D[None, :] ** 2)) < tol:
            break
        J = 2.0 * _K[None, :, :] * np.einsum("nkc,nlc->nkl", s, r0)
        g -= np.linalg.solve(J, sig[..., None])[..., 0]
    _apply(xw, g, r0)
    _apply(vw, g, r0, 1.0 / dt)


class DeviceRigidWaterMD:
    """Everything on the GPU; positions/velocities/forces are torch CUDA tensors."""

    def __init__(self, system: TholeSystem, precision="mixed", dt: float = 0.001, temperature: float = 300.0,
                 seed: int = 0, warm_start: bool = True, device: str = "cuda:0", ewald: bool = False):
        import torch

        self.torch = torch
        self.n = system.n
        self.nw = system.n // 3
        self.dt = dt
        self.dev = torch.device(device)
        self.lib = A.lib()
        self.kernel = CudaCalcTholeDipoleForceKernel(system, precision=precision, warm_start=warm_start, ewald=ewald)
        self.stream = torch.cuda.current_stream(self.dev)
        self.kernel.setStream(self.stream.cuda_stream)
        self.pos = torch.tensor(system.positions, dtype=torch.float64, device=self.dev).contiguous()
        self.vel = torch.tensor(maxwell_boltzmann(self.nw, temperature, seed), dtype=torch.float64,
                                device=self.dev).contiguous()
        self.frc = torch.zeros_like(self.pos)
        self._ke = torch.zeros(1, dtype=torch.float64, device=self.dev)
        self._chk(self.lib.tdp_md_constrain_velocities(self.nw, D_OH, D_HH, MASS_O, MASS_H, self._p(self.pos),
                                                       self._p(self.vel), self._s()))
        self.energy = self._forces()
        self.steps = 0

    def _p(self, t):
        return C.c_void_p(t.data_ptr())

    def _s(self):
        return C.c_void_p(self.stream.cuda_stream)

    def _chk(self, rc):
        A.check(rc, None)

    def _forces(self) -> float:
        self.frc.zero_()
        return self.kernel.execute_device(self.pos.data_ptr(), A.F64, self.frc.data_ptr(), A.F64)

    def step(self, n: int = 1) -> float:
        for _ in range(n):
            self._chk(self.lib.tdp_md_kick_drift(self.nw, D_OH, D_HH, MASS_O, MASS_H, self.dt, self._p(self.pos),
                                                 self._p(self.vel), self._p(self.frc), self._s()))
            self.energy = self._forces()
            self._chk(self.lib.tdp_md_kick(self.nw, D_OH, D_HH, MASS_O, MASS_H, self.dt, self._p(self.pos),
                                           self._p(self.vel), self._p(self.frc), self._s()))
            self.steps += 1
        return self.energy

    def kinetic_energy(self) -> float:
        self._chk(self.lib.tdp_md_kinetic_energy(self.nw, MASS_O, MASS_H, self._p(self.vel), self._p(self._ke),
                                                 self._s()))
        return float(self._ke.item())

    def temperature(self) -> float:
        dof = 6 * self.nw - 3  # rigid waters, centre of mass removed
        return 2.0 * self.kinetic_energy() / (dof * KB)

    def close(self):
        self.kernel.close()


class HostRigidWaterMD:
    """The same integrator as a user-level loop over host arrays: each step
    hands host positions to the C ABI and reads forces back."""

    def __init__(self, system: TholeSystem, precision="mixed", dt: float = 0.001, temperature: float = 300.0,
                 seed: int = 0, warm_start: bool = True, pinned: Optional[np.ndarray] = None, ewald: bool = False):
        self.n = system.n
        self.nw = system.n // 3
        self.dt = dt
        self.kernel = CudaCalcTholeDipoleForceKernel(system, precision=precision, warm_start=warm_start, ewald=ewald)
        self.pos = np.array(system.positions, dtype=np.float64) if pinned is None else pinned
        if pinned is not None:
            self.pos[...] = system.positions
        self.vel = maxwell_boltzmann(self.nw, temperature, seed)
        self.inv_m = 1.0 / np.tile([MASS_O, MASS_H, MASS_H], self.nw)[:, None]
        _rattle_host(self.pos, self.vel)
        self.frc = np.zeros((self.n, 3))
        self.energy, _ = self.kernel.execute(self.pos, forces=self.frc)
        self.steps = 0

    def step(self, n: int = 1) -> float:
        for _ in range(n):
            self.vel += 0.5 * self.dt * self.frc * self.inv_m
            x0 = self.pos.copy()
            self.pos += self.dt * self.vel
            _shake_host(x0, self.pos, self.vel, self.dt)
            self.frc[...] = 0.0
            self.energy, _ = self.kernel.execute(self.pos, forces=self.frc)
            self.vel += 0.5 * self.dt * self.frc * self.inv_m
            _rattle_host(self.pos, self.vel)
            self.steps += 1
        return self.energy

    def close(self):
        self.kernel.close()
