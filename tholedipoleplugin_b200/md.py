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


def _bonds(xw: np.ndarray) -> np.ndarray:
    """(nw, 3 constraints, 3) bond vectors x_a - x_b."""
    return np.stack([xw[:, a] - xw[:, b] for a, b in _PAIRS], axis=1)


def host_kick_drift(pos: np.ndarray, vel: np.ndarray, frc: np.ndarray, dt: float) -> None:
    """v += dt/2 F/m, x += dt v, SHAKE back onto the rigid-water constraints
    (tdp_md_host_kick_drift: the device step's arithmetic on host threads)."""
    for a in (pos, vel, frc):
        assert a.dtype == np.float64 and a.flags.c_contiguous
    A.check(A.lib().tdp_md_host_kick_drift(pos.shape[0] // 3, D_OH, D_HH, MASS_O, MASS_H, dt,
                                           pos.ctypes.data_as(C.c_void_p), vel.ctypes.data_as(C.c_void_p),
                                           frc.ctypes.data_as(C.c_void_p)), None)


def host_kick(pos: np.ndarray, vel: np.ndarray, frc: Optional[np.ndarray], dt: float) -> None:
    """v += dt/2 F/m (skipped for frc None), then RATTLE (tdp_md_host_kick)."""
    for a in (pos, vel) + ((frc,) if frc is not None else ()):
        assert a.dtype == np.float64 and a.flags.c_contiguous
    fp = frc.ctypes.data_as(C.c_void_p) if frc is not None else None
    A.check(A.lib().tdp_md_host_kick(pos.shape[0] // 3, D_OH, D_HH, MASS_O, MASS_H, dt,
                                     pos.ctypes.data_as(C.c_void_p), vel.ctypes.data_as(C.c_void_p), fp), None)


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
    hands host positions to the C ABI and reads forces back.  The half steps
    (kick, drift, SHAKE/RATTLE) run on host threads (tdp_md_host_*)."""

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
        host_kick(self.pos, self.vel, None, 0.0)
        self.frc = np.zeros((self.n, 3))
        self.energy, _ = self.kernel.execute(self.pos, forces=self.frc)
        self.steps = 0

    def step(self, n: int = 1) -> float:
        for _ in range(n):
            host_kick_drift(self.pos, self.vel, self.frc, self.dt)
            self.frc[...] = 0.0
            self.energy, _ = self.kernel.execute(self.pos, forces=self.frc)
            host_kick(self.pos, self.vel, self.frc, self.dt)
            self.steps += 1
        return self.energy

    def close(self):
        self.kernel.close()
