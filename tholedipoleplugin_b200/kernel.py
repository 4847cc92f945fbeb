"""Python front end of the CUDA kernel object.

:class:`CudaCalcTholeDipoleForceKernel` mirrors the abstract kernel interface
of the reference plugin, CalcTholeDipoleForceKernel
(openmmapi/include/TholeDipoleKernels.h:46-122): ``initialize``, ``execute``,
``copyParametersToContext``, ``getPMEParameters``, ``getInducedDipoles``,
``getLabFramePermanentDipoles``, ``getTotalDipoles``,
``getElectrostaticPotential`` and ``getSystemMultipoleMoments`` -- each a thin
call into the C ABI of include/tholedipole_b200.h.  Errors raise
:class:`TdpError` where the reference throws OpenMMException.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence, Tuple

import numpy as np

from . import _capi as A
from .systems import PME, TholeSystem

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def _iptr(a: np.ndarray):
    return a.ctypes.data_as(_ip)


class _DescBuffers:
    """numpy buffers that a SystemDesc points into (kept alive with it)."""

    def __init__(self, s: TholeSystem, precision: int, solver: int, flags: int):
        n = s.n
        self.q = np.ascontiguousarray(s.charges, dtype=np.float64)
        self.d = np.ascontiguousarray(np.asarray(s.dipoles, dtype=np.float64).reshape(n, 3))
        self.a = np.ascontiguousarray(s.polarizabilities, dtype=np.float64)
        self.t = np.ascontiguousarray(s.tholes, dtype=np.float64)
        ax = np.asarray(s.axis, dtype=np.int32).reshape(n, 4)
        self.types = np.ascontiguousarray(ax[:, 0])
        self.z = np.ascontiguousarray(ax[:, 1])
        self.x = np.ascontiguousarray(ax[:, 2])
        self.y = np.ascontiguousarray(ax[:, 3])
        o12, c12 = s.cov12_csr()
        o13, c13 = s.cov13_csr()
        self.o12, self.c12 = o12.astype(np.int32), np.append(c12, -1).astype(np.int32)
        self.o13, self.c13 = o13.astype(np.int32), np.append(c13, -1).astype(np.int32)
        ex = list(s.extrap) if s.extrap is not None else []
        self.ex = np.array(ex + [0.0], dtype=np.float64)
        desc = A.SystemDesc()
        desc.num_particles = n
        desc.charges, desc.molecular_dipoles = _dptr(self.q), _dptr(self.d)
        desc.polarizabilities, desc.thole_damping = _dptr(self.a), _dptr(self.t)
        desc.axis_types, desc.atom_z = _iptr(self.types), _iptr(self.z)
        desc.atom_x, desc.atom_y = _iptr(self.x), _iptr(self.y)
        desc.covalent12_offsets, desc.covalent12_atoms = _iptr(self.o12), _iptr(self.c12)
        desc.covalent13_offsets, desc.covalent13_atoms = _iptr(self.o13), _iptr(self.c13)
        desc.nonbonded_method = int(s.method)
        desc.polarization_type = int(s.polarization)
        desc.cutoff = float(s.cutoff)
        desc.ewald_error_tolerance = float(s.ewald_tolerance)
        desc.pme_alpha = 0.0
        desc.mutual_target_epsilon = float(s.target_eps)
        desc.mutual_max_iterations = int(s.max_iter)
        desc.num_extrapolation_coefficients = len(ex)
        desc.extrapolation_coefficients = _dptr(self.ex)
        desc.precision = precision
        desc.solver = solver
        desc.flags = flags
        self.desc = desc


def _precision(p) -> int:
    if isinstance(p, int):
        return p
    return {"mixed": A.PRECISION_MIXED, "double": A.PRECISION_DOUBLE}[p]


def _solver(s) -> int:
    if isinstance(s, int):
        return s
    return {"cg": A.SOLVER_CG, "jacobi": A.SOLVER_JACOBI}[s]


class CudaCalcTholeDipoleForceKernel:
    """One TholeDipoleForce evaluated on the GPU (reference semantics)."""

    Name = "CalcTholeDipoleForce"

    def __init__(self, system: TholeSystem, precision="mixed", solver="cg", dd_force_r4: bool = False,
                 warm_start: bool = False, ewald: bool = False, variational: bool = False):
        """``ewald=True`` (PME systems only) runs the library's Ewald mode
        (TDP_FLAG_EWALD: neighbour-list real space + smooth PME) instead of the
        reference's minimum-image all-pairs sum; ``variational=True`` (NoCutoff
        systems only, TDP_FLAG_VARIATIONAL) gives the variational energy and its
        exact gradient over all pairs."""
        self._lib = A.lib()
        self.n = system.n
        self.method = int(system.method)
        flags = ((A.FLAG_DD_FORCE_R4 if dd_force_r4 else 0) | (A.FLAG_WARM_START if warm_start else 0)
                 | (A.FLAG_EWALD if ewald else 0) | (A.FLAG_VARIATIONAL if variational else 0))
        self._buf = _DescBuffers(system, _precision(precision), _solver(solver), flags)
        h = C.c_void_p()
        A.check(self._lib.tdp_create(C.byref(self._buf.desc), C.byref(h)), None)
        self._h = h
        self.positions = np.ascontiguousarray(system.positions, dtype=np.float64).reshape(self.n, 3)
        if system.method == PME:
            self.setBox(system.box)

    # -- lifetime -----------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.tdp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    def _check(self, rc):
        A.check(rc, self._h)

    # -- configuration --------------------------------------------------------
    def setBox(self, box) -> None:
        b = np.asarray(box, dtype=np.float64)
        if b.size == 3:
            b = np.diag(b)
        b = np.ascontiguousarray(b.reshape(9))
        self._check(self._lib.tdp_set_box(self._h, _dptr(b)))

    def setStream(self, stream_ptr: int) -> None:
        self._check(self._lib.tdp_set_stream(self._h, C.c_void_p(stream_ptr)))

    def copyParametersToContext(self, system: TholeSystem) -> None:
        """updateParametersInContext (ReferenceTholeDipoleKernels.cpp:317-339)."""
        b = _DescBuffers(system, 0, 0, 0)
        self._check(self._lib.tdp_update_params(self._h, system.n, _dptr(b.q), _dptr(b.d), _dptr(b.a), _dptr(b.t),
                                                _iptr(b.types), _iptr(b.z), _iptr(b.x), _iptr(b.y)))

    def updateParticleParams(self, charges, dipoles, polarizabilities, tholes) -> None:
        """Per-particle parameters only (axis frames and covalent maps stay):
        host arrays, or contiguous float64 CUDA torch tensors, which then never
        leave the device."""
        arrs = [charges, dipoles, polarizabilities, tholes]
        if all(getattr(a, "is_cuda", False) for a in arrs):
            for a in arrs:
                assert a.dtype.itemsize == 8 and a.is_contiguous()
            rc = self._lib.tdp_update_particle_params(self._h, *[C.c_void_p(a.data_ptr()) for a in arrs], 1)
        else:
            hs = [np.ascontiguousarray(np.asarray(a, dtype=np.float64)) for a in arrs]
            rc = self._lib.tdp_update_particle_params(self._h, *[h.ctypes.data_as(C.c_void_p) for h in hs], 0)
        self._check(rc)

    def enableTiming(self, on: bool = True) -> None:
        self._check(self._lib.tdp_enable_timing(self._h, 1 if on else 0))

    # -- evaluation -----------------------------------------------------------
    def _pos(self, positions):
        if positions is None:
            return self.positions
        p = np.ascontiguousarray(np.asarray(positions, dtype=np.float64).reshape(self.n, 3))
        self.positions = p
        return p

    def execute(self, positions=None, include_forces: bool = True, include_energy: bool = True,
                forces: Optional[np.ndarray] = None, require_convergence: bool = False) -> Tuple[float, np.ndarray]:
        """Energy and forces for host positions; forces are ADDED to ``forces``
        (zeros if None), as the reference adds into the context force array."""
        p = self._pos(positions)
        f = np.zeros((self.n, 3)) if forces is None else forces
        assert f.dtype == np.float64 and f.flags.c_contiguous
        e = C.c_double(0.0)
        flags = (A.COMPUTE_FORCES if include_forces else 0) | (A.COMPUTE_ENERGY if include_energy else 0)
        if require_convergence:
            flags |= A.COMPUTE_REQUIRE_CONVERGENCE
        self._check(self._lib.tdp_compute(self._h, p.ctypes.data_as(C.c_void_p), A.F64, 0,
                                          f.ctypes.data_as(C.c_void_p), A.F64, C.byref(e), flags))
        return e.value, f

    def execute_device(self, pos_ptr: int, pos_dtype: int, forces_ptr: int, force_dtype: int,
                       include_forces: bool = True) -> float:
        """Device-resident positions/forces (raw CUDA pointers, e.g. torch data_ptr())."""
        e = C.c_double(0.0)
        flags = (A.COMPUTE_FORCES if include_forces else 0) | A.COMPUTE_ENERGY
        self._check(self._lib.tdp_compute(self._h, C.c_void_p(pos_ptr), pos_dtype, 1, C.c_void_p(forces_ptr),
                                          force_dtype, C.byref(e), flags))
        return e.value

    def solveDevice(self, pos_ptr: int, pos_dtype: int, out: np.ndarray) -> None:
        """Rotation, permanent field and induced-dipole solve at device-resident
        positions (a raw CUDA pointer); the induced dipoles land in ``out``."""
        assert out.dtype == np.float64 and out.flags.c_contiguous and out.size == 3 * self.n
        self._check(self._lib.tdp_get_dipoles(self._h, A.DIPOLES_INDUCED, C.c_void_p(pos_ptr), pos_dtype, 1,
                                              _dptr(out)))

    def _dipoles(self, which, positions):
        p = self._pos(positions)
        out = np.zeros((self.n, 3))
        self._check(self._lib.tdp_get_dipoles(self._h, which, p.ctypes.data_as(C.c_void_p), A.F64, 0, _dptr(out)))
        return out

    def getInducedDipoles(self, positions=None) -> np.ndarray:
        return self._dipoles(A.DIPOLES_INDUCED, positions)

    def getLabFramePermanentDipoles(self, positions=None) -> np.ndarray:
        return self._dipoles(A.DIPOLES_LAB_PERMANENT, positions)

    def getTotalDipoles(self, positions=None) -> np.ndarray:
        return self._dipoles(A.DIPOLES_TOTAL, positions)

    def getElectrostaticPotential(self, grid, positions=None) -> np.ndarray:
        p = self._pos(positions)
        g = np.ascontiguousarray(np.asarray(grid, dtype=np.float64).reshape(-1, 3))
        out = np.zeros(g.shape[0])
        self._check(self._lib.tdp_get_potential(self._h, p.ctypes.data_as(C.c_void_p), A.F64, 0, _dptr(g),
                                                g.shape[0], _dptr(out)))
        return out

    def getSystemMultipoleMoments(self, masses, positions=None) -> np.ndarray:
        p = self._pos(positions)
        m = np.ascontiguousarray(np.asarray(masses, dtype=np.float64))
        out = np.zeros(13)
        self._check(self._lib.tdp_get_moments(self._h, p.ctypes.data_as(C.c_void_p), A.F64, 0, _dptr(m),
                                              _dptr(out)))
        return out

    def getPMEParameters(self):
        a = C.c_double()
        nx, ny, nz = C.c_int32(), C.c_int32(), C.c_int32()
        self._check(self._lib.tdp_get_pme_parameters(self._h, C.byref(a), C.byref(nx), C.byref(ny), C.byref(nz)))
        return a.value, nx.value, ny.value, nz.value

    def adjoint(self, dL_dF=None, dL_dE: float = 0.0) -> np.ndarray:
        """Per-particle gradients (dq, dalpha, dthole, dmu_mol[3]) of
        dL_dE * E + sum dL_dF . F at the last execute()'s positions."""
        out = np.zeros((self.n, 6))
        g = None if dL_dF is None else np.ascontiguousarray(np.asarray(dL_dF, dtype=np.float64).reshape(self.n, 3))
        self._check(self._lib.tdp_adjoint(self._h, None if g is None else g.ctypes.data_as(C.c_void_p),
                                          float(dL_dE), _dptr(out)))
        return out

    def adjoint_device(self, dL_dF_ptr: int, dL_dE: float, grads_ptr: int) -> None:
        """tdp_adjoint on device memory: dL_dF (n*3, 0 = zero) and grads (n*6) are
        raw CUDA pointers."""
        self._check(self._lib.tdp_adjoint_device(self._h, C.c_void_p(dL_dF_ptr or None), float(dL_dE),
                                                 C.c_void_p(grads_ptr)))

    def solverStats(self):
        it, conv, st = C.c_int32(), C.c_int32(), C.c_int32()
        eps = C.c_double()
        self._check(self._lib.tdp_solver_stats(self._h, C.byref(it), C.byref(eps), C.byref(conv), C.byref(st)))
        return {"iterations": it.value, "epsilon": eps.value, "converged": conv.value, "status": st.value}

    def solverHistory(self) -> np.ndarray:
        """Stopping quantity at every step of the last Mutual solve (start,
        iterations, true-residual checks), oldest first."""
        cnt = C.c_int32()
        self._check(self._lib.tdp_solver_history(self._h, None, 0, C.byref(cnt)))
        out = np.zeros(max(cnt.value, 1))
        self._check(self._lib.tdp_solver_history(self._h, _dptr(out), cnt.value, C.byref(cnt)))
        return out[:cnt.value]

    def stageTimes(self) -> Sequence[float]:
        out = np.zeros(A.NUM_STAGE_TIMES)
        self._check(self._lib.tdp_stage_times(self._h, _dptr(out)))
        return out
