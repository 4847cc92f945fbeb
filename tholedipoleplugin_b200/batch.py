"""Cluster batches: many isolated (NoCutoff) TholeDipoleForce systems
evaluated in one persistent GPU launch (tdp_batch_* in
include/tholedipole_b200.h).

Each cluster is evaluated with exactly the per-system semantics of
:class:`~tholedipoleplugin_b200.kernel.CudaCalcTholeDipoleForceKernel` (the
reference's ReferenceCalcTholeDipoleForceKernel::execute,
platforms/reference/src/ReferenceTholeDipoleKernels.cpp), but the batch has no
reference counterpart: the reference evaluates one System per context.
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import _capi as A
from .kernel import _DescBuffers, _precision
from .systems import TholeSystem, concat_clusters


class ClusterBatch:
    """All clusters' particles concatenated; cluster c owns particles
    ``offsets[c]:offsets[c+1]``.  ``compute`` returns per-cluster energies and
    the forces of every particle (torque mapping included)."""

    def __init__(self, clusters: Sequence[TholeSystem], precision="mixed", dd_force_r4: bool = False):
        self._lib = A.lib()
        self.system, self.offsets = concat_clusters(clusters)
        self.n = self.system.n
        self.num_clusters = len(clusters)
        flags = A.FLAG_DD_FORCE_R4 if dd_force_r4 else 0
        self._buf = _DescBuffers(self.system, _precision(precision), A.SOLVER_CG, flags)
        self._offs = np.ascontiguousarray(self.offsets, dtype=np.int32)
        h = C.c_void_p()
        rc = self._lib.tdp_batch_create(C.byref(self._buf.desc), self.num_clusters,
                                        self._offs.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(h))
        self._check(rc, None)
        self._h = h
        self.positions = np.ascontiguousarray(self.system.positions, dtype=np.float64).reshape(self.n, 3)

    def _check(self, rc: int, h) -> None:
        if rc != A.TDP_OK:
            msg = self._lib.tdp_batch_last_error(h)
            raise A.TdpError(rc, msg.decode() if msg else "")

    # -- lifetime -----------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.tdp_batch_destroy(self._h)
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

    # -- evaluation ---------------------------------------------------------
    def setStream(self, stream) -> None:
        ptr = stream if isinstance(stream, int) else getattr(stream, "cuda_stream", 0)
        self._check(self._lib.tdp_batch_set_stream(self._h, C.c_void_p(ptr)), self._h)

    def compute(self, positions: Optional[np.ndarray] = None):
        """(energies[num_clusters], forces[n, 3]) at ``positions`` (host, nm)."""
        if positions is not None:
            self.positions = np.ascontiguousarray(positions, dtype=np.float64).reshape(self.n, 3)
        forces = np.zeros((self.n, 3))
        energies = np.zeros(self.num_clusters)
        rc = self._lib.tdp_batch_compute(self._h, self.positions.ctypes.data_as(C.c_void_p), 0,
                                         forces.ctypes.data_as(C.c_void_p), energies.ctypes.data_as(C.c_void_p))
        self._check(rc, self._h)
        return energies, forces

    def compute_device(self, positions_ptr: int, forces_ptr: int, energies_ptr: int) -> None:
        """Device-resident call: all three are device pointers (n*3, n*3, num_clusters doubles)."""
        rc = self._lib.tdp_batch_compute(self._h, C.c_void_p(positions_ptr), 1, C.c_void_p(forces_ptr),
                                         C.c_void_p(energies_ptr))
        self._check(rc, self._h)

    def updateParams(self, charges, dipoles, polarizabilities, tholes) -> None:
        """New per-particle parameters (host numpy arrays, or CUDA torch tensors
        of float64 on this batch's device) for every cluster."""
        arrs = [charges, dipoles, polarizabilities, tholes]
        if all(hasattr(a, "data_ptr") and getattr(a, "is_cuda", False) for a in arrs):
            for a in arrs:
                assert a.dtype.itemsize == 8 and a.is_contiguous()
            rc = self._lib.tdp_batch_update_params(self._h, *[C.c_void_p(a.data_ptr()) for a in arrs], 1)
        else:
            hs = [np.ascontiguousarray(np.asarray(a, dtype=np.float64)) for a in arrs]
            rc = self._lib.tdp_batch_update_params(self._h, *[h.ctypes.data_as(C.c_void_p) for h in hs], 0)
        self._check(rc, self._h)

    def adjoint(self, dL_dF=None, dL_dE=None) -> np.ndarray:
        """Per-particle gradients (dq, dalpha, dthole, dmu_mol[3]) of
        sum_c dL_dE[c] E_c + sum_i dL_dF_i . F_i at the last compute (host arrays)."""
        out = np.zeros((self.n, 6))
        gF = None if dL_dF is None else np.ascontiguousarray(np.asarray(dL_dF, dtype=np.float64).reshape(self.n, 3))
        gE = None if dL_dE is None else np.ascontiguousarray(np.asarray(dL_dE, dtype=np.float64).reshape(-1))
        rc = self._lib.tdp_batch_adjoint(self._h, None if gF is None else gF.ctypes.data_as(C.c_void_p),
                                         None if gE is None else gE.ctypes.data_as(C.c_void_p), 0,
                                         out.ctypes.data_as(C.c_void_p))
        self._check(rc, self._h)
        return out

    def adjoint_device(self, dL_dF_ptr: int, dL_dE_ptr: int, grads_ptr: int) -> None:
        """Device-resident reverse pass: raw CUDA pointers (n*3, num_clusters,
        n*6 doubles); 0 for an absent cotangent."""
        rc = self._lib.tdp_batch_adjoint(self._h, C.c_void_p(dL_dF_ptr or None), C.c_void_p(dL_dE_ptr or None), 1,
                                         C.c_void_p(grads_ptr))
        self._check(rc, self._h)

    def adjointStats(self):
        it = np.zeros(self.num_clusters, dtype=np.int32)
        eps = np.zeros(self.num_clusters)
        self._check(self._lib.tdp_batch_adjoint_stats(self._h, it.ctypes.data_as(C.POINTER(C.c_int32)),
                                                      eps.ctypes.data_as(C.POINTER(C.c_double))), self._h)
        return it, eps

    def inducedDipoles(self) -> np.ndarray:
        out = np.zeros((self.n, 3))
        self._check(self._lib.tdp_batch_get_induced_dipoles(self._h, out.ctypes.data_as(C.POINTER(C.c_double))),
                    self._h)
        return out

    def solverStats(self):
        """(iterations[num_clusters], epsilons[num_clusters]) of the last compute."""
        it = np.zeros(self.num_clusters, dtype=np.int32)
        eps = np.zeros(self.num_clusters)
        self._check(self._lib.tdp_batch_solver_stats(self._h, it.ctypes.data_as(C.POINTER(C.c_int32)),
                                                     eps.ctypes.data_as(C.POINTER(C.c_double))), self._h)
        return it, eps

    def tile(self) -> Dict[str, float]:
        t, l, c = C.c_int32(), C.c_int32(), C.c_int32()
        ms = C.c_double()
        self._check(self._lib.tdp_batch_tile(self._h, C.byref(t), C.byref(l), C.byref(c), C.byref(ms)), self._h)
        return {"threads": t.value, "lanes": l.value, "ctas": c.value, "last_ms": ms.value}

    def tileCandidates(self) -> List[Dict[str, float]]:
        cap = 64
        t = np.zeros(cap, dtype=np.int32)
        l = np.zeros(cap, dtype=np.int32)
        ms = np.zeros(cap)
        k = self._lib.tdp_batch_tile_candidates(self._h, cap, t.ctypes.data_as(C.POINTER(C.c_int32)),
                                                l.ctypes.data_as(C.POINTER(C.c_int32)),
                                                ms.ctypes.data_as(C.POINTER(C.c_double)))
        return [{"threads": int(t[i]), "lanes": int(l[i]), "ms": float(ms[i])} for i in range(min(k, cap))]

    def cluster_slice(self, c: int) -> slice:
        return slice(int(self.offsets[c]), int(self.offsets[c + 1]))
