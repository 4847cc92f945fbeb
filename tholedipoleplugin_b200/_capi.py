"""ctypes binding of the C ABI in include/tholedipole_b200.h.

The shared library is built in-tree (tholedipoleplugin_b200/build.py) and
loaded from this package directory.  There is no fallback: if the library is
missing or fails to load, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtholedipole_b200.so")

TDP_OK = 0
TDP_ERR_INVALID_ARGUMENT, TDP_ERR_CUDA, TDP_ERR_NOT_PME, TDP_ERR_SIZE_MISMATCH = -1, -2, -3, -4
TDP_ERR_BOX_TOO_SMALL, TDP_ERR_NOT_CONVERGED, TDP_ERR_NON_FINITE, TDP_ERR_UNSUPPORTED = -5, -6, -7, -8
ERRORS = {
    -1: "invalid argument", -2: "CUDA error", -3: "not PME", -4: "size mismatch", -5: "box too small",
    -6: "not converged", -7: "non-finite", -8: "unsupported",
}
PRECISION_MIXED, PRECISION_DOUBLE = 0, 1
SOLVER_CG, SOLVER_JACOBI = 0, 1
FLAG_DD_FORCE_R4 = 1 << 0
FLAG_WARM_START = 1 << 1
FLAG_EWALD = 1 << 2
FLAG_VARIATIONAL = 1 << 3
NUM_STAGE_TIMES = 14
COMPUTE_FORCES, COMPUTE_ENERGY, COMPUTE_REQUIRE_CONVERGENCE = 1, 2, 4
F64, F32 = 0, 1
DIPOLES_INDUCED, DIPOLES_LAB_PERMANENT, DIPOLES_TOTAL = 0, 1, 2
STATUS_CONVERGED, STATUS_MAX_ITERATIONS, STATUS_NON_FINITE = 0, 1, 2

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


class SystemDesc(C.Structure):
    _fields_ = [
        ("num_particles", C.c_int32),
        ("charges", _dp), ("molecular_dipoles", _dp), ("polarizabilities", _dp), ("thole_damping", _dp),
        ("axis_types", _ip), ("atom_z", _ip), ("atom_x", _ip), ("atom_y", _ip),
        ("covalent12_offsets", _ip), ("covalent12_atoms", _ip),
        ("covalent13_offsets", _ip), ("covalent13_atoms", _ip),
        ("nonbonded_method", C.c_int32), ("polarization_type", C.c_int32),
        ("cutoff", C.c_double), ("ewald_error_tolerance", C.c_double), ("pme_alpha", C.c_double),
        ("pme_grid", C.c_int32 * 3),
        ("mutual_target_epsilon", C.c_double), ("mutual_max_iterations", C.c_int32),
        ("num_extrapolation_coefficients", C.c_int32), ("extrapolation_coefficients", _dp),
        ("precision", C.c_int32), ("solver", C.c_int32), ("flags", C.c_uint32),
    ]


class TdpError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{message} [{ERRORS.get(code, code)}]")
        self.code = code


_lib: Optional[C.CDLL] = None

# name: (restype, argtypes)
PROTOTYPES = {
    "tdp_abi_version": (C.c_int, []),
    "tdp_last_error": (C.c_char_p, [C.c_void_p]),
    "tdp_create": (C.c_int, [C.POINTER(SystemDesc), C.POINTER(C.c_void_p)]),
    "tdp_destroy": (None, [C.c_void_p]),
    "tdp_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "tdp_set_box": (C.c_int, [C.c_void_p, _dp]),
    "tdp_update_params": (C.c_int, [C.c_void_p, C.c_int32, _dp, _dp, _dp, _dp, _ip, _ip, _ip, _ip]),
    "tdp_compute": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_int32, _dp,
                              C.c_uint32]),
    "tdp_compute_openmm": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_void_p, _dp,
                                     C.c_uint32]),
    "tdp_get_dipoles": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_int32, _dp]),
    "tdp_get_potential": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, _dp, C.c_int32, _dp]),
    "tdp_get_moments": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, _dp, _dp]),
    "tdp_potential_noalloc": (C.c_int, [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p,
                                        C.c_int32, _dp, C.c_void_p, C.c_void_p]),
    "tdp_get_pme_parameters": (C.c_int, [C.c_void_p, _dp, _ip, _ip, _ip]),
    "tdp_solver_stats": (C.c_int, [C.c_void_p, _ip, _dp, _ip, _ip]),
    "tdp_solver_history": (C.c_int, [C.c_void_p, _dp, C.c_int32, _ip]),
    "tdp_adjoint": (C.c_int, [C.c_void_p, C.c_void_p, C.c_double, _dp]),
    "tdp_adjoint_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_double, C.c_void_p]),
    "tdp_update_particle_params": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                             C.c_int32]),
    "tdp_enable_timing": (C.c_int, [C.c_void_p, C.c_int32]),
    "tdp_stage_times": (C.c_int, [C.c_void_p, _dp]),
    "tdp_md_kick_drift": (C.c_int, [C.c_int32, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                                    C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "tdp_md_kick": (C.c_int, [C.c_int32, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                              C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "tdp_md_constrain_velocities": (C.c_int, [C.c_int32, C.c_double, C.c_double, C.c_double, C.c_double,
                                              C.c_void_p, C.c_void_p, C.c_void_p]),
    "tdp_md_kinetic_energy": (C.c_int, [C.c_int32, C.c_double, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p]),
    "tdp_md_host_kick_drift": (C.c_int, [C.c_int32, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                                         C.c_void_p, C.c_void_p, C.c_void_p]),
    "tdp_md_host_kick": (C.c_int, [C.c_int32, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                                   C.c_void_p, C.c_void_p, C.c_void_p]),
    "tdp_batch_create": (C.c_int, [C.POINTER(SystemDesc), C.c_int32, _ip, C.POINTER(C.c_void_p)]),
    "tdp_batch_destroy": (None, [C.c_void_p]),
    "tdp_batch_last_error": (C.c_char_p, [C.c_void_p]),
    "tdp_batch_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "tdp_batch_compute": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]),
    "tdp_batch_get_induced_dipoles": (C.c_int, [C.c_void_p, _dp]),
    "tdp_batch_solver_stats": (C.c_int, [C.c_void_p, _ip, _dp]),
    "tdp_batch_tile": (C.c_int, [C.c_void_p, _ip, _ip, _ip, _dp]),
    "tdp_batch_tile_candidates": (C.c_int, [C.c_void_p, C.c_int32, _ip, _ip, _dp]),
    "tdp_batch_update_params": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32]),
    "tdp_batch_adjoint": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]),
    "tdp_batch_adjoint_stats": (C.c_int, [C.c_void_p, _ip, _dp]),
}


def declared_symbols():
    """Entry points declared in include/*.h (parsed from the headers)."""
    import glob
    import re
    names = set()
    inc = os.path.join(os.path.dirname(HERE), "include")
    for path in glob.glob(os.path.join(inc, "*.h")):
        text = open(path).read()
        names.update(re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(tdp\w+)\s*\(", text, re.M))
    return sorted(names)


def lib() -> C.CDLL:
    """Load the in-tree library; raise if it is absent (no fallback path exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run tholedipoleplugin_b200/build.py (nvcc, sm_100a)")
        l = C.CDLL(LIB_PATH)
        for name, (res, args) in PROTOTYPES.items():
            fn = getattr(l, name)
            fn.restype = res
            fn.argtypes = args
        _lib = l
    return _lib


def check(rc: int, handle=None) -> None:
    if rc != TDP_OK:
        msg = lib().tdp_last_error(handle)
        raise TdpError(rc, msg.decode() if msg else "")
