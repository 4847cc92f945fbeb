"""ctypes front end of the CPU oracle.  TEST INFRASTRUCTURE ONLY.

Two back ends share one C struct (oracle/tdp_oracle.h):

* ``port``      -- the plain-C FP64 restatement, oracle/_build/libtdp_oracle.so.
* ``reference`` -- the reference plugin's own ReferenceTholeDipoleForce.cpp,
  compiled unmodified by oracle/Makefile into oracle/_ref/libtdp_ref.so
  (present only where the reference source tree was available at build time).

Both compute the reference semantics of aehogan/tholedipoleplugin
(platforms/reference/src/ReferenceTholeDipoleForce.cpp): all-pairs interactions,
orthorhombic minimum image for the PME flag, Jacobi iteration for Mutual.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_LIB = os.path.join(HERE, "_build", "libtdp_oracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libtdp_ref.so")

RINV4_FILL, RINV4_POWER = 0, 1

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class _Sys(C.Structure):
    _fields_ = [
        ("n", C.c_int), ("pos", _dp), ("charge", _dp), ("dipole", _dp), ("polarity", _dp),
        ("thole", _dp), ("axis", _ip), ("cov12_off", _ip), ("cov12", _ip), ("cov13_off", _ip),
        ("cov13", _ip), ("method", C.c_int), ("box", C.c_double * 3), ("polarization", C.c_int),
        ("target_eps", C.c_double), ("max_iter", C.c_int), ("n_extrap", C.c_int), ("extrap", _dp),
        ("rinv4_mode", C.c_int), ("rinv4_value", C.c_double),
    ]


class _Stats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("epsilon", C.c_double), ("converged", C.c_int)]


# Where this build script looks for the reference plugin's source tree when
# TDP_REFERENCE_DIR is not set (the compiled reference is built only if the
# tree is there; without it the tests use the golden fixtures in tests/golden).
DEFAULT_REFERENCE_DIR = "/root/reference"


def reference_dir() -> Optional[str]:
    d = os.environ.get("TDP_REFERENCE_DIR", DEFAULT_REFERENCE_DIR)
    return d if os.path.isdir(d) else None


def build() -> None:
    """Compile the oracle libraries (oracle/Makefile): the restatement always,
    the compiled reference where its source tree is present."""
    cmd = ["make", "-s", "-C", HERE]
    ref = reference_dir()
    if ref:
        cmd.append(f"REF={ref}")
    subprocess.run(cmd, check=True)


_libs = {}


def _lib(which: str):
    if which not in _libs:
        path = PORT_LIB if which == "port" else REF_LIB
        if not os.path.exists(path):
            build()
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        lib = C.CDLL(path)
        _libs[which] = lib
    return _libs[which]


def reference_available() -> bool:
    try:
        _lib("reference")
        return True
    except (FileNotFoundError, OSError, subprocess.CalledProcessError):
        return False


def _p(a, t=_dp):
    return a.ctypes.data_as(t) if a is not None else None


@dataclass
class Result:
    energy: float
    forces: np.ndarray
    induced: Optional[np.ndarray] = None
    lab: Optional[np.ndarray] = None
    iterations: int = 0
    epsilon: float = 0.0
    converged: int = 0


class _Packed:
    """Keeps the numpy buffers alive while the C struct points at them."""

    def __init__(self, sys, rinv4_mode=RINV4_FILL, rinv4_value=0.0, polarization=None):
        n = sys.n
        self.pos = np.ascontiguousarray(sys.positions, dtype=np.float64).reshape(n, 3)
        self.q = np.ascontiguousarray(sys.charges, dtype=np.float64)
        self.d = np.ascontiguousarray(sys.dipoles, dtype=np.float64).reshape(n, 3)
        self.a = np.ascontiguousarray(sys.polarizabilities, dtype=np.float64)
        self.t = np.ascontiguousarray(sys.tholes, dtype=np.float64)
        self.ax = np.ascontiguousarray(sys.axis, dtype=np.int32).reshape(n, 4)
        self.c12o, self.c12 = sys.cov12_csr()
        self.c13o, self.c13 = sys.cov13_csr()
        self.c12 = np.ascontiguousarray(np.append(self.c12, -1), dtype=np.int32)
        self.c13 = np.ascontiguousarray(np.append(self.c13, -1), dtype=np.int32)
        ex = list(sys.extrap) if sys.extrap is not None else []
        self.ex = np.ascontiguousarray(np.array(ex + [0.0], dtype=np.float64))
        s = _Sys()
        s.n = n
        s.pos, s.charge, s.dipole = _p(self.pos), _p(self.q), _p(self.d)
        s.polarity, s.thole, s.axis = _p(self.a), _p(self.t), _p(self.ax, _ip)
        s.cov12_off, s.cov12 = _p(self.c12o, _ip), _p(self.c12, _ip)
        s.cov13_off, s.cov13 = _p(self.c13o, _ip), _p(self.c13, _ip)
        s.method = int(sys.method)
        for k in range(3):
            s.box[k] = float(sys.box[k])
        s.polarization = int(sys.polarization if polarization is None else polarization)
        s.target_eps = float(sys.target_eps)
        s.max_iter = int(sys.max_iter)
        s.n_extrap = len(ex)
        s.extrap = _p(self.ex)
        s.rinv4_mode = int(rinv4_mode)
        s.rinv4_value = float(rinv4_value)
        self.s = s


def _check(rc, what):
    if rc != 0:
        raise ValueError(f"oracle {what} rejected the input (code {rc})")


def compute(sys, backend: str = "port", rinv4_mode: int = RINV4_FILL, rinv4_value: float = 0.0,
            dipoles: bool = True) -> Result:
    """Energy, forces (added to zero), induced and lab-frame dipoles."""
    pk = _Packed(sys, rinv4_mode, rinv4_value)
    n = sys.n
    forces = np.zeros((n, 3))
    e = C.c_double(0.0)
    st = _Stats()
    if backend == "port":
        lib = _lib("port")
        mu = np.zeros((n, 3))
        lab = np.zeros((n, 3))
        _check(lib.tdpo_compute(C.byref(pk.s), C.byref(e), _p(forces), _p(mu), _p(lab), C.byref(st)), "compute")
        return Result(e.value, forces, mu, lab, st.iterations, st.epsilon, st.converged)
    if rinv4_mode != RINV4_FILL:
        raise ValueError("the compiled reference can only fill the rInvVec[4] word with a constant")
    lib = _lib("reference")
    lib.tdpref_compute.argtypes = [C.c_void_p, C.c_double, _dp, _dp, C.c_void_p]
    _check(lib.tdpref_compute(C.byref(pk.s), rinv4_value, C.byref(e), _p(forces), C.byref(st)), "compute")
    res = Result(e.value, forces, None, None, st.iterations, st.epsilon, st.converged)
    if dipoles:
        res.induced = induced_dipoles(sys, backend)[0]
        res.lab = lab_dipoles(sys, backend)
    return res


def compute_full(sys, rinv4_value: float = 0.0) -> Result:
    """Energy, forces and the induced dipoles of the same solve from the
    compiled reference (one calculateForceAndEnergy call, RTDF.cpp:100-127),
    plus the lab-frame dipoles (no solve)."""
    pk = _Packed(sys)
    n = sys.n
    forces = np.zeros((n, 3))
    mu = np.zeros((n, 3))
    e = C.c_double(0.0)
    st = _Stats()
    lib = _lib("reference")
    lib.tdpref_compute_full.argtypes = [C.c_void_p, C.c_double, _dp, _dp, _dp, C.c_void_p]
    _check(lib.tdpref_compute_full(C.byref(pk.s), rinv4_value, C.byref(e), _p(forces), _p(mu), C.byref(st)),
           "compute_full")
    return Result(e.value, forces, mu, lab_dipoles(sys, "reference"), st.iterations, st.epsilon, st.converged)


def lab_dipoles(sys, backend: str = "port") -> np.ndarray:
    pk = _Packed(sys)
    out = np.zeros((sys.n, 3))
    if backend == "port":
        _check(_lib("port").tdpo_lab_dipoles(C.byref(pk.s), _p(out)), "lab_dipoles")
    else:
        _check(_lib("reference").tdpref_lab_dipoles(C.byref(pk.s), _p(out)), "lab_dipoles")
    return out


def induced_dipoles(sys, backend: str = "port"):
    """(mu_induced, stats)."""
    pk = _Packed(sys)
    n = sys.n
    mu = np.zeros((n, 3))
    st = _Stats()
    if backend == "port":
        lib = _lib("port")
        lab = np.zeros((n, 3))
        fixed = np.zeros((n, 3))
        _check(lib.tdpo_lab_dipoles(C.byref(pk.s), _p(lab)), "lab_dipoles")
        _check(lib.tdpo_induced_dipoles(C.byref(pk.s), _p(lab), _p(fixed), _p(mu), C.byref(st)), "induced")
    else:
        lib = _lib("reference")
        lib.tdpref_induced_dipoles.argtypes = [C.c_void_p, C.c_double, _dp, C.c_void_p]
        _check(lib.tdpref_induced_dipoles(C.byref(pk.s), 0.0, _p(mu), C.byref(st)), "induced")
    return mu, (st.iterations, st.epsilon, st.converged)


def total_dipoles(sys, backend: str = "port") -> np.ndarray:
    if backend == "port":
        return lab_dipoles(sys, "port") + induced_dipoles(sys, "port")[0]
    pk = _Packed(sys)
    out = np.zeros((sys.n, 3))
    _check(_lib("reference").tdpref_total_dipoles(C.byref(pk.s), _p(out)), "total_dipoles")
    return out


def fixed_field(sys, backend: str = "port") -> np.ndarray:
    pk = _Packed(sys, polarization=0)
    out = np.zeros((sys.n, 3))
    if backend == "port":
        lib = _lib("port")
        lab = np.zeros((sys.n, 3))
        _check(lib.tdpo_lab_dipoles(C.byref(pk.s), _p(lab)), "lab_dipoles")
        _check(lib.tdpo_fixed_field(C.byref(pk.s), _p(lab), _p(out)), "fixed_field")
    else:
        _check(_lib("reference").tdpref_fixed_field(C.byref(pk.s), _p(out)), "fixed_field")
    return out


def induced_field(sys, mu: np.ndarray, backend: str = "port") -> np.ndarray:
    """One pass of the mutual field T*mu."""
    pk = _Packed(sys, polarization=0)
    m = np.ascontiguousarray(mu, dtype=np.float64).reshape(sys.n, 3)
    out = np.zeros((sys.n, 3))
    if backend == "port":
        _check(_lib("port").tdpo_induced_field(C.byref(pk.s), _p(m), _p(out)), "induced_field")
    else:
        _check(_lib("reference").tdpref_induced_field(C.byref(pk.s), _p(m), _p(out)), "induced_field")
    return out


def map_torque(sys, torque: np.ndarray) -> np.ndarray:
    """Forces from per-atom torques by the reference's mapTorqueToForce
    (RTDF.cpp:915-1115), restated in the port."""
    pk = _Packed(sys, polarization=0)
    t = np.ascontiguousarray(torque, dtype=np.float64).reshape(sys.n, 3)
    out = np.zeros((sys.n, 3))
    _check(_lib("port").tdpo_map_torque(C.byref(pk.s), _p(t), _p(out)), "map_torque")
    return out


def potential(sys, grid: np.ndarray, backend: str = "port") -> np.ndarray:
    pk = _Packed(sys)
    g = np.ascontiguousarray(grid, dtype=np.float64).reshape(-1, 3)
    out = np.zeros(g.shape[0])
    lib = _lib(backend)
    fn = lib.tdpo_potential if backend == "port" else lib.tdpref_potential
    _check(fn(C.byref(pk.s), _p(g), C.c_int(g.shape[0]), _p(out)), "potential")
    return out


def moments(sys, backend: str = "port") -> np.ndarray:
    pk = _Packed(sys)
    m = np.ascontiguousarray(sys.masses if sys.masses is not None else np.ones(sys.n), dtype=np.float64)
    out = np.zeros(13)
    lib = _lib(backend)
    fn = lib.tdpo_moments if backend == "port" else lib.tdpref_moments
    _check(fn(C.byref(pk.s), _p(m), _p(out)), "moments")
    return out


def validate(sys) -> int:
    pk = _Packed(sys)
    return int(_lib("port").tdpo_validate(C.byref(pk.s)))
