"""The OpenMM-facing adapter: CudaCalcTholeDipoleForceKernel behind the
plugin's CalcTholeDipoleForceKernel interface, created through the CUDA kernel
factory that registerTholeDipoleCudaKernelFactories() installs (the pattern of
platforms/cuda/src/CudaTholeDipoleKernelFactory.cpp:44-73).

The GPU tests run tholedipoleplugin_b200/_build/adapter_driver, which drives the
kernel the way the reference's tests drive a platform
(platforms/reference/tests/TestReferenceTholeDipoleForce.cpp), and compare its
output with the FP64 oracle: energy/forces/dipoles/potential/moments (plain
form: 1e-9 relative), the updateParametersInContext equivalence (:285-313,
tolerance 1e-4 there, 1e-9 here) and the reference's error messages."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as O
from tholedipoleplugin_b200 import build as B
from tholedipoleplugin_b200 import systems as S

from .fixtures import ammonia, water4
from .gpu_util import rel_err, rel_rms


def test_adapter_library_exports_registration_symbols():
    B.build()
    lib = C.CDLL(B.ADAPTER_LIB)
    for name in ("registerPlatforms", "registerKernelFactories", "registerTholeDipoleCudaKernelFactories"):
        assert hasattr(lib, name)
    assert os.access(B.ADAPTER_DRIVER, os.X_OK)


def _write(s, path, grid):
    """System description for the driver; every number as a plain decimal."""
    def num(v):
        return repr(float(v))

    ex = list(s.extrap) if s.extrap is not None else []
    box = np.diag(np.asarray(s.box, dtype=float)) if np.size(s.box) == 3 else np.asarray(s.box).reshape(3, 3)
    masses = s.masses if s.masses is not None else np.ones(s.n)
    lines = [" ".join([str(int(s.n)), str(int(s.method)), str(int(s.polarization)), num(s.cutoff),
                       num(s.ewald_tolerance), num(s.target_eps), str(int(s.max_iter)), str(len(ex))]
                      + [num(c) for c in ex]),
             " ".join(num(b) for b in box.reshape(9))]
    for i in range(s.n):
        a = [int(v) for v in s.axis[i]]
        c12, c13 = [int(v) for v in s.cov12[i]], [int(v) for v in s.cov13[i]]
        fields = [num(s.charges[i])] + [num(v) for v in s.dipoles[i]] + [num(s.polarizabilities[i]),
                                                                        num(s.tholes[i])]
        fields += [str(v) for v in a] + [str(len(c12))] + [str(v) for v in c12] + [str(len(c13))]
        fields += [str(v) for v in c13] + [num(masses[i])] + [num(v) for v in s.positions[i]]
        lines.append(" ".join(fields))
    lines.append(str(len(grid)))
    lines += [" ".join(num(x) for x in g) for g in grid]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def _run(s, grid, tmp_path, precision="double"):
    path = str(tmp_path / "system.txt")
    _write(s, path, grid)
    out = subprocess.run([B.ADAPTER_DRIVER, path, precision], check=True, capture_output=True, text=True,
                         timeout=300).stdout
    res = {}
    for line in out.splitlines():
        tag, _, rest = line.partition(" ")
        res[tag] = rest
    return res


def _arr(s):
    return np.array([float(x) for x in s.split()])


def _scaled(s):
    """The parameter change the driver applies before copyParametersToContext."""
    d = s.dipoles.copy()
    d[:, 0] *= 0.7
    return s.copy(charges=s.charges * 1.1, dipoles=d, polarizabilities=s.polarizabilities * 1.5,
                  tholes=s.tholes * 1.3)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["ammonia_mutual", "water4_pme", "ammonia_extrapolated"])
def test_adapter_matches_oracle(name, tmp_path):
    s = {"ammonia_mutual": ammonia(S.MUTUAL), "water4_pme": water4(S.MUTUAL),
         "ammonia_extrapolated": ammonia(S.EXTRAPOLATED)}[name]
    s = s.copy(target_eps=1e-12, max_iter=3000)
    grid = np.random.default_rng(5).uniform(-0.5, 0.5, size=(9, 3))
    r = _run(s, grid, tmp_path)
    ref = O.compute(s, "port")
    assert rel_err(float(r["energy"]), ref.energy) < 1e-9
    assert rel_rms(_arr(r["forces"]).reshape(-1, 3), ref.forces) < 1e-9
    assert rel_rms(_arr(r["induced"]).reshape(-1, 3), ref.induced) < 1e-9
    assert rel_rms(_arr(r["lab"]).reshape(-1, 3), ref.lab) < 1e-12
    assert rel_rms(_arr(r["total"]).reshape(-1, 3), ref.lab + ref.induced) < 1e-9
    assert rel_rms(_arr(r["potential"]), O.potential(s, grid, "port")) < 1e-9
    assert rel_rms(_arr(r["moments"]), O.moments(s, "port")) < 1e-9
    if s.method == S.PME:
        a, nx, ny, nz = r["pme"].split()
        assert abs(float(a) - np.sqrt(-np.log(2 * s.ewald_tolerance)) / s.cutoff) < 1e-12
        assert int(nx) == int(np.ceil(2 * float(a) * s.box[0] / (3 * s.ewald_tolerance ** 0.2)))
    else:
        assert r["pme_error"] == "getPMEParametersInContext: This Context is not using PME"
    # updateParametersInContext equals a fresh context, and both equal the oracle.
    eu, ef = float(r["energy_updated"]), float(r["energy_fresh"])
    assert rel_err(eu, ef) < 1e-9
    assert rel_rms(_arr(r["forces_updated"]), _arr(r["forces_fresh"])) < 1e-9
    ref2 = O.compute(_scaled(s), "port")
    assert rel_err(eu, ref2.energy) < 1e-9
    assert abs(eu - float(r["energy"])) > 1e-4 * abs(ref2.energy)  # the update changed the result
    assert r["size_error"] == "updateParametersInContext: The number of particles has changed"
    assert r["name_error"] == "Tried to create kernel with illegal kernel name 'NoSuchKernel'"


@pytest.mark.gpu
def test_adapter_mixed_precision(tmp_path):
    s = ammonia(S.MUTUAL).copy(target_eps=1e-9, max_iter=3000)
    r = _run(s, np.zeros((1, 3)) + 2.0, tmp_path, "mixed")
    ref = O.compute(s.copy(target_eps=1e-12), "port")
    assert rel_err(float(r["energy"]), ref.energy) < 1e-6
    assert rel_rms(_arr(r["forces"]).reshape(-1, 3), ref.forces) < 2e-5


# ---------------------------------------------------------------------------
# The adapter compiled against the plugin's own public API (the reference's
# openmmapi headers, TholeDipoleForce.cpp and TholeDipoleForceImpl.cpp built
# unmodified by oracle/Makefile into oracle/_ref/reference_api_driver), driven
# through a Context: TholeDipoleForceImpl::initialize validates and creates
# the kernel by name, calcForcesAndEnergy gates on the force group, the
# queries go through the Force's Context methods, and the CUDA platform's
# buffers (posq, atom index, fixed-point forces) take the device path.
# ---------------------------------------------------------------------------
API_DRIVER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                          "reference_api_driver")
api_driver = pytest.mark.skipif(not os.path.exists(API_DRIVER),
                                reason="the reference-API build of the adapter needs the reference source tree")


def _run_api(s, grid, tmp_path, precision, *extra):
    path = str(tmp_path / "system.txt")
    _write(s, path, grid)
    out = subprocess.run([API_DRIVER, path, precision, *extra], check=True, capture_output=True, text=True,
                         timeout=300).stdout
    res = {}
    for line in out.splitlines():
        tag, _, rest = line.partition(" ")
        res[tag] = rest
    return res


@pytest.mark.gpu
@api_driver
@pytest.mark.parametrize("name,precision", [("water4_pme", "double"), ("ammonia_mutual", "double"),
                                            ("ammonia_extrapolated", "double"), ("water4_pme", "mixed")])
def test_reference_api_context_matches_oracle(name, precision, tmp_path):
    s = {"ammonia_mutual": ammonia(S.MUTUAL), "water4_pme": water4(S.MUTUAL),
         "ammonia_extrapolated": ammonia(S.EXTRAPOLATED)}[name]
    s = s.copy(target_eps=1e-12 if precision == "double" else 1e-9, max_iter=3000)
    grid = np.random.default_rng(6).uniform(-0.5, 0.5, size=(7, 3))
    r = _run_api(s, grid, tmp_path, precision)
    ref = O.compute(s.copy(target_eps=1e-12), "port")
    te, tf = (1e-9, 1e-9) if precision == "double" else (1e-6, 2e-5)
    e = float(r["energy"])
    assert rel_err(e, ref.energy) < te
    assert rel_rms(_arr(r["forces"]).reshape(-1, 3), ref.forces) < tf
    assert rel_rms(_arr(r["induced"]).reshape(-1, 3), ref.induced) < tf
    assert rel_rms(_arr(r["lab"]).reshape(-1, 3), ref.lab) < 1e-12
    assert rel_rms(_arr(r["total"]).reshape(-1, 3), ref.lab + ref.induced) < tf
    assert rel_rms(_arr(r["potential"]), O.potential(s.copy(target_eps=1e-12), grid, "port")) < tf
    if s.method == S.PME:
        assert "pme" in r
    else:
        assert r["pme_error"] == "getPMEParametersInContext: This Context is not using PME"
    # Force groups: the force in group 3 contributes only when group 3 is asked for.
    assert float(r["energy_other_groups"]) == 0.0
    assert float(r["energy_own_group"]) == e
    # The CUDA platform's buffers: same evaluation, forces through the fixed-point accumulator.
    ed = float(r["energy_device"])
    fd = _arr(r["forces_device"]).reshape(-1, 3)
    if precision == "double":
        assert rel_err(ed, e) < 1e-12
        assert np.abs(fd - _arr(r["forces"]).reshape(-1, 3)).max() <= 2.0 ** -31
    else:  # float4 posq: coordinates rounded to FP32
        assert rel_err(ed, ref.energy) < te and rel_rms(fd, ref.forces) < tf
    assert rel_rms(_arr(r["induced_device"]).reshape(-1, 3), ref.induced) < tf
    # updateParametersInContext: kernel.copyParametersToContext + context.systemChanged().
    assert int(r["system_changed"]) >= 1
    ref2 = O.compute(_scaled(s).copy(target_eps=1e-12), "port")
    assert rel_err(float(r["energy_updated"]), ref2.energy) < te
    assert rel_rms(_arr(r["forces_updated"]).reshape(-1, 3), ref2.forces) < tf


@pytest.mark.gpu
@api_driver
def test_reference_api_validation_messages(tmp_path):
    s = water4(S.MUTUAL)
    r = _run_api(s, np.zeros((1, 3)), tmp_path, "double", "validate")
    assert r["particles_error"] == ("TholeDipoleForce must have exactly as many particles as the System it "
                                    "belongs to.")
    assert r["cutoff_error"] == "TholeDipoleForce: The cutoff distance cannot be greater than half the periodic box size."
    assert r["axis_error"].startswith("TholeDipoleForce: axis type=7 not currently handled")
    assert r["zaxis_error"] == f"TholeDipoleForce: invalid z axis particle: {s.n + 5}"
