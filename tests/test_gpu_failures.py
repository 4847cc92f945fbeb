"""Failure statuses of the C ABI, each caused by host-side inputs only: a
non-finite coordinate (host and device buffers), an iteration cap too small
to converge, a periodic box below twice the cutoff, and a field sum beyond the
mixed form's fixed-point accumulator range.  After every failure the same
handle must evaluate a good configuration correctly again.

The reference's behaviour these follow: non-convergence is not an error
(ReferenceTholeDipoleForce.cpp:820-851 just stops at the cap and reports
getMutualInducedDipoleConverged() = 0); the box check and its message are
ReferenceTholeDipoleKernels.cpp:168-172."""
import ctypes as C

import numpy as np
import pytest
import torch

from oracle import oracle as O
from tholedipoleplugin_b200 import _capi as A
from tholedipoleplugin_b200 import systems as S
from tholedipoleplugin_b200.kernel import CudaCalcTholeDipoleForceKernel

from .fixtures import ammonia
from .gpu_util import rel_err, rel_rms

pytestmark = pytest.mark.gpu


def _good_call(k, s, ref):
    e, f = k.execute(s.positions)
    assert rel_err(e, ref.energy) < 1e-6 and rel_rms(f, ref.forces) < 2e-5
    assert k.solverStats()["status"] == A.STATUS_CONVERGED


@pytest.fixture(scope="module")
def water():
    s = S.config_small(target_eps=1e-9, max_iter=500)
    return s, O.compute(s.copy(target_eps=1e-12, max_iter=5000), "port")


@pytest.mark.parametrize("precision", ["double", "mixed"])
@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_nan_host_positions(water, precision, dtype):
    s, ref = water
    with CudaCalcTholeDipoleForceKernel(s, precision=precision) as k:
        bad = s.positions.copy()
        bad[17, 1] = np.nan
        hb = np.ascontiguousarray(bad, dtype=np.float64 if dtype == "f64" else np.float32)
        f = np.zeros((s.n, 3))
        e = C.c_double()
        rc = k._lib.tdp_compute(k.handle, hb.ctypes.data_as(C.c_void_p), A.F64 if dtype == "f64" else A.F32, 0,
                                f.ctypes.data_as(C.c_void_p), A.F64, C.byref(e),
                                A.COMPUTE_FORCES | A.COMPUTE_ENERGY)
        assert rc == A.TDP_ERR_NON_FINITE
        assert "not finite" in k._lib.tdp_last_error(k.handle).decode()
        assert np.all(f == 0.0)  # nothing was added
        _good_call(k, s, ref)


@pytest.mark.parametrize("precision", ["double", "mixed"])
def test_nan_device_positions(water, precision):
    """A non-finite coordinate in a device buffer is not inspected on the host;
    the solve's residual (or a field sum) turns non-finite and the call fails
    with TDP_ERR_NON_FINITE."""
    s, ref = water
    with CudaCalcTholeDipoleForceKernel(s, precision=precision) as k:
        bad = torch.tensor(s.positions, dtype=torch.float64, device="cuda")
        bad[5, 0] = float("inf")
        frc = torch.zeros_like(bad)
        with pytest.raises(A.TdpError) as ei:
            k.execute_device(bad.data_ptr(), A.F64, frc.data_ptr(), A.F64)
        assert ei.value.code == A.TDP_ERR_NON_FINITE
        if precision == "double":
            assert k.solverStats()["status"] == A.STATUS_NON_FINITE
        _good_call(k, s, ref)


@pytest.mark.parametrize("solver", ["cg", "jacobi"])
def test_iteration_cap(water, solver):
    s, ref = water
    with CudaCalcTholeDipoleForceKernel(s.copy(max_iter=1), precision="double", solver=solver) as k:
        e, f = k.execute(s.positions)
        st = k.solverStats()
        assert st["status"] == A.STATUS_MAX_ITERATIONS and st["converged"] == 0
        assert st["iterations"] == 1 and st["epsilon"] > 1e-9
        assert np.isfinite(e) and np.all(np.isfinite(f))
        with pytest.raises(A.TdpError) as ei:
            k.execute(s.positions, require_convergence=True)
        assert ei.value.code == A.TDP_ERR_NOT_CONVERGED


def test_iteration_cap_matches_reference_jacobi():
    # The reference stops at the cap with the dipoles of its last sweep; the
    # Jacobi solver runs the same sweeps, so the unconverged result matches.
    s = ammonia().copy(max_iter=2, target_eps=1e-12)
    ref = O.compute(s, "port")
    assert ref.converged == 0 and ref.iterations == 2
    with CudaCalcTholeDipoleForceKernel(s, precision="double", solver="jacobi") as k:
        e, f = k.execute(s.positions)
        st = k.solverStats()
        assert st["iterations"] == 2 and st["converged"] == 0
        assert rel_err(e, ref.energy) < 1e-10 and rel_rms(f, ref.forces) < 1e-10


@pytest.mark.parametrize("precision", ["double", "mixed"])
def test_box_too_small(water, precision):
    s, ref = water
    with CudaCalcTholeDipoleForceKernel(s, precision=precision) as k:
        k.setBox([1.5, 1.8643, 1.8643])  # below 2 x 0.8 nm in x
        with pytest.raises(A.TdpError) as ei:
            k.execute(s.positions)
        assert ei.value.code == A.TDP_ERR_BOX_TOO_SMALL
        assert "The periodic box size has decreased to less than twice the nonbonded cutoff." in str(ei.value)
        k.setBox(s.box)
        _good_call(k, s, ref)


def test_fixed_point_range():
    """Two charges 1e-4 nm apart give a field of ~1e8 e/nm^2, beyond the mixed
    form's 64-bit fixed-point accumulator range: the call reports it instead of
    wrapping.  The FP64 form has no such range and evaluates it.  The Thole
    factor 1e-3 keeps the pair undamped (a u^3 = 1e3 at 1e-4 nm); with the
    water value 0.39 the damping would cap the field near 1e2."""
    pos = np.array([[0.1, 0.2, 0.3], [0.1, 0.2, 0.3001], [0.6, 0.2, 0.3]])
    s = S.TholeSystem(positions=pos, charges=np.array([1.0, -1.0, 0.5]), dipoles=np.zeros((3, 3)),
                      polarizabilities=np.array([1e-3, 1e-3, 1e-3]), tholes=np.array([1e-3] * 3),
                      axis=np.array([[S.NOAXISTYPE, -1, -1, -1]] * 3, dtype=np.int32), cov12=[[], [], []],
                      cov13=[[], [], []], method=S.NO_CUTOFF, polarization=S.DIRECT)
    with CudaCalcTholeDipoleForceKernel(s, precision="mixed") as k:
        with pytest.raises(A.TdpError) as ei:
            k.execute(pos)
        assert ei.value.code == A.TDP_ERR_NON_FINITE
        assert "fixed-point accumulator range" in str(ei.value)
        far = pos.copy()
        far[1, 2] = 0.45
        good = s.copy(positions=far)
        ref = O.compute(good, "port")
        e, f = k.execute(far)
        assert rel_err(e, ref.energy) < 1e-6 and rel_rms(f, ref.forces) < 2e-5
    with CudaCalcTholeDipoleForceKernel(s, precision="double") as k:
        ref = O.compute(s, "port")
        e, f = k.execute(pos)
        # Energies of ~3e5 from terms that cancel to a part in ~1e3: summation
        # order alone moves the last ~1e-8 of it.
        assert rel_err(e, ref.energy) < 1e-7 and rel_rms(f, ref.forces) < 1e-7
