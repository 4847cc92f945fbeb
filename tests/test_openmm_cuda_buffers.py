"""tdp_compute_openmm: execute on the OpenMM CUDA platform's own buffers --
posq (float4 in single/mixed precision, double4 in double) in the context's
permuted atom order with its atom_index table, and the 64-bit fixed-point force
accumulator (2^32 units, component-major with the padded atom count) -- the
buffers a CUDA-platform kernel reads from its CudaContext
(platforms/cuda/src/CudaTholeDipoleKernelFactory.cpp:68-73).

The buffers are emulated with torch: a seeded permutation, padding slots, and
a force accumulator that already holds other forces' contributions (the kernel
must add, not overwrite).  The result must equal tdp_compute on the same
coordinates (the float4 case with FP32-rounded coordinates) to the fixed-point
resolution."""
import ctypes as C

import numpy as np
import pytest

from tholedipoleplugin_b200 import _capi as A
from tholedipoleplugin_b200 import systems as S
from tholedipoleplugin_b200.kernel import CudaCalcTholeDipoleForceKernel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,posq_double", [("mixed", False), ("double", True), ("double", False)])
def test_openmm_buffers_match_compute(precision, posq_double):
    import torch

    s = S.config_small(target_eps=1e-9, max_iter=500)
    n = s.n
    padded = ((n + 31) // 32) * 32 + 32
    rng = np.random.default_rng(11)
    perm = rng.permutation(n)                       # slot k holds atom perm[k]
    pos = s.positions if posq_double else s.positions.astype(np.float32).astype(np.float64)
    posq = np.zeros((padded, 4))
    posq[:n, :3] = pos[perm]
    posq[:n, 3] = s.charges[perm]
    atom_index = np.full(padded, -1, dtype=np.int32)
    atom_index[:n] = perm
    other = rng.integers(-2**40, 2**40, size=3 * padded, dtype=np.int64)   # earlier forces in the accumulator
    dev = torch.device("cuda", 0)
    t_posq = torch.tensor(posq, dtype=torch.float64 if posq_double else torch.float32, device=dev)
    t_idx = torch.tensor(atom_index, device=dev)
    t_acc = torch.tensor(other, device=dev)
    with CudaCalcTholeDipoleForceKernel(s, precision=precision) as k:
        e_ref, f_ref = k.execute(pos)
    with CudaCalcTholeDipoleForceKernel(s, precision=precision) as k:
        k.setStream(torch.cuda.current_stream(dev).cuda_stream)
        e = C.c_double()
        rc = k._lib.tdp_compute_openmm(k.handle, C.c_void_p(t_posq.data_ptr()), 1 if posq_double else 0,
                                       C.c_void_p(t_idx.data_ptr()), padded, C.c_void_p(t_acc.data_ptr()),
                                       C.byref(e), A.COMPUTE_FORCES | A.COMPUTE_ENERGY)
        assert rc == 0, k._lib.tdp_last_error(k.handle)
    acc = t_acc.cpu().numpy()
    assert np.all(acc[n:padded] == other[n:padded])   # padding slots untouched
    added = (acc - other).reshape(3, padded)[:, :n].T.astype(np.float64) / 2.0**32   # slot order
    f_slots = f_ref[perm]
    assert abs(e.value - e_ref) <= 1e-12 * abs(e_ref)
    # Truncation to 2^-32 per component.
    assert np.abs(added - f_slots).max() <= 2.0 ** -32 * 1.01
