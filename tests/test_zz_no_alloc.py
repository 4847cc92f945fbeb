"""tdp_potential_noalloc: the potential query for callers that cannot call
cudaMalloc -- a host program whose pool allocator owns all device memory, or
a loop that must not pay the implicit device synchronisation of
cudaMalloc/cudaFree.  It takes caller-owned device buffers and keeps its
scratch in a fixed device array (8 MiB, TDP_NOALLOC_SCRATCH_DOUBLES doubles).

Checked through the C ABI against tdp_get_potential (which allocates device
copies of the grid and the result on every call) on two calls in a row, with
the tolerance of the other FP64 query tests (1e-9 RMS relative), and against
the FP64 oracle's potential.  Further cases: a grid of half the scratch size,
where the split over atoms is capped by the scratch array and every slot is
reused; an empty particle set (zeros); the legacy default stream.  This file
is named so that pytest collects it last; it needs nothing from earlier tests."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from tholedipoleplugin_b200 import _capi as A
from tholedipoleplugin_b200 import systems as S
from tholedipoleplugin_b200.kernel import CudaCalcTholeDipoleForceKernel

from .fixtures import ammonia
from .gpu_util import rel_rms

pytestmark = pytest.mark.gpu


def _call(n, pos, q, dip, grid, periodic, box, out, stream):
    b = np.ascontiguousarray(np.asarray(box, dtype=np.float64).reshape(3))
    return A.lib().tdp_potential_noalloc(n, C.c_void_p(pos.data_ptr()), C.c_void_p(q.data_ptr()),
                                         C.c_void_p(dip.data_ptr()), grid.shape[0], C.c_void_p(grid.data_ptr()),
                                         periodic, b.ctypes.data_as(C.POINTER(C.c_double)),
                                         C.c_void_p(out.data_ptr()), C.c_void_p(stream))


@pytest.mark.parametrize("which", ["water216_pme", "ammonia_nocutoff"])
def test_noalloc_potential_matches_allocating_query(which):
    import torch

    s = S.config_small() if which == "water216_pme" else ammonia()
    rng = np.random.default_rng(7)
    lo, hi = s.positions.min(0) - 0.3, s.positions.max(0) + 0.3
    grid = rng.uniform(lo, hi, size=(517, 3))
    with CudaCalcTholeDipoleForceKernel(s.copy(target_eps=1e-11, max_iter=2000), precision="double") as k:
        expected = k.getElectrostaticPotential(grid, s.positions)   # existing, allocating entry point
        total = k.getTotalDipoles()                                 # dipoles of that same evaluation
    dev = torch.device("cuda", 0)
    pos = torch.tensor(s.positions, dtype=torch.float64, device=dev)
    q = torch.tensor(s.charges, dtype=torch.float64, device=dev)
    dip = torch.tensor(total, dtype=torch.float64, device=dev)
    g = torch.tensor(grid, dtype=torch.float64, device=dev)
    out = torch.empty(grid.shape[0], dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    periodic = 1 if s.method == S.PME else 0
    for _ in range(2):  # two calls in a row share the same scratch array
        out.fill_(float("nan"))
        rc = _call(s.n, pos, q, dip, g, periodic, s.box, out, stream)
        torch.cuda.synchronize()
        assert rc == 0, A.lib().tdp_last_error(None)
        got = out.cpu().numpy()
        assert np.all(np.isfinite(got))
        assert rel_rms(got, expected) < 1e-9


def test_noalloc_rejects_oversized_grid():
    import torch

    dev = torch.device("cuda", 0)
    one = torch.zeros(3, dtype=torch.float64, device=dev)
    big = A.lib().tdp_potential_noalloc(1, C.c_void_p(one.data_ptr()), C.c_void_p(one.data_ptr()),
                                        C.c_void_p(one.data_ptr()), (1 << 20) + 1, C.c_void_p(one.data_ptr()), 0,
                                        None, C.c_void_p(one.data_ptr()), None)
    assert big == -1
    assert b"scratch limit" in A.lib().tdp_last_error(None)


def _device(*arrays):
    import torch
    dev = torch.device("cuda", 0)
    return [torch.tensor(np.asarray(a, dtype=np.float64), device=dev) for a in arrays]


def test_noalloc_potential_matches_oracle():
    """The potential of the FP64 oracle (converged dipoles, minimum image) at
    the same grid points, with the GPU's total dipoles from a tight solve."""
    import torch

    s = S.config_small()
    grid = np.random.default_rng(8).uniform(-0.2, 2.0, size=(300, 3))
    ref = O.potential(s.copy(target_eps=1e-12, max_iter=5000), grid, "port")
    with CudaCalcTholeDipoleForceKernel(s.copy(target_eps=1e-12, max_iter=2000), precision="double") as k:
        total = k.getTotalDipoles(s.positions)
    pos, q, dip, g = _device(s.positions, s.charges, total, grid)
    out = torch.full((grid.shape[0],), float("nan"), dtype=torch.float64, device="cuda")
    rc = _call(s.n, pos, q, dip, g, 1, s.box, out, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert rc == 0, A.lib().tdp_last_error(None)
    assert rel_rms(out.cpu().numpy(), ref) < 1e-9


def test_noalloc_scratch_capped_split():
    """num_points = half the scratch: the atom split is capped at two chunks by
    the scratch size, so both halves of the array are written and read; the
    result must equal the allocating query's, twice in a row."""
    import torch

    s = S.water_box(9, 2.8, seed=31, cutoff=0.9)   # 2,187 atoms
    npts = (1 << 20) // 2
    grid = np.random.default_rng(9).uniform(0.0, 2.8, size=(npts, 3))
    with CudaCalcTholeDipoleForceKernel(s.copy(target_eps=1e-10, max_iter=2000), precision="double") as k:
        expected = k.getElectrostaticPotential(grid, s.positions)
        total = k.getTotalDipoles()
    pos, q, dip, g = _device(s.positions, s.charges, total, grid)
    out = torch.empty(npts, dtype=torch.float64, device="cuda")
    for _ in range(2):
        out.fill_(float("nan"))
        rc = _call(s.n, pos, q, dip, g, 1, s.box, out, torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        assert rc == 0, A.lib().tdp_last_error(None)
        assert rel_rms(out.cpu().numpy(), expected) < 1e-9


def test_noalloc_empty_particles_and_default_stream():
    import torch

    grid = np.random.default_rng(10).uniform(-1.0, 1.0, size=(33, 3))
    (g,) = _device(grid)
    out = torch.full((33,), float("nan"), dtype=torch.float64, device="cuda")
    rc = A.lib().tdp_potential_noalloc(0, None, None, None, 33, C.c_void_p(g.data_ptr()), 0, None,
                                       C.c_void_p(out.data_ptr()), None)
    torch.cuda.synchronize()
    assert rc == 0 and torch.all(out == 0.0)
    # Legacy default stream (NULL), non-periodic ammonia, against the allocating query.
    s = ammonia()
    with CudaCalcTholeDipoleForceKernel(s.copy(target_eps=1e-11, max_iter=2000), precision="double") as k:
        expected = k.getElectrostaticPotential(grid, s.positions)
        total = k.getTotalDipoles()
    pos, q, dip = _device(s.positions, s.charges, total)
    out.fill_(float("nan"))
    rc = _call(s.n, pos, q, dip, g, 0, np.zeros(3), out, None)
    torch.cuda.synchronize()
    assert rc == 0, A.lib().tdp_last_error(None)
    assert rel_rms(out.cpu().numpy(), expected) < 1e-9
