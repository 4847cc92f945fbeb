"""Edge cases of the box kernels on the GPU, through the C ABI, against the FP64
oracle: an empty system, a single atom, sizes on either side of the 32-atom
tile, and every band width the pair kernels can run with (one CTA per band
pair of 1, 2, 4, 8 or 16 tiles; 2 I tiles per warp from 8-tile bands on, one
below) on a ragged water box.  Tolerances as in test_gpu_parity.py."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from tholedipoleplugin_b200 import systems as S
from tholedipoleplugin_b200.kernel import CudaCalcTholeDipoleForceKernel

from .fixtures import small_random_system
from .gpu_util import energy_rms_scale, rel_err, rel_rms

pytestmark = pytest.mark.gpu

_ORACLE = {}


def _oracle(key, s):
    if key not in _ORACLE:
        _ORACLE[key] = O.compute(s.copy(target_eps=1e-12, max_iter=5000), "port")
    return _ORACLE[key]


def _check(s, ref, precision, e, f, mu):
    if precision == "double":
        assert rel_err(e, ref.energy) < 1e-9, (e, ref.energy)
        assert rel_rms(f, ref.forces) < 1e-8
        assert rel_rms(mu, ref.induced) < 1e-8
    else:
        c2 = energy_rms_scale(s)
        assert abs(e - ref.energy) < 1e-6 * abs(ref.energy) + 3e-7 * c2, (e, ref.energy, c2)
        assert rel_rms(f, ref.forces) < 2e-5
        assert rel_rms(mu, ref.induced) < 2e-5


def _run(s, precision):
    eps = 1e-11 if precision == "double" else 1e-9
    with CudaCalcTholeDipoleForceKernel(s.copy(target_eps=eps, max_iter=2000), precision=precision) as k:
        e, f = k.execute(s.positions)
        mu = k.getInducedDipoles()
    return e, f, mu


@pytest.mark.parametrize("precision", ["double", "mixed"])
def test_empty_system(precision):
    z = np.zeros((0, 3))
    s = S.TholeSystem(positions=z, charges=np.zeros(0), dipoles=z, polarizabilities=np.zeros(0),
                      tholes=np.zeros(0), axis=np.zeros((0, 4), dtype=np.int32), cov12=[], cov13=[],
                      method=S.NO_CUTOFF)
    with CudaCalcTholeDipoleForceKernel(s, precision=precision) as k:
        e, f = k.execute(z)
        assert e == 0.0 and f.shape == (0, 3)
        assert k.solverStats()["converged"]


@pytest.mark.parametrize("precision", ["double", "mixed"])
@pytest.mark.parametrize("method", [S.NO_CUTOFF, S.PME])
def test_single_atom(precision, method):
    # No pairs: zero energy, force and field; the induced dipole is alpha * 0.
    s = S.TholeSystem(positions=np.array([[0.3, 0.4, 0.5]]), charges=np.array([0.7]),
                      dipoles=np.array([[0.01, -0.02, 0.005]]), polarizabilities=np.array([1.2e-3]),
                      tholes=np.array([0.39]), axis=np.array([[S.NOAXISTYPE, -1, -1, -1]], dtype=np.int32),
                      cov12=[[]], cov13=[[]], method=method, box=np.array([2.0, 2.0, 2.0]), cutoff=0.9)
    e, f, mu = _run(s, precision)
    assert e == 0.0
    assert np.all(f == 0.0) and np.all(mu == 0.0)


@pytest.mark.parametrize("precision", ["double", "mixed"])
@pytest.mark.parametrize("n", [31, 32, 33, 63, 64, 65])
def test_tile_boundary_sizes(precision, n):
    s = small_random_system(n, seed=100 + n, method=S.PME)
    _check(s, _oracle(("tile", n), s), precision, *_run(s, precision))


@pytest.fixture
def band_env():
    old = os.environ.get("TDP_BAND_TILES")
    yield
    if old is None:
        os.environ.pop("TDP_BAND_TILES", None)
    else:
        os.environ["TDP_BAND_TILES"] = old


@pytest.mark.parametrize("band", [1, 2, 4, 8, 16])
def test_every_band_width(band, band_env):
    # 729 waters (2,187 atoms: 69 tiles, the last one ragged) in a 2.8 nm box;
    # the band width is read at create time.
    s = S.water_box(9, 2.8, seed=31, cutoff=0.9)
    ref = _oracle(("band", 9), s)
    os.environ["TDP_BAND_TILES"] = str(band)
    for precision in (["double", "mixed"] if band <= 8 else ["mixed"]):
        _check(s, ref, precision, *_run(s, precision))
