"""C ABI checks that need no GPU: the in-tree library loads, exports every
entry point that include/*.h declares, and rejects invalid systems in its host
validation (TholeDipoleForceImpl.cpp:52-108) before touching the device."""
import ctypes as C

import numpy as np
import pytest

from tholedipoleplugin_b200 import _capi as A
from tholedipoleplugin_b200 import build as B
from tholedipoleplugin_b200 import systems as S
from tholedipoleplugin_b200.kernel import _DescBuffers

from .fixtures import ammonia


@pytest.fixture(scope="module")
def lib():
    B.build()
    return A.lib()


def test_exports_every_declared_symbol(lib):
    declared = A.declared_symbols()
    assert "tdp_create" in declared and "tdp_compute" in declared
    for name in declared:
        assert hasattr(lib, name), name
    assert set(A.PROTOTYPES) <= set(declared)


def test_abi_version(lib):
    assert lib.tdp_abi_version() == 1


def _create(sys_, **kw):
    buf = _DescBuffers(sys_, 0, 0, 0)
    for k, v in kw.items():
        setattr(buf.desc, k, v)
    h = C.c_void_p()
    rc = A.lib().tdp_create(C.byref(buf.desc), C.byref(h))
    return rc, h, buf


@pytest.mark.parametrize("mutate,fragment", [
    (lambda s: s.axis.__setitem__((0, 0), 7), "axis type=7"),
    (lambda s: s.axis.__setitem__((1, 1), 99), "invalid z axis particle: 99"),
    (lambda s: s.axis.__setitem__((2, 2), -1), "invalid x axis particle: -1"),
    (lambda s: s.axis.__setitem__((3, 3), -1), "invalid y axis particle: -1"),
])
def test_invalid_axes_rejected(lib, mutate, fragment):
    s = ammonia()
    mutate(s)
    rc, h, _ = _create(s)
    assert rc == -1
    assert fragment in lib.tdp_last_error(None).decode()


def test_rotation_without_x_atom_rejected(lib):
    s = ammonia()
    s.axis[0] = [S.NOAXISTYPE, 1, -1, -1]  # reference would dereference a null particle
    rc, _, _ = _create(s)
    assert rc == -1 and "no x axis particle" in lib.tdp_last_error(None).decode()


def test_long_covalent_list_rejected(lib):
    s = ammonia()
    s.cov12[0] = [1, 2, 3, 4, 5, 6]
    rc, _, _ = _create(s)
    assert rc == -1 and "only five scale factors" in lib.tdp_last_error(None).decode()


def test_bad_enums_rejected(lib):
    s = ammonia()
    assert _create(s, nonbonded_method=2)[0] == -1
    assert "nonbonded method" in lib.tdp_last_error(None).decode()
    assert _create(s, polarization_type=5)[0] == -1
    assert _create(s, precision=9)[0] == -1
    assert _create(s, solver=9)[0] == -1


def test_null_desc(lib):
    h = C.c_void_p()
    assert lib.tdp_create(None, C.byref(h)) == -1


def test_query_argument_checks(lib):
    # Host-side checks of the solver queries, before any device work.
    cnt = C.c_int32(-5)
    assert lib.tdp_solver_history(None, None, 0, C.byref(cnt)) == -1
    it, conv, st = C.c_int32(), C.c_int32(), C.c_int32()
    eps = C.c_double()
    assert lib.tdp_solver_stats(None, C.byref(it), C.byref(eps), C.byref(conv), C.byref(st)) == -1
    out = (C.c_double * 14)()
    assert lib.tdp_stage_times(None, out) == -1


# -- cluster batches: host validation runs before any device work ----------
def _batch_create(clusters, offsets=None, edit=None, **kw):
    sys_, offs = S.concat_clusters(clusters)
    if offsets is not None:
        offs = np.asarray(offsets, dtype=np.int32)
    if edit is not None:
        edit(sys_)
    buf = _DescBuffers(sys_, 0, 0, 0)
    for k, v in kw.items():
        setattr(buf.desc, k, v)
    offs = np.ascontiguousarray(offs, dtype=np.int32)
    h = C.c_void_p()
    rc = A.lib().tdp_batch_create(C.byref(buf.desc), len(offs) - 1, offs.ctypes.data_as(C.POINTER(C.c_int32)),
                                  C.byref(h))
    return rc, A.lib().tdp_batch_last_error(None).decode()


def test_batch_rejects_periodic_and_jacobi(lib):
    cl = [ammonia(), ammonia()]
    rc, msg = _batch_create(cl, nonbonded_method=S.PME)
    assert rc == A.TDP_ERR_UNSUPPORTED and "NoCutoff" in msg
    rc, msg = _batch_create(cl, solver=A.SOLVER_JACOBI)
    assert rc == A.TDP_ERR_UNSUPPORTED and "conjugate gradients" in msg


def test_batch_rejects_bad_offsets(lib):
    cl = [ammonia(), ammonia()]
    n = sum(c.n for c in cl)
    rc, msg = _batch_create(cl, offsets=[0, 5, n - 1])
    assert rc == -1 and "from 0 to num_particles" in msg
    rc, msg = _batch_create(cl, offsets=[0, n, 4, n])
    assert rc == -1 and "non-decreasing" in msg


def test_batch_rejects_links_across_clusters(lib):
    a, b = ammonia(), ammonia()
    a.cov12[0] = a.cov12[0] + [a.n + 1]  # partner index lands in the second cluster
    rc, msg = _batch_create([a, b])
    assert rc == -1 and "another cluster" in msg
    n_a = ammonia().n

    def z_into_first(sys_):
        sys_.axis[n_a, 1] = 1  # first atom of the second cluster takes its Z atom from the first

    rc, msg = _batch_create([ammonia(), ammonia()], edit=z_into_first)
    assert rc == -1 and "another cluster" in msg


def test_ewald_mode_validation(lib):
    # TDP_FLAG_EWALD needs the PME method, and Thole damping below 1e-12 at the
    # cutoff (exp(-rc^3 / t^5): rc >= 0.63 nm for t = 0.39).
    s = S.config_small()
    rc, _, _ = _create(s.copy(method=S.NO_CUTOFF), flags=A.FLAG_EWALD)
    assert rc == -1 and "needs the PME nonbonded method" in lib.tdp_last_error(None).decode()
    rc, _, _ = _create(s.copy(cutoff=0.6), flags=A.FLAG_EWALD)
    assert rc == -1 and "Thole damping at the cutoff" in lib.tdp_last_error(None).decode()
    rc, _, _ = _create(s, flags=A.FLAG_EWALD, ewald_error_tolerance=0.7)
    assert rc == -1 and "tolerance" in lib.tdp_last_error(None).decode()


def test_gradient_modes_validation(lib):
    s = S.config_small()
    rc, _, _ = _create(s.copy(polarization=S.EXTRAPOLATED), flags=A.FLAG_EWALD)
    assert rc == -8 and "Mutual or Direct polarization" in lib.tdp_last_error(None).decode()
    rc, _, _ = _create(s, flags=A.FLAG_VARIATIONAL)
    assert rc == -1 and "NoCutoff mode" in lib.tdp_last_error(None).decode()
    rc, _, _ = _create(s.copy(method=S.NO_CUTOFF), flags=A.FLAG_VARIATIONAL | A.FLAG_EWALD)
    assert rc == -1 and "exclude each other" in lib.tdp_last_error(None).decode()
