"""Pins the plain-C restatement (oracle/tdp_oracle.c) against the reference
plugin's own ReferenceTholeDipoleForce.cpp.

The two must agree to rounding level on every stage the reference exposes:
lab-frame rotation (RTDF.cpp:477-571), permanent field (:678-733), the mutual
field pass (:766-818), the Jacobi solve (:820-851), extrapolation (:853-909),
the pair energy/force/torque routine with its frame convention (:129-393),
torque mapping (:915-1115), potential (:1315-1372) and moments (:1225-1313).

Where the compiled reference (oracle/_ref) is present the restatement is
compared with it live.  Everywhere, it is also compared with the golden
fixtures that tests/golden/make_golden.py wrote from the compiled reference
(tests/golden/pin.npz), so the pin holds without the reference tree."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from tholedipoleplugin_b200 import systems as S

from .fixtures import reference_test_systems, small_random_system
from .golden.make_golden import QUERY_SYSTEMS, positions_sha, query_grid, seeded_dipoles

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
live = pytest.mark.skipif(not O.reference_available(), reason="compiled reference not available")


def _close(a, b, rtol=1e-12, atol=1e-13):
    a = np.asarray(a)
    b = np.asarray(b)
    scale = max(np.abs(b).max(), 1.0) if b.size else 1.0
    assert np.abs(a - b).max() <= atol + rtol * scale, (np.abs(a - b).max(), scale)


SYSTEMS = dict(reference_test_systems())
SYSTEMS["water216"] = S.config_small(max_iter=60)
SYSTEMS["random_nocutoff"] = small_random_system(40, seed=5, method=S.NO_CUTOFF)
SYSTEMS["random_pme"] = small_random_system(45, seed=6, method=S.PME)


@live
@pytest.mark.parametrize("name", sorted(SYSTEMS))
@pytest.mark.parametrize("fill", [0.0, 1234.5])
def test_compute_matches_reference(name, fill):
    s = SYSTEMS[name]
    a = O.compute(s, "port", rinv4_value=fill)
    b = O.compute(s, "reference", rinv4_value=fill, dipoles=False)
    assert a.iterations == b.iterations and a.converged == b.converged
    _close(a.energy, b.energy)
    _close(a.forces, b.forces)


@live
@pytest.mark.parametrize("name", sorted(SYSTEMS))
def test_stages_match_reference(name):
    s = SYSTEMS[name]
    _close(O.lab_dipoles(s, "port"), O.lab_dipoles(s, "reference"))
    _close(O.fixed_field(s, "port"), O.fixed_field(s, "reference"))
    mu = seeded_dipoles(s.n)
    _close(O.induced_field(s, mu, "port"), O.induced_field(s, mu, "reference"))
    ma, sa = O.induced_dipoles(s, "port")
    mb, sb = O.induced_dipoles(s, "reference")
    assert sa[0] == sb[0]
    _close(ma, mb)
    _close(O.total_dipoles(s, "port"), O.total_dipoles(s, "reference"))


@live
@pytest.mark.parametrize("name", QUERY_SYSTEMS)
def test_queries_match_reference(name):
    s = SYSTEMS[name]
    grid = query_grid()
    _close(O.potential(s, grid, "port"), O.potential(s, grid, "reference"))
    _close(O.moments(s, "port"), O.moments(s, "reference"))


@pytest.fixture(scope="module")
def pin_golden():
    return np.load(os.path.join(GOLDEN, "pin.npz"))


@pytest.mark.parametrize("name", sorted(SYSTEMS))
def test_restatement_matches_golden(name, pin_golden):
    """The restatement against the compiled reference's stored outputs: every
    stage, the iteration count of the Jacobi loop, and the queries."""
    g = {k.split("/", 1)[1]: pin_golden[k] for k in pin_golden.files if k.startswith(name + "/")}
    s = SYSTEMS[name]
    assert positions_sha(s) == str(g["sha"]), "the seeded system changed since the fixtures were made"
    a = O.compute(s, "port")
    assert a.iterations == int(g["iterations"]) and a.converged == int(g["converged"])
    _close(a.energy, g["energy"])
    _close(a.forces, g["forces"])
    _close(O.lab_dipoles(s, "port"), g["lab"])
    _close(O.fixed_field(s, "port"), g["fixed_field"])
    _close(O.induced_field(s, seeded_dipoles(s.n), "port"), g["induced_field"])
    mu, st = O.induced_dipoles(s, "port")
    assert st[0] == int(g["induced_iterations"])
    _close(mu, g["induced"])
    _close(O.total_dipoles(s, "port"), g["total"])
    if name in QUERY_SYSTEMS:
        _close(O.potential(s, query_grid(), "port"), g["potential"])
        _close(O.moments(s, "port"), g["moments"])
