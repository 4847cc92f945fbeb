"""TholeDipoleForce API mirror and XML round trip, after the reference's
serialization test (serialization/tests/TestSerializeTholeDipoleForce.cpp:45-156):
every force-level setting, extrapolation coefficient, particle parameter and
covalent map survives serialize -> deserialize.  Plus the API defaults and
setter validation of openmmapi/src/TholeDipoleForce.cpp:43-61, and (GPU) the
Context queries against the oracle."""
import numpy as np
import pytest

from oracle import oracle as O
from tholedipoleplugin_b200.force import Context, TholeDipoleForce, deserialize, serialize

from .fixtures import ammonia
from .gpu_util import rel_err, rel_rms


def test_defaults():
    f = TholeDipoleForce()
    assert f.getNonbondedMethod() == TholeDipoleForce.NoCutoff
    assert f.getPolarizationType() == TholeDipoleForce.Mutual
    assert f.getPmeBSplineOrder() == 5
    assert f.getCutoffDistance() == 1.0
    assert f.getEwaldErrorTolerance() == 1e-4
    assert f.getMutualInducedMaxIterations() == 60
    assert f.getMutualInducedTargetEpsilon() == 1e-5
    assert f.getExtrapolationCoefficients() == [-0.154, 0.017, 0.658, 0.474]
    assert f.getPMEParameters() == (0.0, 0, 0, 0)
    with pytest.raises(ValueError, match="Illegal value for nonbonded method"):
        f.setNonbondedMethod(2)


def test_serialization_round_trip():
    force = TholeDipoleForce()
    force.setForceGroup(3)
    force.setNonbondedMethod(TholeDipoleForce.PME)
    force.setPolarizationType(TholeDipoleForce.Mutual)
    force.setCutoffDistance(0.9)
    force.setEwaldErrorTolerance(1.0e-05)
    force.setMutualInducedMaxIterations(200)
    force.setMutualInducedTargetEpsilon(1.0e-05)
    force.setPMEParameters(0.5, 32, 32, 32)
    force.setExtrapolationCoefficients([0.0, -0.1, 1.1])
    for i in range(4):
        idx = force.addParticle(i + 1.0, [0.1 * i, 0.2 * i, 0.3 * i], 0.5 + 0.1 * i, 0.8 + 0.05 * i,
                                TholeDipoleForce.ZThenX, i + 1, i + 2, i + 3)
        for j in range(TholeDipoleForce.CovalentEnd):
            force.setCovalentMap(idx, j, [i * j, i * j + 1])
    text = serialize(force)
    copy = deserialize(text)
    for getter in ("getForceGroup", "getNonbondedMethod", "getPolarizationType", "getCutoffDistance",
                   "getEwaldErrorTolerance", "getMutualInducedMaxIterations", "getMutualInducedTargetEpsilon",
                   "getPmeBSplineOrder", "getPMEParameters", "getExtrapolationCoefficients", "getNumParticles"):
        assert getattr(force, getter)() == getattr(copy, getter)(), getter
    for i in range(force.getNumParticles()):
        assert force.getParticleParameters(i) == copy.getParticleParameters(i)
        for j in range(TholeDipoleForce.CovalentEnd):
            assert force.getCovalentMap(i, j) == copy.getCovalentMap(i, j)
    assert serialize(copy) == text
    assert '<Force ' in text and 'type="TholeDipoleForce"' in text and 'version="1"' in text
    assert "<CovalentMap type=" in text and "<Dipole " in text and "<Coefficient c=" in text


def test_version_check():
    text = serialize(TholeDipoleForce()).replace('version="1"', 'version="2"')
    with pytest.raises(ValueError, match="Unsupported version number"):
        deserialize(text)


def _ammonia_force():
    s = ammonia()
    f = TholeDipoleForce()
    f.setNonbondedMethod(s.method)
    f.setPolarizationType(s.polarization)
    f.setMutualInducedTargetEpsilon(1e-11)
    f.setMutualInducedMaxIterations(500)
    for i in range(s.n):
        f.addParticle(s.charges[i], s.dipoles[i], s.polarizabilities[i], s.tholes[i], *[int(v) for v in s.axis[i]])
        f.setCovalentMap(i, TholeDipoleForce.Covalent12, s.cov12[i])
        f.setCovalentMap(i, TholeDipoleForce.Covalent13, s.cov13[i])
    return s, f


def test_to_system_matches_fixture():
    s, f = _ammonia_force()
    t = f.toSystem(s.positions)
    assert np.array_equal(t.axis, s.axis) and t.cov12 == s.cov12 and t.cov13 == s.cov13
    ref = O.compute(s.copy(target_eps=1e-11, max_iter=500), "port")
    got = O.compute(t, "port")
    assert got.energy == ref.energy


@pytest.mark.gpu
def test_context_matches_oracle():
    s, f = _ammonia_force()
    ctx = Context(f, s.positions, masses=s.masses, precision="double")
    e, forces = ctx.getState()
    ref = O.compute(s.copy(target_eps=1e-12, max_iter=3000), "port")
    assert rel_err(e, ref.energy) < 1e-9 and rel_rms(forces, ref.forces) < 1e-9
    assert rel_rms(ctx.getInducedDipoles(), ref.induced) < 1e-9
    # updateParametersInContext: a changed charge changes the energy as a fresh context says.
    q, d, pol, th, t, z, x, y = f.getParticleParameters(0)
    f.setParticleParameters(0, 1.2 * q, d, pol, th, t, z, x, y)
    ctx.updateParametersInContext()
    e2, _ = ctx.getState()
    fresh = Context(f, s.positions, precision="double")
    e3, _ = fresh.getState()
    assert rel_err(e2, e3) < 1e-9 and abs(e2 - e) > 1e-6
    ctx.close()
    fresh.close()
