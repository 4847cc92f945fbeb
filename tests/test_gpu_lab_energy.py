"""The lab-frame energy walk (pair_energy_lab, energy_walk_x2_fast) against the
general quasi-internal-frame walk and the FP64 oracle.

Tile pairs that Thole damping cannot reach take the lab-frame form of the
reference's pair routine (ReferenceTholeDipoleForce.cpp:129-366) unless
TDP_LAB_ENERGY=0.  The two forms are algebraically identical, so they must
agree to rounding: FP64 to 1e-12, FP32 within the mixed form's own rounding
(forces 2e-6 RMS; energy 1e-6 relative plus the FP32 rounding of the pair
terms, 3e-7 sqrt(sum (q_i q_j / r_ij)^2), which matters where the total nearly
cancels, as for the 1000-water cluster: 13.2 against a scale of several
hundred).  Both are also checked against the oracle
with the parity tolerances, for Mutual and Direct polarization and for a box
whose tiles straddle the half-box (folded tile pairs)."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from tholedipoleplugin_b200 import systems as S
from tholedipoleplugin_b200.kernel import CudaCalcTholeDipoleForceKernel

from .gpu_util import energy_rms_scale, rel_err, rel_rms

pytestmark = pytest.mark.gpu


@pytest.fixture
def lab_env():
    old = os.environ.get("TDP_LAB_ENERGY")
    yield
    if old is None:
        os.environ.pop("TDP_LAB_ENERGY", None)
    else:
        os.environ["TDP_LAB_ENERGY"] = old


def _run(s, precision, lab):
    os.environ["TDP_LAB_ENERGY"] = "1" if lab else "0"
    eps = 1e-11 if precision == "double" else 1e-9
    with CudaCalcTholeDipoleForceKernel(s.copy(target_eps=eps, max_iter=2000), precision=precision) as k:
        e, f = k.execute(s.positions)
    return e, f


SYSTEMS = {
    "water729_mutual": lambda: S.water_box(9, 2.8, seed=31, cutoff=0.9),
    "water729_direct": lambda: S.water_box(9, 2.8, seed=32, cutoff=0.9, polarization=S.DIRECT),
    "water1000_nocutoff": lambda: S.water_box(10, 3.1, seed=33, cutoff=0.9, method=S.NO_CUTOFF),
}


@pytest.mark.parametrize("name", sorted(SYSTEMS))
@pytest.mark.parametrize("precision", ["double", "mixed"])
def test_lab_energy_matches_general_walk_and_oracle(name, precision, lab_env):
    s = SYSTEMS[name]()
    e0, f0 = _run(s, precision, lab=False)
    e1, f1 = _run(s, precision, lab=True)
    if precision == "double":
        assert rel_err(e1, e0) < 1e-12 and rel_rms(f1, f0) < 1e-12
    else:
        c2 = energy_rms_scale(s)
        assert abs(e1 - e0) < 1e-6 * abs(e0) + 3e-7 * c2 and rel_rms(f1, f0) < 2e-6
    ref = O.compute(s.copy(target_eps=1e-12, max_iter=5000), "port")
    if precision == "double":
        assert rel_err(e1, ref.energy) < 1e-9 and rel_rms(f1, ref.forces) < 1e-8
    else:
        c2 = energy_rms_scale(s)
        assert abs(e1 - ref.energy) < 1e-6 * abs(ref.energy) + 3e-7 * c2
        assert rel_rms(f1, ref.forces) < 2e-5
