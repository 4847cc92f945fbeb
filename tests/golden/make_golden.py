"""Generates the golden fixtures in tests/golden from the reference plugin's own
ReferenceTholeDipoleForce.cpp, compiled unmodified by oracle/Makefile into
oracle/_ref/libtdp_ref.so (run where the reference source tree is present):

    python tests/golden/make_golden.py [--only pin|water2187|water12288]

pin.npz          every system of tests/test_oracle_pin.py at its own settings:
                 energy, forces and iteration count of calculateForceAndEnergy
                 (RTDF.cpp:100-127), lab-frame dipoles, permanent field, one
                 mutual-field pass on seeded dipoles, induced and total dipoles,
                 and the potential and multipole moments of three of them.  The
                 pin test checks the restatement against these when the compiled
                 reference is absent.
water2187.npz    729 waters in a 2.8 nm box (PME flag = minimum image), and
water12288.npz   the 4,096-water box of the 12,288-atom workload (4.968 nm):
                 energy, forces and induced dipoles of one evaluation with the
                 Jacobi loop run to an RMS dipole change of 1e-12, i.e. the
                 converged fixed point.  The GPU tests compare both precision
                 forms against these.

Each file stores the SHA-256 of the float64 positions it was made from, so a
change of the seeded generator shows up as a fixture mismatch, not as a
numerical failure.  The 12,288-atom solve takes about 15 minutes on one core.
"""
from __future__ import annotations

import argparse
import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from tholedipoleplugin_b200 import systems as S  # noqa: E402


def positions_sha(s) -> str:
    return hashlib.sha256(np.ascontiguousarray(s.positions, dtype=np.float64).tobytes()).hexdigest()


def pin_systems():
    """The systems of tests/test_oracle_pin.py (same names, same settings)."""
    from tests.fixtures import reference_test_systems, small_random_system
    systems = dict(reference_test_systems())
    systems["water216"] = S.config_small(max_iter=60)
    systems["random_nocutoff"] = small_random_system(40, seed=5, method=S.NO_CUTOFF)
    systems["random_pme"] = small_random_system(45, seed=6, method=S.PME)
    return systems


QUERY_SYSTEMS = ("ammonia_mutual", "water4_pme", "random_nocutoff")


def seeded_dipoles(n: int) -> np.ndarray:
    return np.random.default_rng(1).normal(scale=0.01, size=(n, 3))


def query_grid() -> np.ndarray:
    return np.random.default_rng(2).uniform(-1.0, 1.0, size=(17, 3))


def make_pin() -> None:
    out = {}
    for name, s in sorted(pin_systems().items()):
        r = O.compute(s, "reference", dipoles=False)
        out[f"{name}/sha"] = np.array(positions_sha(s))
        out[f"{name}/energy"] = np.array(r.energy)
        out[f"{name}/forces"] = r.forces
        out[f"{name}/iterations"] = np.array(r.iterations)
        out[f"{name}/converged"] = np.array(r.converged)
        out[f"{name}/lab"] = O.lab_dipoles(s, "reference")
        out[f"{name}/fixed_field"] = O.fixed_field(s, "reference")
        out[f"{name}/induced_field"] = O.induced_field(s, seeded_dipoles(s.n), "reference")
        mu, st = O.induced_dipoles(s, "reference")
        out[f"{name}/induced"] = mu
        out[f"{name}/induced_iterations"] = np.array(st[0])
        out[f"{name}/total"] = O.total_dipoles(s, "reference")
        if name in QUERY_SYSTEMS:
            out[f"{name}/potential"] = O.potential(s, query_grid(), "reference")
            out[f"{name}/moments"] = O.moments(s, "reference")
        print(f"pin {name}: n={s.n} E={r.energy:.12g} it={r.iterations}", flush=True)
    np.savez_compressed(os.path.join(HERE, "pin.npz"), **out)


def box_system(name: str):
    if name == "water2187":
        return S.water_box(9, 2.8, seed=31, cutoff=0.9)
    if name == "water12288":
        return S.config_medium(seed=1)
    raise KeyError(name)


def make_box(name: str) -> None:
    s = box_system(name).copy(target_eps=1e-12, max_iter=20000)
    t = time.perf_counter()
    r = O.compute_full(s)
    dt = time.perf_counter() - t
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), sha=np.array(positions_sha(s)), energy=np.array(r.energy),
                        forces=r.forces, induced=r.induced, iterations=np.array(r.iterations),
                        epsilon=np.array(r.epsilon), seconds=np.array(dt))
    print(f"{name}: n={s.n} E={r.energy:.12g} it={r.iterations} eps={r.epsilon:.3g} {dt:.0f}s", flush=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", choices=["pin", "water2187", "water12288"])
    a = ap.parse_args()
    if not O.reference_available():
        raise SystemExit("the compiled reference (oracle/_ref/libtdp_ref.so) is needed; build it with oracle/Makefile")
    if a.only in (None, "pin"):
        make_pin()
    for name in ("water2187", "water12288"):
        if a.only in (None, name):
            make_box(name)


if __name__ == "__main__":
    main()
