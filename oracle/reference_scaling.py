"""Checks the model the bench's reference arm uses to time the compiled
reference (oracle/_ref) on boxes too large to run whole: samples on the
6,591-atom box (13^3 waters at the 32^3 box's density) of the permanent field,
one mutual-field pass and the energy/force pass, scaled by the pair count
(N(N-1) ratio) and the Jacobi sweep count.  Here the model's prediction for the
12,288-atom box (4,096 waters, 4.968 nm) is compared with one full timed
evaluation of that box by the same compiled reference, on one core.  TEST AND
MEASUREMENT INFRASTRUCTURE ONLY.

    python oracle/reference_scaling.py > profiles/reference_scaling_water12288.md
"""
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402
from oracle import oracle as O  # noqa: E402
from tholedipoleplugin_b200 import systems as S  # noqa: E402


def main():
    if not O.reference_available():
        raise SystemExit("needs the compiled reference (oracle/_ref/libtdp_ref.so)")
    tf = min(bench._ref_sample("fixed") for _ in range(2))
    tp = min(bench._ref_sample("pass") for _ in range(2))
    te = min(bench._ref_sample("energy") for _ in range(2))
    box = S.config_medium(seed=1)   # target 1e-6, the workload's
    t0 = time.perf_counter()
    r = O.compute(box, "reference", dipoles=False)
    full = time.perf_counter() - t0
    pred, t_pass = bench.reference_step_seconds(tf, tp, te, box.n, r.iterations)
    ns = bench._sample_system().n
    print("# Reference timing model vs a full run (12,288-atom water box)\n")
    print("Command: `python oracle/reference_scaling.py` (compiled reference, oracle/_ref, one core).\n")
    print(f"- sample box: {ns} atoms; permanent field {tf:.3f} s, one mutual-field pass {t_pass:.3f} s, "
          f"energy/force pass {te - tf:.3f} s")
    print(f"- full box: {box.n} atoms, Jacobi sweeps to 1e-6: {r.iterations}")
    print(f"- model prediction (pair-count scaling x {r.iterations} sweeps): {pred:.1f} s")
    print(f"- measured full evaluation: {full:.1f} s")
    print(f"- measured / predicted: {full / pred:.3f}")


if __name__ == "__main__":
    main()
