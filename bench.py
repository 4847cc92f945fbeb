#!/usr/bin/env python
"""Benchmark of the TholeDipoleForce hot path on B200.

Workload (per GPU): the 98,304-atom water box -- 32,768 rigid 3-site waters on
a 32^3 lattice in a 9.936 nm cubic box, seeded jitter and orientations,
minimum-image all-pairs electrostatics with Thole-damped mutual polarization
converged to an RMS dipole change below 1e-6 e*nm -- integrated by velocity
Verlet (1 fs, rigid waters, Maxwell-Boltzmann start at 300 K).  One "step" is
one MD step: kick-drift-SHAKE, the full force/energy evaluation (lab-frame
rotation, permanent field, CG solve, pair energy/force/torque, torque
mapping) and kick-RATTLE.

Reported (one JSON line, rank 0):
  value        ns/day of the mixed form, summed over ranks (replicas; weak scaling)
  e2e          the same metric through the public C ABI with host buffers
               (positions copied in from pinned memory and forces read back
               every step, integration on the host)
  plain        ns/day and SCF solves/s of the FP64 form; mixed solves/s beside it
  errors       mixed vs plain on this box; both vs the FP64 oracle on 216 waters
  roofline     the dominant kernel against the FP32 issue rate of the GPU
               (FP32 SGEMM measured here); roofline_hbm: the same kernel
               against the measured HBM copy bandwidth
  cpu_baseline the reference's own FP64 code (compiled oracle/_ref), 1 core,
               timed on a 6,591-atom sample and scaled to this box
  clusters     the batched-cluster workload (1024 NoCutoff water clusters of
               4-64 waters in one persistent launch): clusters/s mixed and
               plain, device-resident and end to end, the autotuner's table,
               per-cluster errors against the FP64 oracle, and the compiled
               reference on one core over 384 of the clusters

`--impl reference` times the reference's CPU implementation on all host cores
instead (rank 0 only).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NS_PER_DAY = 1e-6 * 86400.0  # per (step/s) at 1 fs
# Algorithmic operation counts per unordered pair (reference semantics):
# mutual-field pass (both sides) 57 FLOP + 9 FLOP minimum image;
# energy/force/torque pair 280 FLOP; permanent-field pair 70 FLOP.
FLOP_MATVEC_PAIR = 66
FLOP_ENERGY_PAIR = 280
FLOP_FIXED_PAIR = 70
# Algorithmic HBM bytes per atom and launch: matvec 16 (posq) + 12 (operand) +
# 12 (result) + 48 (four CG vectors); energy pass 16 (posq) + 16 (dipole,
# thole) + 16 (induced) + 16 (raw y, z) + 56 (seven FP64 outputs).
BYTES_MATVEC_ATOM = 88
# FP64 records of the plain form: posq 32 + operand 32 + result 24 + CG vectors 48.
BYTES_MATVEC_ATOM_FP64 = 136
BYTES_ENERGY_ATOM = 120
# CPU samples of the reference run on 13^3 = 2,197 waters (6,591 atoms) at the
# density of the 32^3 box and are scaled to the full box by the pair count.
SAMPLE_SIDE = 13


class Ranks:
    """Rank plumbing of one bench process under torchrun (RANK, WORLD_SIZE,
    LOCAL_RANK, MASTER_ADDR/PORT): with more than one rank, a process group with
    a short timeout (NCCL on the GPUs; gloo in the multi-process CPU test), a
    barrier and the maximum of a host float over ranks.  The box workload is
    replicated -- each rank integrates its own seeded box -- so nothing but these
    timing reductions crosses ranks, and every rank takes them in the same order."""

    def __init__(self, backend: str = "nccl", timeout_s: int = 600):
        import torch
        import torch.distributed as dist
        self._dist = dist
        self._torch = torch
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        if backend == "nccl":
            torch.cuda.set_device(self.local)
            self.device = torch.device("cuda", self.local)
        else:
            self.device = torch.device("cpu")
        if self.world > 1:
            import datetime
            kw = {"device_id": self.device} if backend == "nccl" else {}
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)

    def barrier(self) -> None:
        if self.world > 1:
            self._dist.barrier()

    def max_over_ranks(self, x: float) -> float:
        if self.world == 1:
            return x
        t = self._torch.tensor([x], dtype=self._torch.float64, device=self.device)
        self._dist.all_reduce(t, op=self._dist.ReduceOp.MAX)
        return float(t.item())

    def close(self) -> None:
        if self.world > 1:
            self._dist.destroy_process_group()


def box_seed(config: str, rank: int) -> int:
    """Seed of rank's replica of the box (each rank integrates a different box)."""
    return {"small": 0, "medium": 1, "profile": 5, "large": 2}[config] + 100 * rank


def parse(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--config", default="large", choices=["small", "medium", "profile", "large"],
                   help="small 648, medium 12,288, profile 41,472 (24^3 waters, kernel profiling), large 98,304 atoms")
    p.add_argument("--no-extras", action="store_true", help="only the timed MD (used under ncu)")
    p.add_argument("--ewald-md", action="store_true",
                   help="profiling: the timed MD runs in the Ewald mode (with --no-extras)")
    p.add_argument("--clusters-profile", type=int, default=0, metavar="N",
                   help="profiling: only the batched-cluster workload, N clusters of the same seeded "
                        "size distribution, mixed form, a few evaluations")
    return p.parse_args(argv)


# ---------------------------------------------------------------------------
# Clock sampling during the timed region.
# ---------------------------------------------------------------------------
class Clocks:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                rows.append(f)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def fp32_sgemm_tflops(torch) -> float:
    """Measured FP32 (non-tensor) throughput: cuBLAS SGEMM 8192^3 with TF32 off, best of 5."""
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    n = 8192
    a = torch.randn(n, n, device="cuda", dtype=torch.float32)
    b = torch.randn(n, n, device="cuda", dtype=torch.float32)
    c = torch.empty_like(a)
    best = 0.0
    for it in range(7):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b, out=c)
        e.record()
        torch.cuda.synchronize()
        if it >= 2:
            best = max(best, 2 * n ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    torch.backends.cuda.matmul.allow_tf32 = prev
    del a, b, c
    torch.cuda.empty_cache()
    return best


def fp64_dgemm_tflops(torch) -> float:
    """Measured FP64 throughput: cuBLAS DGEMM 4096^3, best of 5 (the plain form's denominator)."""
    n = 4096
    a = torch.randn(n, n, device="cuda", dtype=torch.float64)
    b = torch.randn(n, n, device="cuda", dtype=torch.float64)
    c = torch.empty_like(a)
    best = 0.0
    for it in range(7):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b, out=c)
        e.record()
        torch.cuda.synchronize()
        if it >= 2:
            best = max(best, 2 * n ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    del a, b, c
    torch.cuda.empty_cache()
    return best


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        return {}


def profile_traffic(kernel: str):
    """DRAM bytes per launch from the committed ncu summary (profiles/), or None."""
    path = os.path.join(ROOT, "profiles", "dram_traffic_water98304.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        f = line.split()
        if len(f) >= 2 and f[0] == kernel:
            try:
                return float(f[1])
            except ValueError:
                return None
    return None


# ---------------------------------------------------------------------------
# CPU: the reference's own FP64 code (compiled oracle/_ref), bounded samples.
# ---------------------------------------------------------------------------
def _sample_system():
    from tholedipoleplugin_b200 import systems as S
    side = SAMPLE_SIDE
    box = 9.936 * side / 32.0  # same density as the 32^3 box
    return S.water_box(side, box, seed=7, cutoff=0.9 if box >= 1.8 else 0.45 * box)


def _ref_sample(which: str):
    """One timed sample on this core: 'fixed' (rotation + permanent field),
    'pass' (setup + one mutual-field pass), 'energy' (Direct evaluation:
    setup + energy/force/torque + torque mapping)."""
    sys.path.insert(0, ROOT)
    import numpy as np
    from oracle import oracle as O
    from tholedipoleplugin_b200 import systems as S
    s = _sample_system()
    t = time.perf_counter()
    if which == "fixed":
        O.fixed_field(s, "reference")
    elif which == "pass":
        O.induced_field(s, np.full((s.n, 3), 1e-3), "reference")
    else:
        O.compute(s.copy(polarization=S.DIRECT), "reference", dipoles=False)
    return time.perf_counter() - t


def reference_step_seconds(t_fixed, t_pass_total, t_energy_total, n_atoms, sweeps):
    """Seconds of one reference evaluation of the n_atoms box (FP64, 1 core),
    from samples on the smaller box: the pair loops scale with the pair count."""
    ns = _sample_system().n
    scale = (n_atoms * (n_atoms - 1)) / (ns * (ns - 1))
    t_pass = max(t_pass_total - t_fixed, 1e-9)
    t_energy = max(t_energy_total - t_fixed, 1e-9)
    return scale * (t_fixed + sweeps * t_pass + t_energy), t_pass


def cpu_baseline_single(n_atoms, sweeps):
    from oracle import oracle as O
    if not O.reference_available():
        return None
    tf = _ref_sample("fixed")
    tp = _ref_sample("pass")
    te = _ref_sample("energy")
    step, t_pass = reference_step_seconds(tf, tp, te, n_atoms, sweeps)
    ns = _sample_system().n
    return {"value": NS_PER_DAY / step, "unit": "ns/day", "cores": 1, "kind": "reference",
            "sample": (f"reference ReferenceTholeDipoleForce.cpp (compiled oracle/_ref), 1 core: permanent field "
                       f"{tf:.2f}s, one mutual-field pass {t_pass:.2f}s, energy/force pass {te - tf:.2f}s on a "
                       f"{ns}-atom water box; scaled by the pair count to {n_atoms} atoms and {sweeps} Jacobi "
                       f"sweeps per evaluation ({step:.0f} s/evaluation)"),
            "seconds_per_step": step}


def run_reference(args):
    """--impl reference: the reference CPU code on every host core (rank 0 only)."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    import multiprocessing as mp
    from oracle import oracle as O
    from tholedipoleplugin_b200 import systems as S
    n_atoms = {"small": 648, "medium": 12288, "profile": 41472, "large": 98304}[args.config]
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    base = {"metric": "ns/day", "unit": "ns/day", "impl": "reference", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic"}
    if not O.reference_available():
        base["unavailable"] = "compiled reference (oracle/_ref/libtdp_ref.so) not present"
        print(json.dumps(base))
        return
    sweeps = _recorded_sweeps(args.config)
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        for _ in range(max(args.warmup, 1)):
            pool.map(_ref_sample, ["fixed"] * cores)
        tf = statistics.mean(pool.map(_ref_sample, ["fixed"] * cores))
        te = statistics.mean(pool.map(_ref_sample, ["energy"] * cores))
        t0 = time.perf_counter()
        tps = []
        for _ in range(args.steps):
            tps.append(statistics.mean(pool.map(_ref_sample, ["pass"] * cores)))
        wall = time.perf_counter() - t0
    tp = statistics.mean(tps)
    step, t_pass = reference_step_seconds(tf, tp, te, n_atoms, sweeps)
    value = cores * NS_PER_DAY / step
    base.update({
        "value": value, "ms_per_step": step * 1e3 / cores,
        "config": {"workload": f"{n_atoms}-atom water box MD step (reference platform semantics)",
                   "n_atoms": n_atoms, "jacobi_sweeps": sweeps},
        "cpu_baseline": {"value": value, "unit": "ns/day", "cores": cores, "kind": "reference",
                         "sample": (f"{cores} concurrent processes of the compiled reference; per process: "
                                    f"permanent field {tf:.2f}s, mutual-field pass {t_pass:.2f}s (mean of "
                                    f"{args.steps} steps, {wall:.0f}s wall), energy pass {te - tf:.2f}s on "
                                    f"{_sample_system().n} atoms, scaled by pair count to {n_atoms} atoms with "
                                    f"{sweeps} Jacobi sweeps")},
        "e2e": {"value": value, "unit": "ns/day", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    })
    print(json.dumps(base))


# Jacobi sweeps the reference's loop (RTDF.cpp:820-851) takes to an RMS dipole
# change below 1e-6 on each seeded box, as counted by the library's Jacobi
# solver, which runs that loop sweep for sweep (the iteration count is tested
# against the reference's): 216 waters 39, 4,096 waters 92, 32,768 waters 134
# (the last re-measured by every default bench run, config.reference_jacobi_sweeps).
REFERENCE_JACOBI_SWEEPS = {"small": 39, "medium": 92, "large": 134}


def _recorded_sweeps(config: str = "large") -> int:
    return REFERENCE_JACOBI_SWEEPS.get(config, 134)


# ---------------------------------------------------------------------------
# Cluster batches: 1024 isolated water clusters, sizes uniform in [4, 64]
# waters, NoCutoff, mutual polarization to 1e-6, one persistent launch.
# ---------------------------------------------------------------------------
N_CLUSTERS = 1024


def _cluster_workload(seed):
    from tholedipoleplugin_b200 import systems as S
    return S.cluster_batch(N_CLUSTERS, 4, 64, seed=seed, target_eps=1e-6, max_iter=500)


def _ref_clusters(args):
    """(seconds, clusters) of the compiled reference over a slice of the cluster workload."""
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    seed, lo, hi = args
    clusters = _cluster_workload(seed)[lo:hi]
    t = time.perf_counter()
    for c in clusters:
        O.compute(c, "reference", dipoles=False)
    return time.perf_counter() - t, len(clusters)


def run_clusters(args, rank, world, barrier, max_over_ranks, stream):
    import numpy as np
    import torch
    from tholedipoleplugin_b200.batch import ClusterBatch

    clusters = _cluster_workload(3 + 100 * rank)
    res = {"workload": f"{N_CLUSTERS} isolated water clusters, 4-64 waters each (seeded), NoCutoff, "
                       "mutual polarization to 1e-6, one persistent graph-captured launch per evaluation"}
    reps = max(5, args.steps)
    for prec in ("mixed", "double"):
        with ClusterBatch(clusters, precision=prec) as b:
            b.setStream(stream.cuda_stream)
            b.compute()  # autotunes the tile shape, captures the graph
            pos = torch.tensor(b.positions, dtype=torch.float64, device="cuda")
            frc = torch.zeros_like(pos)
            en = torch.zeros(b.num_clusters, dtype=torch.float64, device="cuda")
            for _ in range(max(3, args.warmup)):
                b.compute_device(pos.data_ptr(), frc.data_ptr(), en.data_ptr())
            torch.cuda.synchronize()
            barrier()
            s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s0.record(stream)
            for _ in range(reps):
                b.compute_device(pos.data_ptr(), frc.data_ptr(), en.data_ptr())
            s1.record(stream)
            torch.cuda.synchronize()
            t_ms = max_over_ranks(s0.elapsed_time(s1) / reps)
            # End to end: host positions in, host forces and energies out, every call.
            hpos = torch.empty((b.n, 3), dtype=torch.float64, pin_memory=True).numpy()
            hpos[...] = b.positions
            barrier()
            t0 = time.perf_counter()
            for _ in range(reps):
                b.compute(hpos)
            t_e2e = max_over_ranks((time.perf_counter() - t0) / reps)
            it, ep = b.solverStats()
            tile = b.tile()
            cand = b.tileCandidates()
            res[prec] = {"clusters_per_s": world * N_CLUSTERS / (t_ms * 1e-3), "ms_per_launch": t_ms,
                         "e2e_clusters_per_s": world * N_CLUSTERS / t_e2e, "n_atoms": b.n,
                         "cg_iterations_mean": float(it.mean()), "cg_iterations_max": int(it.max()),
                         "max_epsilon": float(ep.max()),
                         "tile": {"threads": tile["threads"], "lanes_per_atom": tile["lanes"], "ctas": tile["ctas"]},
                         "autotuner_ms": {f"{c['threads']}x{c['lanes']}": round(c["ms"], 4) for c in cand}}
            if prec == "mixed":
                e_mixed, f_mixed = b.compute()
                offs = b.offsets
    res["mixed_over_plain"] = res["mixed"]["clusters_per_s"] / res["double"]["clusters_per_s"]
    # Pair work of one evaluation: every cluster's fixed field, its matvecs and its energy pass.
    sizes = np.diff(offs).astype(np.float64)
    pairs = float((sizes * (sizes - 1) / 2).sum())
    res["unordered_pairs"] = pairs
    if rank == 0:
        from oracle import oracle as O
        # Per-cluster error against the FP64 oracle (converged to 1e-12) on a seeded sample.
        sample = np.random.default_rng(0).choice(N_CLUSTERS, 32, replace=False)
        e_rel, f_rel = [], []
        for k in sample:
            c = clusters[k]
            ref = O.compute(c.copy(target_eps=1e-12, max_iter=5000), "port")
            sl = slice(int(offs[k]), int(offs[k + 1]))
            e_rel.append(abs(e_mixed[k] - ref.energy) / abs(ref.energy))
            f_rel.append(rel_rms(f_mixed[sl], ref.forces))
        res["errors_mixed_vs_fp64_oracle"] = {
            "clusters_sampled": len(sample), "energy_rel_median": float(np.median(e_rel)),
            "energy_rel_max": float(np.max(e_rel)), "force_rms_rel_median": float(np.median(f_rel)),
            "force_rms_rel_max": float(np.max(f_rel)),
            "note": "batch at the workload's 1e-6 target; oracle converged to 1e-12"}
        if world == 1 and O.reference_available():
            t, m = _ref_clusters((3, 0, 384))
            res["cpu_baseline"] = {"value": m / t, "unit": "clusters/s", "cores": 1, "kind": "reference",
                                   "sample": f"compiled reference on the first {m} clusters of the workload, "
                                             f"1 core, {t:.1f}s"}
    return res


# ---------------------------------------------------------------------------
# Our arm.
# ---------------------------------------------------------------------------
def rel_rms(a, b):
    import numpy as np
    return float(np.sqrt(np.mean((a - b) ** 2) / np.mean(b ** 2)))


def ewald_section(system, K, W, stream, world, barrier, max_over_ranks, rank):
    """The box in the library's Ewald mode (no reference counterpart: the
    reference's PME is the all-pairs minimum image): MD ns/day and SCF solves/s
    for the mixed and plain forms, errors mixed vs plain on this box and both
    vs the FP64 Ewald oracle (smooth-PME restatement) on 216 waters."""
    import numpy as np
    import torch
    from tholedipoleplugin_b200 import _capi as A
    from tholedipoleplugin_b200 import systems as S
    from tholedipoleplugin_b200.kernel import CudaCalcTholeDipoleForceKernel
    from tholedipoleplugin_b200.md import DeviceRigidWaterMD
    n = system.n
    res = {"workload": f"{n}-atom water box, Ewald mode: real space within {system.cutoff} nm over a 32-atom tile "
                       f"neighbour list + order-5 smooth PME (tolerance {system.ewald_tolerance}), mutual "
                       "polarization to 1e-6, velocity Verlet 1 fs"}

    def md_rate(precision, steps, warm):
        md = DeviceRigidWaterMD(system, precision=precision, warm_start=True, seed=11 + rank, ewald=True)
        md.kernel.enableTiming(True)
        md.step(warm)
        torch.cuda.synchronize()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        mv_ms, mv_n, en_ms, tot_ms, its, launches = 0.0, 0, 0.0, 0.0, [], 0
        e0.record(stream)
        for _ in range(steps):
            md.step()
            st = md.kernel.stageTimes()
            mv_ms += st[7]
            mv_n += int(st[6])
            en_ms += st[8]
            tot_ms += st[5]
            launches += int(st[9]) + 2
            its.append(md.kernel.solverStats()["iterations"])
        e1.record(stream)
        torch.cuda.synchronize()
        t = max_over_ranks(e0.elapsed_time(e1))
        params = md.kernel.getPMEParameters()
        md.close()
        return {"ns_per_day": world * steps / (t * 1e-3) * NS_PER_DAY, "ms_per_step": t / steps, "steps": steps,
                "cg_iterations_mean": statistics.mean(its), "matvec_ms_per_launch": mv_ms / max(mv_n, 1),
                "matvec_share": mv_ms / t, "energy_force_ms": en_ms / steps, "energy_force_share": en_ms / t,
                "launches_per_step": launches / steps}, params

    mixed, params = md_rate("mixed", K, max(W, 3))
    plain, _ = md_rate("double", max(3, K // 2), 3)
    res["pme"] = {"alpha_per_nm": params[0], "grid": list(params[1:]), "order": 5}
    res["mixed"] = mixed
    res["plain"] = plain
    res["md_ns_per_day_mixed_over_plain"] = mixed["ns_per_day"] / plain["ns_per_day"]

    def solves_per_s(precision, reps):
        with CudaCalcTholeDipoleForceKernel(system, precision=precision, ewald=True) as k:
            k.setStream(stream.cuda_stream)
            dev_pos = torch.tensor(system.positions, dtype=torch.float64, device="cuda")
            buf = np.zeros((n, 3))
            for _ in range(2):
                k.solveDevice(dev_pos.data_ptr(), A.F64, buf)
            torch.cuda.synchronize()
            s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s0.record(stream)
            for _ in range(reps):
                k.solveDevice(dev_pos.data_ptr(), A.F64, buf)
            s1.record(stream)
            torch.cuda.synchronize()
            return world * reps / (max_over_ranks(s0.elapsed_time(s1)) * 1e-3), k.solverStats()["iterations"]

    reps = max(5, K)
    sm, im = solves_per_s("mixed", reps)
    sp, ip = solves_per_s("double", reps)
    res["scf_solves_per_s"] = {"mixed": sm, "plain": sp, "mixed_over_plain": sm / sp,
                               "cg_iterations": {"mixed": im, "plain": ip},
                               "what": "rotation + permanent field + CG to 1e-6 from mu0 = alpha E (Ewald)"}
    if rank == 0:
        def rel_rms(a, b):
            return float(np.sqrt(np.mean((a - b) ** 2) / np.mean(b ** 2)))

        errs = {}
        with CudaCalcTholeDipoleForceKernel(system.copy(target_eps=1e-9), precision="mixed", ewald=True) as km:
            em, fm = km.execute(system.positions)
            mum = km.getInducedDipoles()
        with CudaCalcTholeDipoleForceKernel(system.copy(target_eps=1e-11), precision="double", ewald=True) as kp:
            ep, fp = kp.execute(system.positions)
            mup = kp.getInducedDipoles()
        errs["mixed_vs_plain_this_box"] = {"energy_rel": abs(em - ep) / abs(ep), "force_rms_rel": rel_rms(fm, fp),
                                           "induced_rms_rel": rel_rms(mum, mup)}
        from oracle import ewald as EW
        small = S.config_small(target_eps=1e-12, max_iter=500)
        alpha, grid = EW.pme_parameters(small.cutoff, small.ewald_tolerance, small.box)
        ref = EW.Ewald(small, alpha, recip="pme", grid=grid).evaluate()
        for prec, eps in (("mixed", 1e-9), ("double", 1e-11)):
            with CudaCalcTholeDipoleForceKernel(small.copy(target_eps=eps), precision=prec, ewald=True) as k:
                e, f = k.execute(small.positions)
                mu = k.getInducedDipoles()
            errs[f"{prec}_vs_fp64_ewald_oracle_216_waters"] = {
                "energy_rel": abs(e - ref.energy) / abs(ref.energy), "force_rms_rel": rel_rms(f, ref.forces),
                "induced_rms_rel": rel_rms(mu, ref.induced)}
        res["errors"] = errs
    return res


def run_ours(args):
    import numpy as np
    import torch

    from tholedipoleplugin_b200 import _capi as A
    from tholedipoleplugin_b200 import systems as S
    from tholedipoleplugin_b200.kernel import CudaCalcTholeDipoleForceKernel
    from tholedipoleplugin_b200.md import DeviceRigidWaterMD, HostRigidWaterMD

    ranks = Ranks("nccl")
    rank, world, local = ranks.rank, ranks.world, ranks.local
    barrier, max_over_ranks = ranks.barrier, ranks.max_over_ranks

    make = {"small": S.config_small, "medium": S.config_medium, "large": S.config_large,
            "profile": lambda seed: S.water_box(24, 9.936 * 24 / 32, seed=seed, cutoff=0.9)}[args.config]
    system = make(seed=box_seed(args.config, rank))
    n = system.n
    pairs = n * (n - 1) / 2
    K, W = args.steps, args.warmup
    stream = torch.cuda.current_stream()

    # ---- mixed form, device-resident MD (the headline) --------------------------------
    md = DeviceRigidWaterMD(system, precision="mixed", warm_start=True, seed=11 + rank, ewald=args.ewald_md)
    md.kernel.enableTiming(True)
    md.step(W)
    torch.cuda.synchronize()
    barrier()
    clocks = Clocks(local)
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    mv_ms, mv_n, en_ms, launches, its = 0.0, 0, 0.0, 0, []
    ev0.record(stream)
    for _ in range(K):
        md.step()
        st = md.kernel.stageTimes()
        mv_ms += st[7]
        mv_n += int(st[6])
        en_ms += st[8]
        launches += int(st[9]) + 2  # + kick-drift and kick kernels
        its.append(md.kernel.solverStats()["iterations"])
    ev1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    barrier()
    t_ms = max_over_ranks(ev0.elapsed_time(ev1))
    value = world * K / (t_ms * 1e-3) * NS_PER_DAY
    temperature = md.temperature()
    md.close()
    del md
    torch.cuda.empty_cache()

    out = {"metric": "ns/day", "value": value, "unit": "ns/day", "n_gpus": world, "steps": K, "warmup": W,
           "ms_per_step": t_ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f32", "data": "synthetic",
           "config": {"workload": f"{n}-atom rigid water box ({n // 3} waters, {system.box[0]} nm cubic, "
                                  + ("Ewald mode: cutoff + smooth PME" if args.ewald_md else "minimum-image all-pairs")
                                  + ", mutual polarization to 1e-6), velocity Verlet 1 fs, "
                                  "mixed form (FP32 pair arithmetic, FP64 accumulation/CG)",
                      "n_atoms": n, "parallelism": f"replicas x{world}",
                      "l2": "inputs+working set per pass ~ 10 MB (L2-resident); every step re-reads all of it",
                      "solver": "CG, warm start from the previous step", "cg_iterations_mean": statistics.mean(its)},
           "gpu_launches": launches, "clocks": clk}

    if args.no_extras:
        if rank == 0:
            print(json.dumps(out), flush=True)
        ranks.close()
        return

    # ---- e2e: the public C ABI with host buffers --------------------------------------
    K_e2e = max(3, K // 4)
    pinned = torch.empty((n, 3), dtype=torch.float64, pin_memory=True).numpy()
    hmd = HostRigidWaterMD(system, precision="mixed", warm_start=True, seed=11 + rank, pinned=pinned)
    hmd.frc = torch.empty((n, 3), dtype=torch.float64, pin_memory=True).numpy()
    hmd.frc[...] = 0.0
    hmd.step(max(1, W))
    barrier()
    t0 = time.perf_counter()
    hmd.step(K_e2e)
    t_e2e = max_over_ranks(time.perf_counter() - t0)
    hmd.close()
    out["e2e"] = {"value": world * K_e2e / t_e2e * NS_PER_DAY, "unit": "ns/day", "h2d_bytes_per_step": n * 3 * 8,
                  "d2h_bytes_per_step": n * 3 * 8 + 8, "steps": K_e2e,
                  "what": "host velocity Verlet + SHAKE/RATTLE (tdp_md_host_*, host threads); tdp_compute on pinned host positions/forces"}

    # ---- plain (FP64) form, same MD -------------------------------------------------
    K_pl = max(3, K // 4)
    pmd = DeviceRigidWaterMD(system, precision="double", warm_start=True, seed=11 + rank)
    pmd.kernel.enableTiming(True)
    pmd.step(max(1, W // 2))
    torch.cuda.synchronize()
    barrier()
    pl_mv_ms, pl_mv_n, pl_en_ms = 0.0, 0, 0.0
    ev0.record(stream)
    for _ in range(K_pl):
        pmd.step()
        st = pmd.kernel.stageTimes()
        pl_mv_ms += st[7]
        pl_mv_n += int(st[6])
        pl_en_ms += st[8]
    ev1.record(stream)
    torch.cuda.synchronize()
    t_pl = max_over_ranks(ev0.elapsed_time(ev1))
    pmd.close()
    del pmd

    # ---- SCF solves/s (rotation + permanent field + CG to 1e-6, cold start) ------------
    def solves_per_s(precision, reps):
        with CudaCalcTholeDipoleForceKernel(system, precision=precision) as k:
            k.setStream(stream.cuda_stream)
            dev_pos = torch.tensor(system.positions, dtype=torch.float64, device="cuda")
            buf = np.zeros((n, 3))
            k.solveDevice(dev_pos.data_ptr(), A.F64, buf)
            torch.cuda.synchronize()
            s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s0.record(stream)
            for _ in range(reps):
                k.solveDevice(dev_pos.data_ptr(), A.F64, buf)
            s1.record(stream)
            torch.cuda.synchronize()
            return reps / (s0.elapsed_time(s1) * 1e-3), k.solverStats()["iterations"]

    reps = max(3, K // 4)
    sps_mixed, it_mixed = solves_per_s("mixed", reps)
    sps_plain, it_plain = solves_per_s("double", reps)
    sps_mixed *= world
    out["plain"] = {"ns_per_day": world * K_pl / (t_pl * 1e-3) * NS_PER_DAY, "ms_per_step": t_pl / K_pl,
                    "steps": K_pl, "matvec_avg_ms": pl_mv_ms / max(pl_mv_n, 1), "energy_avg_ms": pl_en_ms / K_pl}
    out["scf_solves_per_s"] = {"mixed": sps_mixed, "plain": world * sps_plain,
                               "mixed_over_plain": sps_mixed / (world * sps_plain),
                               "cg_iterations": {"mixed": it_mixed, "plain": it_plain},
                               "what": "rotation + permanent field + CG to 1e-6 from mu0 = alpha E"}
    out["md_ns_per_day_mixed_over_plain"] = value / out["plain"]["ns_per_day"]

    # ---- Ewald mode (TDP_FLAG_EWALD): the same box with real-space cutoff + smooth PME ---------
    out["ewald"] = ewald_section(system, K, W, stream, world, barrier, max_over_ranks, rank)

    # ---- cluster batches (1024 NoCutoff clusters of 4-64 waters, one launch) -------------
    out["clusters"] = run_clusters(args, rank, world, barrier, max_over_ranks, stream)

    # ---- errors (rank 0) ---------------------------------------------------------------
    if rank == 0:
        errs = {}
        with CudaCalcTholeDipoleForceKernel(system.copy(target_eps=1e-9, max_iter=500), precision="mixed") as km:
            em, fm = km.execute(system.positions)
            mum = km.getInducedDipoles()
        with CudaCalcTholeDipoleForceKernel(system.copy(target_eps=1e-11, max_iter=500), precision="double") as kp:
            ep, fp = kp.execute(system.positions)
            mup = kp.getInducedDipoles()
        errs["mixed_vs_plain_this_box"] = {"energy_rel": abs(em - ep) / abs(ep), "force_rms_rel": rel_rms(fm, fp),
                                           "induced_rms_rel": rel_rms(mum, mup)}
        with CudaCalcTholeDipoleForceKernel(system, precision="mixed") as km6:
            e6, f6 = km6.execute(system.positions)
        errs["mixed_eps1e-6_vs_plain_tight_this_box"] = {"energy_rel": abs(e6 - ep) / abs(ep),
                                                         "force_rms_rel": rel_rms(f6, fp)}
        from oracle import oracle as O
        small = S.config_small()
        ref = O.compute(small.copy(target_eps=1e-12, max_iter=5000), "port")
        for prec, eps in (("mixed", 1e-9), ("double", 1e-11)):
            with CudaCalcTholeDipoleForceKernel(small.copy(target_eps=eps, max_iter=2000), precision=prec) as k:
                e, f = k.execute(small.positions)
                mu = k.getInducedDipoles()
            errs[f"{prec}_vs_fp64_oracle_216_waters"] = {"energy_rel": abs(e - ref.energy) / abs(ref.energy),
                                                        "force_rms_rel": rel_rms(f, ref.forces),
                                                        "induced_rms_rel": rel_rms(mu, ref.induced)}
        out["errors"] = errs

        # Reference Jacobi sweeps on this box (GPU Jacobi = the reference loop).
        with CudaCalcTholeDipoleForceKernel(system, precision="double", solver="jacobi") as kj:
            kj.getInducedDipoles(system.positions)
            sweeps = kj.solverStats()["iterations"]
        out["config"]["reference_jacobi_sweeps"] = sweeps

        # ---- roofline --------------------------------------------------------------------
        peaks = measured_peaks()
        fp32 = fp32_sgemm_tflops(torch)
        mv_avg = mv_ms / max(mv_n, 1)
        en_avg = en_ms / K
        dominant = "energy" if en_ms >= mv_ms else "matvec"
        if dominant == "energy":
            flops, avg, bytes_ = pairs * FLOP_ENERGY_PAIR, en_avg, n * BYTES_ENERGY_ATOM
            kname = "k_energy_sym<float>"
        else:
            flops, avg, bytes_ = pairs * FLOP_MATVEC_PAIR, mv_avg, n * BYTES_MATVEC_ATOM
            kname = "k_field_sym<float,1>"
        ach = flops / (avg * 1e-3) / 1e12
        hbm_peak = peaks.get("hbm_gbs", 6650.0)
        out["roofline"] = {"bound": "fp32", "kernel": kname, "achieved": ach, "peak": fp32, "unit": "TFLOP/s",
                           "frac": ach / fp32, "traffic": profile_traffic(kname),
                           "peak_source": "FP32 cuBLAS SGEMM 8192^3 (TF32 off), measured in this run",
                           "algorithmic": f"{FLOP_ENERGY_PAIR if dominant == 'energy' else FLOP_MATVEC_PAIR} "
                                          f"FLOP per unordered pair x {pairs:.4g} pairs per launch",
                           "avg_launch_ms": avg,
                           "share_of_step": (en_ms if dominant == "energy" else mv_ms) / t_ms}
        out["roofline_hbm"] = {"bound": "hbm", "kernel": kname, "achieved": bytes_ / (avg * 1e-3) / 1e9,
                               "peak": hbm_peak, "unit": "GB/s",
                               "frac": bytes_ / (avg * 1e-3) / 1e9 / hbm_peak,
                               "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks else "fallback"}
        # Plain (FP64) form: the same kernels against the FP64 rate (DGEMM measured here) and HBM.
        fp64 = fp64_dgemm_tflops(torch)
        pmv = out["plain"]["matvec_avg_ms"]
        pen = out["plain"]["energy_avg_ms"]
        out["plain"]["roofline"] = {
            "bound": "fp64", "kernel": "k_field_sym<double,1>",
            "achieved": pairs * FLOP_MATVEC_PAIR / (pmv * 1e-3) / 1e12, "peak": fp64, "unit": "TFLOP/s",
            "frac": pairs * FLOP_MATVEC_PAIR / (pmv * 1e-3) / 1e12 / fp64,
            "peak_source": "FP64 cuBLAS DGEMM 4096^3, measured in this run",
            "energy_tflops": pairs * FLOP_ENERGY_PAIR / (pen * 1e-3) / 1e12}
        out["plain"]["roofline_hbm"] = {
            "bound": "hbm", "kernel": "k_field_sym<double,1>",
            "achieved": n * BYTES_MATVEC_ATOM_FP64 / (pmv * 1e-3) / 1e9, "peak": hbm_peak, "unit": "GB/s",
            "frac": n * BYTES_MATVEC_ATOM_FP64 / (pmv * 1e-3) / 1e9 / hbm_peak}
        out["kernels"] = {"matvec_avg_ms": mv_avg, "matvec_launches": mv_n, "matvec_share": mv_ms / t_ms,
                          "matvec_tflops": pairs * FLOP_MATVEC_PAIR / (mv_avg * 1e-3) / 1e12,
                          "energy_avg_ms": en_avg, "energy_share": en_ms / t_ms,
                          "energy_tflops": pairs * FLOP_ENERGY_PAIR / (en_avg * 1e-3) / 1e12}
        out["md_temperature_K"] = temperature

        # ---- CPU baseline (N = 1 only) ------------------------------------------------------
        if world == 1:
            out["cpu_baseline"] = cpu_baseline_single(n, sweeps)
        print(json.dumps(out), flush=True)
    barrier()
    ranks.close()


def run_clusters_profile(args):
    """A small case of the batched-cluster kernel for ncu: N clusters drawn like
    the 1024-cluster workload, a few evaluations of the mixed form."""
    import torch
    from tholedipoleplugin_b200 import systems as S
    from tholedipoleplugin_b200.batch import ClusterBatch
    clusters = S.cluster_batch(args.clusters_profile, 4, 64, seed=3, target_eps=1e-6, max_iter=500)
    with ClusterBatch(clusters, precision="mixed") as b:
        b.compute()
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        s0.record()
        for _ in range(max(1, args.steps)):
            b.compute()
        s1.record()
        torch.cuda.synchronize()
        it, _ = b.solverStats()
        print(json.dumps({"clusters": args.clusters_profile, "atoms": b.n, "tile": b.tile(),
                          "ms_per_evaluation_incl_copies": s0.elapsed_time(s1) / max(1, args.steps),
                          "cg_iterations_mean": float(it.mean())}))


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.clusters_profile > 0:
        run_clusters_profile(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
