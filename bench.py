"""Benchmark of the MAISE NN-potential hot path on B200.

Workload (one GPU): Cu-Pd-Ag random fcc alloy, 10x10x10 conventional cells,
4000 atoms, a = 3.8 A, equal fractions, species-resolved 282-input
Behler-Parrinello basis (8 G2 + 43 G4 per pair/triple), 282-10-10-1 tanh
networks with random N(0, 1/fan_in) FP64 weights, Rc = 6 A; NVT molecular
dynamics at 600 K, dt = 1 fs, tau = 25 fs.  A step = one NVT step: wrap,
neighbour list, descriptors + MLP + forces + virial, thermostat, integrator.

  value   atom-steps/s of device-resident MD (mb_md_nvt), per-step CUDA events,
          L2 overwritten between steps outside the timed events
  e2e     atom-steps/s of MD driven through the C-ABI (mb_efs, the call behind
          CALL_MAISE) with host positions in and host forces out every step
  roofline  the fused descriptor/force kernel against the FP64 FMA peak
  cpu_baseline  the reference MAISE sources (oracle/_ref) on the host cores

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

With --gpus N > 1 (launched by torchrun) every rank runs an independent
replica on its own GPU; value = atom-steps of all ranks / max time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "atom-steps/s (E+F+stress) & relaxed structures/s vs plain GPU path"
UNIT = "atom-steps/s"
WORKLOAD = "CuPdAg fcc 10x10x10 (4000 atoms), 282-10-10-1 FP64, Rc 6 A, NVT 600 K, dt 1 fs"


def workload(seed=0):
    from maise_b200 import models, workloads

    w = workloads.random_alloy(n=10, a=3.8, seed=seed, species=(29, 46, 47))
    return w, models.Basis()


def make_model(td, w, basis, seed=1):
    from maise_b200 import models

    path = os.path.join(td, "model")
    models.random_model(path, w["spcz"], basis, (w["X"], w["LAT"], w["atmn"], 3), seed=seed)
    return path


def algorithmic_flops(basis, nspc, pairs, triplets, N):
    """FLOPs of one E+F+S evaluation by the counting rule frozen for this
    path: per pair 37 + 12 N_G2, per triplet 112 + 2 N_eta + 6 N_zl + 11 N_G4,
    per atom 4 (D H1 + H1 H2 + H2) + 4 (H1 + H2); exp/cos/pow/tanh count 1
    each in a separate tally that is not included here."""
    ng2, ne, nzl, ng4 = basis.ng2, len(basis.eta4), len(basis.zetas) * len(basis.lambdas), basis.ng4
    D, h1, h2 = basis.ncmp(nspc), 10, 10
    return (pairs * (37 + 12 * ng2) + triplets * (112 + 2 * ne + 6 * nzl + 11 * ng4)
            + N * (4 * (D * h1 + h1 * h2 + h2) + 4 * (h1 + h2)))


class ClockSampler:
    """nvidia-smi sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except Exception:
        return {}


def profile_traffic():
    """DRAM bytes per launch of the fused kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "k_efs_md4000.md")
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":")[1])
    except Exception:
        pass
    return None


def cpu_baseline(w, model_dir, max_seconds=40.0):
    """Reference MAISE (compiled sources) E+F+S via CALL_MAISE on all host cores."""
    from oracle import RefOracle, ref_available

    if not ref_available():
        return None
    cores = os.cpu_count() or 1
    ref = RefOracle(model_dir, cores)
    X, L, at = w["X"], w["LAT"], w["atmn"]
    t0 = time.perf_counter()
    ref.efs(X, L, at, 3, NM=100)  # first call allocates everything (excluded)
    t_first = time.perf_counter() - t0
    times = []
    while len(times) < 3 and sum(times) < max_seconds:
        t0 = time.perf_counter()
        ref.efs(X, L, at, 3, NM=100)
        times.append(time.perf_counter() - t0)
    per = float(np.median(times))
    return {"value": len(at) / per, "unit": UNIT, "cores": cores, "kind": "reference",
            "sample": f"{len(times)} CALL_MAISE E+F+S calls on the 4000-atom structure (first call, "
                      f"{t_first:.1f} s incl. allocation, excluded); median {per:.3f} s per call"}


def run_reference(args, rank, world):
    """--impl reference: the reference CPU implementation on the same workload."""
    from oracle import RefOracle, ref_available

    if rank != 0:
        return
    if not ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "reference sources were not compiled (oracle/_ref)"}))
        return
    w, basis = workload()
    cores = os.cpu_count() or 1
    with tempfile.TemporaryDirectory() as td:
        make_model(td, w, basis)
        ref = RefOracle(td, cores)
        from maise_b200 import atomic_mass, maxwell

        V = maxwell([atomic_mass(w["spcz"][s]) for s in w["atmn"]], 600.0, seed=7)
        t0 = time.perf_counter()
        ref.nvt(w["X"], w["LAT"], w["atmn"], 3, 600.0, 1.0, 25.0, max(1, min(args.warmup, 1)), V=V, NM=100)
        t_warm = time.perf_counter() - t0
        steps = args.steps
        per_est = t_warm / max(1, min(args.warmup, 1))
        budget = 150.0
        if per_est * steps > budget:
            steps = max(1, int(budget / per_est))
        t0 = time.perf_counter()
        ref.nvt(w["X"], w["LAT"], w["atmn"], 3, 600.0, 1.0, 25.0, steps, V=V, NM=100)
        dt = time.perf_counter() - t0
    value = len(w["atmn"]) * steps / dt
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * dt / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "impl": "reference MAISE sources, CELL_FRC + NVT step, OpenMP"},
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                             "sample": f"{steps} NVT steps of the 4000-atom structure (first CALL_MAISE excluded)"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=50)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    if args.impl == "reference":
        run_reference(args, rank, world)
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return

    import torch

    import maise_b200
    from maise_b200 import atomic_mass, maxwell

    torch.cuda.set_device(local)
    w, basis = workload()
    N = len(w["atmn"])
    td = tempfile.mkdtemp()
    model = make_model(td, w, basis)
    pot = maise_b200.Potential(model, device=local)
    pot.reserve(N, 72)
    V0 = maxwell([atomic_mass(w["spcz"][s]) for s in w["atmn"]], 600.0, seed=7 + rank)

    # warm-up (also settles the neighbour capacity)
    st = pot.md_nvt(w["X"], w["LAT"], w["atmn"], V0, 600.0, dt=1.0, tau=25.0, nsteps=args.warmup, NM=100,
                    trace=False)
    X, V, xi = st["X"], st["V"], st["xi"]

    peaks = measured_peaks()
    l2_flush = 256 << 20
    sampler = ClockSampler(local)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    sampler.start()
    launches0 = pot.launches
    pot.md_profile(True, capacity=args.steps + 16, flush_bytes=l2_flush)
    pot.profile(True, capacity=args.steps + 16)
    st = pot.md_nvt(X, w["LAT"], w["atmn"], V, 600.0, dt=1.0, tau=25.0, nsteps=args.steps, NM=100, xi=xi,
                    trace=True)
    torch.cuda.synchronize()
    launches = pot.launches - launches0
    steps_t = pot.md_profile_read()
    kern = pot.profile_read()
    pot.md_profile(False)
    pot.profile(False)
    clocks = sampler.stop()
    step_s = steps_t["ms_total"] / 1e3
    if dist is not None:
        t = torch.tensor([step_s], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        step_s = float(t.item())
    value = world * N * args.steps / step_s

    # end to end through the C-ABI: host positions in, host forces out, host NVT update
    amu = np.array([atomic_mass(w["spcz"][s]) for s in w["atmn"]])[:, None] * 103.6427
    Xe, Ve, xie = st["X"].copy(), st["V"].copy(), st["xi"]
    kT = 600.0 / 11604.0
    stream = torch.cuda.ExternalStream(pot.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    k2 = min(args.e2e_steps, args.steps)
    e0.record(stream)
    for _ in range(k2):
        r = pot.efs(Xe, w["LAT"], w["atmn"], ND=3, NM=100)
        K = 0.5 * (amu * Ve * Ve).sum()
        xie += 1.0 / (25.0 * 25.0) * (2.0 * K / (3.0 * N * kT) - 1.0)
        f = r["F"] / amu - xie * Ve
        Xe = r["X"] + Ve + 0.5 * f
        Ve = Ve + f
    e1.record(stream)
    e1.synchronize()
    e2e_s = e0.elapsed_time(e1) / 1e3
    if dist is not None:
        t = torch.tensor([e2e_s], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e = {"value": world * N * k2 / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 3 * N * 8 + N * 4 + 9 * 8,
           "d2h_bytes_per_step": 3 * N * 8 + N * 8 + 3 * N * 8 + 16 * 8}

    # roofline of the fused descriptor/MLP/force kernel
    launches_k = max(1, kern["launches"])
    ms_k = kern["ms_total"] / launches_k
    flops = algorithmic_flops(basis, 3, kern["pairs"] / launches_k, kern["triplets"] / launches_k, N)
    fp64_peak = maise_b200.fp64_peak_tflops(local)
    achieved = flops / (ms_k * 1e-3) / 1e12
    roof = {"bound": "fp64", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
            "frac": achieved / fp64_peak, "traffic": profile_traffic(),
            "kernel": "k_efs (fused descriptors + MLP + forces + virial)", "ms_per_launch": ms_k,
            "flops_per_launch": flops, "pairs_per_atom": kern["pairs"] / launches_k / N,
            "triplets_per_atom": kern["triplets"] / launches_k / N,
            "peak_source": "FP64 FMA-chain probe measured in this run (MEASURED_PEAKS.json has no FP64 figure)",
            "hbm_peak_gbs_measured": peaks.get("hbm_gbs")}

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * step_s / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "atoms": N, "parallelism": f"replicas x{world}",
                       "l2": "256 MiB buffer overwritten between timed steps (outside the step events)",
                       "model": "random N(0,1/fan_in) weights, input ranges from the structure"},
            "e2e": e2e, "roofline": roof, "gpu_launches": launches, "clocks": clocks}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(w, td)
    if rank == 0:
        print(json.dumps(line))
    pot.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
