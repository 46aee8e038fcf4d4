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
SETTLE_STEPS = 20  # untimed NVT steps from the ideal lattice before the warm-up
KERNEL_NAME = ("descriptor pass: k_legs (leg tables) + k_trip (triplet lists) + k_efs_leg (fused descriptors + "
               "MLP + forces + virial), timed together")
KERNEL_NAME_NOLEGS = "descriptor pass: k_efs (fused descriptors + MLP + forces + virial)"


def tuned_kernel(pot):
    """(kernel name, the autotuner's E/F/S entries) of a potential after its passes."""
    tt = [e for e in pot.tune_table() if e["mode"] == "efs"]
    legs = tt[-1]["legs"] if tt else True
    return (KERNEL_NAME if legs else KERNEL_NAME_NOLEGS), tt


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


def _nvml_index(local):
    """NVML / nvidia-smi index of CUDA device `local` (CUDA_VISIBLE_DEVICES
    renumbers the CUDA devices, not NVML's)."""
    cvd = os.environ.get("CUDA_VISIBLE_DEVICES", "")
    parts = [x.strip() for x in cvd.split(",") if x.strip()]
    if local < len(parts) and parts[local].isdigit():
        return int(parts[local])
    return local


class ClockSampler:
    """SM clock and clock-event reasons sampled during the timed region:
    NVML read every 10 ms from a thread (read-only queries), else
    nvidia-smi every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, device):
        self.device = _nvml_index(device)
        self.proc = None
        self.nv = None
        self.lines = []
        self.samples = []  # (sm MHz, max MHz, set of reasons) from NVML
        self.stop_flag = threading.Event()

    def start(self):
        try:
            import pynvml as nv

            nv.nvmlInit()
            self.nv = nv
            self.h = nv.nvmlDeviceGetHandleByIndex(self.device)
            self.bits = [nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                         nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap]
            self._sample_nvml()
            self.t = threading.Thread(target=self._poll_nvml, daemon=True)
            self.t.start()
            return
        except Exception:
            self.nv = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _sample_nvml(self):
        nv = self.nv
        sm = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
        mx = nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM)
        r = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
        self.samples.append((float(sm), float(mx), {n for n, b in zip(self.NAMES, self.bits) if r & b}))

    def _poll_nvml(self):
        while not self.stop_flag.wait(0.01):
            try:
                self._sample_nvml()
            except Exception:
                return

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.nv is not None:
            self.stop_flag.set()
            self.t.join(timeout=5)
            try:
                self._sample_nvml()
            except Exception:
                pass
            try:
                self.nv.nvmlShutdown()
            except Exception:
                pass
            if not self.samples:
                return None
            reasons = set().union(*(x[2] for x in self.samples))
            return {"sm_mhz": float(np.median([x[0] for x in self.samples])), "sm_max_mhz": self.samples[-1][1],
                    "reasons": sorted(reasons), "samples": len(self.samples), "source": "NVML, 10 ms"}
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for k, nm in enumerate(self.NAMES):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm),
                "source": "nvidia-smi, 200 ms"}


def max_over_ranks(seconds, dist=None):
    """The slowest rank's time: the job finishes when its last replica does.
    Works over NCCL (CUDA tensor) or gloo (CPU tensor)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(seconds)
    import torch

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(seconds)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except Exception:
        return {}


def profile_traffic():
    """DRAM bytes of one descriptor pass (k_legs + k_trip + k_efs_leg, one
    ncu capture each) from the committed summary."""
    path = os.path.join(ROOT, "profiles", "descriptor_pass_md4000.md")
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_pass:"):
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
            "sample": f"{len(times)} CALL_MAISE E+F+S calls on the 4000-atom structure at the end of the timed "
                      f"MD (first call, "
                      f"{t_first:.1f} s incl. allocation, excluded); median {per:.3f} s per call"}


POP_WORKLOAD = ("EA population relax: 256 Mg-Ca structures of 8-64 atoms, 20 A^3/atom +-15%, angles 60-120 deg, "
                "2.0 A minimum distance, random compositions; 145-10-10-1 tanh model; RLXT 3 (positions and cell) "
                "to max |F| < 0.01 eV/A, UREP 100 eV")
GEN_WORKLOAD = ("surrogate-screened EA generation: 4096 Cu-Pd-Ag offspring of 16-48 atoms generated as the "
                "population relax; 128-bin per-pair histograms -> 768-128-64-64-1 SiLU FP32 MLP trained by Adam on "
                "20000 relaxed offspring (16000 fitted, 4000 held out to set the keep fraction); the best fraction "
                "by prediction is relaxed")


def workloads_basis():
    """The G2/G4 basis every workload's model uses (the reference bases' shape)."""
    from maise_b200 import models

    return models.Basis()


def _binding_model(td, name, structures, spcz, seed, angular=0.3):
    from maise_b200 import models

    big = max(structures, key=lambda s: len(s["atmn"]))
    path = os.path.join(td, name)
    os.makedirs(path, exist_ok=True)
    models.random_model(os.path.join(path, "model"), list(spcz), models.Basis(), (big["X"], big["LAT"], big["atmn"], 3),
                        seed=seed, binding=True, angular=angular)
    return os.path.join(path, "model")


def population_relax(local, td, plain_sample=64, mitr=1000, fmax=0.01, urep=100.0):
    """Relaxed structures/s of the persistent batched relax (FP32 descriptors
    and MLP, FP64 reductions and BFGS) against the plain one-structure FP64
    path (host BFGS over the GPU E/F/S) on a seeded random sample of 64
    structures of the same population; every batched minimum is
    re-evaluated by the FP64 path."""
    import maise_b200
    from maise_b200 import workloads

    pop = workloads.ea_population(count=256, seed=3)
    nat = np.array([len(s["atmn"]) for s in pop])
    pot = maise_b200.Potential(_binding_model(td, "pop", pop, (12, 20), 5), device=local)
    pot.relax_batch(pop[:4], urep=urep, rlxt=3, mitr=3, fmax=fmax)  # module load, launch set-up
    t0 = time.perf_counter()
    rb = pot.relax_batch(pop, urep=urep, rlxt=3, mitr=mitr, fmax=fmax)
    wall = time.perf_counter() - t0
    dE, f64 = [], []
    for k, s in enumerate(pop):
        r = pot.efs(rb["X"][k], rb["LAT"][k], s["atmn"], ND=3, NM=300, urep=urep)
        dE.append(abs(rb["H"][k] - r["H"]) / nat[k])
        f64.append(float(np.abs(r["F"]).max()))
    dE, f64 = np.array(dE), np.array(f64)
    conv = rb["status"] == 0
    sample = np.sort(np.random.default_rng(17).choice(len(pop), plain_sample, replace=False))
    t0 = time.perf_counter()
    plain = [pot.relax_fmax(pop[k]["X"], pop[k]["LAT"], pop[k]["atmn"], ND=3, NM=300, urep=urep, rlxt=3, mitr=mitr,
                            fmax=fmax) for k in sample]
    t_plain = time.perf_counter() - t0
    batched = len(pop) / (rb["ms"] / 1e3)
    plain_sps = plain_sample / t_plain
    # the same launch with the reference's line-search curvature constant
    # (0.1; the batched default is 0.5), separating the batching's gain from
    # the line search's
    os.environ["MAISE_B200_BATCH_SIGMA"] = "0.1"
    try:
        r01 = pot.relax_batch(pop, urep=urep, rlxt=3, mitr=mitr, fmax=fmax)
    finally:
        del os.environ["MAISE_B200_BATCH_SIGMA"]
    at_ref = {"sigma": 0.1, "batched_structures_per_s": len(pop) / (r01["ms"] / 1e3),
              "speedup_vs_plain": len(pop) / (r01["ms"] / 1e3) / plain_sps,
              "evals_per_iteration": r01["evals"] / max(1, int(r01["iters"].sum())),
              "converged": int((r01["status"] == 0).sum()),
              "enthalpy_per_atom_median_abs_diff": float(np.median(np.abs(r01["H"] - rb["H"]) / nat))}
    pot.close()
    # FP32 roofline of k_relax_batch: the frozen counting rule over the pairs,
    # forward triplets and atom evaluations the kernel counted, over its time
    basis = workloads_basis()
    flops = algorithmic_flops(basis, 2, rb["pairs"], rb["triplets"], rb["atom_evals"])
    fp32 = maise_b200.fp32_peak_tflops(local)
    ach = flops / (rb["ms"] * 1e-3) / 1e12
    roof = {"bound": "fp32", "achieved": ach, "peak": fp32, "unit": "TFLOP/s", "frac": ach / fp32,
            "kernel": "k_relax_batch (whole persistent launch: evaluations, BFGS, line search)",
            "atom_evaluations": rb["atom_evals"], "pairs_per_atom_eval": rb["pairs"] / max(1, rb["atom_evals"]),
            "triplets_per_atom_eval": rb["triplets"] / max(1, rb["atom_evals"]), "flops": flops,
            "peak_source": "FP32 FMA-chain probe measured in this run"}
    return {"workload": POP_WORKLOAD, "structures": len(pop), "atoms": int(nat.sum()),
            "batched_structures_per_s": batched, "batched_e2e_structures_per_s": len(pop) / wall,
            "plain_structures_per_s": plain_sps, "speedup_vs_plain": batched / plain_sps,
            "plain_sample": f"{plain_sample} structures drawn at random (seed 17) from the population, one "
                            f"mb_relax_fmax each; their atom counts average {nat[sample].mean():.1f} against "
                            f"{nat.mean():.1f} for all",
            "batched_converged": int(conv.sum()), "plain_converged": int(sum(r["converged"] for r in plain)),
            "batched_evals": rb["evals"], "kernel_ms": rb["ms"], "roofline": roof,
            "line_search": {"sigma": 0.5, "evals_per_iteration": rb["evals"] / max(1, int(rb["iters"].sum())),
                            "plain_path_sigma": 0.1},
            "at_reference_sigma": at_ref,
            "fp32_vs_fp64_ev_per_atom_max_converged": float(dE[conv].max()) if conv.any() else None,
            "fp64_max_force_converged_ev_per_a": float(f64[conv].max()) if conv.any() else None,
            "dtype": "descriptors/MLP fp32, reductions/BFGS fp64"}


def plain_relax_many(model, structures, device, urep, mitr, fmax, threads=8):
    """Relaxed enthalpies of `structures` by the plain FP64 path (mb_relax_fmax),
    one handle per host thread so that independent relaxations overlap on
    the GPU (the handle API is per thread)."""
    import concurrent.futures as cf

    import maise_b200

    chunks = [list(range(k, len(structures), threads)) for k in range(threads)]
    H = np.zeros(len(structures))

    def run(idx):
        pot = maise_b200.Potential(model, device=device)
        for k in idx:
            s = structures[k]
            H[k] = pot.relax_fmax(s["X"], s["LAT"], s["atmn"], ND=3, NM=300, urep=urep, rlxt=3, mitr=mitr,
                                  fmax=fmax)["H"]
        pot.close()

    with cf.ThreadPoolExecutor(threads) as ex:
        list(ex.map(run, chunks))
    return H


def surrogate_generation(local, td, n_train=20000, n_gen=4096, epochs=60, mitr=300, fmax=0.01, urep=100.0,
                         plain_judge=256, holdout=0.2, keep_fixed=0.25):
    """One EA generation with and without the surrogate screen: relax every
    offspring, or predict all, keep the best fraction and relax those; the
    full relaxation of every offspring judges the screen's recall of the
    best 10%.  Training pairs come from relaxing 20000 other offspring; a
    held-out fifth of them, not fitted, sets the keep fraction (the smallest
    that recalls 99% of the held-out best tenth, plus 0.02).  The same
    generation screened with a fixed quarter kept is reported beside it."""
    import maise_b200
    from maise_b200 import workloads
    from maise_b200.surrogate import Surrogate, calibrate_keep, keep_best, recall

    spc = (29, 46, 47)
    train = workloads.ea_population_chunked(n_train, seed=11, nmin=16, nmax=48, species=spc)
    gen = workloads.ea_population_chunked(n_gen, seed=12, nmin=16, nmax=48, species=spc)
    model_gen = _binding_model(td, "gen", train, spc, 5)
    pot = maise_b200.Potential(model_gen, device=local)
    t0 = time.perf_counter()
    rt = pot.relax_batch(train, urep=urep, rlxt=3, mitr=mitr, fmax=fmax)
    t_data = time.perf_counter() - t0
    y = rt["H"] / np.array([len(s["atmn"]) for s in train])
    perm = np.random.default_rng(13).permutation(n_train)
    ho, fit_idx = np.sort(perm[:int(holdout * n_train)]), np.sort(perm[int(holdout * n_train):])
    sur = Surrogate(3, device=local)
    t0 = time.perf_counter()
    feat = sur.features(train)
    loss = sur.fit(feat[fit_idx], y[fit_idx], epochs=epochs, batch=256, lr=1e-3)
    t_fit = time.perf_counter() - t0
    keep = calibrate_keep(sur.predict(feat[ho]), y[ho])
    nat = np.array([len(s["atmn"]) for s in gen])
    t0 = time.perf_counter()
    ra = pot.relax_batch(gen, urep=urep, rlxt=3, mitr=mitr, fmax=fmax)
    t_all = time.perf_counter() - t0
    truth = ra["H"] / nat
    t0 = time.perf_counter()
    pred = sur.screen(gen)
    kept = keep_best(pred, keep)
    t_pred = time.perf_counter() - t0
    rk = pot.relax_batch([gen[i] for i in kept], urep=urep, rlxt=3, mitr=mitr, fmax=fmax)
    t_scr = time.perf_counter() - t0
    # the same screen keeping a fixed quarter
    t0 = time.perf_counter()
    kept_q = keep_best(sur.screen(gen), keep_fixed)
    rq = pot.relax_batch([gen[i] for i in kept_q], urep=urep, rlxt=3, mitr=mitr, fmax=fmax)
    t_q = time.perf_counter() - t0
    e0 = np.array([pot.energy(s["X"], s["LAT"], s["atmn"], ND=3, NM=300, urep=urep)["H"] for s in gen]) / nat
    # composition alone: least squares of the training labels on the species fractions
    def frac(ss):
        return np.array([[np.mean(np.asarray(s["atmn"]) == k) for k in range(len(spc))] + [1.0] for s in ss])

    coef, *_ = np.linalg.lstsq(frac([train[k] for k in fit_idx]), y[fit_idx], rcond=None)
    pcomp = frac(gen) @ coef
    # the plain FP64 relax (host BFGS over the GPU E+F+S, one structure at a
    # time per handle, 8 handles on host threads) of a random sample judges
    # the screen on that sample
    sample = np.sort(np.random.default_rng(23).choice(n_gen, plain_judge, replace=False))
    t0 = time.perf_counter()
    plain = plain_relax_many(model_gen, [gen[k] for k in sample], local, urep=urep, mitr=mitr, fmax=fmax)
    t_plain = time.perf_counter() - t0
    truth_plain = plain / nat[sample]
    in_kept = np.zeros(n_gen, bool)
    in_kept[kept] = True
    ntop = max(1, int(round(0.10 * len(sample))))
    top = np.argsort(truth_plain, kind="stable")[:ntop]
    recall_plain = float(in_kept[sample[top]].mean())
    sur.close()
    # the same screen trained only on pairs the plain FP64 path produced
    try:
        plain_trained = _plain_trained_screen(model_gen, local, pot, train, feat, gen, truth, sample, top, t_all,
                                              urep=urep, mitr=mitr, fmax=fmax, epochs=epochs)
    except Exception as e:  # noqa: BLE001 -- reported in the field, the generation's own numbers stand
        plain_trained = {"error": f"{type(e).__name__}: {e}"}
    try:
        fixed = fixed_composition_generation(pot, local, urep=urep, mitr=mitr, fmax=fmax, epochs=epochs,
                                             holdout=holdout, keep_fixed=keep_fixed)
    except Exception as e:  # noqa: BLE001 -- reported in the field, the generation's own numbers stand
        fixed = {"error": f"{type(e).__name__}: {e}"}
    pot.close()
    return {"workload": GEN_WORKLOAD, "offspring": n_gen, "train_pairs": n_train - len(ho),
            "keep": keep,
            "keep_rule": f"smallest fraction recalling 99% of the best 10% of {len(ho)} held-out training pairs "
                         f"(seed 13, not fitted), + 0.02",
            "recall_top10": recall(pred, truth, keep), "recall_top10_by_unrelaxed_energy": recall(e0, truth, keep),
            "recall_top10_by_composition": recall(pcomp, truth, keep),
            "mae_ev_per_atom": {"surrogate": float(np.abs(pred - truth).mean()),
                                "composition": float(np.abs(pcomp - truth).mean())},
            "recall_top10_plain_judged": recall_plain,
            "plain_judge_sample": f"{len(sample)} offspring drawn at random (seed 23), each relaxed by the plain FP64 "
                                  f"path (mb_relax_fmax) in {t_plain:.1f} s; recall = share of the sample's best "
                                  f"{ntop} that the screen keeps",
            "plain_vs_batched_ev_per_atom_median": float(np.median(np.abs(truth_plain - truth[sample]))),
            "recall_top10_random_expectation": keep,
            "generation_s_relax_all": t_all, "generation_s_screened": t_scr, "speedup": t_all / t_scr,
            "screen_s": t_pred, "relax_all_kernel_ms": ra["ms"], "relax_kept_kernel_ms": rk["ms"],
            "work_kept_share": {"structures": len(kept) / n_gen,
                                "atom_evaluations": rk["atom_evals"] / max(1, ra["atom_evals"]),
                                "triplets": rk["triplets"] / max(1, ra["triplets"]),
                                "kernel_time": rk["ms"] / max(1e-9, ra["ms"])},
            "fixed_keep": {"keep": keep_fixed, "recall_top10": recall(pred, truth, keep_fixed),
                           "generation_s_screened": t_q, "speedup": t_all / t_q,
                           "kernel_time_share": rq["ms"] / max(1e-9, ra["ms"])},
            "train_data_relax_s": t_data, "fit_s": t_fit, "epochs": epochs, "final_loss": float(loss[-1]),
            "judge": "batched relax of every offspring (FP32 descriptors/MLP, FP64 BFGS)",
            "plain_trained": plain_trained,
            "fixed_composition": fixed}


def _plain_trained_screen(model, local, pot, train, feat, gen, truth, sample, top, t_all, urep, mitr, fmax, epochs,
                          n_plain=2000, holdout=0.2):
    """The surrogate trained on unrelaxed/relaxed pairs of the plain FP64
    path (mb_relax_fmax, 8 handles on host threads) for the first 2000
    training offspring, its keep fraction calibrated on a held-out fifth of
    them, then screening the same generation (kept offspring relaxed by the
    batched launch)."""
    from maise_b200.surrogate import Surrogate, calibrate_keep, keep_best, recall

    sub = train[:n_plain]
    nt = np.array([len(s["atmn"]) for s in sub])
    t0 = time.perf_counter()
    yp = plain_relax_many(model, sub, local, urep=urep, mitr=mitr, fmax=fmax) / nt
    t_pairs = time.perf_counter() - t0
    perm = np.random.default_rng(14).permutation(n_plain)
    ho, fit_idx = np.sort(perm[:int(holdout * n_plain)]), np.sort(perm[int(holdout * n_plain):])
    sur = Surrogate(3, device=local)
    fs = feat[:n_plain]
    sur.fit(fs[fit_idx], yp[fit_idx], epochs=4 * epochs, batch=256, lr=1e-3)
    keep = calibrate_keep(sur.predict(fs[ho]), yp[ho])
    t0 = time.perf_counter()
    pred = sur.screen(gen)
    kept = keep_best(pred, keep)
    if keep < 1.0:
        pot.relax_batch([gen[i] for i in kept], urep=urep, rlxt=3, mitr=mitr, fmax=fmax)
        t_scr = time.perf_counter() - t0
    else:
        t_scr = t_all + (time.perf_counter() - t0)
    sur.close()
    in_kept = np.zeros(len(gen), bool)
    in_kept[kept] = True
    return {"train_pairs": len(fit_idx), "held_out": len(ho),
            "pairs": f"the first {n_plain} training offspring relaxed by the plain FP64 path in {t_pairs:.1f} s",
            "epochs": 4 * epochs, "keep": keep, "recall_top10": recall(pred, truth, keep),
            "recall_top10_plain_judged": float(in_kept[sample[top]].mean()), "speedup": t_all / t_scr}


def fixed_composition_generation(pot, local, urep, mitr, fmax, epochs, holdout, keep_fixed, n_train=4096,
                                 n_gen=1024):
    """The screen where composition says nothing: every offspring Cu:Pd:Ag
    1:1:1 (18-48 atoms), a surrogate trained on relaxed offspring of that
    composition, the keep fraction calibrated on held-out pairs as in the
    main generation; recall of the best 10% of 1024 others against ranking
    by unrelaxed enthalpy and against random, and the generation's speed-up."""
    from maise_b200 import workloads
    from maise_b200.surrogate import Surrogate, calibrate_keep, keep_best, recall

    spc = (29, 46, 47)
    kw = dict(nmin=18, nmax=48, species=spc, composition=(1, 1, 1))
    train = workloads.ea_population_chunked(n_train, seed=21, **kw)
    gen = workloads.ea_population_chunked(n_gen, seed=22, **kw)
    rt = pot.relax_batch(train, urep=urep, rlxt=3, mitr=mitr, fmax=fmax)
    t0 = time.perf_counter()
    ra = pot.relax_batch(gen, urep=urep, rlxt=3, mitr=mitr, fmax=fmax)
    t_all = time.perf_counter() - t0
    nt = np.array([len(s["atmn"]) for s in train])
    ng = np.array([len(s["atmn"]) for s in gen])
    y = rt["H"] / nt
    perm = np.random.default_rng(24).permutation(n_train)
    ho, fit_idx = np.sort(perm[:int(holdout * n_train)]), np.sort(perm[int(holdout * n_train):])
    sur = Surrogate(3, device=local)
    feat = sur.features(train)
    sur.fit(feat[fit_idx], y[fit_idx], epochs=epochs, batch=256, lr=1e-3)
    keep = calibrate_keep(sur.predict(feat[ho]), y[ho])
    t0 = time.perf_counter()
    pred = sur.screen(gen)
    kept = keep_best(pred, keep)
    t_pred = time.perf_counter() - t0
    if keep < 1.0:
        rk = pot.relax_batch([gen[i] for i in kept], urep=urep, rlxt=3, mitr=mitr, fmax=fmax)
        t_scr = time.perf_counter() - t0
    else:
        # nothing can be pruned at the target recall: the generation relaxes
        # every offspring after the screen, as without it
        rk = ra
        t_scr = t_all + t_pred
    sur.close()
    truth = ra["H"] / ng
    e0 = np.array([pot.energy(s["X"], s["LAT"], s["atmn"], ND=3, NM=300, urep=urep)["H"] for s in gen]) / ng
    return {"offspring": n_gen, "train_pairs": n_train - len(ho), "composition": "Cu:Pd:Ag 1:1:1, 18-48 atoms",
            "keep": keep, "recall_top10": recall(pred, truth, keep),
            "recall_top10_by_unrelaxed_energy": recall(e0, truth, keep),
            "recall_top10_random_expectation": keep,
            "speedup": t_all / t_scr, "screen_s": t_pred,
            "relax_all_kernel_ms": ra["ms"], "relax_kept_kernel_ms": rk["ms"],
            "relax_all_iters_max": int(ra["iters"].max()), "relax_kept_iters_max": int(rk["iters"].max()),
            "at_fixed_keep": {"keep": keep_fixed, "recall_top10": recall(pred, truth, keep_fixed),
                              "recall_top10_by_unrelaxed_energy": recall(e0, truth, keep_fixed)},
            "mae_ev_per_atom": float(np.abs(pred - truth).mean()),
            "spread_ev_per_atom": float(truth.std())}


def _efs_rate(pot, w, ND, calls, NM):
    """atom-steps/s of E+F+S through mb_efs (host arrays in and out), plus
    the fused kernel's time and pair/triplet counts over those calls."""
    pot.efs(w["X"], w["LAT"], w["atmn"], ND=ND, NM=NM)  # tuning, capacity, graph capture
    pot.efs(w["X"], w["LAT"], w["atmn"], ND=ND, NM=NM)
    pot.profile(True, capacity=calls + 4)
    t0 = time.perf_counter()
    for _ in range(calls):
        pot.efs(w["X"], w["LAT"], w["atmn"], ND=ND, NM=NM)
    dt = time.perf_counter() - t0
    k = pot.profile_read()
    pot.profile(False)
    return len(w["atmn"]) * calls / dt, k


def _roofline(basis, nspc, k, N, peak, pot):
    n = max(1, k["launches"])
    ms = k["ms_total"] / n
    fl = algorithmic_flops(basis, nspc, k["pairs"] / n, k["triplets"] / n, N)
    ach = fl / (ms * 1e-3) / 1e12
    kname, tuned = tuned_kernel(pot)
    return {"bound": "fp64", "achieved": ach, "peak": peak, "unit": "TFLOP/s", "frac": ach / peak,
            "kernel": kname, "tuned_shapes": tuned, "ms_per_launch": ms, "flops_per_launch": fl,
            "pairs_per_atom": k["pairs"] / n / N, "triplets_per_atom": k["triplets"] / n / N}


CFG1_WORKLOAD = ("Cu fcc 2x2x2 conventional (32 atoms, a = 3.61 A, Gaussian 0.05 A jitter), 51-10-10-1 tanh FP64, "
                 "Rc 6 A: E+F+S, then a 200-iteration BFGS cell relax (RLXT 3)")
CFG4_WORKLOAD = ("Au fcc particle (a = 4.08 A, 5% vacancies, 0.05 A jitter, 15 A vacuum padding, no periodic "
                 "directions), 51-10-10-1 tanh FP64, Rc 6 A: E+F+S, then 500 NVT steps at 300 K")


def config1_leg(local, td, peak, cpu=True):
    """The small plain-method case: E+F+S atom-steps/s and a 200-iteration
    BFGS relax (structures/s) through the C-ABI, against the reference
    sources (CALL_MAISE and CELL_RELX over the project BFGS) on the host
    cores in the same run."""
    import maise_b200
    from maise_b200 import models, workloads

    w = workloads.fcc_supercell(n=2, a=3.61, jitter=0.05, seed=0)
    d = os.path.join(td, "cfg1")
    os.makedirs(d, exist_ok=True)
    basis = models.Basis()
    # a plain random network has no minimum for the cell to relax into (the
    # 9 lattice DOF collapse it until an atom has hundreds of neighbours);
    # the binding sign structure gives one (the cell contracts to ~151 A^3)
    models.random_model(os.path.join(d, "model"), w["spcz"], basis, (w["X"], w["LAT"], w["atmn"], 3), seed=1,
                        binding=True)
    NM = 400
    pot = maise_b200.Potential(os.path.join(d, "model"), device=local)
    rate, k = _efs_rate(pot, w, 3, 2000, NM)
    roof = _roofline(basis, 1, k, 32, peak, pot)  # before the relax adds its own tuner entries
    pot.relax(w["X"], w["LAT"], w["atmn"], ND=3, NM=NM, rlxt=3, mitr=5, etol=0.0)  # warm-up
    reps = 5
    t0 = time.perf_counter()
    for _ in range(reps):
        r = pot.relax(w["X"], w["LAT"], w["atmn"], ND=3, NM=NM, rlxt=3, mitr=200, etol=0.0)
    t_relax = (time.perf_counter() - t0) / reps
    out = {"workload": CFG1_WORKLOAD, "atoms": 32, "efs_atom_steps_per_s": rate,
           "model": "random weights with the binding sign structure (seed 1)",
           "roofline": roof, "relax_structures_per_s": 1.0 / t_relax,
           "relax_iterations": r["iters"], "relax_H": r["H"], "relax_calls": [r["n_energy"], r["n_force"]]}
    pot.close()
    if cpu:
        from oracle import RefOracle, ref_available

        if ref_available():
            cores = os.cpu_count() or 1
            ref = RefOracle(d, cores)
            ref.efs(w["X"], w["LAT"], w["atmn"], 3, NM=NM)
            n, t0 = 0, time.perf_counter()
            while n < 20 or time.perf_counter() - t0 < 2.0:
                ref.efs(w["X"], w["LAT"], w["atmn"], 3, NM=NM)
                n += 1
            ref_rate = 32 * n / (time.perf_counter() - t0)
            t0 = time.perf_counter()
            rr = ref.relax(w["X"], w["LAT"], w["atmn"], 3, rlxt=3, mitr=200, etol=0.0, NM=NM)
            t_ref = time.perf_counter() - t0
            out["cpu_baseline"] = {"efs_atom_steps_per_s": ref_rate, "relax_structures_per_s": 1.0 / t_ref,
                                   "relax_iterations": rr["iters"], "relax_H": rr["H"], "cores": cores,
                                   "kind": "reference",
                                   "sample": f"{n} CALL_MAISE calls; one CELL_RELX of up to 200 iterations"}
    return out


def particle_leg(local, td, peak, md_steps=500, cpu=True):
    """The large cluster: E+F+S atom-steps/s through mb_efs and 500 NVT steps
    at 300 K on the device (mb_md_nvt), against one reference CALL_MAISE on
    the host cores (first call, which allocates, excluded)."""
    import maise_b200
    from maise_b200 import atomic_mass, maxwell, models, workloads

    w = workloads.fcc_particle()
    N = len(w["atmn"])
    d = os.path.join(td, "cfg4")
    os.makedirs(d, exist_ok=True)
    basis = models.Basis()
    models.random_model(os.path.join(d, "model"), w["spcz"], basis, (w["X"], w["LAT"], w["atmn"], 0), seed=1)
    pot = maise_b200.Potential(os.path.join(d, "model"), device=local)
    rate, k = _efs_rate(pot, w, 0, 50, 100)
    V0 = maxwell([atomic_mass(w["spcz"][s]) for s in w["atmn"]], 300.0, seed=7)
    st = pot.md_nvt(w["X"], w["LAT"], w["atmn"], V0, 300.0, nsteps=10, ND=0, NM=100, trace=False)  # warm-up
    pot.md_profile(True, capacity=md_steps + 16)
    st = pot.md_nvt(st["X"], w["LAT"], w["atmn"], st["V"], 300.0, nsteps=md_steps, ND=0, NM=100, xi=st["xi"],
                    trace=True)
    md = pot.md_profile_read()
    pot.md_profile(False)
    out = {"workload": CFG4_WORKLOAD, "atoms": N, "efs_atom_steps_per_s": rate,
           "roofline": _roofline(basis, 1, k, N, peak, pot),
           "md_atom_steps_per_s": N * md["steps"] / (md["ms_total"] / 1e3), "md_steps": md["steps"],
           "md_final_K_eV": float(st["K"][-1])}
    pot.close()
    if cpu:
        from oracle import RefOracle, ref_available

        if ref_available():
            cores = os.cpu_count() or 1
            ref = RefOracle(d, cores)
            ref.efs(w["X"], w["LAT"], w["atmn"], 0, NM=100)
            t0 = time.perf_counter()
            ref.efs(w["X"], w["LAT"], w["atmn"], 0, NM=100)
            t_ref = time.perf_counter() - t0
            out["cpu_baseline"] = {"efs_atom_steps_per_s": N / t_ref, "cores": cores, "kind": "reference",
                                   "sample": "one CALL_MAISE E+F+S of the whole particle (first call excluded)"}
    return out


def profile_case(case):
    """Small cases sized for an ncu capture (a few MB on the device):
    md           the 4000-atom workload: the bench's 20 settle steps, then 10 NVT
                 steps at the settled neighbour counts (descriptor-pass launches;
                 the autotuner's trial launches all come before the last 10)
    relax-batch  64 Mg-Ca structures of the population relax, 20 BFGS iterations
    surrogate    features of 512 Cu-Pd-Ag offspring and 5 training epochs
    small-cell   the 32-atom Cu cell: 60 E+F+S passes (the autotuner's trial
                 launches come first, then the shape it keeps)"""
    import maise_b200
    from maise_b200 import atomic_mass, maxwell, workloads

    td = tempfile.mkdtemp()
    if case == "md":
        w, basis = workload()
        pot = maise_b200.Potential(make_model(td, w, basis))
        V = maxwell([atomic_mass(w["spcz"][s]) for s in w["atmn"]], 600.0, seed=7)
        st = pot.md_nvt(w["X"], w["LAT"], w["atmn"], V, 600.0, nsteps=SETTLE_STEPS, NM=100, trace=False)
        pot.md_nvt(st["X"], w["LAT"], w["atmn"], st["V"], 600.0, nsteps=10, NM=100, xi=st["xi"], trace=False)
    elif case == "small-cell":
        from maise_b200 import models

        w = workloads.fcc_supercell(n=2, a=3.61, jitter=0.05, seed=0)
        models.random_model(os.path.join(td, "model"), w["spcz"], models.Basis(), (w["X"], w["LAT"], w["atmn"], 3),
                            seed=1, binding=True)
        pot = maise_b200.Potential(os.path.join(td, "model"))
        for _ in range(60):
            pot.efs(w["X"], w["LAT"], w["atmn"], ND=3, NM=400)
        print("small-cell: tuned", pot.tune_table())
    elif case == "relax-batch":
        pop = workloads.ea_population(count=64, seed=3)
        pot = maise_b200.Potential(_binding_model(td, "pop", pop, (12, 20), 5))
        r = pot.relax_batch(pop, urep=100.0, rlxt=3, mitr=20, fmax=0.01)
        print(f"relax-batch: {r['evals']} evaluations in {r['ms']:.1f} ms")
    else:
        from maise_b200.surrogate import Surrogate

        pop = workloads.ea_population_chunked(512, seed=11, nmin=16, nmax=48, species=(29, 46, 47))
        sur = Surrogate(3)
        feat = sur.features(pop)
        sur.fit(feat, np.linspace(-4.0, -3.0, len(pop)), epochs=5, batch=256)
        sur.screen(pop)


def bench_config(N, world):
    """The `config` of both arms' lines (they run the same protocol)."""
    return {"workload": WORKLOAD, "atoms": N, "parallelism": f"replicas x{world}", "settle_steps": SETTLE_STEPS,
            "l2": "256 MiB buffer overwritten between timed steps (outside the step events)",
            "model": "random N(0,1/fan_in) weights, input ranges from the structure"}


REF_MAX_STEPS = 60  # longest timed run of the reference arm (about 4.4 s per step on 16 cores)


def run_reference(args, rank, world):
    """--impl reference: the reference MAISE sources (oracle/_ref, compiled from
    the reference's own files) run the same protocol as the GPU arm on the
    host cores -- the reference's Maxwell velocities (seed 7), SETTLE_STEPS
    untimed NVT steps, W untimed warm-up steps, then K timed steps of
    CELL_FRC + the NVT update of Dynamics (src/cmod.c:403-453).  Nothing of
    libmaise_b200 is loaded.  Ranks other than 0 exit without work."""
    from oracle import RefOracle, ref_available

    if rank != 0:
        return
    if not ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "reference sources were not compiled (oracle/_ref)"}))
        return
    w, basis = workload()
    N = len(w["atmn"])
    cores = os.cpu_count() or 1
    steps = min(args.steps, REF_MAX_STEPS)
    with tempfile.TemporaryDirectory() as td:
        make_model(td, w, basis)
        ref = RefOracle(td, cores)
        V = ref.maxwell(w["X"], w["LAT"], w["atmn"], 3, 600.0, seed=7, NM=100)
        st = ref.nvt(w["X"], w["LAT"], w["atmn"], 3, 600.0, 1.0, 25.0, SETTLE_STEPS + args.warmup, V=V, NM=100)
        t0 = time.perf_counter()
        st = ref.nvt(st["X"], w["LAT"], w["atmn"], 3, 600.0, 1.0, 25.0, steps, V=st["V"], xi=st["xi"], NM=100)
        dt = time.perf_counter() - t0
    value = N * steps / dt
    sample = (f"{steps} timed NVT steps of the 4000-atom structure (CELL_FRC + NVT update, OpenMP) after "
              f"{SETTLE_STEPS} settle and {args.warmup} warm-up steps from the reference's Maxwell velocities")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * dt / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": bench_config(N, world), "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference", "sample": sample},
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
    ap.add_argument("--no-population", action="store_true", help="skip the population relax and surrogate legs")
    ap.add_argument("--no-extra-legs", action="store_true", help="skip the 32-atom cell and 20000-atom particle legs")
    ap.add_argument("--profile-case", choices=["md", "relax-batch", "surrogate", "small-cell"],
                    help="run one small case of a hot kernel for an ncu capture and exit (no bench line)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    t_start = time.perf_counter()

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

    if args.profile_case:
        profile_case(args.profile_case)
        return
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

    # The timed steps are those of the thermostatted run: the random-weight
    # potential heats the ideal lattice in its first steps (about 85 neighbours
    # per atom against 65 later), so the workload starts after SETTLE_STEPS of
    # NVT, and then come the W warm-up steps (which also settle the neighbour
    # capacity and the kernel shape) and the K timed ones, whatever W is.
    st = pot.md_nvt(w["X"], w["LAT"], w["atmn"], V0, 600.0, dt=1.0, tau=25.0, nsteps=SETTLE_STEPS, NM=100,
                    trace=False)
    st = pot.md_nvt(st["X"], w["LAT"], w["atmn"], st["V"], 600.0, dt=1.0, tau=25.0, nsteps=args.warmup, NM=100,
                    xi=st["xi"], trace=False)
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
    step_s = max_over_ranks(steps_t["ms_total"] / 1e3, dist)
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
    e2e_s = max_over_ranks(e0.elapsed_time(e1) / 1e3, dist)
    e2e = {"value": world * N * k2 / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 3 * N * 8 + N * 4 + 9 * 8,
           "d2h_bytes_per_step": 3 * N * 8 + N * 8 + 3 * N * 8 + 16 * 8}

    # roofline of the fused descriptor/MLP/force kernel
    launches_k = max(1, kern["launches"])
    ms_k = kern["ms_total"] / launches_k
    flops = algorithmic_flops(basis, 3, kern["pairs"] / launches_k, kern["triplets"] / launches_k, N)
    fp64_peak = maise_b200.fp64_peak_tflops(local)
    achieved = flops / (ms_k * 1e-3) / 1e12
    kname, tuned = tuned_kernel(pot)
    roof = {"bound": "fp64", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
            "frac": achieved / fp64_peak, "traffic": profile_traffic(),
            "kernel": kname, "tuned_shapes": tuned, "ms_per_launch": ms_k,
            "flops_per_launch": flops, "pairs_per_atom": kern["pairs"] / launches_k / N,
            "triplets_per_atom": kern["triplets"] / launches_k / N,
            "peak_source": "FP64 FMA-chain probe measured in this run (MEASURED_PEAKS.json has no FP64 figure)",
            "hbm_peak_gbs_measured": peaks.get("hbm_gbs")}

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * step_s / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": bench_config(N, world),
            "e2e": e2e, "roofline": roof, "gpu_launches": launches, "clocks": clocks}
    def leg(name, fn):
        """one extra leg; a leg that raises is reported in its key, not fatal"""
        t0 = time.perf_counter()
        try:
            r = fn()
        except Exception as e:  # noqa: BLE001 -- the headline line must still print
            import traceback

            traceback.print_exc()
            r = {"error": f"{type(e).__name__}: {e}"}
        print(f"[bench] {name}: {time.perf_counter() - t0:.1f} s", file=sys.stderr, flush=True)
        return r

    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = leg("cpu_baseline", lambda: cpu_baseline(dict(w, X=st["X"]), td))
    if rank == 0 and not args.no_population:
        line["population_relax"] = leg("population_relax", lambda: population_relax(local, td))
        line["surrogate_generation"] = leg("surrogate_generation", lambda: surrogate_generation(local, td))
    if rank == 0 and not args.no_extra_legs:
        cpu = world == 1 and not args.no_cpu_baseline
        line["small_cell"] = leg("small_cell", lambda: config1_leg(local, td, fp64_peak, cpu=cpu))
        line["particle"] = leg("particle", lambda: particle_leg(local, td, fp64_peak, cpu=cpu))
    if rank == 0:
        print(json.dumps(line))
        print(f"[bench] total: {time.perf_counter() - t_start:.1f} s", file=sys.stderr, flush=True)
    pot.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
