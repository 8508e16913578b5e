#!/usr/bin/env python3
"""GFN-FF energy + gradient throughput on B200.

Default workload: the 20,480-atom cluster (6000 H2O + 40 C20H42, 6040 fragments; the largest
single-GPU configuration and one of the two the mixed-vs-FP64 target is quoted on), mixed
form, with the FP64 form measured beside it; the 512-conformer batch (20-300 atoms, the
other target configuration) is measured in the same run and reported under "configs".  One
step = one energy + analytic gradient evaluation of a fresh geometry (MD-like perturbation of
the structure; for the batch, of every molecule).

* ``value``: evaluations/s with coordinates resident in HBM, through the device entry
  point ``gfnff_energy_and_gradient_device``; each step timed with CUDA events on the
  handle's stream, L2 flushed (256 MiB write) before every timed step.
* ``e2e``: evaluations/s through the host C-ABI call ``gfnff_energy_and_gradient``
  (host coordinates in, energy + gradient + terms out, copies inside the timed region).
* ``roofline``: the dominant phase of the step against its arithmetic (FP64 FMA, measured
  by the library's microbenchmark) or HBM (MEASURED_PEAKS.json) bound.
* ``error_vs_oracle``: both forms against the CPU oracle (FP64 restatement of curcuma's CPU
  path) at the workload's own geometry, computed in the CPU-baseline leg.
* ``cpu_baseline``: the CPU oracle on the same workload at all host threads and at one
  thread (bounded samples: whole evaluations for the single structures, a time-bounded
  number of molecules for the batch); rank 0 at N=1 only.

``--impl reference`` times that CPU restatement alone as the reference arm (the
reference's own CPU code cannot be built here: Eigen and friends are fetched at configure
time).  Multi-GPU: ``--gpus N`` under torchrun runs independent replicas of the single
structures (weak scaling, no collective on the data path) and splits one conformer ensemble
into cost-balanced molecule shards gathered on rank 0; timings are reduced with MAX over
ranks.
"""
import argparse
import ctypes
import json
import os
import statistics
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "GFN-FF E+grad evals/s: mixed vs FP64 GPU at \u0394E\u22641e-6 Eh, \u0394F\u22641e-5 Eh/bohr"
UNIT = "evals/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", type=int, default=5)
    ap.add_argument("--also", default="4",
                    help="comma-separated further configs measured in the same run ('' = none)")
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile", action="store_true",
                    help="only set up the workload and run warmup + steps evaluations through the "
                         "public API (a short command for ncu captures); prints one line")
    return ap.parse_args()


def workload(cfg, rank=0, world=1):
    """The structure(s) of a config.  Under torchrun the single structures are replicas (every
    rank evaluates the same structure) and the conformer batch is one ensemble (seed 1004)
    split into cost-balanced molecule shards, one per rank (``shard_by_cost``); the fourth
    entry of a batch is (molecules of this rank, their indices in the ensemble, the
    ensemble)."""
    from curcuma_b200 import workloads as W
    from curcuma_b200.sharding import shard_by_cost
    if cfg == 1:
        return "n-C64H130 all-trans, 0.05 A noise (seed 1001)", *W.alkane(64, 1001)
    if cfg == 2:
        return "1000 H2O cluster, 1.0 g/cm3 (seed 1002)", *W.water_cluster(1000, 1002)
    if cfg == 3:
        return "Gly50 + 1500 H2O (seed 1003)", *W.solvated_peptide(50, 1500, 1003)
    if cfg == 5:
        return "6000 H2O + 40 C20H42 (seed 1005)", *W.large_cluster(6000, 40, 20, 1005)
    if cfg == 4:
        ens = W.conformer_batch(512, 1004)
        idx = shard_by_cost([len(z) for z, _ in ens], world)[rank]
        mols = [ens[i] for i in idx]
        Z = np.concatenate([z for z, _ in mols])
        X = np.concatenate([x for _, x in mols])
        return ("512 saturated C/N/O chains, 20-300 atoms log-uniform (seed 1004)", Z, X,
                (mols, idx, ens))
    raise SystemExit(f"unknown config {cfg}")


def max_over_ranks(x, dist, device):
    """The largest value over all ranks (times are reported for the slowest rank)."""
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def perturbed(X, k, sigma=0.01, seed=7):
    rng = np.random.default_rng(seed + k)
    return X + rng.normal(scale=sigma, size=X.shape)


class Clocks:
    """SM clock and clock-event reasons sampled through NVML (read-only queries) every
    5 ms by a background thread while the measurement runs; nvidia-smi's own polling
    loop is too coarse for timed regions of a few tens of milliseconds."""

    NAMES = {"hw_slowdown": "nvmlClocksEventReasonHwSlowdown",
             "hw_thermal_slowdown": "nvmlClocksEventReasonHwThermalSlowdown",
             "sw_thermal_slowdown": "nvmlClocksEventReasonSwThermalSlowdown",
             "sw_power_cap": "nvmlClocksEventReasonSwPowerCap"}

    def __init__(self, device):
        import threading
        self.samples, self.reasons, self.max_mhz = [], set(), 0.0
        self._stop = threading.Event()
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            vis = os.environ.get("CUDA_VISIBLE_DEVICES")
            idx = int(vis.split(",")[device]) if vis else device
            self.h = pynvml.nvmlDeviceGetHandleByIndex(idx)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM))
        except Exception:
            self.nv = None
            return
        self.t = threading.Thread(target=self._run, daemon=True)
        self.t.start()

    def _run(self):
        nv = self.nv
        while not self._stop.is_set():
            try:
                self.samples.append(float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)))
                mask = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                for k, attr in self.NAMES.items():
                    if mask & getattr(nv, attr):
                        self.reasons.add(k)
            except Exception:
                pass
            time.sleep(0.005)

    def stop(self):
        if self.nv is None:
            return None
        self._stop.set()
        self.t.join()
        if not self.samples:
            return None
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples), "source": "nvml"}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def pair_counts(Z, X):
    """Unique pairs evaluated per step: Coulomb r <= 100 bohr, D4 r <= 50 bohr within the
    60 bohr setup list (same geometry)."""
    Xb = X / 0.529177210903
    n = len(Z)
    nc = nd = 0
    for i0 in range(0, n, 512):
        d = np.linalg.norm(Xb[i0:i0 + 512, None, :] - Xb[None, :, :], axis=-1)
        idx = np.arange(i0, min(n, i0 + 512))[:, None] < np.arange(n)[None, :]
        nc += int(((d <= 100.0) & idx).sum())
        nd += int(((d <= 50.0) & idx).sum())
    return nc, nd


def roofline(phase_avg, info, fp64_peak, hbm_peak, hbm_src):
    """Algorithmic work per launch of the dominant phase.  FLOP conventions (erf/exp/
    sqrt/div = 1 op): Coulomb E+G 40/pair, D4 E+G 45/pair, repulsion 30/pair, CN+dCN
    35/pair, EEQ element 20; Cholesky n^3/3 + 2 n^2 (solve).  Pair counts are unique pairs
    (i < j): the algorithmic work, whatever the kernel evaluates."""
    name = max(phase_avg, key=phase_avg.get)
    ms = phase_avg[name]
    n, nred = info["n"], info["nred"]
    if name == "pairs":
        flops = 40.0 * info["coulomb_pairs"] + 45.0 * info["disp_pairs"]
        bound, unit, peak = "fp64", "TFLOP/s", fp64_peak
        achieved = flops / (ms * 1e-3) / 1e12
    elif name == "eeq_solve" and info.get("solver") == "pcg":
        # PCG: the reduced matrix is streamed once per matrix-vector product (the
        # iterations, the warm start and the true-residual check); only its lower
        # triangle from 4096 unknowns on
        mbytes = 8.0 * nred * (nred + 1) / 2.0 if info["pcg_lower"] else 8.0 * nred * nred
        if info.get("prod64", -1) >= 0:
            # mixed refinement solver: the inner iterations stream the FP32 copy (half the
            # bytes), the true-residual checks the FP64 triangle
            bytes_ = info["iters"] * mbytes / 2.0 + info["prod64"] * mbytes
        else:
            bytes_ = (info["iters"] + 2) * mbytes
        bound, unit, peak = "hbm", "GB/s", hbm_peak
        achieved = bytes_ / (ms * 1e-3) / 1e9
    elif name == "eeq_solve":
        flops = info.get("eeq_flops", nred ** 3 / 3.0 + 2.0 * nred ** 2)
        bound, unit, peak = "fp64", "TFLOP/s", fp64_peak
        achieved = flops / (ms * 1e-3) / 1e12
    elif name == "eeq_matrix":
        # lower triangle of the reduced matrix, four EEQ elements (20 FLOP each) per entry
        flops = 80.0 * nred * (nred + 1) / 2.0
        bound, unit, peak = "fp64", "TFLOP/s", fp64_peak
        achieved = flops / (ms * 1e-3) / 1e12
    else:
        # list-driven phases: term records + 24 B coordinates + 24 B gradient per atom ref
        bytes_ = info.get(f"bytes_{name}", 0.0)
        bound, unit, peak = "hbm", "GB/s", hbm_peak
        achieved = bytes_ / (ms * 1e-3) / 1e9 if bytes_ else 0.0
    traffic = None
    tf = ROOT / "profiles" / "traffic.json"
    if tf.exists():
        traffic = json.loads(tf.read_text()).get(f"config{info['config']}", {}).get(name)
    return {"kernel": name, "bound": bound, "achieved": achieved, "peak": peak, "unit": unit,
            "frac": achieved / peak if peak else None, "traffic": traffic, "ms": ms,
            "peak_source": "measured (fma microbenchmark)" if bound == "fp64" else hbm_src}


def cpu_model():
    try:
        for l in open("/proc/cpuinfo"):
            if l.startswith("model name"):
                return l.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def oracle_results(Z, X, mols, nthreads=0):
    """The CPU oracle at the workload's own geometry: (total energies per molecule,
    gradient N x 3, seconds of the oracle evaluations)."""
    from tests.oracle_api import Oracle
    parts = mols if mols else [(Z, X)]
    E, G, secs = [], [], 0.0
    for z, x in parts:
        o = Oracle(z, x)
        t = time.perf_counter()
        T, g, q, cn = o.engrad(x, nthreads)
        secs += time.perf_counter() - t
        E.append(T["total"])
        G.append(g)
    return np.array(E), np.concatenate(G), secs


def cpu_rate(Z, X, mols, nthreads, budget_s, max_evals=64):
    """Evaluations/s of the CPU oracle on a bounded sample of the workload: whole evaluations
    of the structure (at least one, more while the budget lasts), or molecules of the batch
    in ensemble order until the budget is spent (oracle set-up not timed).  Returns
    (rate, seconds, evaluations, description)."""
    from tests.oracle_api import Oracle
    if mols:
        k, secs = 0, 0.0
        while secs < budget_s and k < len(mols):
            z, x = mols[k]
            o = Oracle(z, x)
            t = time.perf_counter()
            o.engrad(perturbed(x, 2000 + k), nthreads)
            secs += time.perf_counter() - t
            k += 1
        return k / secs, secs, k, f"{k} molecules of the ensemble, one E+grad each"
    o = Oracle(Z, X)
    t = time.perf_counter()
    k = 0
    while k < 1 or (time.perf_counter() - t < budget_s and k < max_evals):
        o.engrad(perturbed(X, 2000 + k), nthreads)
        k += 1
    dt = time.perf_counter() - t
    return k / dt, dt, k, f"{k} full E+grad evaluation(s) of the structure"


def cpu_baseline(Z, X, mols, budget_s=20.0, t1_limit_s=60.0):
    """T = all host threads and T = 1 (the latter only where one evaluation at one thread
    fits t1_limit_s, estimated from the all-thread time)."""
    threads = os.cpu_count()
    rate, dt, k, what = cpu_rate(Z, X, mols, 0, budget_s)
    out = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port", "cpu": cpu_model(),
           "sample": f"{what} ({dt:.1f} s)", "what": "CPU restatement of curcuma's gfnff path (oracle/)"}
    est1 = (dt / k) * threads
    if mols or est1 <= t1_limit_s:
        r1, d1, k1, w1 = cpu_rate(Z, X, mols, 1, budget_s)
        out["t1"] = {"value": r1, "unit": UNIT, "cores": 1, "sample": f"{w1} ({d1:.1f} s)"}
    else:
        out["t1"] = {"value": None, "cores": 1,
                     "skipped": f"one evaluation at one thread estimated at {est1:.0f} s"}
    return out


def run_reference(args):
    """The reference arm: the CPU restatement of curcuma's path on all host threads, on the
    default workload; a bounded sample (at least one whole evaluation, at most ~60 s of
    evaluations, or molecules of the batch) stands for --steps K (echoed as given)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    wl = workload(args.config)
    desc, Z, X = wl[:3]
    mols = wl[3][0] if len(wl) > 3 else None
    threads = os.cpu_count()
    rate, dt, k, what = cpu_rate(Z, X, mols, 0, 60.0)
    line = {"metric": METRIC, "value": rate, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / rate,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": f"config {args.config}: {desc}", "natoms": int(len(Z))},
            "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": "port", "cpu": cpu_model(),
                             "sample": f"{what} ({dt:.1f} s); --steps/--warmup bound nothing here"},
            "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "CPU restatement of curcuma's gfnff path (oracle/), all host threads; the "
                    "reference's own build needs network-fetched Eigen and is unavailable here"}
    print(json.dumps(line), flush=True)


def measure(args, precision, Z, X, torch, dist, world, local, mols=None, units=None):
    """Device-timed and end-to-end throughput of one precision form on the workload
    (molecule evaluations per second; a batch handle evaluates all molecules per step).
    units: molecule evaluations per step over all ranks (default: world x this rank's)."""
    from curcuma_b200 import GFNFF, _lib

    n = len(Z)
    nmol = len(mols) if mols else 1
    units = units if units is not None else world * nmol
    gpu = GFNFF(precision=0 if precision == "fp64" else 1, device=local)
    t0 = time.perf_counter()
    ok = gpu.setMoleculeBatch(mols) if mols else gpu.setMolecule(Z, X)
    if not ok:
        raise SystemExit(gpu.getErrorMessage())
    setup_s = time.perf_counter() - t0
    lib, h = gpu._lib, gpu.handle
    stream = torch.cuda.ExternalStream(lib.gfnff_stream(h), device=torch.device("cuda", local))
    steps, warm = args.steps, args.warmup
    geoms = torch.tensor(np.stack([perturbed(X, k) / 0.529177210903 for k in range(steps + warm)]),
                         dtype=torch.float64, device="cuda")
    d_e = torch.zeros(nmol, dtype=torch.float64, device="cuda")
    d_g = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
    d_st = torch.zeros(nmol, dtype=torch.int32, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    P = ctypes.c_void_p

    def step(k):
        rc = lib.gfnff_energy_and_gradient_device(h, P(geoms[k].data_ptr()), P(d_e.data_ptr()),
                                                 P(d_g.data_ptr()), P(d_st.data_ptr()))
        if rc != 0:
            raise SystemExit(lib.gfnff_last_error(h).decode())

    clocks = Clocks(local)
    for k in range(warm):
        step(k)
    torch.cuda.synchronize()
    events = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    worst = 0
    # timed region: the step as the library runs it (graph replay), L2 flushed before each
    with torch.cuda.stream(stream):
        for k in range(steps):
            flush.zero_()
            events[k][0].record(stream)
            step(warm + k)
            events[k][1].record(stream)
            events[k][1].synchronize()
            worst = max(worst, int(d_st.max().item()))
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    step_ms = [a.elapsed_time(b) for a, b in events]
    kpe = gpu.kernelsPerEvaluation()   # of the graph the timed steps replayed
    # phase split: the same steps again with CUDA events between the phases (direct
    # launches), for the roofline of the dominant kernel
    phases = np.zeros(len(_lib.PHASES))
    buf = (ctypes.c_double * len(_lib.PHASES))()
    lib.gfnff_set_phase_timing(h, 1)
    step(0)
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        for k in range(steps):
            flush.zero_()
            step(warm + k)
            lib.gfnff_phase_times(h, buf, len(buf))
            phases += np.array(buf[:])
    torch.cuda.synchronize()
    total_ms = float(sum(step_ms))
    if world > 1:
        total_ms = max_over_ranks(total_ms, dist, "cuda")
    lib.gfnff_set_phase_timing(h, 0)
    # end to end through the host C ABI: host coordinates in, energy + gradient out
    hostX = [perturbed(X, 5000 + k) for k in range(steps)]
    evaluate = gpu.calculateEnergyBatch if mols else (lambda: gpu.calculateEnergy(True))
    for k in range(min(3, warm)):
        gpu.updateGeometry(perturbed(X, 4000 + k))
        evaluate()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t = time.perf_counter()
    for k in range(steps):
        gpu.updateGeometry(hostX[k])
        evaluate()
        if gpu.hasError():
            raise SystemExit(gpu.getErrorMessage())
    e2e_s = time.perf_counter() - t
    clk = clocks.stop()
    if world > 1:
        e2e_s = max_over_ranks(e2e_s, dist, "cuda")
    return {"gpu": gpu, "value": units * steps / (total_ms * 1e-3), "total_ms": total_ms, "step_ms": step_ms,
            "phase_avg": {k: v / steps for k, v in zip(_lib.PHASES, phases)}, "status": worst,
            "e2e": {"value": units * steps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 3 * n * 8,
                    "d2h_bytes_per_step": (3 * n + 16 * nmol) * 8 + 4 * nmol},
            "clocks": clk, "setup_s": setup_s, "solver": gpu.eeqSolver(), "iters": gpu.eeqIterations(),
            "prod64": gpu.eeqFP64Products() if nmol == 1 else -1, "kernels_per_eval": kpe}


def per_molecule_loop(mols, local):
    """The plain FP64 form called one molecule at a time through the host C ABI (one
    handle per molecule, set up beforehand): the way a per-molecule loop over a conformer
    set runs without batching."""
    from curcuma_b200 import GFNFF

    handles = []
    for z, x in mols:
        g = GFNFF(device=local)
        if not g.setMolecule(z, x):
            raise SystemExit(g.getErrorMessage())
        handles.append((g, x))
    for g, x in handles:
        g.calculateEnergy(True)
    t = time.perf_counter()
    for k, (g, x) in enumerate(handles):
        g.updateGeometry(perturbed(x, 7000 + k))
        g.calculateEnergy(True)
    dt = time.perf_counter() - t
    for g, _ in handles:
        g.close()
    return {"value": len(mols) / dt, "unit": UNIT, "seconds": dt,
            "what": "one host-API E+grad call per molecule, FP64, every molecule once"}


def md_run(gpu, Z, X, steps=1000, dt_fs=0.5):
    """NVE velocity Verlet from 300 K Maxwell-Boltzmann velocities (seed 1003), the
    E+grad step replayed as a CUDA graph; energy drift from a linear fit."""
    from curcuma_b200 import atomic_masses, maxwell_boltzmann

    gpu.updateGeometry(X)
    v0 = maxwell_boltzmann(atomic_masses(Z), 300.0, 1003)
    t = time.perf_counter()
    ep, ek = gpu.runMD(steps, dt_fs, v0)
    dt = time.perf_counter() - t
    if gpu.hasError():
        return {"error": gpu.getErrorMessage()}
    et = ep + ek
    slope = float(np.polyfit(np.arange(steps + 1) * dt_fs * 1e-3, et, 1)[0])
    return {"steps": steps, "dt_fs": dt_fs, "ms_per_step": 1e3 * dt / steps,
            "drift_eh_per_ps": slope, "drift_eh_per_ps_per_atom": slope / len(Z),
            "max_abs_dE_total_eh": float(np.abs(et - et[0]).max()), "T0_K": "300 (Maxwell-Boltzmann, seed 1003)"}


def fd_check(gpu, X, n_atoms=64, h_bohr=1e-4):
    """Central finite differences (h = 1e-4 bohr) on 64 seeded atoms against the analytic
    gradient of the FP64 form."""
    gpu.updateGeometry(X)
    gpu.calculateEnergy(True)
    G = gpu.getGradient()
    rng = np.random.default_rng(64)
    atoms = rng.choice(len(X), size=min(n_atoms, len(X)), replace=False)
    h = h_bohr * 0.529177210903
    err = []
    for a in atoms:
        for d in range(3):
            Xp, Xm = X.copy(), X.copy()
            Xp[a, d] += h
            Xm[a, d] -= h
            gpu.updateGeometry(Xp)
            ep = gpu.calculateEnergy(True)
            gpu.updateGeometry(Xm)
            em = gpu.calculateEnergy(True)
            err.append(abs((ep - em) / (2 * h_bohr) - G[a, d]))
    return {"atoms": len(atoms), "h_bohr": h_bohr, "max_abs_err_eh_per_bohr": float(max(err)),
            "rms_err_eh_per_bohr": float(np.sqrt(np.mean(np.square(err))))}


def run_config(args, cfg, torch, dist, world, rank, local):
    """Both precision forms on one config: device-timed and end-to-end throughput, phase split,
    roofline of the dominant phase, both forms at the workload's own geometry (gathered in
    ensemble order for a sharded batch), and at N=1 the CPU leg (the oracle's results for the
    error of both forms, and the timed CPU baselines).  Returns rank 0's summary (None on the
    other ranks); every rank takes the same collective steps."""
    from curcuma_b200.sharding import gather_ensemble

    wl = workload(cfg, rank, world)
    desc, Z, X = wl[:3]
    shard = wl[3] if len(wl) > 3 else None
    mols = shard[0] if shard else None
    n = len(Z)
    units = len(shard[2]) if shard else world
    forms = [args.precision] + [p for p in ("mixed", "fp64") if p != args.precision]
    res = {p: measure(args, p, Z, X, torch, dist, world, local, mols, units=units) for p in forms}
    main = res[args.precision]
    gpu = main["gpu"]
    natoms, nfrag = gpu.sizes()
    # both forms at the workload's own geometry: energies per molecule and gradients
    at_x = {}
    for p in forms:
        g = res[p]["gpu"]
        g.updateGeometry(X)
        e = np.atleast_1d(g.calculateEnergyBatch()[0] if mols else g.calculateEnergy(True))
        if g.hasError():
            raise SystemExit(g.getErrorMessage())
        at_x[p] = (e, g.getGradient())
    gathered = None
    if shard and world > 1:
        sizes = [len(z) for z, _ in shard[2]]
        at_x = {p: gather_ensemble(shard[1], e, G, sizes, dist.all_gather_object, world) for p, (e, G) in at_x.items()}
        gathered = {"molecules": len(sizes), "ranks": world, "energy_sum_eh": float(at_x[args.precision][0].sum())}
    launches = main["kernels_per_eval"]
    loop = per_molecule_loop(mols, local) if (mols and world == 1) else None
    if rank != 0:
        return None
    if mols:
        nc = nd = 0
        for z, x in mols:
            a_, b_ = pair_counts(z, x)
            nc += a_
            nd += b_
        hbs = []
        counts = {"molecules": len(mols)}
    else:
        nc, nd = pair_counts(Z, X)
        hbs = gpu.topology(6, 4)
        counts = {k: len(gpu.topology(kind, w)) for k, kind, w in
                  [("bonds", 0, 2), ("angles", 1, 3), ("torsions", 2, 4), ("inversions", 3, 4), ("hbonds", 6, 4),
                   ("xbonds", 7, 3), ("atm", 12, 3), ("batm", 13, 3)]}
    sym = os.environ.get("GFNFF_PCG_SYM")
    info = {"n": n, "nred": n - nfrag, "config": cfg, "coulomb_pairs": nc, "disp_pairs": nd,
            "solver": main["solver"], "iters": main["iters"], "prod64": main["prod64"],
            "pcg_lower": (sym != "0") if sym is not None else (n - nfrag) >= 4096,
            "bytes_hbonds": len(hbs) * (19 * 8 + 3 * 48 + 2 * 48)}
    if mols:   # block-diagonal EEQ: one reduced system per molecule (one fragment each)
        info["eeq_flops"] = sum((len(z) - 1) ** 3 / 3.0 + 2.0 * (len(z) - 1) ** 2 for z, _ in mols)
    hbm_peak, hbm_src = measured_peaks()
    fp64_peak = gpu._lib.gfnff_fma_peak_tflops(local, 1)
    roof = roofline(main["phase_avg"], info, fp64_peak, hbm_peak, hbm_src)
    if roof["kernel"] == "eeq_solve" and main["solver"] == "pcg" and main["iters"] > 0:
        # the solve as iteration latency (what bounds it while M stays in L2)
        nprod = main["iters"] + (main["prod64"] if main["prod64"] >= 0 else 2)
        roof["us_per_iteration"] = 1e3 * roof["ms"] / nprod
        if main["prod64"] >= 0:
            roof["fp32_inner_iterations"] = main["iters"]
            roof["fp64_products"] = main["prod64"]
        roof["matrix_in_l2"] = not info["pcg_lower"]
    summary = {
        "workload": f"config {cfg}: {desc}", "natoms": natoms, "nfrag": nfrag,
        "value": main["value"], "e2e": main["e2e"], "ms_per_step": main["total_ms"] / args.steps,
        "step_ms_median": statistics.median(main["step_ms"]), "status": main["status"],
        "setup_s": round(main["setup_s"], 3), "gpu_launches_per_step": launches, "roofline": roof,
        "forms": {p: {"value": r["value"], "e2e": r["e2e"]["value"], "eeq_solver": r["solver"],
                      "eeq_iterations_last_step": r["iters"],
                      "phase_ms": {k: round(v, 4) for k, v in r["phase_avg"].items()}}
                  for p, r in res.items()},
        "mixed_vs_fp64": res["mixed"]["value"] / res["fp64"]["value"],
        "mixed_vs_fp64_e2e": res["mixed"]["e2e"]["value"] / res["fp64"]["e2e"]["value"],
        "pairs": {"coulomb": nc, "dispersion": nd}, "terms": counts, "clocks": main["clocks"],
        "parallelism": (f"one ensemble in {world} cost-balanced molecule shards, gathered on the host" if mols
                        else f"replicas x{world}"),
        "scaling": "strong" if mols and world > 1 else "weak",
    }
    if gathered:
        summary["gathered"] = gathered
    if loop:
        summary["per_molecule_loop_fp64"] = loop
        summary["batch_vs_loop"] = main["value"] / loop["value"]
    if cfg == 3:
        from curcuma_b200 import GFNFF
        exact = {}
        for p in ("mixed", "fp64"):
            g = GFNFF(precision=0 if p == "fp64" else 1, device=local, exact_gradient=True)
            if not g.setMolecule(Z, X):
                raise SystemExit(g.getErrorMessage())
            exact[p] = g
        summary["md"] = {p: md_run(g, Z, X) for p, g in exact.items()}
        summary["md"]["gradient"] = "exact (derivative of the energy)"
        summary["md"]["note"] = ("C3 spans 274 bohr: ~500 atom pairs cross the 100 bohr Coulomb cut of the "
                                 "reference's energy every step, each a jump of up to ~2e-3 Eh, so E_total "
                                 "random-walks independently of dt; systems without cut pairs conserve it")
        summary["fd_check"] = {"exact_fp64": fd_check(exact["fp64"], X),
                               "reference_fp64": fd_check(res["fp64"]["gpu"], X)}
    if world == 1 and not args.no_cpu_baseline:
        # CPU leg: the oracle at the workload's geometry gives the error of both forms, then
        # the timed baselines
        E_o, G_o, _ = oracle_results(Z, X, mols)
        summary["error_vs_oracle"] = {
            p: {"dE_eh": float(np.abs(e - E_o).max()), "max_dF_eh_per_bohr": float(np.abs(G - G_o).max())}
            for p, (e, G) in at_x.items()}
        summary["error_vs_oracle"]["geometry"] = "the workload's own geometry" + (
            ", every molecule" if mols else "")
        summary["cpu_baseline"] = cpu_baseline(Z, X, mols)
    return summary


def run_ours(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    cfgs = [args.config] + [int(c) for c in args.also.split(",") if c.strip() and int(c) != args.config]
    summaries = {c: run_config(args, c, torch, dist, world, rank, local) for c in cfgs}
    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return
    head = summaries[args.config]
    hbm_peak, hbm_src = measured_peaks()
    from curcuma_b200 import _lib
    lib = _lib.load()
    fp64_peak = lib.gfnff_fma_peak_tflops(local, 1)
    fp32_peak = lib.gfnff_fma_peak_tflops(local, 0)
    steps = args.steps
    launches = head["gpu_launches_per_step"]
    line = {"metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": world, "steps": steps,
            "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True,
            "scaling": head["scaling"], "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "mixed(f32 short-range, f64 long-range/EEQ/sums)",
            "data": "synthetic",
            "config": {"workload": head["workload"], "natoms": head["natoms"], "nfrag": head["nfrag"],
                       "precision": args.precision, "eeq_solver": head["forms"][args.precision]["eeq_solver"],
                       "eeq_iterations_last_step": head["forms"][args.precision]["eeq_iterations_last_step"],
                       "l2": "flushed before every timed step (256 MiB write)",
                       "parallelism": head["parallelism"], "setup_s": head["setup_s"]},
            "e2e": head["e2e"], "gpu_launches": launches * steps if launches and launches > 0 else None,
            "kernels_per_step": launches, "roofline": head["roofline"],
            "phase_ms": head["forms"][args.precision]["phase_ms"], "step_ms_median": head["step_ms_median"],
            "status": head["status"], "forms": head["forms"], "mixed_vs_fp64": head["mixed_vs_fp64"],
            "mixed_vs_fp64_e2e": head["mixed_vs_fp64_e2e"], "clocks": head["clocks"],
            "peaks": {"fp64_fma_tflops": fp64_peak, "fp32_fma_tflops": fp32_peak, "hbm_gbs": hbm_peak,
                      "source": "FMA: library microbenchmark (csrc/device/peaks.cu); HBM: " + hbm_src},
            "configs": {str(c): v for c, v in summaries.items()}}
    for k in ("error_vs_oracle", "cpu_baseline"):
        if k in head:
            line[k] = head[k]
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def run_profile(args):
    """Set-up plus warmup + steps evaluations of the workload and nothing else: the launch
    sequence a profiler should see (set-up's solver probes, then the evaluations)."""
    import torch

    from curcuma_b200 import GFNFF

    torch.cuda.set_device(0)
    wl = workload(args.config)
    desc, Z, X = wl[:3]
    mols = wl[3][0] if len(wl) > 3 else None
    g = GFNFF(precision=0 if args.precision == "fp64" else 1, device=0)
    if not (g.setMoleculeBatch(mols) if mols else g.setMolecule(Z, X)):
        raise SystemExit(g.getErrorMessage())
    for k in range(args.warmup + args.steps):
        g.updateGeometry(perturbed(X, k))
        if mols:
            g.calculateEnergyBatch()
        else:
            g.calculateEnergy(True)
        if g.hasError():
            raise SystemExit(g.getErrorMessage())
    print(json.dumps({"profile": f"config {args.config}: {desc}", "precision": args.precision,
                      "evals": args.warmup + args.steps, "eeq_solver": g.eeqSolver()}), flush=True)


def main():
    args = parse()
    if args.profile:
        run_profile(args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
