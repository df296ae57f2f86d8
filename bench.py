#!/usr/bin/env python
"""Throughput of the B200 MD timestep hot path (atom-steps/s).

Headline workload (value): 1,048,576-atom LJ fluid (FCC 64^3 cells, rho* 0.8442,
T* 0.72, rc 2.5 sigma, skin 0.3 sigma, dt 0.005), mixed precision (FP32 pair math,
FP64 positions and sums).  The same line carries, for the metric's other
halves: the FP64 GPU form of the same kernels, the 8000-ion Ewald electrolyte
(L = 40, alpha 0.3, rc 10, kmax 8) in both precisions, and the relative force
error of the mixed form against the FP64 form on identical states.

A step is one velocity-Verlet step of the whole system (list maintenance,
forces, integration).  Inputs (positions, list) are far larger than L2 for the
headline workload, so no flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

N > 1 (under torchrun): every rank advances its own replica of the workload
(the path does not shard; replicas only), timing is the max over ranks.
`--impl reference` times the reference's own CPU implementation
(oracle/_ref/ref_harness, the unmodified reference compiled from its sources)
on the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "atom-steps/s: 1M LJ + 8K-ion Ewald, mixed vs FP64 GPU at ≤1e-5 rel force err"
UNIT = "atom-steps/s"


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class Clocks:
    """SM clocks and clock-event (throttle) reasons sampled during a region:
    NVML polled every 20 ms from a thread (read-only queries), else
    nvidia-smi at its 200 ms minimum."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index: int):
        self.index = index
        self.p = None
        self.f = None
        self.samples = None
        self.mx = None
        self.stop = None
        self.t = None

    def _nvml_start(self):
        import threading
        import pynvml
        pynvml.nvmlInit()
        h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
        self.mx = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
        bits = [pynvml.nvmlClocksEventReasonHwSlowdown, pynvml.nvmlClocksEventReasonHwThermalSlowdown,
                pynvml.nvmlClocksEventReasonSwThermalSlowdown, pynvml.nvmlClocksEventReasonSwPowerCap]
        self.samples = []
        self.stop = threading.Event()

        def poll():
            while not self.stop.is_set():
                try:
                    sm = float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM))
                    r = int(pynvml.nvmlDeviceGetCurrentClocksEventReasons(h))
                    self.samples.append((sm, [nm for nm, bit in zip(self.NAMES, bits) if r & bit]))
                except Exception:
                    pass
                self.stop.wait(0.02)

        self.t = threading.Thread(target=poll, daemon=True)
        self.t.start()

    def __enter__(self):
        try:
            self._nvml_start()
            return self
        except Exception:
            self.samples = None
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.t:
            self.stop.set()
            self.t.join(timeout=2)
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()

    def summary(self):
        if self.samples is not None:
            if not self.samples:
                return None
            reasons = sorted({nm for _, rs in self.samples for nm in rs})
            return {"sm_mhz": statistics.median([sm for sm, _ in self.samples]), "sm_max_mhz": self.mx,
                    "reasons": reasons, "samples": len(self.samples), "source": "nvml, 20 ms"}
        if not self.f:
            return None
        try:
            self.f.seek(0)
            rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        except Exception:
            return None
        finally:
            try:
                os.unlink(self.f.name)
            except Exception:
                pass
        sm, mx, reasons = [], None, set()
        for r in rows:
            r = [x.strip() for x in r]
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except (ValueError, IndexError):
                continue
            for k, nm in enumerate(self.NAMES):
                if len(r) > 5 + k and r[5 + k].lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm),
                "source": "nvidia-smi, 200 ms"}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def fma_peaks(abi, device: int):
    """FP32 and FP64 FMA-pipe peaks of this GPU, measured now (cvr_measure_fma_peak:
    FMA-only kernel filling every SM, best of 5, CUDA events), TFLOP/s."""
    try:
        f32, _ = abi.fma_peak(device, False, 2000)
        f64, _ = abi.fma_peak(device, True, 1000)
        return {"fp32_tflops": f32, "fp64_tflops": f64, "source": "cvr_measure_fma_peak, measured in this run"}
    except Exception as e:  # pragma: no cover - reported, not hidden
        return {"fp32_tflops": None, "fp64_tflops": None, "source": f"failed: {e}"}


def lj_pair_flops_per_atom(n_cand: float, density: float, rc: float) -> float:
    """Algorithmic FP32 flops of one atom's row in the LJ pair kernel: 8 per
    list entry (displacement 3, r^2 5) and 15 more per pair inside rc (1/r^2,
    (s/r)^6, the force coefficient and three force FMAs), FMA = 2; the pairs
    inside rc of a uniform fluid number rho (4/3) pi rc^3."""
    n_rc = density * 4.0 / 3.0 * np.pi * rc ** 3
    return 8.0 * n_cand + 15.0 * n_rc


def profiled_traffic(name: str):
    """dram bytes per launch of a kernel, from a committed ncu summary (profiles/)."""
    path = os.path.join(ROOT, "profiles", name)
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("dram_bytes_per_launch_full_size:"):
                    return float(line.split(":", 1)[1].split()[0])
    except Exception:
        pass
    return None


# ---------------------------------------------------------------- GPU arm

def time_run(sim, torch, steps: int, warmup: int, dist=None, thermo_every: int = 0):
    """Device time of exactly `steps` steps on the context's stream (CUDA
    events), bracketed by barrier + synchronize; returns ms."""
    stream = torch.cuda.ExternalStream(sim.stream)
    sim.run(warmup)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sim.run(steps, thermo_every)
    e1.record(stream)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    return e0.elapsed_time(e1)


def max_over_ranks(x: float, dist, torch, device: str = "cuda"):
    """The slowest rank's time (replicas: the job ends when the last one does)."""
    if dist is None:
        return x
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(ms_local: float, atoms_per_rank: int, steps: int, dist, torch, device: str = "cuda"):
    """(max-over-ranks ms, whole-job atom-steps/s): every rank advances its own
    replica of atoms_per_rank atoms for `steps` steps."""
    world = dist.get_world_size() if dist is not None else 1
    ms_max = max_over_ranks(ms_local, dist, torch, device)
    return ms_max, world * atoms_per_rank * steps / (ms_max / 1e3)


def force_error(abi, s):
    """Mixed-form accelerations against the FP64 form on the same state:
    (global ||dF||/||F||, max_i |dF_i| / rms|F|)."""
    a = abi.Simulation(s, precision=abi.PREC_MIXED)
    b = abi.Simulation(s, precision=abi.PREC_FP64)
    fa, _ = a.compute_forces()
    fb, _ = b.compute_forces()
    a.close()
    b.close()
    d = np.linalg.norm(fa - fb, axis=1)
    nb = np.linalg.norm(fb, axis=1)
    return float(np.linalg.norm(d) / np.linalg.norm(nb)), float(d.max() / np.sqrt(np.mean(nb ** 2)))


def ions_line(abi, W, torch, steps: int, warmup: int, device: int = 0):
    """8000 ions (LJ + Ewald r + k), both precisions: K graph-launched steps
    timed with CUDA events, then K more steps with per-kernel events (stream
    launches) for the k-space / pair breakdown."""
    s_ion = W.config_ions_8000(seed=2)
    ion = {}
    for nm, p in (("mixed", abi.PREC_MIXED), ("fp64", abi.PREC_FP64)):
        si = abi.Simulation(s_ion, precision=p, device=device)
        si.run(warmup)
        b0 = si.info()["builds"]
        msi = time_run(si, torch, steps, 0)
        nbuilds = si.info()["builds"] - b0
        si.set_kernel_timing(True)
        msk = time_run(si, torch, steps, 0)
        kms, kn = si.kernel_time(abi.KT_KSPACE)
        pms, pn = si.kernel_time(abi.KT_PAIR)
        bms, _ = si.kernel_time(abi.KT_BUILD)
        info = si.info()
        nk = info["nk"]
        ion[nm] = {"value": s_ion.n * steps / (msi / 1e3), "ms_per_step": msi / steps, "list_builds": nbuilds,
                   "kspace_force": "tcgen05 TF32 hi/lo" if info["kspace_tensor_cores"] else "CUDA cores",
                   "kernel_window_ms_per_step": msk / steps, "kspace_ms_per_step": kms / max(kn, 1),
                   "pair_ms_per_step": pms / max(pn, 1), "build_ms_per_step": bms / steps,
                   # algorithmic flops of the k-space pass: S(k) and the force each 4 FMA
                   # (8 flops) per (k-vector, atom); of the pair pass: ~45 per list entry
                   "kspace_flops_per_step": 2 * 8.0 * nk * s_ion.n,
                   "kspace_tflops": 2 * 8.0 * nk * s_ion.n / (kms / max(kn, 1) / 1e3) / 1e12 if kms > 0 else None,
                   "pair_tflops": 45.0 * si.info()["list_entries"] * 1.0 / (pms / max(pn, 1) / 1e3) / 1e12
                   if pms > 0 else None}
        si.close()
    return ion


def replica_line(abi, W, torch, nsteps: int):
    """1024 replicas (64-2048 atoms, rho* 0.8, half charged +-1, alpha 0.35,
    k_max 6, T 0.7-1.5) advanced nsteps steps in one graph launch; device time
    with CUDA events on the batch stream, after the autotuning run."""
    b = W.replica_batch()
    bt = abi.Batch(b.n, b.box, b.mass, b.charge)
    bt.set_forces(b.epsilon, b.sigma, b.rc_lj, b.rc_r, b.alpha, b.kmax, b.k_e, b.dt)
    bt.set_state(b.pos, b.vel, b.type)
    bt.run(3)
    stream = torch.cuda.ExternalStream(bt.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    out = bt.run(nsteps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    info = bt.info()
    bt.close()
    return {"value": float(b.n.sum()) * nsteps / (ms / 1e3), "unit": UNIT, "steps_in_one_launch": nsteps,
            "ms_per_step": ms / nsteps, "atoms": int(b.n.sum()), "replicas": len(b.n),
            "classes": info["classes"], "nan": bool(np.isnan(out).any()),
            "note": "rc_r = L/2 (minimum image), rc_lj = min(2.5, L/2)"}


def adjoint_line(abi, W, torch, nsteps: int = 500):
    """Loss + gradient of the 4000-atom two-species mixture over 500 steps
    (dt 0.002), checkpoints every 50, mixed and FP64; wall time of the
    synchronous C-ABI call (forward, re-run segments, reverse sweep)."""
    s = W.adjoint_mixture()
    out = {}
    for nm, prec in (("mixed", abi.PREC_MIXED), ("fp64", abi.PREC_FP64)):
        a = abi.Adjoint.from_system(s, prec)
        a.loss_grad(min(20, nsteps), 10)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        J, g = a.loss_grad(nsteps, 50)
        dt = time.perf_counter() - t0
        out[nm] = {"seconds": dt, "steps": nsteps, "gradient_atom_steps_per_s": 4000 * nsteps / dt, "loss": J}
        a.close()
    out["fp64_over_mixed_time"] = out["fp64"]["seconds"] / out["mixed"]["seconds"]
    return out


def gpu_arm(args):
    import torch
    rank, world, local = dist_env()
    dist = None
    if world > 1:
        import torch.distributed as td
        torch.cuda.set_device(local)
        td.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
        dist = td
    else:
        torch.cuda.set_device(0)
    from caviar_b200 import build as B
    B.build()
    from caviar_b200 import _abi as abi
    from caviar_b200 import workloads as W

    steps, warmup = args.steps, max(3, args.warmup)
    peaks = fma_peaks(abi, local)
    s_lj = W.config_lj_1m(seed=3 + rank)
    n = s_lj.n

    # --- headline: 1M LJ, mixed, device-resident inputs
    sim = abi.Simulation(s_lj, precision=abi.PREC_MIXED, device=local)
    sim.run(warmup)
    l0 = sim.launches
    b0 = sim.info()["builds"]
    # timed region: one CUDA graph per step (list build in a conditional node), no per-kernel events
    with Clocks(local) as clk:
        ms = time_run(sim, torch, steps, 0, dist)
    launches = sim.launches - l0
    info = sim.info()
    builds = info["builds"] - b0
    ms_max, value = whole_job_rate(ms, n, steps, dist, torch)
    # kernel breakdown: the next K steps of the same run with CUDA events around every kernel
    # (stream launches instead of the graph, so these steps run a little slower than the timed ones)
    sim.set_kernel_timing(True)
    ms_k = time_run(sim, torch, steps, 0, dist)
    pair_ms, pair_n = sim.kernel_time(abi.KT_PAIR)
    build_ms, build_n = sim.kernel_time(abi.KT_BUILD)
    integ_ms, integ_n = sim.kernel_time(abi.KT_INTEGRATE)
    sim.set_kernel_timing(False)

    # --- e2e through the public API: host (pinned) buffers in, results out
    pos_h = torch.from_numpy(np.ascontiguousarray(s_lj.pos)).pin_memory()
    vel_h = torch.from_numpy(np.ascontiguousarray(s_lj.vel)).pin_memory()
    typ_h = torch.from_numpy(np.ascontiguousarray(s_lj.type, np.int32)).pin_memory()
    out_p = torch.empty((n, 3), dtype=torch.float64).pin_memory()
    out_v = torch.empty((n, 3), dtype=torch.float64).pin_memory()
    thermo = torch.empty((steps, abi.N_THERMO), dtype=torch.float64).pin_memory()
    sim2 = abi.Simulation(s_lj, precision=abi.PREC_MIXED, device=local)
    sim2.run(warmup)
    # three whole end-to-end jobs (state in from host, K steps, state out to
    # host), each timed by the host clock around the public calls; the
    # median is reported, all three are listed
    e2e_runs = []
    for _ in range(3):
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        t0 = time.perf_counter()
        sim2.set_state_ptr(n, pos_h.data_ptr(), vel_h.data_ptr(), typ_h.data_ptr())
        sim2.run_ptr(steps, 1, thermo.data_ptr())
        sim2.get_state_ptr(out_p.data_ptr(), out_v.data_ptr(), 0)
        torch.cuda.synchronize()
        e2e_runs.append(max_over_ranks(time.perf_counter() - t0, dist, torch))
    e2e_s = statistics.median(e2e_runs)
    e2e = world * n * steps / e2e_s
    h2d = n * (3 * 8 + 3 * 8 + 4)
    d2h = n * (3 * 8 + 3 * 8)
    sim2.close()

    # --- secondary lines (FP64 form, 8K ions, replicas, adjoint, force error)
    # and the CPU baseline: single-GPU runs only (under torchrun the other
    # ranks would wait for them at the closing barrier)
    sec = {}
    if world == 1:
        sim64 = abi.Simulation(s_lj, precision=abi.PREC_FP64, device=local)
        ms64 = time_run(sim64, torch, steps, warmup)
        sec["lj_1m_fp64"] = {"value": n * steps / (ms64 / 1e3), "ms_per_step": ms64 / steps}
        sim64.close()
        ion = ions_line(abi, W, torch, steps, warmup, local)
        sec["ions_8k_mixed"] = ion["mixed"]
        sec["ions_8k_fp64"] = ion["fp64"]
        sec["mixed_over_fp64"] = {"lj_1m": value / world / sec["lj_1m_fp64"]["value"],
                                  "ions_8k": ion["mixed"]["value"] / ion["fp64"]["value"]}
        sec["replicas_1024"] = replica_line(abi, W, torch, args.replica_steps)
        sec["adjoint_4000"] = adjoint_line(abi, W, torch, args.adjoint_steps)
        g1, m1 = force_error(abi, W.fcc_lattice(64, 0.8442, 0.72, seed=3, jitter=0.1))
        g2, m2 = force_error(abi, W.config_ions_8000(seed=2))
        sec["force_rel_err_mixed_vs_fp64"] = {"lj_1m": {"global": g1, "max_over_rms": m1},
                                              "ions_8k": {"global": g2, "max_over_rms": m2}}

    # --- roofline of the dominant kernel (the pair kernel on the headline workload)
    peak, peak_kind = measured_peaks()
    real_b = 4
    mean_cnt = info["list_entries"] / n
    bytes_launch = n * (4 * real_b + 4 + 3 * real_b) + 4.0 * mean_cnt * n
    pair_avg_ms = pair_ms / max(pair_n, 1)
    achieved = bytes_launch / (pair_avg_ms / 1e3) / 1e9
    traffic = profiled_traffic("pair_lj1m.txt")
    density = n / float(np.prod(np.asarray(s_lj.hi) - np.asarray(s_lj.lo)))
    flops_launch = n * lj_pair_flops_per_atom(mean_cnt, density, s_lj.lj.cutoff)
    fp32_achieved = flops_launch / (pair_avg_ms / 1e3) / 1e12
    fp32_peak = peaks["fp32_tflops"]
    # roofline: the pair kernel's arithmetic intensity against the ridge point
    # (FP32 peak / HBM peak) says which roof binds it
    ai = flops_launch / bytes_launch
    ridge = (fp32_peak * 1e12) / (peak * 1e9) if fp32_peak else None
    bound = "hbm" if (ridge is None or ai < ridge) else "fp32"
    sim.close()

    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(s_lj, budget_s=args.cpu_budget)
        sec["ions_8k_mixed"]["cpu_baseline"] = cpu_baseline_ions(min(15.0, args.cpu_budget))
        sec["replicas_1024"]["cpu_baseline"] = cpu_baseline_replicas(min(10.0, args.cpu_budget))
        sec["adjoint_4000"]["cpu_baseline"] = cpu_baseline_adjoint()

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": steps, "warmup": warmup,
            "ms_per_step": ms_max / steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "fp32",
            "precision": "fp32 pair/k-space math, fp64 positions + S(k) + energy/virial sums",
            "data": "synthetic (seeded FCC lattice + Maxwell-Boltzmann velocities)",
            "config": {"workload": "LJ fluid N=1048576 (FCC 64^3, rho*=0.8442, T*=0.72, rc=2.5, skin=0.3, dt=0.005), "
                                   "mixed precision", "n_atoms": n, "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (list ~%d MB, positions %d MB)" % (
                           int(4 * mean_cnt * n / 1e6), int(n * 24 / 1e6)),
                       "rebuild_policy": "displacement (skin/2)", "list_builds_in_window": builds,
                       "mean_neighbours": mean_cnt},
            "roofline": {"bound": bound, "kernel": "k_pair (LJ, full Verlet list)", "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                         "peak_source": peak_kind, "bytes_per_launch": bytes_launch,
                         "fp32": {"achieved": fp32_achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                                  "frac": fp32_achieved / fp32_peak if fp32_peak else None,
                                  "flops_per_launch": flops_launch, "peak_source": peaks["source"]},
                         "arithmetic_intensity_flop_per_byte": ai, "ridge_flop_per_byte": ridge,
                         "limiter": "neither roof: latency of the neighbour gathers (ncu: long-scoreboard "
                                    "stalls, profiles/pair_lj1m.txt)",
                         "avg_launch_ms": pair_avg_ms, "launches": pair_n,
                         "share_of_step": pair_ms / ms_k if ms_k > 0 else None,
                         "timing": "pair kernel bracketed by CUDA events on the context stream over a second "
                                   "K-step window of the same run (stream launches, ms_per_step %.4f)" % (
                                       ms_k / steps)},
            "kernel_ms_per_step": {"pair": pair_ms / max(steps, 1), "build": build_ms / max(steps, 1),
                                   "integrate": integ_ms / max(steps, 1)},
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": h2d / steps, "d2h_bytes_per_step":
                    d2h / steps + 8 * abi.N_THERMO,
                    "note": "cvr_set_state from pinned host buffers + cvr_run (setup, K steps, per-step thermo "
                            "record read back) + cvr_get_state to pinned host buffers; median of three whole jobs",
                    "seconds_per_job": e2e_runs},
            "gpu_launches": launches,
            "fma_peaks": peaks,
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
            "secondary": sec,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


# ----------------------------------------------------- reference CPU arm

def reference_step_time(s, max_steps: int, budget_s: float):
    """Run the unmodified reference on `s` until `budget_s` seconds of steps
    (at least 2, at most max_steps + 1) and return (seconds per step after the
    first, steps timed, seconds of the first step, which includes setup)."""
    from oracle import oracle as O
    if not O.harness_available():
        return None
    r = O.run_reference(s, "run", nsteps=max_steps + 1, budget_s=budget_s, timeout=budget_s * 10 + 600)
    k = int(r["steps_done"]) - 1
    return float(r["wall_rest"]) / k, k, float(r["wall_first"])


def cpu_baseline(s, budget_s: float = 20.0):
    try:
        res = reference_step_time(s, 1000, budget_s)
    except Exception as e:  # pragma: no cover - reported, not hidden
        return {"value": None, "unit": UNIT, "cores": 1, "kind": "reference", "sample": f"failed: {e}"}
    if res is None:
        return {"value": None, "unit": UNIT, "cores": 1, "kind": "reference", "sample": "harness not built"}
    per, k, first = res
    return {"value": s.n / per, "unit": UNIT, "cores": 1, "kind": "reference",
            "sample": f"{k} velocity-Verlet steps of the same {s.n}-atom system after a setup step "
                      f"({first:.1f} s); serial reference (its OpenMP build does not compile)"}


def cpu_baseline_ions(budget_s: float = 15.0):
    """The unmodified reference on the 8000-ion Ewald system (config of the
    ions line): whole steps after its setup step until budget_s, 1 core."""
    from caviar_b200 import workloads as W
    s = W.config_ions_8000(seed=2)
    try:
        res = reference_step_time(s, 100, budget_s)
    except Exception as e:  # pragma: no cover - reported, not hidden
        return {"value": None, "unit": UNIT, "cores": 1, "kind": "reference", "sample": f"failed: {e}"}
    if res is None:
        return {"value": None, "unit": UNIT, "cores": 1, "kind": "reference", "sample": "harness not built"}
    per, k, first = res
    return {"value": s.n / per, "unit": UNIT, "cores": 1, "kind": "reference",
            "sample": f"{k} velocity-Verlet steps of the same 8000-ion system after a setup step ({first:.1f} s)"}


def cpu_baseline_replicas(budget_s: float = 10.0, procs: int = 8):
    """The unmodified reference on replicas of the batch, one process per
    core running concurrently: the replicas at the batch's size octiles
    (its sizes are uniform, so they represent it), each advanced whole steps
    until budget_s after its setup step; aggregate = sum of each process's
    atom-steps/s.  Each replica runs with neighbour-list radius = ghost
    cutoff = L/2 (cutoff_extra_coef 1), the largest its one-ghost-image
    scheme allows (workloads.replica_system)."""
    from concurrent.futures import ThreadPoolExecutor
    from caviar_b200 import workloads as W
    from oracle import oracle as O
    if not O.harness_available():
        return {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": "harness not built"}
    procs = max(1, min(procs, os.cpu_count() or 1))
    b = W.replica_batch()
    order = np.argsort(b.n, kind="stable")
    picks = [int(order[min(len(order) - 1, int((q + 0.5) * len(order) / procs))]) for q in range(procs)]

    def one(r):
        s = W.replica_system(b, r)
        res = O.run_reference(s, "run", nsteps=100000, budget_s=budget_s, timeout=budget_s * 10 + 300)
        k = int(res["steps_done"]) - 1
        return s.n, float(res["wall_rest"]) / max(k, 1), k
    try:
        with ThreadPoolExecutor(procs) as ex:
            got = list(ex.map(one, picks))
    except Exception as e:  # pragma: no cover - reported, not hidden
        return {"value": None, "unit": UNIT, "cores": procs, "kind": "reference", "sample": f"failed: {e}"}
    value = sum(n / per for n, per, _ in got)
    return {"value": value, "unit": UNIT, "cores": procs, "kind": "reference",
            "sample": f"{procs} concurrent reference processes, replicas of " +
                      ", ".join(f"{n} atoms ({k} steps)" for n, _, k in got) +
                      " (the batch's size octiles), aggregate of their atom-steps/s"}


def cpu_baseline_adjoint(nsteps: int = 3):
    """The FP64 C restatement of the trajectory adjoint (oracle/adjoint.c; the
    reference has no gradients) on the 4000-atom mixture: loss and full
    gradient of an nsteps-step trajectory with a checkpoint every step
    (forward, re-run segments, reverse sweep), 1 core."""
    from caviar_b200 import workloads as W
    from oracle import oracle as O
    s = W.adjoint_mixture()
    try:
        a = O.AdjOracle(s)
        t0 = time.perf_counter()
        a.loss_grad(s.pos, s.vel, nsteps, 1)
        dt = time.perf_counter() - t0
    except Exception as e:  # pragma: no cover - reported, not hidden
        return {"value": None, "unit": "gradient atom-steps/s", "cores": 1, "kind": "port", "sample": f"failed: {e}"}
    return {"value": 4000 * nsteps / dt, "unit": "gradient atom-steps/s", "cores": 1, "kind": "port",
            "sample": f"loss + gradient over {nsteps} steps, checkpoint every step ({dt:.1f} s), FP64 restatement"}


def reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from caviar_b200 import workloads as W
    from oracle import oracle as O
    s = W.config_lj_1m(seed=3)
    if not O.harness_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_harness not built"}), flush=True)
        return
    # warm-up is the reference's setup step plus W steps is too long for 1M
    # atoms at ~5 s/step; time a bounded number of whole steps instead.
    budget = max(20.0, args.cpu_budget * 3)
    per, k, first = reference_step_time(s, args.steps, budget)
    value = s.n / per
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": k, "warmup": 1,
            "ms_per_step": per * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "fp64", "data": "synthetic (seeded FCC lattice + Maxwell-Boltzmann velocities)",
            "config": {"workload": "LJ fluid N=1048576 (FCC 64^3, rho*=0.8442, T*=0.72, rc=2.5, skin=0.3, "
                                   "dt=0.005)", "n_atoms": s.n, "parallelism": "serial CPU"},
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference",
                             "sample": f"{k} steps after one setup step ({first:.1f} s); unmodified reference "
                                       "compiled from its own sources, serial"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--replica-steps", type=int, default=1000)
    ap.add_argument("--adjoint-steps", type=int, default=500)
    ap.add_argument("--only", default="all", choices=["all", "replicas", "adjoint", "ions"],
                    help="run one secondary workload alone and print its JSON (profiling runs)")
    args = ap.parse_args()
    if args.impl == "reference":
        reference_arm(args)
    elif args.only != "all":
        import torch
        torch.cuda.set_device(0)
        from caviar_b200 import build as B
        B.build()
        from caviar_b200 import _abi as abi
        from caviar_b200 import workloads as W
        if args.only == "replicas":
            res = replica_line(abi, W, torch, args.replica_steps)
        elif args.only == "ions":
            res = ions_line(abi, W, torch, args.steps, max(3, args.warmup))
        else:
            res = adjoint_line(abi, W, torch, args.adjoint_steps)
        print(json.dumps({"only": args.only, **res}), flush=True)
    else:
        gpu_arm(args)


if __name__ == "__main__":
    main()
