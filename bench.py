#!/usr/bin/env python
"""Benchmark of the force/integration hot path on B200.

Headline workload (one "step" = one kick-drift-kick leapfrog step):
  LBVH Barnes-Hut, N = 2^20 Plummer sphere (lognormal masses mu=0 sigma=0.5,
  renormalised to 1), 30-bit Morton codes on the bounding cube, stable radix
  sort, Karras tree, monopole cells at theta = 0.5, eps = 0.005, FP32
  interactions on double-single positions, FP64 state, dt = 5e-4.
metric: LBVH-BH steps/s at N = 2^20 (higher is better).

Also reported on the same JSON line: the all-pairs pair-interaction rates of
the FP64 and mixed kernels on the cold-disk workload (N = 262144) and the
mixed-vs-FP64 force error, the FP64-walk LBVH step rate at the same theta
(equal approximation error), the roofline of the dominant kernel (the tree
walk), a CPU baseline (the reference's own Barnes_Hut + update_leapfrog,
compiled from its sources) and SM clocks sampled during the timed region.

`--impl reference` times the reference CPU implementation of the same
workload on the host cores (the reference has no usable GPU path here).

Multi-GPU: the LBVH path does not shard (the tree is global), so N GPUs run N
independent replicas of the workload ("replicas only"); value = total steps/s.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

N_C2 = 1 << 20
THETA, EPS, DT = 0.5, 0.005, 5e-4
SEED_C2 = 1002
N_C3, EPS_C3, SEED_C3 = 262144, 0.002, 1003
# the workload both arms (this library and the reference CPU code) run
C2_WORKLOAD = ("C2 LBVH Barnes-Hut KDK step, Plummer N=1048576 lognormal(0,0.5) masses, 30-bit Morton on the "
               "bounding cube, theta=0.5, eps=0.005, dt=5e-4")
FLOP_PER_PAIR = 20  # Newtonian pair, Nyland et al. GPU Gems 3 ch. 31 convention
# 1PN pair term (compute_gravitational with get_pn1): the Newtonian 20 + unit
# vector 3, v_i - v_j 3, v_i.v_j 5, n.v_i 5, n.v_j 5, bracket A 13, bracket B 3,
# prefactor 2, the three components 12 = 71 FLOP
FLOP_PER_PN1_PAIR = 71
# EIH 1PN pair (two passes over the system): pass 1 the Newtonian 20 plus the
# potential 2; pass 2 separation 3, r^2 with softening 6, rsqrt 1, r^-2 1,
# v_i.v_j, d.v_i, d.v_j, d.A_j 20, n.v_j 1, bracket B 10, W 4, prefactors 6,
# the three components 21 = 73; 95 FLOP
FLOP_PER_EIH_PAIR = 95
# Adjoint pair term (J^T w and the mass gradient, one pair): separation 3,
# r^2 with softening 6, rsqrt 1, s^3 and s^5 3, u = m_k w_j - m_j w_k 9,
# d.u 5, 3 s^5 (d.u) 2, the three components 12, w_j.d 5, mass-gradient
# term 2 = 48 FLOP
FLOP_PER_ADJ_PAIR = 48
# Tree build, algorithmic bytes per body: Morton 32 (read the position 24,
# write code and index 8) + sort 16 (one read and one write of the 8-byte
# key/value, whatever the pass count) + Karras 24 (read the code, write links
# and ranges) + leaf gather 48 (read position and mass 32, write 16) +
# bottom-up 120 (per internal node: read two 40-byte child records, write 40)
BUILD_BYTES_PER_BODY = 240

# dram__bytes_read.sum + dram__bytes_write.sum of one k_walk launch captured with
# ncu at N = 2^19 (103.82 + 17.07 MB read + written, the fused next drift's
# position read and write included), scaled by the number of bodies to
# N = 2^20 (the walk reads each tree node about once).
WALK_TRAFFIC_BYTES = 120.89e6 * 2


def fp_peaks(f_mhz: float):
    """FP32 and FP64 pipe peaks in TFLOP/s (an FMA counted as 2) at SM clock f_mhz:
    148 SMs x 128 FP32 lanes, x 64 FP64 lanes."""
    return 148 * 128 * 2 * f_mhz * 1e6 / 1e12, 148 * 64 * 2 * f_mhz * 1e6 / 1e12


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


class ClockSampler:
    """SM clock and clock-event reasons sampled while the timed region runs.

    NVML polled every ~2 ms from a thread (the timed C-ABI call releases the
    GIL), so that even a timed region of a few tens of milliseconds gets
    samples; the GPU is found by its PCI bus id, which stays right when
    CUDA_VISIBLE_DEVICES renumbers devices. Falls back to `nvidia-smi -lms 200`
    when NVML is unavailable. Read-only: no clock or other setting is changed."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4))

    def __init__(self, device: int, interval_s: float = 0.002):
        self.device = device
        self.interval = interval_s
        self.proc = None
        self.lines: list[str] = []
        self.nvml = None
        self.handle = None
        self.samples: list[tuple[float, int]] = []
        self.max_mhz = None
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            pr = torch.cuda.get_device_properties(device)
            try:
                bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
                self.handle = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
            except Exception:
                self.handle = pynvml.nvmlDeviceGetHandleByIndex(device)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.handle, pynvml.NVML_CLOCK_SM)
            self.nvml = pynvml
        except Exception:
            self.nvml = None

    def start(self):
        if self.nvml is not None:
            self._stop = threading.Event()
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
            return
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None

    def _poll(self):
        nv = self.nvml
        while not self._stop.is_set():
            try:
                mhz = nv.nvmlDeviceGetClockInfo(self.handle, nv.NVML_CLOCK_SM)
                rs = nv.nvmlDeviceGetCurrentClocksEventReasons(self.handle)
                self.samples.append((float(mhz), int(rs)))
            except Exception:
                pass
            time.sleep(self.interval)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    @staticmethod
    def _summary(sm, smax, reasons, source):
        loaded = [x for x in sm if smax and x > 0.5 * smax] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm), "source": source}

    def stop(self) -> dict:
        if self.nvml is not None:
            self._stop.set()
            self.t.join(timeout=5)
            reasons = {nm for nm, bit in self.REASONS for _, r in self.samples if r & bit}
            return self._summary([m for m, _ in self.samples], float(self.max_mhz), reasons,
                                 f"nvml every {self.interval * 1e3:.0f} ms")
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = [nm for nm, _ in self.REASONS]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return self._summary(sm, smax, reasons, "nvidia-smi every 200 ms")


def max_over_ranks(ms: float, dist=None, device: str = "cpu") -> float:
    """Largest per-rank device time of the timed region (MAX all-reduce);
    the rank's own value when not distributed."""
    if dist is None:
        return ms
    import torch
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world: int, steps: int, ms_max: float) -> float:
    """Steps per second of the whole job: every rank runs `steps` steps of its
    own replica, the job lasts as long as the slowest rank."""
    return world * steps / (ms_max / 1e3)


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text()), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0}, "fallback"


def cpu_baseline_c2(pos, vel, m, steps: int = 1):
    """The reference's Barnes_Hut + update_leapfrog on the host cores, one
    step at full N (2 tree builds + walks)."""
    from oracle.oracle import Ref
    if not Ref.available():
        return None
    ref = Ref()
    ref.setup(pos, vel, m, G=1.0, dt=DT, eps2=EPS * EPS, theta=THETA, box=float(np.abs(pos).max()), solver="bh")
    t0 = time.perf_counter()
    ref.leapfrog(steps)
    dt = time.perf_counter() - t0
    return {"value": steps / dt, "unit": "steps/s", "cores": ref.threads(), "kind": "reference",
            "cpu_model": cpu_model(),
            "sample": f"{steps} update_leapfrog step(s) of Barnes_Hut at N={len(m)} (full workload), "
                      f"reference sources compiled unmodified with a std::thread TBB stand-in"}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    from aster_b200 import gen
    from oracle.oracle import Ref
    if not Ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU build oracle/_ref missing"}))
        return 0
    pos, vel, m = gen.plummer(N_C2, SEED_C2, masses="lognormal")
    ref = Ref()
    ref.setup(pos, vel, m, G=1.0, dt=DT, eps2=EPS * EPS, theta=THETA, box=float(np.abs(pos).max()), solver="bh")
    for _ in range(args.warmup):
        ref.leapfrog(1)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ref.leapfrog(1)
    el = time.perf_counter() - t0
    v = args.steps / el
    line = {
        "impl": "reference", "metric": "LBVH-BH steps/s @N=1M", "value": v, "unit": "steps/s", "n_gpus": 0,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": C2_WORKLOAD, "n": N_C2,
                   "precision": "FP64 throughout (the reference CPU Barnes_Hut)"},
        "cpu_baseline": {"value": v, "unit": "steps/s", "cores": ref.threads(), "kind": "reference",
                         "cpu_model": cpu_model(),
                         "sample": f"full N={N_C2} update_leapfrog steps with Barnes_Hut (2 tree builds + walks "
                                   f"each), reference sources compiled unmodified, std::thread TBB stand-in"},
        "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    rank, world, local = dist_env()
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from aster_b200 import gen
    from aster_b200.api import FP64, MIXED, SOLVER_LBVH, Context, Params

    device = local if world > 1 else 0
    pos, vel, m = gen.plummer(args.n, SEED_C2, masses="lognormal")
    p = Params(G=1.0, eps2=EPS * EPS, theta=THETA, dt=DT)
    ctx = Context(device)
    ctx.upload(pos, vel, m)

    def barrier():
        if dist:
            dist.barrier()

    e_start = ctx.energy(p) if not args.quick else None
    # warm-up (also primes the cached acceleration)
    ctx.kdk_steps(p, args.warmup, SOLVER_LBVH, MIXED)
    barrier()
    clocks = ClockSampler(device)
    clocks.start()
    ctx.kdk_steps(p, args.steps, SOLVER_LBVH, MIXED)   # device-timed inside (CUDA events)
    st = ctx.stats()
    barrier()
    clk = clocks.stop()
    ms = max_over_ranks(st["ms_total"], dist, f"cuda:{device}")
    value = whole_job_rate(world, args.steps, ms)
    drift = None
    if e_start is not None:
        e_end = ctx.energy(p)
        drift = {"steps": args.warmup + args.steps, "energy_rel": abs(e_end[0] - e_start[0]) / abs(e_start[0]),
                 "momentum_abs": float(np.abs(e_end[1] - e_start[1]).max()),
                 "note": "FP64 O(N^2) energy with the Plummer potential, before warm-up and after the timed steps"}
    walk_ms = st["ms_force"] / max(args.steps, 1)
    build_ms = st["ms_build"] / max(args.steps, 1)
    inter_per_step = st["interactions"] / max(args.steps, 1)
    kernels = st["kernels"]

    # e2e through the C ABI with pinned host buffers: H2D state, one step, D2H state
    e2e = None if args.no_e2e else e2e_c2(ctx, p, pos, vel, m, args)
    line = {}
    if rank == 0:
        peaks, src = measured_peaks()
        f_mhz = clk.get("sm_mhz") or peaks.get("sm_max_mhz", 1965.0)
        sms = 148
        fp32_peak = sms * 128 * 2 * f_mhz * 1e6 / 1e12
        achieved = inter_per_step * FLOP_PER_PAIR / (walk_ms / 1e3) / 1e12
        build_gbs = BUILD_BYTES_PER_BODY * args.n / (build_ms / 1e3) / 1e9 if build_ms > 0 else None
        args.sm_mhz = f_mhz
        extra = secondary(ctx, args) if not args.quick else {}
        line = {
            "metric": "LBVH-BH steps/s @N=1M", "value": value, "unit": "steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 pairs / f64 state", "data": "synthetic",
            "config": {"workload": (C2_WORKLOAD if args.n == N_C2 else
                                    C2_WORKLOAD.replace("C2 LBVH", "C2 at reduced size: LBVH")
                                    .replace("N=1048576", f"N={args.n}")),
                       "n": args.n, "precision": "mixed: FP32 interactions on double-single positions, FP64 state", "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "l2": "per-step working set > L2: the tree rebuild writes ~0.4 GB every step"},
            "phases_ms": {"build": build_ms, "walk": walk_ms, "other": ms / args.steps - build_ms - walk_ms},
            "interactions_per_step": inter_per_step,
            "drift": drift,
            "walk_stack_high_water": st["max_stack"],
            "roofline": {"bound": "fp32", "kernel": "k_walk (tree walk + interactions)",
                         "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s", "frac": achieved / fp32_peak,
                         "traffic": args.walk_traffic,
                         "peak_source": f"148 SMs x 128 FP32 lanes x 2 x "
                                        + (f"median SM clock {f_mhz:.0f} MHz sampled during the timed region"
                                           if clk.get("sm_mhz") else f"max SM clock {f_mhz:.0f} MHz (no clock samples)")
                                        + " (no FP32 figure in MEASURED_PEAKS.json)",
                         "flop_per_interaction": FLOP_PER_PAIR},
            "build_roofline": None if build_gbs is None else {
                "bound": "hbm", "kernels": "tree build (Morton, sort, Karras, bottom-up, node records)",
                "achieved": build_gbs, "peak": peaks.get("hbm_gbs", 6650.0), "unit": "GB/s",
                "frac": build_gbs / peaks.get("hbm_gbs", 6650.0), "bytes_per_body": BUILD_BYTES_PER_BODY,
                "peak_source": f"{src} copy bandwidth (MEASURED_PEAKS.json)" if src == "measured"
                else "fallback copy bandwidth"},
            "e2e": e2e,
            "gpu_launches": kernels,
            "clocks": clk,
        }
        line.update(extra)
        if not args.no_cpu_baseline and world == 1:
            line["cpu_baseline"] = cpu_baseline_c2(pos, vel, m)
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def e2e_c2(ctx, p, pos, vel, m, args):
    """Same metric through the public C ABI with host buffers, as a host loop
    keeping its state in host memory would drive it: every step copies the
    state (positions, velocities, masses and the bodies' accelerations, the
    reference BodyArray's fields) host->device from pinned memory, runs one KDK
    step, and copies positions, velocities and accelerations back into the
    same host arrays, which are the next step's input (aster_kdk_steps_host:
    the positions' copy back overlaps the step's force evaluation)."""
    import ctypes
    from aster_b200.api import MIXED, SOLVER_LBVH
    n = len(m)
    lib = ctx.lib
    # page-locked host buffers (torch's pinned allocator; same primary context)
    pinned = []
    try:
        import torch
        hp = torch.from_numpy(np.ascontiguousarray(pos)).pin_memory()
        hv = torch.from_numpy(np.ascontiguousarray(vel)).pin_memory()
        hm = torch.from_numpy(np.ascontiguousarray(m)).pin_memory()
        ha = torch.zeros((n, 3), dtype=torch.float64).pin_memory()
        arrs = [t.numpy() for t in (hp, hv, hm, ha)]
        pinned = [hp, hv, hm, ha]
    except Exception:
        arrs = [np.ascontiguousarray(pos).copy(), np.ascontiguousarray(vel).copy(), np.ascontiguousarray(m),
                np.zeros((n, 3))]
    hp, hv, hm, ha = arrs
    vp = ctypes.c_void_p
    cp = p.c_struct()
    # the accelerations of the initial state (one force evaluation, untimed)
    st = lib.aster_state_upload(ctx.h, n, vp(hp.ctypes.data), vp(hv.ctypes.data), vp(hm.ctypes.data))
    st = st or lib.aster_lbvh_forces(ctx.h, ctypes.byref(cp), MIXED, vp(ha.ctypes.data), None)
    if st:
        raise RuntimeError(f"e2e setup failed: {st}")

    def one():
        # upload, one KDK step, download, in one call (the positions' copy back
        # overlaps the force evaluation)
        st = lib.aster_kdk_steps_host(ctx.h, ctypes.byref(cp), SOLVER_LBVH, MIXED, 1, n, vp(hp.ctypes.data),
                                      vp(hv.ctypes.data), vp(ha.ctypes.data), vp(hm.ctypes.data))
        if st:
            raise RuntimeError(f"e2e step failed: {st}")

    for _ in range(2):
        one()
    k = max(2, min(args.steps, 10))
    t0 = time.perf_counter()
    for _ in range(k):
        one()
    el = time.perf_counter() - t0
    del pinned
    return {"value": k / el, "unit": "steps/s", "h2d_bytes_per_step": n * (24 + 24 + 8 + 24),
            "d2h_bytes_per_step": n * (24 + 24 + 24), "steps": k,
            "note": "host wall clock around synchronous C-ABI calls (each call ends with a stream sync); the "
                    "state round-trips through pinned host memory every step"}


def secondary(ctx, args):
    """All-pairs rates (C3 disk) and the FP64-walk LBVH rate (same theta)."""
    from aster_b200 import gen
    from aster_b200.api import FP64, MIXED, SOLVER_LBVH, Params
    out = {}
    # FP64 LBVH at the same theta: same tree, same interaction lists
    pos, vel, m = gen.plummer(N_C2, SEED_C2, masses="lognormal")
    p = Params(G=1.0, eps2=EPS * EPS, theta=THETA, dt=DT)
    ctx.upload(pos, vel, m)
    a32 = ctx.lbvh_forces(p, MIXED)
    a64 = ctx.lbvh_forces(p, FP64)
    tg = np.random.default_rng(4096).choice(N_C2, 4096, replace=False)
    exact = ctx.allpairs_targets(p, tg, FP64)
    ctx.kdk_steps(p, 1, SOLVER_LBVH, FP64)
    ctx.kdk_steps(p, 3, SOLVER_LBVH, FP64)
    s64 = ctx.stats()
    err_bh = float(np.linalg.norm(a32[tg] - exact) / np.linalg.norm(exact))
    out["lbvh_precision"] = {
        "fp64_walk_steps_per_s": 3 / (s64["ms_total"] / 1e3),
        "mixed_vs_fp64_walk_rel_l2": float(np.linalg.norm(a32 - a64) / np.linalg.norm(a64)),
        "approx_rel_l2_vs_fp64_allpairs_4096_sample": err_bh,
    }
    # all-pairs on the C3 cold disk
    pos, vel, m = gen.exponential_disk(N_C3, SEED_C3)
    p3 = Params(G=1.0, eps2=EPS_C3 ** 2, dt=1e-4)
    ctx.upload(pos, vel, m)
    res = {}
    accs = {}
    for name, prec in (("fp64", FP64), ("mixed", MIXED)):
        accs[name] = ctx.allpairs(p3, prec)
        times = []
        for _ in range(3):
            ctx.allpairs(p3, prec)
            times.append(ctx.stats()["ms_force"])
        t = min(times)
        res[name] = {"ms_per_eval": t, "pairs_per_s": N_C3 * (N_C3 - 1) / (t / 1e3)}
    f32p, f64p = fp_peaks(getattr(args, "sm_mhz", 1965.0))
    for name, peak in (("fp64", f64p), ("mixed", f32p)):
        tf = res[name]["pairs_per_s"] * FLOP_PER_PAIR / 1e12
        res[name]["roofline"] = {"bound": "fp64" if name == "fp64" else "fp32", "achieved": tf, "peak": peak,
                                 "unit": "TFLOP/s", "frac": tf / peak}
    res["mixed_vs_fp64_rel_l2"] = float(np.linalg.norm(accs["mixed"] - accs["fp64"]) / np.linalg.norm(accs["fp64"]))
    res["workload"] = "C3 cold exponential disk N=262144 (+central mass 0.1), eps=0.002, one force evaluation"
    try:
        from oracle.oracle import Ref
        if Ref.available():  # the reference's Parallelized solver, sources [0, 4096) only
            ref = Ref().setup(pos, vel, m, G=1.0, dt=1e-4, eps2=EPS_C3 ** 2).set_bounds(0, 4096)
            t0 = time.perf_counter()
            ref.forces()
            el = time.perf_counter() - t0
            res["cpu_reference"] = {"pairs_per_s": N_C3 * 4096 / el, "cores": ref.threads(), "cpu_model": cpu_model(),
                                    "sample": f"all {N_C3} targets against sources [0, 4096) (Solver::set_bounds), "
                                              "one force evaluation, reference sources compiled unmodified"}
    except Exception as exc:  # the CPU figure is reported beside the GPU one, never instead of it
        res["cpu_reference"] = {"unavailable": str(exc)[:200]}
    res["c3_drift"] = c3_drift(ctx)
    out["allpairs"] = res
    out["allpairs_1m"] = allpairs_1m(ctx, getattr(args, "sm_mhz", 1965.0))
    out["ensemble"] = ensemble_c4(ctx, sm_mhz=getattr(args, "sm_mhz", 1965.0))
    out["adjoint"] = adjoint_c5(ctx, getattr(args, "sm_mhz", 1965.0))
    out["c1"] = kdk_c1(ctx)
    out["next_rows"] = next_rows(ctx)
    return out


def next_rows(ctx):
    """The rows beyond the headline path, each on its parity-test setup at a
    measurable size (device time, CUDA events): SABA4 (C1 all-pairs, and C2
    LBVH), Wisdom-Holman (8 planets + 262,144 test particles), device-resident
    stepping with collectors against plain stepping (C1), the C4 ensemble with
    every post-Newtonian term, and the post-Newtonian LBVH walk (C2)."""
    from aster_b200 import gen
    from aster_b200.api import (COLLECT_CENTER, COLLECT_ENERGY, COLLECT_MOMENTUM, FP64, MIXED, NEWTON,
                                PN1, PN2, PN25, SOLVER_ALLPAIRS, SOLVER_LBVH, UPDATER_KDK, YOSHIDA4, Params)
    out = {}
    # SABA4: 4 force evaluations a step
    pos, vel, m = gen.plummer(4096, 1001)
    p = Params(eps2=1e-4, dt=1e-3)
    saba = {"workload": "SABA4, C1 Plummer N=4096 all-pairs, 100 steps; C2 N=1048576 LBVH mixed, 2 steps"}
    for name, prec in (("c1_fp64", FP64), ("c1_mixed", MIXED)):
        ctx.upload(pos, vel, m)
        e0, _ = ctx.energy(p)
        ctx.saba_steps(p, 4, 100, SOLVER_ALLPAIRS, prec)
        ms = ctx.stats()["ms_total"]
        e1, _ = ctx.energy(p)
        saba[name] = {"ms_per_step": ms / 100, "energy_drift": abs(e1 - e0) / abs(e0)}
    pos2, vel2, m2 = gen.plummer(N_C2, SEED_C2, masses="lognormal")
    p2 = Params(G=1.0, eps2=EPS * EPS, theta=THETA, dt=DT)
    ctx.upload(pos2, vel2, m2)
    ctx.saba_steps(p2, 4, 1, SOLVER_LBVH, MIXED)
    ctx.saba_steps(p2, 4, 2, SOLVER_LBVH, MIXED)
    saba["c2_lbvh_mixed"] = {"ms_per_step": ctx.stats()["ms_total"] / 2}
    out["saba4"] = saba
    # post-Newtonian LBVH walk at C2 (KDK, mixed, 1PN and every term; c = 100)
    pnl = {"workload": "C2 LBVH KDK mixed with post-Newtonian laws, c=100, 3 steps (Newtonian step for scale)"}
    for name, law in (("newton", NEWTON), ("pn1", NEWTON | PN1), ("all_terms", NEWTON | PN1 | PN2 | PN25)):
        q = Params(G=1.0, eps2=EPS * EPS, theta=THETA, dt=DT, c=100.0, force_law=law)
        ctx.upload(pos2, vel2, m2)
        ctx.kdk_steps(q, 1, SOLVER_LBVH, MIXED)
        ctx.kdk_steps(q, 3, SOLVER_LBVH, MIXED)
        pnl[name] = {"ms_per_step": ctx.stats()["ms_total"] / 3}
    out["pn_lbvh"] = pnl
    # Wisdom-Holman
    pw, vw, mw = gen.planetary_system(8, 262144, 1023)
    ctx.upload(pw, vw, mw)
    pwh = Params(G=1.0, dt=0.02)
    ctx.wh_steps(pwh, 2)
    ctx.wh_steps(pwh, 200)
    ms = ctx.stats()["ms_total"]
    out["wisdom_holman"] = {"workload": "star + 8 planets + 262144 test particles, FP64, dt=0.02, 200 steps",
                            "ms_per_step": ms / 200, "body_steps_per_s": len(mw) * 200 / (ms / 1e3)}
    # device-resident stepping with collectors vs plain stepping (C1)
    rec = {"workload": "C1 Plummer N=4096 KDK all-pairs FP64, 100 steps; energy+momentum+centre every 10 steps"}
    ctx.upload(pos, vel, m)
    ctx.kdk_steps(p, 100, SOLVER_ALLPAIRS, FP64)
    rec["plain_ms"] = ctx.stats()["ms_total"]
    ctx.upload(pos, vel, m)
    ctx.record(p, 100, updater=UPDATER_KDK, solver=SOLVER_ALLPAIRS, precision=FP64, rate=10,
               collect=COLLECT_ENERGY | COLLECT_MOMENTUM | COLLECT_CENTER)
    rec["recorded_ms"] = ctx.stats()["ms_total"]
    out["record"] = rec
    # C4 ensemble with every post-Newtonian term
    pe, ve, me, off = gen.hierarchical_ensemble(16384, 1004)
    ens = {"workload": "C4 16384 systems n~U[3,64], Newton+1PN+2PN+2.5PN c=100, Yoshida-4, dt=1e-4, 1000 steps"}
    q = Params(G=1.0, c=100.0, eps2=0.0, dt=1e-4, force_law=NEWTON | PN1 | PN2 | PN25)
    cfg = {"warps_per_block": 8, "unroll": 2, "use_graph": 1}
    ctx.ensemble_upload(off, pe, ve, me)
    ctx.ensemble_run(q, 20, YOSHIDA4, MIXED, cfg)
    ctx.ensemble_run(q, 1000, YOSHIDA4, MIXED, cfg)
    st = ctx.stats()
    ens.update(steps_per_s=1000 / (st["ms_total"] / 1e3), pair_terms_per_s=st["interactions"] / (st["ms_total"] / 1e3))
    out["pn_ensemble"] = ens
    return out


def kdk_c1(ctx):
    """C1: Plummer N=4096, eps=0.01, dt=1e-3, 100 KDK all-pairs steps, FP64
    and mixed: device time per step, energy drift, momentum."""
    from aster_b200 import gen
    from aster_b200.api import FP64, MIXED, SOLVER_ALLPAIRS, Params
    pos, vel, m = gen.plummer(4096, 1001)
    p = Params(eps2=1e-4, dt=1e-3)
    out = {"workload": "C1 Plummer N=4096, eps=0.01, dt=1e-3, 100 KDK steps (one force evaluation per step)"}
    for name, prec in (("fp64", FP64), ("mixed", MIXED)):
        ctx.upload(pos, vel, m)
        e0, _ = ctx.energy(p)
        ctx.kdk_steps(p, 100, SOLVER_ALLPAIRS, prec)
        ms = ctx.stats()["ms_total"]
        e1, mom = ctx.energy(p)
        out[name] = {"ms_per_step": ms / 100, "pairs_per_s": 100 * 4096 * 4095 / (ms / 1e3),
                     "energy_drift": abs(e1 - e0) / abs(e0), "momentum_abs": float(np.abs(mom).max())}
    try:
        from oracle.oracle import Ref
        if Ref.available():  # the reference's Parallelized + update_leapfrog (2 force evaluations a step)
            ref = Ref().setup(pos, vel, m, G=1.0, dt=1e-3, eps2=1e-4)
            t0 = time.perf_counter()
            ref.leapfrog(10)
            el = time.perf_counter() - t0
            out["cpu_reference"] = {"steps_per_s": 10 / el, "cores": ref.threads(), "cpu_model": cpu_model(),
                                    "sample": "10 of the 100 steps, reference sources compiled unmodified"}
    except Exception as exc:  # the CPU figure is reported beside the GPU one, never instead of it
        out["cpu_reference"] = {"unavailable": str(exc)[:200]}
    return out


def allpairs_1m(ctx, sm_mhz: float):
    """One mixed and one FP64 all-pairs evaluation of the C2 bodies (N = 2^20
    lognormal Plummer, eps = 0.005): pair rates against the FP32 and FP64
    pipe peaks, and the mixed-vs-FP64 force error over all bodies. Each
    precision is first run once on a 2^14-body state (module load, first-use
    allocation), then timed on one full evaluation (CUDA events)."""
    from aster_b200 import gen
    from aster_b200.api import FP64, MIXED, Params
    p = Params(G=1.0, eps2=EPS * EPS)
    pw, vw, mw = gen.plummer(1 << 14, 7, masses="lognormal")
    ctx.upload(pw, vw, mw)
    for prec in (FP64, MIXED):
        ctx.allpairs(p, prec)
    pos, vel, m = gen.plummer(N_C2, SEED_C2, masses="lognormal")
    ctx.upload(pos, vel, m)
    f32p, f64p = fp_peaks(sm_mhz)
    out = {"workload": "C2 bodies: Plummer N=1048576, lognormal(0,0.5) masses, eps=0.005, one all-pairs "
                       "force evaluation per precision (N(N-1) pairs)"}
    accs = {}
    for name, prec, peak in (("mixed", MIXED, f32p), ("fp64", FP64, f64p)):
        accs[name] = ctx.allpairs(p, prec)
        t = ctx.stats()["ms_force"]
        rate = N_C2 * (N_C2 - 1) / (t / 1e3)
        tf = rate * FLOP_PER_PAIR / 1e12
        out[name] = {"ms_per_eval": t, "pairs_per_s": rate,
                     "roofline": {"bound": "fp32" if prec == MIXED else "fp64", "achieved": tf, "peak": peak,
                                  "unit": "TFLOP/s", "frac": tf / peak, "flop_per_pair": FLOP_PER_PAIR}}
    out["mixed_vs_fp64_rel_l2"] = float(np.linalg.norm(accs["mixed"] - accs["fp64"]) /
                                        np.linalg.norm(accs["fp64"]))
    out["mixed_speedup_over_fp64"] = out["fp64"]["ms_per_eval"] / out["mixed"]["ms_per_eval"]
    return out


def c3_drift(ctx, nsteps: int = 1000):
    """C3 long run: 1000 KDK steps (dt = 1e-4) of the N = 262144 cold disk
    with FP64 and with mixed all-pairs forces; energy drift of each (FP64
    O(N^2) energy with the Plummer-softened potential that the force is the
    gradient of), the momentum at the end and how far apart the two runs'
    final positions are."""
    from aster_b200 import gen
    from aster_b200.api import FP64, MIXED, SOLVER_ALLPAIRS, Params
    pos, vel, m = gen.exponential_disk(N_C3, SEED_C3)
    p = Params(G=1.0, eps2=EPS_C3 ** 2, dt=1e-4)
    out = {"workload": f"C3 disk N={N_C3}, eps=0.002, dt=1e-4, {nsteps} KDK steps"}
    finals = {}
    for name, prec in (("fp64", FP64), ("mixed", MIXED)):
        ctx.upload(pos, vel, m)
        e0, _ = ctx.energy(p)
        ctx.kdk_steps(p, nsteps, SOLVER_ALLPAIRS, prec)
        ms = ctx.stats()["ms_total"]
        e1, mom = ctx.energy(p)
        finals[name] = ctx.download()[0]
        out[name] = {"s": ms / 1e3, "energy_drift": abs(e1 - e0) / abs(e0), "momentum_abs": float(np.abs(mom).max())}
    out["final_pos_mixed_vs_fp64_rel_l2"] = float(np.linalg.norm(finals["mixed"] - finals["fp64"]) /
                                                  np.linalg.norm(finals["fp64"]))
    return out


def ensemble_c4(ctx, nsteps: int = 10_000, sm_mhz: float = 1965.0):
    """C4: 16384 hierarchical systems (n in [3, 64]), 1PN (c = 100) in the
    N-body Einstein-Infeld-Hoffmann form the configuration names, Yoshida-4,
    dt = 1e-4, nsteps in one persistent graph-captured launch with the
    autotuned launch shape and schedule; FP32 pair terms, FP64 state. The
    reference's pairwise get_pn1 law is run the same way beside it. Energy
    drift per system: |dE/E0| over all systems, and |dE| / (K + |U|) over the
    resolved ones (inner-binary pericentre time >= 20 dt, no other pair
    closer than 0.5 at the start)."""
    from aster_b200 import gen
    from aster_b200.api import EIH, MIXED, NEWTON, PN1, YOSHIDA4, Params
    from aster_b200.autotune import tune_ensemble
    pos, vel, m, off = gen.hierarchical_ensemble(16384, 1004)
    tp, dmin, scale = gen.ensemble_measures(pos, vel, m, off)
    resolved = (tp >= 20 * 1e-4) & (dmin >= 0.5)
    f32p = fp_peaks(sm_mhz)[0]
    out = {"workload": "C4 16384 systems n~U[3,64], lognormal(0,1) masses, hierarchical, c=100, Yoshida-4, "
                       "dt=1e-4, one graph-captured launch", "steps": nsteps,
           "resolved_systems": int(resolved.sum())}
    for name, law, fpp in (("eih", NEWTON | PN1 | EIH, FLOP_PER_EIH_PAIR), ("pairwise", NEWTON | PN1,
                                                                            FLOP_PER_PN1_PAIR)):
        p = Params(G=1.0, c=100.0, eps2=0.0, dt=1e-4, force_law=law)
        ctx.ensemble_upload(off, pos, vel, m)
        cfg = tune_ensemble(ctx, off, p, steps=40, cache=None)
        cfg = {k: cfg[k] for k in ("warps_per_block", "unroll", "check_every", "use_graph", "schedule")}
        e0 = ctx.ensemble_energy(p)
        ctx.ensemble_run(p, nsteps, YOSHIDA4, MIXED, cfg)
        st = ctx.stats()
        e1 = ctx.ensemble_energy(p)
        de = np.abs((e1 - e0) / e0)
        ds = np.abs(e1 - e0) / scale
        rate = st["interactions"] / (st["ms_total"] / 1e3)
        tf = rate * fpp / 1e12
        out[name] = {"ms": st["ms_total"], "steps_per_s": nsteps / (st["ms_total"] / 1e3), "pair_terms_per_s": rate,
                     "config": cfg,
                     "roofline": {"bound": "fp32", "achieved": tf, "peak": f32p, "unit": "TFLOP/s",
                                  "frac": tf / f32p, "flop_per_pair": fpp},
                     "energy_drift_median": float(np.median(de)), "energy_drift_p90": float(np.percentile(de, 90)),
                     "resolved_drift_per_scale_median": float(np.median(ds[resolved])),
                     "resolved_drift_per_scale_p90": float(np.percentile(ds[resolved], 90))}
    return out


def adjoint_c5(ctx, sm_mhz: float = 1965.0):
    """C5: N=16384 Plummer, eps=0.01, dt=1e-3, 1000 KDK steps, checkpoints
    every 32; forward + reverse sweep time for dL/d(x0, v0, m). Roofline over
    the whole run: the forward pass and the per-segment recomputation each
    evaluate N(N-1) force pairs per step (20 FLOP), the reverse sweep one
    adjoint pair term per pair per step (48 FLOP), against the FP32 pipe
    (mixed) or FP64 pipe (FP64) peak at the sampled SM clock."""
    from aster_b200 import gen
    from aster_b200.api import FP64, MIXED, SOLVER_ALLPAIRS, Params
    n, T = 16384, 1000
    p = Params(eps2=1e-4, dt=1e-3)
    x0, v0, m = gen.plummer(n, 1005)
    rng = np.random.default_rng(1005)
    ctx.upload(x0 + rng.normal(0, 1e-3, x0.shape), v0, m)
    ctx.kdk_steps(p, T, SOLVER_ALLPAIRS, FP64)
    target, _, _ = ctx.download()
    ctx.upload(x0, v0, m)
    out = {"workload": "C5 Plummer N=16384, eps=0.01, dt=1e-3, 1000 KDK steps, loss=mean|x_T-x*|^2, K=32"}
    f32p, f64p = fp_peaks(sm_mhz)
    pairs = n * (n - 1)
    flop = pairs * T * (2 * FLOP_PER_PAIR + FLOP_PER_ADJ_PAIR)
    for name, prec, peak in (("mixed", MIXED, f32p), ("fp64", FP64, f64p)):
        loss, *_ = ctx.adjoint(p, T, target, prec, 32)
        ms = ctx.stats()["ms_total"]
        tf = flop / (ms / 1e3) / 1e12
        out[name] = {"ms_forward_plus_adjoint": ms, "loss": loss,
                     "roofline": {"bound": "fp32" if prec == MIXED else "fp64", "achieved": tf, "peak": peak,
                                  "unit": "TFLOP/s", "frac": tf / peak,
                                  "flop_per_step": f"N(N-1) x (2 x {FLOP_PER_PAIR} + {FLOP_PER_ADJ_PAIR})"}}
    return out


def run_case(args):
    """One secondary workload, briefly: C3 all-pairs (a warm-up then one
    FP64 and one mixed evaluation), C4 ensemble (a 50-step launch), C5 adjoint
    (8 steps, checkpoints every 4)."""
    from aster_b200 import gen
    from aster_b200.api import EIH, FP64, MIXED, NEWTON, PN1, YOSHIDA4, Context, Params
    ctx = Context(0)
    out = {"case": args.case}
    if args.case == "allpairs":
        pos, vel, m = gen.exponential_disk(N_C3, SEED_C3)
        p3 = Params(G=1.0, eps2=EPS_C3 ** 2, dt=1e-4)
        ctx.upload(pos, vel, m)
        for prec in (FP64, MIXED):
            ctx.allpairs(p3, prec)
            ctx.allpairs(p3, prec)
            out[f"ms_{prec}"] = ctx.stats()["ms_force"]
    elif args.case == "c3drift":
        out.update(c3_drift(ctx))
    elif args.case == "wh":
        # Wisdom-Holman: a star, 8 planets and 262,144 massless test particles, 20 steps
        pos, vel, m = gen.planetary_system(8, 262144, 1023)
        ctx.upload(pos, vel, m)
        p = Params(G=1.0, dt=0.02)
        ctx.wh_steps(p, 2)
        ctx.wh_steps(p, 20)
        out["ms_20_steps"] = ctx.stats()["ms_total"]
    elif args.case == "scale":
        # the C2 step (mixed LBVH KDK, theta = 0.5, eps = 0.005) at larger N
        from aster_b200.api import SOLVER_LBVH
        out["runs"] = []
        for lg in (22, 24, 25):
            n = 1 << lg
            pos, vel, m = gen.plummer(n, SEED_C2, masses="lognormal")
            p = Params(G=1.0, eps2=EPS * EPS, theta=THETA, dt=DT)
            ctx.upload(pos, vel, m)
            ctx.kdk_steps(p, 1, SOLVER_LBVH, MIXED)
            ctx.kdk_steps(p, 3, SOLVER_LBVH, MIXED)
            st = ctx.stats()
            run = {"n": n, "ms_per_step": st["ms_total"] / 3, "ms_build": st["ms_build"] / 3,
                   "ms_walk": st["ms_force"] / 3, "interactions_per_step": st["interactions"] / 3,
                   "walk_stack_high_water": st["max_stack"]}
            if lg == 24:
                tg = np.random.default_rng(4096).choice(n, 4096, replace=False)
                a = ctx.lbvh_forces(p, MIXED)
                exact = ctx.allpairs_targets(p, tg, FP64)
                run["approx_rel_l2_vs_fp64_allpairs_4096_sample"] = float(
                    np.linalg.norm(a[tg] - exact) / np.linalg.norm(exact))
            out["runs"].append(run)
            del pos, vel, m
    elif args.case == "pnlbvh":
        # the C2 step with Newton + 1PN (c = 100) at args.n bodies: one step, then three
        from aster_b200.api import SOLVER_LBVH
        pos, vel, m = gen.plummer(args.n, SEED_C2, masses="lognormal")
        p = Params(G=1.0, eps2=EPS * EPS, theta=THETA, dt=DT, c=100.0, force_law=NEWTON | PN1)
        ctx.upload(pos, vel, m)
        ctx.kdk_steps(p, 1, SOLVER_LBVH, MIXED)
        ctx.kdk_steps(p, 3, SOLVER_LBVH, MIXED)
        st = ctx.stats()
        out.update(n=args.n, ms_per_step=st["ms_total"] / 3, interactions_per_step=st["interactions"] / 3)
    elif args.case in ("ensemble", "ensemble_eih"):
        # the C4 ensemble (16384 systems), pairwise or EIH 1PN, plain launches
        # with a launch shape the autotuner picks on B200: a 20-step launch,
        # then one of 300 steps
        eih = args.case == "ensemble_eih"
        pos, vel, m, off = gen.hierarchical_ensemble(16384, 1004)
        p = Params(G=1.0, c=100.0, eps2=0.0, dt=1e-4, force_law=NEWTON | PN1 | (EIH if eih else 0))
        ctx.ensemble_upload(off, pos, vel, m)
        cfg = {"warps_per_block": 2, "unroll": 1 if eih else 2, "use_graph": 0}
        ctx.ensemble_run(p, 20, YOSHIDA4, MIXED, cfg)
        ctx.ensemble_run(p, 300, YOSHIDA4, MIXED, cfg)
        out["ms_300_steps"] = ctx.stats()["ms_total"]
    else:
        x0, v0, m = gen.plummer(16384, 1005)
        p = Params(eps2=1e-4, dt=1e-3)
        ctx.upload(x0, v0, m)
        ctx.adjoint(p, 8, x0 + 1e-3, MIXED, 4)
        out["ms"] = ctx.stats()["ms_total"]
    ctx.close()
    print(json.dumps(out), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--quick", action="store_true", help="skip the secondary measurements")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end (host buffer) measurement")
    ap.add_argument("--n", type=int, default=N_C2,
                    help="bodies in the headline workload (default 2^20; smaller only for profiling captures)")
    ap.add_argument("--walk-traffic", type=float, default=WALK_TRAFFIC_BYTES,
                    help="DRAM bytes per walk launch from an ncu capture (reported as roofline.traffic)")
    ap.add_argument("--case", default=None,
                    choices=["allpairs", "ensemble", "ensemble_eih", "adjoint", "c3drift", "wh", "scale", "pnlbvh"],
                    help="run one secondary workload briefly (used for profiling captures) and exit")
    args = ap.parse_args()
    if args.warmup < 3:
        log("warm-up raised to 3 steps (timing rule)")
        args.warmup = 3
    if args.case:
        return run_case(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
