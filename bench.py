#!/usr/bin/env python
"""SPM steps/s at 128^3 with 256 colloids on B200: mixed precision vs FP64.

Workload (one box per GPU): 128^3 periodic grid, 256 spheres a=5, xi=2,
kBT=1e-3 thermal kicks, dt=0.01, seeded non-overlapping positions
(kapsel_old_b200.workload.mixed_128_256).  A step is one
Time_evolution_hydro of the reference (sp_3d_ns.cxx:61-212).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Our arm: W untimed steps, then K timed steps.  Before every timed step a
256 MiB buffer is written (L2 flush, the L2 is 126 MB); each step is timed
with CUDA events on the library's stream; the state is device resident.
`e2e` repeats K steps through the public C ABI with the per-step host work
(thermostat normals generated on the host and copied in, particle records
copied out) inside a wall-clock timed region.  Under torchrun each rank runs
an independent replica (the SPM step runs on one GPU: replicas only);
the timed region is bracketed by a barrier and the max over ranks is used.

Reference arm: the unmodified KAPSEL sources built by oracle/Makefile
(oracle/_ref, OpenMP loops on all host cores) timed by wall clock on the same
workload, min(K, 30) steps after min(W, 10) warm-up steps; rank 0 only.
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
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "SPM steps/s at 128³, 256 colloids: mixed vs FP64 on B200, % of HBM roofline"
UNIT = "steps/s"
WORKLOAD = "SPM Navier-Stokes step, 128^3 grid, 256 spheres a=5 xi=2, kBT=1e-3, dt=0.01"
REF_MAX_STEPS = 30


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# algorithmic bytes of each launch (compulsory reads + writes of the stored
# operands; complex values 2R, real values R bytes)
# profiling slots of a step (kapsel_gpu_profile_step), labelled with the
# kernel names the library reports; repeated kernels get the suffixes below
SLOT_SUFFIX = {3: "#5", 5: "#2", 11: "#3"}
# y-pass variants of the batch autotuner (kapsel_batch_variants)
Y_VARIANTS = ["warp", "block wide tile", "block narrow tile", "warp, fused y/z planes"]


def slot_labels(names):
    return [(n + SLOT_SUFFIX.get(i, "")) if n else "" for i, n in enumerate(names)]


def kernel_bytes(cfg, R: int):
    NX, NY, NZ = [1 << p for p in cfg["np_xyz"]]
    T = [(n + 2) // 3 for n in (NX, NY, NZ)]
    KXc, KYc, TZ = 2 * T[0] - 1, 2 * T[1] - 1, T[2]
    C = 2 * R
    N = NX * NY * NZ
    zeta = 2 * KXc * KYc * TZ * C
    I1 = NX * KYc * TZ * C  # one component after the x pass
    I2 = NX * NY * TZ * C  # one component after the y pass
    Np = len(cfg["particles"])
    S = sekibun_count(cfg)
    part = Np * 26 * 8
    return {
        "k_x_zeta_to_u": zeta + 3 * I1,
        "k_y_pass<inv>": 3 * I1 + 3 * I2,
        "k_z_products": 3 * I2 + 5 * I2,
        "k_y_pass<fwd>#5": 5 * I2 + 5 * I1,
        "k_x_advect_update": 5 * I1 + 2 * zeta + 3 * I1,
        "k_y_pass<inv>#2": 3 * I1 + 3 * I2,
        "k_z_c2r": 3 * I2 + 3 * N * R,
        "k_particles_position": 2 * part,
        "k_particles_hydro_velocity": 3 * Np * S * R + 2 * part,
        "k_particles_scatter": 2 * 4 * Np * S * R + part,
        "k_z_force": 7 * N * R + 3 * I2,
        "k_y_pass<fwd>#3": 3 * I2 + 3 * I1,
        "k_x_force_to_zeta": 3 * I1 + 2 * zeta,
        # fused y/z plane kernels: the y pass's intermediate stays on chip
        "k_yzw_c2r": 3 * I1 + 3 * N * R,
        "k_zyw_force": 7 * N * R + 3 * I1,
    }


def sekibun_count(cfg):
    a, axi = float(cfg.get("a", 5.0)), float(cfg.get("a_xi", 2.0))
    nh = int(a) + int(axi) + 2
    rmax = a + 0.5 * axi + 1.7321
    n = 0
    for i in range(-nh, nh + 1):
        for j in range(-nh, nh + 1):
            for k in range(-nh, nh + 1):
                if math.sqrt(i * i + j * j + k * k) < rmax:
                    n += 1
    return n


def step_bytes_model(cfg, R: int):
    """Compulsory bytes of one step: 40.6 field passes of N*R at 128^3 with
    256 spheres (stages: 5+7+5 spectral, 0.71 gather, 4 phi/up reset,
    1.89 scatter, 10 force, 7 zeta update)."""
    NX, NY, NZ = [1 << p for p in cfg["np_xyz"]]
    N = NX * NY * NZ
    Np = len(cfg["particles"])
    S = sekibun_count(cfg)
    frac = Np * S / N
    passes = 5 + 7 + 5 + 3 * frac + 4 + 4 * 2 * frac + 10 + 7
    return passes * N * R, passes


def reduce_max(value: float, dist=None, device="cuda") -> float:
    """Max over ranks of a per-rank timing (the whole-job time of replicas)."""
    if dist is None:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(units_per_rank: int, world: int, max_seconds: float) -> float:
    """Whole-job throughput of independent replicas: all ranks' units over the
    slowest rank's time."""
    return units_per_rank * world / max_seconds


class NvmlClockSampler:
    """SM clock and clock-event reasons read through NVML every 5 ms on a host
    thread while the timed steps run (read-only queries; the timed region of
    the headline is well under a second, shorter than nvidia-smi's sampling
    interval)."""

    early = False  # started right before the timed steps

    def __init__(self, index: int):
        import pynvml

        self.nv = pynvml
        pynvml.nvmlInit()
        # the CUDA device's own GPU (by PCI address: NVML counts all GPUs of
        # the node, CUDA only the visible ones), else NVML's device `index`
        try:
            import torch

            pr = torch.cuda.get_device_properties(index)
            bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
            self.h = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            self.h = pynvml.nvmlDeviceGetHandleByIndex(index)
        self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM))
        self.sm, self.bits, self.stop_ev, self.t = [], 0, None, None

    def start(self):
        import threading

        self.stop_ev = threading.Event()

        def run():
            nv = self.nv
            while not self.stop_ev.is_set():
                self.sm.append(float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)))
                self.bits |= int(nv.nvmlDeviceGetCurrentClocksEventReasons(self.h))
                self.stop_ev.wait(0.005)

        self.t = threading.Thread(target=run, daemon=True)
        self.t.start()

    def stop(self):
        self.stop_ev.set()
        self.t.join()
        nv = self.nv
        names = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                 "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                 "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                 "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
        reasons = sorted(k for k, b in names.items() if self.bits & b)
        try:
            nv.nvmlShutdown()
        except Exception:
            pass
        if not self.sm:
            return None
        return {"sm_mhz": statistics.median(self.sm), "sm_max_mhz": self.max_mhz, "reasons": reasons,
                "samples": len(self.sm), "source": "nvml"}


class ClockSampler:
    early = True  # started before the warm-up
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.f.name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
def run_ours(args, rank, world, local_rank):
    import ctypes

    import numpy as np
    import torch

    import kapsel_old_b200 as kg
    from kapsel_old_b200 import workload

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist

    cfg = workload.mixed_128_256()
    hbm, peak_kind = peaks()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    L = kg.load_library()

    def timed(precision, steps, warmup, cfg=cfg, setup=None, sampler=None):
        sim = kg.Simulation(cfg, precision=precision)
        if setup is not None:
            setup(sim)
        sp = ctypes.c_void_p()
        sim._check(L.kapsel_gpu_get_stream(sim.h, ctypes.byref(sp)))
        stream = torch.cuda.ExternalStream(sp.value)
        sim.step(max(warmup, 3), graph=True)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        if sampler is not None and not sampler.early:
            sampler.start()
        for k in range(steps):
            with torch.cuda.stream(stream):
                flush.fill_(float(k))
                evs[k][0].record(stream)
            sim._check(L.kapsel_gpu_step_graph(sim.h, 1))
            evs[k][1].record(stream)
        torch.cuda.synchronize()
        if sampler is not None:
            sampler.result = sampler.stop()
        ms = reduce_max(sum(a.elapsed_time(b) for a, b in evs), dist)
        return sim, stream, ms

    # ---- mixed precision (headline) with clocks sampled during the timed
    # region (NVML, else nvidia-smi)
    try:
        clk = NvmlClockSampler(local_rank)
    except Exception:
        clk = ClockSampler(local_rank)
        clk.start()  # nvidia-smi starts slowly: it samples from the warm-up on
    sim_m, stream_m, ms_m = timed(kg.MIXED, args.steps, args.warmup, sampler=clk)
    clocks = clk.result
    # ---- FP64 path, same workload
    sim_d, _, ms_d = timed(kg.FP64, args.steps, args.warmup)
    sim_d.close()
    # ---- mixed-precision error of the headline configuration over its full
    # run, against the FP64 GPU path (which the tests pin to the reference)
    parity = parity_curve(kg, cfg, args.parity_steps) if args.parity_steps > 0 else None

    # ---- per-kernel durations (CUDA events between launches on the library stream)
    nker = kg.load_library().kapsel_gpu_launches_per_step(sim_m.h)
    prof_steps = max(5, min(args.steps, 20))
    acc = np.zeros(13)
    buf = (ctypes.c_float * 13)()
    for k in range(prof_steps):
        with torch.cuda.stream(stream_m):
            flush.fill_(float(k))
        torch.cuda.synchronize()
        sim_m._check(L.kapsel_gpu_profile_step(sim_m.h, buf))
        acc += np.frombuffer(buf, dtype=np.float32)
    acc /= prof_steps
    names = slot_labels(sim_m.step_kernel_names())
    # profiling slots: the kernels of a step, each launched on its own (in
    # the timed graph the position update runs inside the c2r launch); a slot
    # with no launch (a y pass inside a fused y/z kernel) is left out
    nslot = len(names)
    shares = {names[i]: float(acc[i]) for i in range(nslot) if names[i]}
    top = max((i for i in range(nslot) if names[i]), key=lambda i: acc[i])
    kb = kernel_bytes(cfg, 4)
    top_name = names[top]
    achieved = kb[top_name] / (acc[top] * 1e-3) / 1e9

    # ---- end to end through the public API: host noise + H2D, step, particle D2H
    Np = sim_m.Np
    rec = np.zeros((Np, kg.P_STRIDE))
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    # every step: the next step's thermostat normals drawn on the host and
    # copied up, the graph step, and the particle records copied back
    # (kapsel_gpu_step_graph_particles: one host synchronisation per step)
    for _ in range(args.steps):
        sim_m._check(L.kapsel_gpu_step_graph_particles(sim_m.h, 1,
                                                       rec.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
    torch.cuda.synchronize()
    e2e_s = reduce_max(time.perf_counter() - t0, dist)
    sim_m.close()

    # ---- the other workloads, same timing rules, fewer steps
    extra = {}
    if not args.no_extra:
        k2 = max(10, min(args.steps, 50))
        c1 = workload.plain_64_16()
        s1, _, ms1 = timed(kg.FP64, k2, args.warmup, cfg=c1)
        s1.close()
        c3 = workload.electrolyte_128_64()
        s3m, _, ms3m = timed(kg.MIXED, k2, args.warmup, cfg=c3)
        s3m.close()
        s3d, _, ms3d = timed(kg.FP64, k2, args.warmup, cfg=c3)
        s3d.close()
        c6 = workload.shear_le_128_256()
        s6m, _, ms6m = timed(kg.MIXED, k2, args.warmup, cfg=c6)
        s6m.close()
        s6d, _, ms6d = timed(kg.FP64, k2, args.warmup, cfg=c6)
        s6d.close()
        extra = {
            "plain_64cubed_16_fp64": {"value": round(k2 * world / (ms1 * 1e-3), 2), "unit": UNIT, "steps": k2,
                                      "workload": "64^3, 16 spheres a=5, kBT=0, body force 1e-3 along -z, FP64"},
            "electrolyte_128cubed_64": {"mixed": round(k2 * world / (ms3m * 1e-3), 2),
                                        "fp64": round(k2 * world / (ms3d * 1e-3), 2), "unit": UNIT, "steps": k2,
                                        "workload": "128^3, 64 spheres a=5 Z=-100, salt Debye 4, Bjerrum 0.7, "
                                                    "E_x=0.05"},
            "shear_le_128cubed_256": {"mixed": round(k2 * world / (ms6m * 1e-3), 2),
                                      "fp64": round(k2 * world / (ms6d * 1e-3), 2), "unit": UNIT, "steps": k2,
                                      "workload": "128^3, 256 spheres a=5, kBT=1e-3, Lees-Edwards shear rate 0.01 "
                                                  "(oblique grid)"},
        }
        # batched ensemble: 48 boxes of 4 shapes, one graph launch per step
        boxes = workload.batched()
        sims = [kg.Simulation(c, precision=kg.MIXED) for c in boxes]
        batch = kg.Batch(sims, autotune=True)
        batch.step(max(args.warmup, 3))
        bstream = torch.cuda.ExternalStream(batch.stream())
        torch.cuda.synchronize()
        kbat = max(5, min(args.steps, 20))
        bms = 0.0
        for k in range(kbat):
            with torch.cuda.stream(bstream):
                flush.fill_(float(k))
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(bstream)
            batch.step(1)
            e1.record(bstream)
            torch.cuda.synchronize()
            bms += e0.elapsed_time(e1)
        bms = reduce_max(bms, dist)
        msd = batch.msd()
        chosen = batch.variants()
        batch.close()
        for sm_ in sims:
            sm_.close()
        pts = sum((1 << c["np_xyz"][0]) * (1 << c["np_xyz"][1]) * (1 << c["np_xyz"][2]) for c in boxes)
        extra["batched_48_boxes"] = {
            "value": round(kbat * world / (bms * 1e-3), 2), "unit": "ensemble steps/s", "steps": kbat,
            "grid_points_steps_per_s": round(kbat * world * pts / (bms * 1e-3), 1),
            "boxes": len(boxes), "particles": sum(len(c["particles"]) for c in boxes),
            "msd_mean": float(np.mean(msd)),
            "autotune": [{"shape": list(v[:3]), "z_pass": ["warp", "block"][v[3]],
                          "y_pass": Y_VARIANTS[v[4]], "x_split": ["default", "other"][v[5]]} for v in chosen],
            "workload": "48 boxes from {32^3, 64^3, 64x64x128, 128^3}, 1-64 spheres a in [4,6], kBT=1e-3, mixed"}
        # learned near-contact correction: trained on the GPU from the committed
        # pair set (method runs at a=5 and a=10), then the 256^3 / 2048-sphere
        # mixed step timed without and with the network attached
        from kapsel_old_b200 import nearcontact as ncm

        pairs = os.path.join(ROOT, "tests", "golden", "nearcontact_pairs.npz")
        if os.path.exists(pairs):
            d = dict(np.load(pairs))
            npair = len(d["gap"])
            ntest = npair // 8
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            net, hist = ncm.fit(d, np.arange(npair - ntest), epochs=600)
            t_fit = time.perf_counter() - t0
            err = ncm.errors(net, d, np.arange(npair - ntest, npair))
            c5 = workload.nearcontact_256_2048()
            k5 = max(10, min(args.steps, 40))
            s5a, _, ms5a = timed(kg.MIXED, k5, args.warmup, cfg=c5)
            s5a.close()
            s5b, _, ms5b = timed(kg.MIXED, k5, args.warmup, cfg=c5, setup=lambda sm_: ncm.attach(sm_, net))
            n_corr = ncm.corrected_pairs(s5b)
            s5b.close()
            extra["nearcontact_256cubed_2048"] = {
                "plain": round(k5 * world / (ms5a * 1e-3), 2), "learned": round(k5 * world / (ms5b * 1e-3), 2),
                "unit": UNIT, "steps": k5, "extra_step_time": round(ms5b / ms5a - 1.0, 4),
                "pairs_corrected_last_step": n_corr,
                "train": {"pairs": int(npair - ntest), "epochs": 600, "seconds": round(t_fit, 2),
                          "final_loss": float(hist[-1])},
                "test_rms": {k: round(v, 6) for k, v in err.items()}, "test_pairs": int(ntest),
                "force_error_reduction": round(err["force_plain"] / err["force_learned"], 2),
                "torque_error_reduction": round(err["torque_plain"] / err["torque_learned"], 2),
                "workload": "256^3, 2048 spheres a=5 (volume fraction 0.064), min gap 0.05a, kBT=1e-3, mixed; "
                            "network 16-128-128-128-16 SiLU, tcgen05 BF16"}
            # the same network at the deployment density (volume fraction
            # 0.27): neighbour lists for the pair searches
            cd = workload.nearcontact_256_dense()
            s6a, _, ms6a = timed(kg.MIXED, k5, args.warmup, cfg=cd)
            s6a.close()
            s6b, _, ms6b = timed(kg.MIXED, k5, args.warmup, cfg=cd, setup=lambda sm_: ncm.attach(sm_, net))
            n_corr6 = ncm.corrected_pairs(s6b)
            s6b.close()
            extra["nearcontact_256cubed_dense"] = {
                "plain": round(k5 * world / (ms6a * 1e-3), 2), "learned": round(k5 * world / (ms6b * 1e-3), 2),
                "unit": UNIT, "steps": k5, "extra_step_time": round(ms6b / ms6a - 1.0, 4),
                "pairs_corrected_last_step": n_corr6,
                "force_error_reduction": round(err["force_plain"] / err["force_learned"], 2),
                "workload": "256^3, 8600 spheres a=5 (volume fraction 0.268), min gap 0.05a, kBT=1e-3, mixed; "
                            "the network trained above"}
            net.close()
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            extra["batched_48_boxes"]["cpu_baseline"] = cpu_baseline_batch(boxes)
            extra["plain_64cubed_16_fp64"]["cpu_baseline"] = cpu_baseline(c1, warmup=1, steps=30)
            extra["electrolyte_128cubed_64"]["cpu_baseline"] = cpu_baseline(c3, warmup=1, steps=4)
            extra["shear_le_128cubed_256"]["cpu_baseline"] = cpu_baseline(c6, warmup=1, steps=8)

    steps_total = args.steps * world
    traffic = ncu_traffic(top_name)
    value = replica_value(args.steps, world, ms_m * 1e-3)
    fp64_value = replica_value(args.steps, world, ms_d * 1e-3)
    bstep, passes = step_bytes_model(cfg, 4)
    line = {
        "metric": METRIC,
        "value": round(value, 3),
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_m / args.steps, 5),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded positions, PCG64 seed 2; MT19937 seed 0 thermostat)",
        "config": {
            "workload": WORKLOAD,
            "grid": [128, 128, 128],
            "particles": 256,
            "precision": "mixed: f32 fields/FFTs/stencil fields, f64 particles, reductions, k=0 mode",
            "l2": "256 MiB buffer written before every timed step (L2 126 MB)",
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
            "cuda_graph": True,
        },
        "fp64": {"value": round(fp64_value, 3), "ms_per_step": round(ms_d / args.steps, 5),
                 "mixed_over_fp64": round(value / fp64_value, 3)},
        "fp64_value": round(fp64_value, 3),
        "mixed_over_fp64": round(value / fp64_value, 3),
        # the same throughput in grid points advanced per second (all ranks)
        "grid_point_steps_per_s": round(value * (1 << sum(cfg["np_xyz"])), 1),
        "parity": parity,
        "roofline": {"bound": "hbm", "kernel": top_name, "achieved": round(achieved, 1), "peak": hbm,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / hbm, 4),
                     "algorithmic_bytes_per_launch": kb[top_name], "avg_launch_ms": round(float(acc[top]), 5),
                     "traffic": traffic[0], "traffic_source": traffic[1]},
        "step_roofline": {"bytes_per_step_model": int(bstep), "field_passes": round(passes, 2),
                          "achieved_gbs": round(bstep / (ms_m / args.steps * 1e-3) / 1e9, 1),
                          "frac": round(bstep / (ms_m / args.steps * 1e-3) / 1e9 / hbm, 4)},
        "kernel_ms": {k: round(v, 5) for k, v in shares.items()},
        "e2e": {"value": round(steps_total / e2e_s, 3), "unit": UNIT, "h2d_bytes_per_step": 6 * 8 * Np,
                "d2h_bytes_per_step": kg.P_STRIDE * 8 * Np + 4},
        "gpu_launches": nker * args.steps,
        "clocks": clocks,
        "other_workloads": extra,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(cfg, warmup=1, steps=min(args.steps, 12))
        # the serial build (the oracle) on one core, reported beside it
        line["cpu_baseline_serial"] = cpu_baseline(cfg, warmup=1, steps=min(args.steps, 8), serial=True)
    return line


# ---------------------------------------------------------------------------
def ncu_traffic(kernel: str):
    """DRAM bytes per launch of `kernel` as an ncu capture recorded them in the
    committed summary (profiles/<kernel without the leading k_>_*.md, line
    `traffic_bytes_per_launch`), with the summary's name and the build it was
    captured on (line `captured_at`): (bytes, source) or (None, None).  The
    figure is not measured by this run."""
    import glob
    import re

    stem = kernel[2:] if kernel.startswith("k_") else kernel
    here = os.path.dirname(os.path.abspath(__file__))
    for f in sorted(glob.glob(os.path.join(here, "profiles", f"k_*{stem.replace('z_', 'z*_')}*.md"))):
        text = open(f).read()
        m = re.search(r"\|\s*traffic_bytes_per_launch\s*\|\s*([0-9]+)\s*\|", text)
        if m:
            at = re.search(r"captured_at:\s*(\S+)", text)
            src = "ncu capture in " + os.path.relpath(f, here) + (f" (build {at.group(1)})" if at else "")
            return int(m.group(1)), src
    return None, None


def parity_curve(kg, cfg, steps: int, points=(1, 10, 100, 250, 500, 1000, 1500, 2000)):
    """Mixed-precision state against the FP64 GPU path from the same initial
    state, both replayed from CUDA graphs: velocity-field relative L2,
    particle velocity relative L2 and the largest position difference at
    checkpoints up to `steps`."""
    import numpy as np

    def rel(a, b):
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))

    a = kg.Simulation(cfg, precision=kg.FP64)
    b = kg.Simulation(cfg, precision=kg.MIXED)
    curve, done = [], 0
    for at in [p for p in points if p <= steps] + ([steps] if steps not in points else []):
        a.step(at - done, graph=True)
        b.step(at - done, graph=True)
        done = at
        pa, pb = a.particles(), b.particles()
        curve.append({"step": at, "u_rel_l2": rel(b.velocity(), a.velocity()), "v_rel_l2": rel(pb["v"], pa["v"]),
                      "x_max_abs": float(np.abs(pb["x_nopbc"] - pa["x_nopbc"]).max())})
    a.close()
    b.close()
    return {"mixed_u_rel_l2": curve[-1]["u_rel_l2"], "mixed_v_rel_l2": curve[-1]["v_rel_l2"],
            "mixed_x_max_abs": curve[-1]["x_max_abs"], "steps": steps,
            "against": "FP64 GPU step from the same state (FP64 pinned to the reference <= 1e-10)",
            "curve": curve}


def cpu_baseline(cfg, warmup: int, steps: int, threads: int | None = None, serial: bool = False):
    """Reference CPU timing on the host cores (oracle/_ref; else the numpy port):
    the OpenMP build on all cores, or with `serial` the serial build (the
    oracle) on one core."""
    from oracle import ref, udf

    threads = 1 if serial else (threads or os.cpu_count() or 1)
    exe = os.path.join(ref.REF_DIR, "kapsel_ref" if serial else "kapsel_ref_omp")
    if os.path.exists(exe):
        with tempfile.TemporaryDirectory() as td:
            kv = udf.write_udf(os.path.join(td, "in.kv"), cfg)
            env = dict(os.environ, OMP_NUM_THREADS=str(threads))
            out = subprocess.run([exe, kv, str(warmup), str(steps)], capture_output=True, text=True, env=env,
                                 timeout=900)
            d = json.loads(out.stdout.strip().splitlines()[-1])
        build = "serial build, one core" if serial else "OpenMP loops"
        return {"value": round(1.0 / d["s_per_step"], 4), "unit": UNIT, "cores": threads, "kind": "reference",
                "sample": f"{steps} steps of the same workload after {warmup} warm-up, "
                          f"unmodified KAPSEL sources ({build}, Ooura FFT), wall clock"}
    from oracle import spm

    o = spm.SpmOracle(cfg)
    o.run(warmup)
    t = time.perf_counter()
    n = max(1, min(steps, 3))
    o.run(n)
    dt = (time.perf_counter() - t) / n
    return {"value": round(1.0 / dt, 4), "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"{n} steps of the same workload, numpy restatement"}


def cpu_baseline_batch(boxes):
    """Estimated reference time of one ensemble step: the reference runs each
    box as its own process, so one box of each shape is timed (2 steps after
    1 warm-up) and the per-shape times are summed over the boxes."""
    per_shape = {}
    for c in boxes:
        key = tuple(c["np_xyz"])
        if key not in per_shape:
            per_shape[key] = 1.0 / cpu_baseline(c, warmup=1, steps=2)["value"]
    total = sum(per_shape[tuple(c["np_xyz"])] for c in boxes)
    return {"value": round(1.0 / total, 5), "unit": "ensemble steps/s", "cores": os.cpu_count() or 1,
            "kind": "reference",
            "sample": "one box per shape timed for 2 steps (OpenMP build, all cores), summed over the 48 boxes"}


def run_reference(args, world: int = 1):
    from kapsel_old_b200 import workload

    cfg = workload.mixed_128_256()
    steps = max(1, min(args.steps, REF_MAX_STEPS))
    # the warm-up the caller asked for (as the GPU arm takes it), at most 10
    warmup = max(1, min(args.warmup, 10))
    cb = cpu_baseline(cfg, warmup=warmup, steps=steps)
    return {
        "impl": "reference",
        "metric": METRIC,
        "value": cb["value"],
        "unit": UNIT,
        "n_gpus": world,  # the launch's N; the work runs on rank 0's host cores (cpu_baseline.cores)
        "steps": steps,
        "warmup": warmup,
        "ms_per_step": round(1000.0 / cb["value"], 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded positions, PCG64 seed 2; MT19937 seed 0 thermostat)",
        "config": {"workload": WORKLOAD, "grid": [128, 128, 128], "particles": 256,
                   "precision": "reference FP64 CPU",
                   "l2": "no flush (host CPU run)",
                   "parallelism": f"OpenMP on {cb['cores']} host cores",
                   "cuda_graph": False},
        "cpu_baseline": cb,
        "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="skip the 64^3 FP64 and electrolyte workloads")
    ap.add_argument("--parity-steps", type=int, default=2000,
                    help="steps of the mixed-vs-FP64 error curve (0: skip)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args, world)), flush=True)
        return

    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    line = run_ours(args, rank, world, local_rank)
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
