#!/usr/bin/env python
"""Benchmark of the per-slot uplink hot path on B200.

Workload (one "step" = one uplink slot of one cell): 256 antennas x 32 users,
4096-point FFT with 3276 data subcarriers, 14 OFDM symbols (2 comb-pilot
symbols + 12 data symbols), 64-QAM at 25 dB SNR over an 8-tap exponential
power-delay-profile channel with antenna correlation 0.5; int8 time-domain
IQ samples in by default (the reference's production sample type; --iq picks
int16, complex float32 or FP16).  Per slot: pilot FFT + LS estimate, per-group ZF
(Gram, inverse, detector), uplink FFT, equalize + FP16 LLR demod + descrambled
hard bits.  Inputs are seeded synthetic slots (megastation_b200.datagen).
The mixed ZF starts its two Newton-Schulz steps from the learned polynomial
initial iterate (its network trained in the run by the library's kernels;
--init exact for the Gauss-Jordan inverse), so the headline is the mixed +
learned path of the metric, with the plain FP32 path timed beside it.

Lines printed (rank 0): one JSON object.  Multi-GPU (torchrun): replicas, one
independent slot stream per GPU (the path has no exchange step).
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(M=256, K=32, N=4096, S=3276, sg=16, Qm=6, U=12, snr_db=25.0, channel="tdl",
                n_taps=8, tap_decay=2.0, rho=0.5, iq_dtype="int8", seed=2024)
# bytes per IQ sample of each input format
IQ_BYTES = {"c64": 8, "int16": 4, "int8": 2, "f16": 4}
METRIC = "slots/s"
# the arithmetic of the mixed path, stage by stage
MIXED_DTYPE = ("bf16 operands with f32 accumulation (Gram, detector W = X C, equalizer GEMV); "
               "f32 inverse + Newton-Schulz; fp16 operands and an fp16 twiddled intermediate with f32 "
               "accumulation in the N=4096 tensor-core FFT (bf16 rows out); fp16 LLRs")
UNIT = "slots/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="cell256x32",
                    choices=["cell256x32", "cells32", "full256x64", "learned128x16", "learned256x32", "ldpc256x32"],
                    help="cells32: 32 seeded uneven cells in one graph launch per slot (autotuned); "
                         "full256x64: uplink + downlink slot, 256-QAM, latency percentiles; "
                         "learned128x16: per-subcarrier ZF with the learned initialiser")
    ap.add_argument("--uplink-symbols", type=int, default=None,
                    help="data symbols per slot of the cell256x32 workload (default 12, the headline); "
                         "with --sym-batch at least as large and U x 16 <= 128 the slot equalizes "
                         "inside its ZF kernel")
    ap.add_argument("--precision", default="mixed", choices=["fp32", "mixed"])
    ap.add_argument("--no-plain", action="store_true", help="skip timing the plain FP32 path")
    ap.add_argument("--no-evm", action="store_true")
    ap.add_argument("--ns-iters", type=int, default=2, help="Newton-Schulz steps of the mixed ZF (config 2 names 2)")
    ap.add_argument("--sym-batch", type=int, default=12)
    ap.add_argument("--init", default="learned", choices=["learned", "exact"],
                    help="initial iterate of the mixed ZF's Newton-Schulz steps: the learned polynomial "
                         "(network trained in the run by the library's kernels) or the exact inverse")
    ap.add_argument("--init-realisations", type=int, default=2440,
                    help="channel realisations per training shape (x 205 groups x 2 shapes)")
    ap.add_argument("--init-steps", type=int, default=3000, help="Adam steps of the initial-iterate network")
    ap.add_argument("--iq", default="int8", choices=["int8", "int16", "c64", "f16"],
                    help="sample format of the cell256x32 workload: int8 is the reference's production "
                         "QuanT (utils/types.h:26), int16 the other integer format its FFT takes")
    ap.add_argument("--rotate", type=int, default=4, help="distinct input slots cycled (L2 flush)")
    ap.add_argument("--windows", type=int, default=10,
                    help="minimum number of repeated K-slot windows timed after the headline window")
    ap.add_argument("--min-slots", type=int, default=1000,
                    help="full256x64: consecutive slots timed for the latency percentiles (at least --steps)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-inflight", action="store_true", help="skip timing two slots in flight")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the short runs of the full-slot (256x64) and 32-cell workloads in the default line")
    return ap.parse_args()


def algorithmic_bytes(cfg, b_in=None):
    """Compulsory bytes of one uplink slot: samples in (b_in bytes each, by
    default those of the workload's sample format), FP16 LLRs and packed
    hard bits out (intermediates excluded)."""
    b_in = IQ_BYTES[cfg.iq_dtype] if b_in is None else b_in
    cb, zeros, stride = cfg.ldpc()
    n_valid = min(cfg.S * cfg.Qm, cb)
    return (cfg.P + cfg.U) * cfg.M * cfg.N * b_in + cfg.U * cfg.K * n_valid * 2 + \
        cfg.U * cfg.K * ((n_valid + 7) // 8)


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, smax, reasons, power = [], None, set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
                power.append(float(f[3]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm),
                "power_w_max": max(power) if power else None}


def max_over_ranks(ms, dist, device="cuda"):
    """The slowest rank's time (every rank takes this collective step at the
    same point, in warm-up and timing alike); ms itself with one process."""
    if not dist:
        return ms
    import torch
    t = torch.tensor([ms], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_value(world, steps, ms):
    """Whole-job throughput: every rank ran `steps` slots of its own stream
    (weak scaling), the job took the slowest rank's `ms`."""
    return world * steps / (ms / 1e3)


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), d.get("bf16_tflops", 1590.0), "measured"
    return 6650.0, 1590.0, "fallback"


def profile_traffic(name, unit_name, units):
    """DRAM bytes per launch from the committed ncu summary profiles/<name>.md
    (its line "dram bytes per <unit_name>: B", scaled by the units of one
    launch), or None when the summary is absent."""
    import re
    path = os.path.join(ROOT, "profiles", name + ".md")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        m = re.search(r"dram bytes per " + re.escape(unit_name) + r": *([0-9.eE+]+)", f.read())
    return float(m.group(1)) * units if m else None


def fused_equalize(cfg, sym_batch, mixed):
    """Whether the mixed slot equalizes inside its ZF kernel (the library's
    rule: the tensor-core FFT of pilots and every uplink symbol in one
    launch, K <= 32, M <= 256, sc_group a multiple of 16, and all of a
    group's (symbol, subcarrier) columns in one 128-column tile)."""
    if not (mixed and cfg.N == 4096 and cfg.U >= 1 and sym_batch >= cfg.U):
        return False
    return cfg.K <= 32 and cfg.M <= 256 and cfg.sg % 16 == 0 and cfg.U * cfg.sg <= 128


def slot_launches(cfg, sym_batch, mixed, downlink=False):
    """Kernels one uplink slot launches: the pilot FFT (inside the first
    uplink FFT launch in the mixed path at N = 4096), the ZF, one uplink FFT
    and one equalize per symbol batch (none when the ZF kernel equalizes);
    with a downlink also the precode and the IFFT, and in the mixed path the
    precoder scaling and its BF16 images (the FP32 path's Cholesky kernel
    writes the precoder itself)."""
    batches = max(1, -(-cfg.U // max(sym_batch, 1)))
    n = (0 if mixed and cfg.N == 4096 else 1) + 1 + 2 * batches
    if fused_equalize(cfg, sym_batch, mixed):
        n -= 1
    return n + ((4 if mixed else 2) if downlink else 0)


def roofline(cfg, args, st, n_valid, hrow):
    """Per-kernel times alone (CUDA events, timing mode) and the roofline of
    the kernel with the largest share of the slot."""
    hbm_peak, tc_peak, peak_kind = measured_peaks()
    calls = max(st["calls"], 1)
    mixed = args.precision == "mixed"
    fused = mixed and st["n_eq"] == 0                  # equalized inside the ZF kernel
    n_fft = max(st["n_fft"], 1)                        # launches over all recorded slots
    n_eq = calls if fused else max(st["n_eq"], 1)
    rows = cfg.U * cfg.M * calls / n_fft               # antenna rows per uplink FFT launch
    syms = cfg.U * calls / n_eq                        # symbols per equalize launch
    out_b = 4 if mixed else 8                          # BF16 planar or c32 per subcarrier
    bps = IQ_BYTES[cfg.iq_dtype]                       # bytes per input sample
    tc = {"MM": 64 if 2 * cfg.K <= 64 else 128, "Mp": (cfg.M + 63) // 64 * 64}
    img_group = 2 * tc["Mp"] * tc["MM"] * 2
    tc_fft = mixed and cfg.N == 4096  # the tensor-core FFT takes the mixed uplink at N = 4096 ...
    # ... and, in the slot, the pilot rows too (one launch with the first batch)
    pilot_rows = cfg.P * cfg.M * calls / n_fft if tc_fft else 0
    k = {
        "fft_uplink": {"ms": st["uplink_fft"] / n_fft, "per_slot_ms": st["uplink_fft"] / calls,
                       "bound": "hbm", "units": rows + pilot_rows, "unit_name": "antenna row",
                       "bytes": rows * (cfg.N * bps + cfg.S * out_b)
                       + pilot_rows * cfg.N * bps + (cfg.G * cfg.M * cfg.K * 8 * calls / n_fft if tc_fft else 0)},
        "fft_pilot": {"ms": st["pilot_fft"] / calls, "per_slot_ms": st["pilot_fft"] / calls,
                      "bound": "hbm", "units": cfg.P * cfg.M, "unit_name": "pilot row",
                      "bytes": cfg.P * cfg.M * (cfg.N * bps) + cfg.G * cfg.M * cfg.K * 8},
        "zf": {"ms": st["zf"] / calls, "per_slot_ms": st["zf"] / calls, "bound": "tensor",
               "units": cfg.G, "unit_name": "subcarrier group",
               "flops": cfg.G * (16.0 * cfg.K ** 2 * cfg.M + 40.0 * cfg.K ** 3)},
        "equalize": {"ms": st["equalize"] / n_eq, "per_slot_ms": st["equalize"] / calls,
                     "bound": "hbm", "units": syms, "unit_name": "symbol",
                     "bytes": (cfg.G * img_group if mixed else cfg.G * cfg.M * cfg.K * 8)
                     + syms * (cfg.M * cfg.S * out_b + cfg.K * (n_valid * 2 + hrow))},
    }
    if tc_fft:
        del k["fft_pilot"]  # the pilot rows go through the uplink FFT launch
    if fused:
        # one kernel: the ZF (latency-bound, its FLOPs stated) and the
        # equalize's bytes (CSI in, samples in, LLRs and hard bits out; the
        # detector image never leaves shared memory), held to HBM
        eq = k.pop("equalize")
        k["zf"].update({"bound": "hbm", "units": cfg.G,
                        "bytes": cfg.G * cfg.M * cfg.K * 8 + eq["bytes"] - cfg.G * img_group})
    names = {"fft_uplink": ("fft_tc_kernel<pilot + uplink rows>" if tc_fft else "fft_kernel<12, uplink LP>") if mixed
             else "fft_kernel<12, uplink>",
             "fft_pilot": "fft_kernel<12, pilot>",
             "zf": (f"zf_mixed_kernel<64, {cfg.Qm}> (ZF + equalize)" if fused else "zf_mixed_kernel<64, 0>")
             if mixed else "zf_chol_kernel<float>",
             "equalize": f"equalize_tc_kernel<64, {cfg.Qm}>" if mixed else "equalize_fp32_kernel"}
    # the tensor-core FFT's traffic depends on the sample format: int8
    # workloads read the int8 capture, the others the int16 one
    fft_tc_prof = "fft_tc_uplink_4096x256" + ("_int8" if cfg.iq_dtype == "int8" else "")
    profiles = {"fft_uplink": fft_tc_prof if tc_fft else "fft_uplink_lp_4096x256",
                "equalize": "equalize_tc_256x32",
                "zf": "zf_eq_fused_256x32" if fused else "zf_mixed_256x32", "fft_pilot": "fft_uplink_lp_4096x256"}
    for key, v in k.items():
        sec = v["ms"] / 1e3
        if v["bound"] == "hbm":
            v["achieved"] = v["bytes"] / sec / 1e9 if sec > 0 else 0.0
            v["frac"] = v["achieved"] / hbm_peak
        else:
            v["achieved"] = v["flops"] / sec / 1e12 if sec > 0 else 0.0
            v["frac"] = v["achieved"] / tc_peak
        if "flops" in v and v["bound"] == "hbm":
            v["tensor_frac"] = v["flops"] / sec / 1e12 / tc_peak if sec > 0 else 0.0
    dom = max(k, key=lambda x: k[x]["per_slot_ms"])
    v = k[dom]
    hbm = v["bound"] == "hbm"
    traffic = profile_traffic(profiles[dom], v["unit_name"], v["units"]) if mixed else None
    roof = {"kernel": names[dom], "bound": v["bound"], "achieved": v["achieved"],
            "peak": hbm_peak if hbm else tc_peak, "unit": "GB/s" if hbm else "TFLOP/s",
            "frac": v["frac"], "traffic": traffic,
            "algorithmic": (f"{v['bytes'] / v['units']:.0f} bytes per {v['unit_name']} x {v['units']:.0f}"
                            if hbm else f"{v['flops'] / v['units']:.0f} flops per {v['unit_name']} x "
                                        f"{v['units']:.0f}"),
            "ms_per_launch": v["ms"],
            "peak_source": f"{peak_kind} (MEASURED_PEAKS.json)" if peak_kind == "measured" else "fallback",
            "per_kernel": {names[x]: {"ms_per_launch": k[x]["ms"], "ms_per_slot": k[x]["per_slot_ms"],
                                      "bound": k[x]["bound"], "achieved": k[x]["achieved"],
                                      "frac": k[x]["frac"]} for x in k},
            "serial_slot_ms": st["slot"] / calls}
    return roof


def cpu_baseline(cfg, slot_np, seconds):
    """Host C++/OpenMP restatement of the same slot (oracle), all host threads."""
    from oracle import oracle as orc
    cb, zeros, stride = cfg.ldpc()
    ps = orc.pilot_sign(cfg.S)
    seq = slot_np["seq"][0]
    threads = os.cpu_count() or 1
    n, t0 = 0, time.perf_counter()
    while True:
        orc.slot_uplink_cpu(slot_np["iq"], cfg.P, cfg.U, cfg.K, cfg.N, cfg.S, cfg.sg, cfg.Qm, cb, stride,
                            zeros, ps, seq, threads=threads)
        n += 1
        el = time.perf_counter() - t0
        if el >= seconds or n >= 200:
            break
    return {"value": n / el, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{n} full slots of the bench workload (FP32, OpenMP, {threads} threads) in {el:.1f} s"}


def _standalone_datagen():
    """megastation_b200/datagen.py loaded as a module of its own, without
    running the package's __init__ (which loads libmegastation_b200.so)."""
    import importlib.util
    path = os.path.join(ROOT, "megastation_b200", "datagen.py")
    spec = importlib.util.spec_from_file_location("_mb_datagen_standalone", path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[spec.name] = mod  # dataclasses resolve the module by name
    spec.loader.exec_module(mod)
    return mod


def run_reference(args, rank, world):
    """The reference arm.  The reference implements this path only as CUDA
    operators (cuFFT, cuBLAS/cuSOLVER, its SIMT equalizer); where they were
    built from the reference tree (oracle/_ref, kind "reference") they run on
    this GPU in process.cc's order on the same slot shapes and integer
    samples as --iq (int8 by default; int16 stands in for the float formats,
    since the reference FFT takes integer IQ only).  Otherwise the FP32
    host C++/OpenMP restatement (kind "port") runs on all host cores.  Rank 0
    only.  This arm never imports the megastation_b200 package, so the
    process maps the reference's library and none of this project's: the
    seeded slot generator (plain numpy) is loaded from its file alone."""
    if rank != 0:
        return
    datagen = _standalone_datagen()
    cfg = datagen.CellConfig(**{**workload_dict(args), "iq_dtype": args.iq})
    from oracle import ref_ops
    cb, zeros, stride = cfg.ldpc()
    import torch
    if ref_ops.available() and torch.cuda.is_available():
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        # the reference FFT takes integer samples only (fft_op.cu:194-200)
        iq_ref = args.iq if args.iq in ("int8", "int16") else "int16"
        cfg = datagen.CellConfig(**{**cfg.__dict__, "iq_dtype": iq_ref})
        R = rotation(cfg, args)
        iqs = [torch.from_numpy(datagen.make_slot(datagen.CellConfig(**{**cfg.__dict__, "seed": cfg.seed + r}))["iq"]
                                ).cuda() for r in range(R)]
        llr = [torch.zeros(cfg.U, cfg.K, stride, dtype=torch.float16, device="cuda") for _ in range(2)]
        ref = ref_ops.RefSlot(cfg.M, cfg.K, cfg.N, cfg.S, cfg.sg, cfg.Qm, cfg.P, cfg.U, cb, zeros, stride,
                              iq=iq_ref)
        stream = torch.cuda.Stream()
        for k in range(max(args.warmup, 3)):
            ref.uplink(iqs[k % R].data_ptr(), llr[k % 2].data_ptr(), stream.cuda_stream)
        stream.synchronize()
        clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
        clocks.start()
        time.sleep(0.3)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for k in range(args.steps):
            ref.uplink(iqs[k % R].data_ptr(), llr[k % 2].data_ptr(), stream.cuda_stream)
        e1.record(stream)
        e1.synchronize()
        clk = clocks.stop()
        ms = e0.elapsed_time(e1)
        v = args.steps / (ms / 1e3)
        line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": f"synthetic (seeded, megastation_b200.datagen), {iq_ref} samples",
                "config": {**workload_config(cfg, args, R), "iq_dtype": iq_ref},
                "clocks": clk,
                "cpu_baseline": {"value": v, "unit": UNIT, "cores": 0, "kind": "reference",
                                 "sample": f"{args.steps} slots through the reference's own CUDA operators "
                                           "(fft_op.cu, beamform.cu, equalize.cu built from the reference "
                                           "tree) on this GPU, process.cc order, one stream"},
                "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return
    d = datagen.make_slot(cfg)
    from oracle import oracle as orc
    ps = orc.pilot_sign(cfg.S)
    threads = os.cpu_count() or 1
    # bounded sample per step: one full slot per step
    for _ in range(max(0, min(args.warmup, 1))):
        orc.slot_uplink_cpu(d["iq"], cfg.P, cfg.U, cfg.K, cfg.N, cfg.S, cfg.sg, cfg.Qm, cb, stride, zeros, ps,
                            d["seq"][0], threads=threads)
    steps = max(1, min(args.steps, 20))
    t0 = time.perf_counter()
    for _ in range(steps):
        orc.slot_uplink_cpu(d["iq"], cfg.P, cfg.U, cfg.K, cfg.N, cfg.S, cfg.sg, cfg.Qm, cb, stride, zeros, ps,
                            d["seq"][0], threads=threads)
    el = time.perf_counter() - t0
    v = steps / el
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
            "steps": steps, "warmup": min(args.warmup, 1), "ms_per_step": 1e3 * el / steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": workload_config(cfg, args),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{steps} full slots, FP32 host C++/OpenMP restatement of the "
                                       f"reference operators ({threads} threads)"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def repeat_windows(step, stream, args, ms_first, dist, world):
    """Times windows of args.steps slots back to back (CUDA events per
    window on the slot stream) until about one second of slots or
    args.windows windows, whichever is more; every rank runs the same
    count, and each window's time is the maximum over ranks."""
    import torch
    n = max(args.windows, int(1000.0 / max(ms_first, 1e-3)))
    n = min(n, 2000)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n)]
    k = 0
    for a, b in ev:
        a.record(stream)
        for _ in range(args.steps):
            step(k)
            k += 1
        b.record(stream)
    stream.synchronize()
    w_ms = torch.tensor([a.elapsed_time(b) for a, b in ev], dtype=torch.float64)
    if dist:
        w_ms = w_ms.cuda()
        dist.all_reduce(w_ms, op=dist.ReduceOp.MAX)
        w_ms = w_ms.cpu()
    vals = np.array([job_value(world, args.steps, m) for m in w_ms.tolist()])
    return {"windows": n, "slots_per_window": args.steps, "value_median": float(np.median(vals)),
            "value_min": float(vals.min()), "value_max": float(vals.max()),
            "value_p10": float(np.percentile(vals, 10)), "value_p90": float(np.percentile(vals, 90)),
            "us_per_slot_median": float(1e3 * np.median(w_ms.numpy()) / args.steps)}


def train_zf_init(args):
    """The learned initial iterate's network (6 -> 64 -> 64 -> 4), trained on
    the GPU by the library's own forward, backward and Adam kernels on the
    quadratic residual targets of every group of seeded channel
    realisations of 256 x 32 and 128 x 16 cells (8-tap channel, correlation
    0.3-0.7, SNR 18-30 dB); returns the network and a training record with
    its held-out residual against the fixed Neumann polynomial."""
    import torch
    from megastation_b200 import learned
    t0 = time.perf_counter()
    data = learned.zf_init_training_set([(256, 32), (128, 16)], n_real=args.init_realisations, seed=1)
    torch.cuda.synchronize()
    t_data = time.perf_counter() - t0
    net = learned.make_zf_init_net(width=64, seed=3)
    t0 = time.perf_counter()
    hist = learned.train(net, data, steps=args.init_steps, batch=4096, lr=2e-3, seed=5, log_every=1000)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    held = learned.zf_init_training_set([(256, 32)], n_real=20, seed=77, rho=(0.5, 0.5), tap_decay=(2.0, 2.0),
                                        snr_db=(25.0, 25.0))
    r_l, r_n = learned.poly_residual(net, held)
    info = {"network": "6 -> 64 -> 64 -> 4, ReLU, BF16 weights, FP32 accumulation",
            "samples": int(data[0].shape[0]), "realisations": 2 * args.init_realisations,
            "steps": args.init_steps, "batch": 4096, "data_s": t_data, "train_s": t_train,
            "loss_history": hist,
            "heldout_residual": {"learned": r_l, "neumann": r_n,
                                 "note": "mean ||I - Gn p(Gn)||_F^2 / K on 4100 groups of the bench channel"}}
    del data
    return net, info


def time_slots(slot_mod, cfg, precision, sym_batch, iq_dev, llr, hard, stream, steps, warmup, dist, net=None):
    """K graph-replayed slots on device-resident inputs; returns ms."""
    import torch
    R = len(iq_dev)
    run = slot_mod.UplinkSlot(cfg, precision=precision, sym_batch=sym_batch, use_graph=True)
    if net is not None:
        run.set_zf_init(net)
    with torch.cuda.stream(stream):
        for k in range(max(warmup, 2 * R)):
            run(iq_dev[k % R], llr[k % 2], hard[k % 2], stream=stream)
    stream.synchronize()
    if dist:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for k in range(steps):
        run(iq_dev[k % R], llr[k % 2], hard[k % 2], stream=stream)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1)


def time_in_flight(slot_mod, cfg, args, iq_dev, stride, hrow, dist, D=2, net=None):
    """The same slots with D of them in flight: D slot runners, each a
    captured graph on its own stream, taking every D-th slot; reported beside
    the headline (one slot at a time), not instead of it."""
    import torch
    R = len(iq_dev)
    streams = [torch.cuda.Stream() for _ in range(D)]
    runs = [slot_mod.UplinkSlot(cfg, precision=args.precision, sym_batch=args.sym_batch, use_graph=True,
                                ns_iters=args.ns_iters) for _ in range(D)]
    if net is not None:
        for r in runs:
            r.set_zf_init(net)
    llr = [torch.zeros(cfg.U, cfg.K, stride, dtype=torch.float16, device="cuda") for _ in range(2 * D)]
    hard = [torch.zeros(cfg.U, cfg.K, hrow, dtype=torch.uint8, device="cuda") for _ in range(2 * D)]

    def step(k):
        i = k % D
        o = (k // D) % 2 * D + i
        runs[i](iq_dev[k % R], llr[o], hard[o], stream=streams[i])

    for k in range(max(args.warmup, 2 * R * D)):
        step(k)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    master = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(master)
    for s in streams:
        s.wait_stream(master)
    for k in range(args.steps):
        step(k)
    for s in streams:
        master.wait_stream(s)
    e1.record(master)
    e1.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), dist)
    return {"slots_in_flight": D, "value": job_value(1 if not dist else dist.get_world_size(), args.steps, ms),
            "unit": UNIT, "us_per_slot": 1e3 * ms / args.steps}


def evm_report(cfg, d, sym_batch, ns_iters=2, net=None):
    """EVM (dB) of the equalized symbols against the transmitted ones for the
    plain FP32 path, the mixed path and an FP64-ZF variant, on one slot.  The
    mixed row follows the mixed slot's arithmetic: the mixed-precision pilot
    and uplink FFTs (tensor cores at N = 4096) and their BF16 rows."""
    import torch
    import megastation_b200 as mb
    iq = torch.from_numpy(d["iq"]).cuda()
    cb, zeros, stride = cfg.ldpc()
    out = {}
    rows = [("fp64_zf", 2, None), ("plain_fp32", 0, None), ("mixed", 1, net)]
    if net is not None:
        rows.append(("mixed_exact_init", 1, None))
    for name, prec, nt in rows:
        csi = torch.zeros(cfg.G, cfg.M, cfg.K, dtype=torch.complex64, device="cuda")
        pf = mb.PilotFFT(cfg.start, cfg.N, cfg.S, cfg.M, cfg.K, cfg.sg)
        (pf.mixed if prec == 1 else pf)(iq[:cfg.P], csi)
        mb.Beamform(cfg.M, cfg.K, cfg.G, precision=prec, ns_iters=ns_iters, init_net=nt).beamform_uplink(
            csi, S=cfg.S, sc_group=cfg.sg)
        uf = mb.UplinkFFT(cfg.start, cfg.N, cfg.S, cfg.M)
        if prec == 1:
            pitch = (cfg.S + 7) // 8 * 8
            ylp = torch.zeros(cfg.U, 2, cfg.M, pitch, dtype=torch.bfloat16, device="cuda")
            uf.uplink_bf16(iq[cfg.P:], ylp, pitch)
            y = torch.complex(ylp[:, 0, :, :cfg.S].float(), ylp[:, 1, :, :cfg.S].float()).contiguous()
        else:
            y = torch.zeros(cfg.U, cfg.M, cfg.S, dtype=torch.complex64, device="cuda")
            uf(iq[cfg.P:], y)
        llr = torch.zeros(cfg.U, cfg.K, stride, dtype=torch.float16, device="cuda")
        x = torch.zeros(cfg.U, cfg.K, cfg.S, dtype=torch.complex64, device="cuda")
        eq = mb.Equalize.equalize_tc if prec == 1 else mb.Equalize.equalize
        eq(csi, y, llr, cfg.sg, cfg.Qm, cb, zeros, 1, x=x)
        torch.cuda.synchronize()
        xs = x.cpu().numpy()
        err = np.mean(np.abs(xs - d["x"]) ** 2) / np.mean(np.abs(d["x"]) ** 2)
        out[name] = float(10 * np.log10(err))
    out["mixed_minus_fp64_db"] = out["mixed"] - out["fp64_zf"]
    out["plain_minus_fp64_db"] = out["plain_fp32"] - out["fp64_zf"]
    return out


def hard_bits_report(cfg, d, sym_batch, ns_iters=2, tol=4.0, net=None):
    """The mixed slot's descrambled hard bits against the plain FP32 slot's
    on the same samples (both through the slot runner the bench times): the
    number of bits that differ where the plain path's |LLR| > tol, the total
    number of differing bits, and the uncoded BER of each path against the
    transmitted bits."""
    import torch
    from megastation_b200 import slot
    cb, zeros, stride = cfg.ldpc()
    n_valid = min(cfg.S * cfg.Qm, cb)
    iq = torch.from_numpy(d["iq"]).cuda()
    out = {}
    for name in ("fp32", "mixed"):
        run = slot.UplinkSlot(cfg, precision=name, sym_batch=sym_batch, ns_iters=ns_iters)
        if name == "mixed" and net is not None:
            run.set_zf_init(net)
        llr, hard = run(iq)
        torch.cuda.synchronize()
        bits = np.unpackbits(hard.cpu().numpy(), axis=-1)[..., :n_valid]
        out[name] = (llr.cpu().numpy().astype(np.float32)[..., zeros:zeros + n_valid], bits)
    lp, bp = out["fp32"]
    _, bm = out["mixed"]
    sure = np.abs(lp) > tol
    sent = d["bits"][..., :n_valid]
    return {"tol_abs_llr": tol, "bits": int(bp.size), "bits_above_tol": int(sure.sum()),
            "mismatch_above_tol": int((bm != bp)[sure].sum()), "mismatch_all": int((bm != bp).sum()),
            "uncoded_ber_plain": float(np.mean(bp != sent)), "uncoded_ber_mixed": float(np.mean(bm != sent))}


def rotation(cfg, args):
    """Distinct input slots cycled through the timed steps: at least
    --rotate, and enough that the rotated samples alone exceed 1.25x the
    126 MB L2, so every step reads its samples from HBM."""
    slot_bytes = cfg.symbols * cfg.M * cfg.N * IQ_BYTES[cfg.iq_dtype]
    return max(2, args.rotate, -(-int(1.25 * 126e6) // slot_bytes))


def workload_dict(args):
    """The cell256x32 workload, with --uplink-symbols data symbols when given."""
    u = getattr(args, "uplink_symbols", None)
    return {**WORKLOAD, "U": u} if u else dict(WORKLOAD)


def workload_config(cfg, args, R=None):
    R = rotation(cfg, args) if R is None else R
    return {"workload": f"uplink slot 256x32, N=4096, S=3276, 2 pilot + {cfg.U} data symbols, 64-QAM, "
                        f"8-tap exp-PDP rho=0.5, 25 dB, {cfg.iq_dtype} samples",
            "M": cfg.M, "K": cfg.K, "N": cfg.N, "S": cfg.S, "sg": cfg.sg, "Qm": cfg.Qm, "P": cfg.P,
            "U": cfg.U, "iq_dtype": cfg.iq_dtype, "precision": args.precision, "sym_batch": args.sym_batch,
            "ns_iters": args.ns_iters,
            "zf_init": ("learned polynomial (network trained in the run), exact inverse as fallback"
                        if args.precision == "mixed" and args.init == "learned" else "exact inverse"),
            "l2": f"inputs {cfg.symbols * cfg.M * cfg.N * IQ_BYTES[cfg.iq_dtype] / 1e6:.1f} MB per slot, {R} "
                  "slots rotated (larger than the 126 MB L2)",
            "seed": cfg.seed}


def measure_full(args, n_min=None):
    """Uplink + downlink slots of a 256-antenna, 64-user cell (N = 4096,
    S = 3276, P = 4 pilot, U = 5 uplink, D = 5 downlink symbols, 256-QAM at
    30 dB, correlated 8-tap channel): uplink FP16 LLRs and descrambled hard
    bits, downlink ZF precoding of seeded 256-QAM symbols and IFFT to complex
    FP16 antenna samples; per-slot latency percentiles over the run."""
    import torch
    from megastation_b200 import datagen, slot
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    cfg = datagen.CellConfig(M=256, K=64, N=4096, S=3276, sg=16, Qm=8, U=5, snr_db=30.0, channel="tdl",
                             n_taps=8, tap_decay=2.0, rho=0.5, seed=5050)
    D = 5
    R = 4
    data = [datagen.make_slot(datagen.CellConfig(**{**cfg.__dict__, "seed": cfg.seed + r})) for r in range(R)]
    iqs = [torch.from_numpy(d["iq"]).cuda() for d in data]
    rng = np.random.default_rng(cfg.seed)
    table = datagen.mod_table(8)
    syms = [torch.from_numpy(table[rng.integers(0, 256, (D, cfg.K, cfg.S))].astype(np.complex64)).cuda()
            for _ in range(R)]
    run = slot.UplinkSlot(cfg, precision=args.precision, sym_batch=cfg.U, use_graph=True, D=D, out_dtype="f16")
    cb, zeros, stride = cfg.ldpc()
    hrow = (min(cfg.S * cfg.Qm, cb) + 7) // 8
    llr = [torch.zeros(cfg.U, cfg.K, stride, dtype=torch.float16, device="cuda") for _ in range(2)]
    hard = [torch.zeros(cfg.U, cfg.K, hrow, dtype=torch.uint8, device="cuda") for _ in range(2)]
    out = [torch.zeros(D, cfg.M, cfg.N, 2, dtype=torch.float16, device="cuda") for _ in range(2)]
    stream = torch.cuda.Stream()
    # the workload's latency percentiles are over at least 1000 consecutive
    # slots (the distinct seeded inputs rotated)
    n = max(args.steps, args.min_slots if n_min is None else n_min)

    def step(k):
        run(iqs[k % R], llr[k % 2], hard[k % 2], stream=stream)
        run.downlink(syms[k % R], out[k % 2], stream=stream)

    with torch.cuda.stream(stream):
        for k in range(max(args.warmup, 2 * R)):
            step(k)
    stream.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n)]
    clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    clocks.start()
    time.sleep(0.3)
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        for k in range(n):
            ev[k][0].record(stream)
            step(k)
            ev[k][1].record(stream)
    stream.synchronize()
    clk = clocks.stop()
    lat = np.array([a.elapsed_time(b) * 1e3 for a, b in ev])
    total_ms = ev[0][0].elapsed_time(ev[-1][1])
    # uplink EVM of the last slot against its transmitted symbols
    k = (n - 1) % R
    x = torch.zeros(cfg.U, cfg.K, cfg.S, dtype=torch.complex64, device="cuda")
    evm = None
    try:
        import megastation_b200 as mb
        csi = torch.zeros(cfg.G, cfg.M, cfg.K, dtype=torch.complex64, device="cuda")
        mb.PilotFFT(cfg.start, cfg.N, cfg.S, cfg.M, cfg.K, cfg.sg)(iqs[k][:cfg.P], csi)
        mb.Beamform(cfg.M, cfg.K, cfg.G, precision=1).beamform_uplink(csi, S=cfg.S, sc_group=cfg.sg)
        y = torch.zeros(cfg.U, cfg.M, cfg.S, dtype=torch.complex64, device="cuda")
        mb.UplinkFFT(cfg.start, cfg.N, cfg.S, cfg.M)(iqs[k][cfg.P:], y)
        l = torch.zeros(cfg.U, cfg.K, stride, dtype=torch.float16, device="cuda")
        mb.Equalize.equalize_tc(csi, y, l, cfg.sg, cfg.Qm, cb, zeros, 1, x=x)
        torch.cuda.synchronize()
        xs = x.cpu().numpy()
        evm = float(10 * np.log10(np.mean(np.abs(xs - data[k]["x"]) ** 2) / np.mean(np.abs(data[k]["x"]) ** 2)))
    except Exception as e:  # reported, not fatal for the timing
        evm = f"unavailable: {e}"
    line = {"metric": "slots/s (uplink + downlink)", "value": n / (total_ms / 1e3), "unit": "slots/s",
            "n_gpus": 1, "steps": n, "warmup": args.warmup, "ms_per_step": total_ms / n,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": MIXED_DTYPE if args.precision == "mixed" else "f32",
            "data": "synthetic (seeded, megastation_b200.datagen)",
            "config": {"workload": "full slot 256x64, N=4096, S=3276, P=4 U=5 D=5, 256-QAM, 30 dB, 8-tap "
                                   "exp-PDP rho=0.5; uplink LLRs + hard bits, downlink precode + IFFT to "
                                   "complex FP16", "slots": n, "distinct_inputs": R,
                       "l2": f"{sum(i.numel() * 8 for i in iqs) / 1e6:.0f} MB of samples rotated"},
            "latency_us": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                           "max": float(lat.max()), "mean": float(lat.mean())},
            "uplink_evm_db": evm, "clocks": clk,
            "gpu_launches": n * slot_launches(cfg, cfg.U, args.precision == "mixed", downlink=True),
            "downlink": ("tcgen05 precode (BF16 operands, FP32 accumulation) into FP16 spectra, then the "
                         "tensor-core inverse FFT (FP16 operands) with the output quantiser"
                         if args.precision == "mixed" else "FP32 precode and FP32 Stockham inverse FFT"),
            "note": "ZF from the exact initial iterate: the learned polynomial's network is trained for "
                    "K/M = 1/8 cells, and at K/M = 1/4 most groups would fall back to the exact inverse"}
    return line


def run_full(args):
    """Prints measure_full's line (config 5 as a workload of its own)."""
    print(json.dumps(measure_full(args)), flush=True)


def run_learned(args, shape="128x16"):
    """Per-subcarrier ZF with the learned initialiser, on a 128-antenna,
    16-user cell (N = 2048, S = 1200, 16-QAM, 25 dB; config 4) or, with
    shape "256x32", on the headline cell (N = 4096, S = 3276, 64-QAM, 25 dB),
    over the delay-spread TDL channel (8 taps, delay spread uniform in
    50-300 ns): the MLP is trained on the GPU (library kernels) on pilot CSI
    of seeded channel realisations, about 1e6 subcarrier samples with exact
    FP64 inverse labels; then EVM and uncoded BER of per-group ZF, exact
    per-subcarrier ZF, and the learned and coarse iterates with 0-2
    Newton-Schulz steps on slots of 50-300 ns, and slots/s of each detector
    path (graph-replayed FP32 slot: pilot FFT, ZF, uplink FFT, equalize)."""
    import torch
    import megastation_b200 as mb
    from megastation_b200 import datagen, learned
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    if shape == "256x32":
        cfg = datagen.CellConfig(M=256, K=32, N=4096, S=3276, sg=16, Qm=6, U=12, snr_db=25.0, channel="tdl_ds",
                                 seed=4041)
        n_default, n_held = 305, 4  # x 3276 subcarriers ~ 1e6 samples
    else:
        cfg = datagen.CellConfig(M=128, K=16, N=2048, S=1200, sg=16, Qm=4, U=13, snr_db=25.0, channel="tdl_ds",
                                 seed=4040)
        n_default, n_held = 834, 16  # x 1200 subcarriers ~ 1e6 samples
    lz = learned.LearnedZF(cfg.M, cfg.K, cfg.S, cfg.sg)
    net = learned.make_mlp(cfg.sg, seed=1)
    n_real = int(os.environ.get("MB_LEARNED_REALISATIONS", str(n_default)))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    parts = []
    for i0 in range(0, n_real, 32):  # pilot CSI in chunks (256 x 32: 54 MB per realisation)
        parts.append(learned.training_set(lz, learned.pilot_csi(cfg, min(32, n_real - i0), seed=7 + 1000 * i0)))
    data = tuple(torch.cat([p[k] for p in parts]) for k in range(4))
    del parts
    held = learned.training_set(lz, learned.pilot_csi(cfg, n_held, seed=8))
    torch.cuda.synchronize()
    t_data = time.perf_counter() - t0
    t0 = time.perf_counter()
    steps = int(os.environ.get("MB_LEARNED_STEPS", "3000"))
    hist = learned.train(net, data, steps=steps, batch=4096, lr=1e-3, seed=9, log_every=500)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    loss_learned, loss_coarse = learned.blend_loss(net, held)

    cb, zeros, stride = cfg.ldpc()
    n_valid = min(cfg.S * cfg.Qm, cb)
    pfft = mb.PilotFFT(cfg.start, cfg.N, cfg.S, cfg.M, cfg.K, cfg.sg)
    ufft = mb.UplinkFFT(cfg.start, cfg.N, cfg.S, cfg.M)
    bf = mb.Beamform(cfg.M, cfg.K, cfg.G)
    modes = [("group_zf", None, 0), ("exact", learned.EXACT, 0)] + \
        [(f"{n}_ns{i}", m, i) for n, m in (("learned", learned.LEARNED), ("coarse", learned.COARSE))
         for i in (0, 1, 2)]
    csi = torch.zeros(cfg.G, cfg.M, cfg.K, dtype=torch.complex64, device="cuda")
    y = torch.zeros(cfg.U, cfg.M, cfg.S, dtype=torch.complex64, device="cuda")
    W = torch.zeros(cfg.S, cfg.M, cfg.K, dtype=torch.complex64, device="cuda")
    llr = torch.zeros(cfg.U, cfg.K, stride, dtype=torch.float16, device="cuda")
    x = torch.zeros(cfg.U, cfg.K, cfg.S, dtype=torch.complex64, device="cuda")

    def slot_ops(iq, mode, init, ns, with_x):
        pfft(iq[:cfg.P], csi)
        ufft(iq[cfg.P:], y)
        if mode == "group_zf":
            Wg = csi
            bf.beamform_uplink(Wg, S=cfg.S, sc_group=cfg.sg)
            sg = cfg.sg
        else:
            Wg = lz.run(csi, init=init, ns_iters=ns, mlp=net, W=W)
            sg = 1
        mb.Equalize.equalize(Wg, y, llr, sg, cfg.Qm, cb, zeros, 1, x=x if with_x else None)

    quality = {}
    for ds in (50.0, 100.0, 150.0, 200.0, 250.0, 300.0):
        c = datagen.CellConfig(**{**cfg.__dict__, "delay_spread_ns": ds, "seed": cfg.seed + int(ds)})
        d = datagen.make_slot(c)
        iq = torch.from_numpy(d["iq"]).cuda()
        for name, init, ns in modes:
            slot_ops(iq, name, init, ns, True)
            torch.cuda.synchronize()
            xs = x.cpu().numpy()
            evm = 10 * np.log10(np.mean(np.abs(xs - d["x"]) ** 2) / np.mean(np.abs(d["x"]) ** 2))
            # uncoded BER: hard decisions (LLR < 0) descrambled, against the sent bits
            lr = llr.cpu().numpy().astype(np.float32)[..., zeros:zeros + n_valid]
            seq = np.broadcast_to(d["seq"], d["bits"].shape)[..., :n_valid]
            bits = (lr < 0).astype(np.uint8) ^ seq
            ber = float(np.mean(bits != d["bits"][..., :n_valid]))
            q = {"evm_db": float(evm), "ber": ber}
            if name not in ("group_zf", "exact") and ns > 0:
                # subcarriers whose start was too far off for Newton-Schulz
                # (the exact inverse taken instead)
                q["exact_fallback"] = float((lz.flags() == 2).float().mean())
            quality.setdefault(name, {})[f"{int(ds)}ns"] = q

    # throughput of each detector path, graph-replayed on device-resident slots
    R = 2
    iqs = [torch.from_numpy(datagen.make_slot(datagen.CellConfig(**{**cfg.__dict__, "delay_spread_ns": 200.0,
                                                                    "seed": 77 + r}))["iq"]).cuda()
           for r in range(R)]
    speed = {}
    stream = torch.cuda.Stream()
    for name, init, ns in (("group_zf", None, 0), ("exact", learned.EXACT, 0), ("learned_ns0", learned.LEARNED, 0),
                           ("learned_ns1", learned.LEARNED, 1), ("learned_ns2", learned.LEARNED, 2),
                           ("coarse_ns1", learned.COARSE, 1)):
        graphs = []
        with torch.cuda.stream(stream):
            for r in range(R):
                slot_ops(iqs[r], name, init, ns, False)
            stream.synchronize()
            for r in range(R):
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g, stream=stream):
                    slot_ops(iqs[r], name, init, ns, False)
                graphs.append(g)
            for k in range(5):
                graphs[k % R].replay()
        stream.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
            for k in range(args.steps):
                graphs[k % R].replay()
            e1.record(stream)
        e1.synchronize()
        speed[name] = {"slots_per_s": args.steps / (e0.elapsed_time(e1) / 1e3),
                       "us_per_slot": 1e3 * e0.elapsed_time(e1) / args.steps}
        del graphs
    mean = lambda n, k: float(np.mean([v[k] for v in quality[n].values()]))
    wl = ("256x32, N=4096, S=3276, 64-QAM, 25 dB, 8-tap TDL, delay spread 50-300 ns" if shape == "256x32"
          else "128x16, N=2048, S=1200, 16-QAM, 25 dB, 8-tap TDL, delay spread 50-300 ns")
    line = {"metric": "slots/s (per-subcarrier ZF, learned init + 1 Newton-Schulz step)",
            "value": speed["learned_ns1"]["slots_per_s"], "unit": "slots/s", "n_gpus": 1, "steps": args.steps,
            "warmup": 5, "ms_per_step": speed["learned_ns1"]["us_per_slot"] / 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 detector, bf16 MLP weights",
            "data": "synthetic (seeded, megastation_b200.datagen / learned.pilot_csi)",
            "config": {"workload": wl,
                       "mlp": "22 -> 256 -> 256 -> 4, ReLU, BF16 weights, FP32 accumulate",
                       "training_realisations": n_real, "training_samples": int(data[0].shape[0]),
                       "steps": steps, "batch": 4096},
            "training": {"data_s": t_data, "train_s": t_train, "loss_history": hist,
                         "heldout_blend_error": {"learned": loss_learned, "coarse": loss_coarse}},
            "quality": quality,
            "mean_evm_db": {n: mean(n, "evm_db") for n in quality},
            "mean_ber": {n: mean(n, "ber") for n in quality},
            "speed": speed}
    print(json.dumps(line), flush=True)


def measure_cells(args, steps=None, reps=10):
    """The batched uneven-cells workload: 32 seeded cells (antennas, users,
    subcarriers, QAM drawn per cell), one CUDA graph launch per slot, tile
    choices from the autotuner; value = batched slots (all 32 cells) per
    second, compared with the same cells launched one slot handle at a time."""
    import torch
    from megastation_b200 import cells, datagen, slot
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    cfgs = datagen.make_cells(n=32, seed=3)
    data = [datagen.make_slot(c) for c in cfgs]
    R = 2
    steps = args.steps if steps is None else steps
    iqs = [[torch.from_numpy(d["iq"]).cuda() for d in data] for _ in range(R)]
    stream = torch.cuda.Stream()
    cs = cells.Cells(cfgs, precision=args.precision)
    with torch.cuda.stream(stream):
        choice, tuned_us = cs.autotune(iqs[0], reps=reps, stream=stream)
        for k in range(max(args.warmup, 2 * R)):
            cs(iqs[k % R], stream=stream)
    stream.synchronize()
    clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    clocks.start()
    time.sleep(0.3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for k in range(steps):
        cs(iqs[k % R], stream=stream)
    e1.record(stream)
    e1.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    # the same cells as 32 separately graph-captured slot handles on one stream
    runs = [slot.UplinkSlot(c, precision=args.precision, sym_batch=max(c.U, 1), use_graph=True) for c in cfgs]
    with torch.cuda.stream(stream):
        for k in range(2 * R):
            for c, r in enumerate(runs):
                r(iqs[k % R][c], stream=stream)
    stream.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for k in range(steps):
        for c, r in enumerate(runs):
            r(iqs[k % R][c], stream=stream)
    f1.record(stream)
    f1.synchronize()
    ms_seq = f0.elapsed_time(f1)
    launches = sum(slot_launches(c, max(c.U, 1), args.precision == "mixed") for c in cfgs)
    line = {"metric": "batched slots/s (32 uneven cells)", "value": steps / (ms / 1e3),
            "unit": "slots/s", "n_gpus": 1, "steps": steps, "warmup": args.warmup,
            "ms_per_step": ms / steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": MIXED_DTYPE if args.precision == "mixed" else "f32",
            "data": "synthetic (seeded, megastation_b200.datagen.make_cells)",
            "config": {"workload": "32 uneven cells: M in {32,64,128}, K in {4,8,16,32}, S in {600,1200,3276} "
                                   "with N in {1024,2048,4096}, QAM {4,16,64}, i.i.d. Rayleigh, 15-25 dB, seed 3",
                       "cells": [[c.M, c.K, c.N, c.S, c.Qm] for c in cfgs],
                       "l2": f"{sum(d['iq'].nbytes for d in data) / 1e6:.0f} MB of samples per slot, {R} slots rotated"},
            "clocks": clk, "gpu_launches": launches * steps, "graph_launches_per_slot": 1,
            "autotune": {"us_per_slot_tuned": tuned_us, "choices": choice},
            "one_handle_per_cell": {"value": steps / (ms_seq / 1e3), "unit": "slots/s",
                                    "note": "32 graph launches per slot on one stream"}}
    return line


def run_cells(args):
    """Prints measure_cells's line (config 3 as a workload of its own)."""
    print(json.dumps(measure_cells(args)), flush=True)


def measure_ldpc(args, steps=20):
    """LDPC decode and encode of one slot's code blocks at the headline
    cell's sizing (config.cc:84-135: BG1, rate 1/3, S = 3276, 64-QAM -> Z =
    288, 46 parity rows; one block per (symbol, user): 12 x 32 = 384).  The
    library ships no TS 38.212 tables, so the graph is base graph 1's
    circulant pattern (the committed fixture recovered from the reference's
    encoder) with seeded shifts mod 288; the cost depends on the pattern
    and Z, not on the shift values.  LLRs: BPSK codewords through AWGN
    (sigma 0.6), 8 min-sum passes."""
    import numpy as np
    import torch

    import megastation_b200 as mb
    from megastation_b200 import datagen
    cfg = datagen.CellConfig(**{**workload_dict(args), "iq_dtype": args.iq})
    cb, zeros, stride = cfg.ldpc()
    Z, kb = zeros // 2, 22
    m = cb // Z - (kb - 2)
    pat = np.load(os.path.join(ROOT, "tests", "golden", "ldpc", "bg1_z16.npz"))["entries"]
    rng = np.random.default_rng(5)
    code = None
    while code is None:
        e = pat.copy()
        e[:, 2] = np.where(e[:, 1] >= kb + 4, 0, rng.integers(0, Z, len(e)))
        try:
            code = mb.Ldpc(e, kb, Z, m, max_batch=cfg.U * cfg.K)
        except mb._lib.MbError:
            code = None  # a singular core block: other shifts
    B = cfg.U * cfg.K
    info = torch.randint(0, 256, (B, code.info_bytes), dtype=torch.uint8, device="cuda")
    cw = code.encode(info)
    bits = np.unpackbits(cw.cpu().numpy(), axis=1)[:, :code.cw_bits].astype(np.float32)
    llr = np.zeros((B, stride), np.float16)
    y = (1.0 - 2.0 * bits) + 0.6 * rng.standard_normal(bits.shape).astype(np.float32)
    llr[:, zeros:zeros + cb] = (2.0 * y / 0.36).astype(np.float16)
    llr_d = torch.from_numpy(llr).cuda()
    out = torch.zeros(B, code.info_bytes, dtype=torch.uint8, device="cuda")

    def timed(fn):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        e1.synchronize()
        return e0.elapsed_time(e1) / steps

    dec_ms = timed(lambda: code.decode(llr_d, max_iter=8, out=out))
    enc_ms = timed(lambda: code.encode(info, out=cw))
    ok = int((out == info).all(dim=1).sum().item())
    return {"metric": "LDPC code blocks/s (decode, 8 passes)", "value": B / (dec_ms / 1e3),
            "unit": "code blocks/s", "ms_per_slot_decode": dec_ms, "ms_per_slot_encode": enc_ms,
            "encode_blocks_per_s": B / (enc_ms / 1e3), "code_blocks_per_slot": B,
            "decoded_correctly": ok, "steps": steps,
            "workload": f"BG1 pattern, Z = {Z}, {m} parity rows, {B} code blocks per slot, AWGN sigma 0.6"}


def run_ldpc(args):
    print(json.dumps(measure_ldpc(args, steps=max(args.steps, 3))), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.workload != "cell256x32":
        if rank == 0:
            {"cells32": run_cells, "full256x64": run_full, "learned128x16": run_learned,
             "learned256x32": lambda a: run_learned(a, "256x32"), "ldpc256x32": run_ldpc}[args.workload](args)
        return

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    import megastation_b200 as mb
    from megastation_b200 import datagen, slot
    cfg = datagen.CellConfig(**{**workload_dict(args), "iq_dtype": args.iq})
    d = datagen.make_slot(cfg)
    cb, zeros, stride = cfg.ldpc()
    n_valid = min(cfg.S * cfg.Qm, cb)
    hrow = (n_valid + 7) // 8

    R = rotation(cfg, args)
    iq_host = torch.from_numpy(d["iq"]).pin_memory()
    iq_dev = [iq_host.cuda() for _ in range(R)]
    stream = torch.cuda.Stream()
    net, init_info = None, None
    if args.precision == "mixed" and args.init == "learned":
        net, init_info = train_zf_init(args)
    run = slot.UplinkSlot(cfg, precision=args.precision, sym_batch=args.sym_batch, use_graph=True,
                          ns_iters=args.ns_iters)
    if net is not None:
        run.set_zf_init(net)
    llr = [torch.zeros(cfg.U, cfg.K, stride, dtype=torch.float16, device="cuda") for _ in range(2)]
    hard = [torch.zeros(cfg.U, cfg.K, hrow, dtype=torch.uint8, device="cuda") for _ in range(2)]

    def step(k, s=stream):
        run(iq_dev[k % R], llr[k % 2], hard[k % 2], stream=s)

    # graphs are per pointer set: capture every (input, output) combination
    with torch.cuda.stream(stream):
        for k in range(max(args.warmup, 2 * R)):
            step(k)
    stream.synchronize()
    if dist:
        dist.barrier()

    # ---- timed region: K slots, device-resident inputs, graph replay
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    # the sampler's start leaves the GPU idle for a moment: warm up again
    # right before the timed window
    with torch.cuda.stream(stream):
        for k in range(max(args.warmup, 2 * R)):
            step(k)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e0.record(stream)
    for k in range(args.steps):
        step(k)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms = max_over_ranks(e0.elapsed_time(e1), dist)
    value = job_value(world, args.steps, ms)
    # the same K-slot window repeated back to back for about a second (and at
    # least --windows times), each timed by its own events, so that the
    # headline window is seen against the spread of many; the clock samples
    # cover all of them
    repeat = repeat_windows(step, stream, args, ms, dist, world)
    clk = clocks.stop()
    # groups the last timed slot solved from the learned iterate (status 3)
    st_last = run.status.cpu().numpy()
    if init_info is not None:
        init_info["groups_from_learned_iterate"] = f"{int((st_last == 3).sum())} of {st_last.size}"
    exact = None
    if net is not None:
        ems_x = max_over_ranks(time_slots(slot, cfg, "mixed", args.sym_batch, iq_dev, llr, hard, stream,
                                          args.steps, args.warmup, dist), dist)
        exact = {"value": job_value(world, args.steps, ems_x), "unit": UNIT, "us_per_slot": 1e3 * ems_x / args.steps,
                 "note": "the same mixed slot with the exact (Gauss-Jordan) initial iterate"}
    plain = None
    if args.precision == "mixed" and not args.no_plain:
        pms = time_slots(slot, cfg, "fp32", args.sym_batch, iq_dev, llr, hard, stream, args.steps,
                         args.warmup, dist)
        pms = max_over_ranks(pms, dist)
        pv = job_value(world, args.steps, pms)
        plain = {"value": pv, "unit": UNIT, "us_per_slot": 1e3 * pms / args.steps,
                 "speedup_mixed_over_plain": value / pv}
    evm = None if args.no_evm or rank != 0 else evm_report(cfg, d, args.sym_batch, args.ns_iters, net=net)
    hb = None if args.no_evm or rank != 0 else hard_bits_report(cfg, d, args.sym_batch, args.ns_iters, net=net)
    inflight = None if args.no_inflight else time_in_flight(slot, cfg, args, iq_dev, stride, hrow, dist, net=net)
    launches_per_slot = slot_launches(cfg, args.sym_batch, args.precision == "mixed")

    # ---- roofline pass: the same slots with every kernel alone on the slot
    # stream (timing mode serialises the side-stream FFT) and CUDA events at
    # the stage boundaries
    run_t = slot.UplinkSlot(cfg, precision=args.precision, sym_batch=args.sym_batch, use_graph=False)
    if net is not None:
        run_t.set_zf_init(net)
    with torch.cuda.stream(stream):
        for k in range(3):
            run_t(iq_dev[k % R], llr[0], hard[0], stream=stream)
        stream.synchronize()
        run_t.timing(args.steps)
        for k in range(args.steps):
            run_t(iq_dev[k % R], llr[k % 2], hard[k % 2], stream=stream)
    stream.synchronize()
    roof = roofline(cfg, args, run_t.stage_ms(), n_valid, hrow)
    slot_bytes = algorithmic_bytes(cfg)
    hbm_peak = measured_peaks()[0]
    roof["slot"] = {"bytes": slot_bytes, "GB_s": slot_bytes * value / world / 1e9,
                    "frac_of_hbm": slot_bytes * value / world / 1e9 / hbm_peak}

    # ---- e2e: the public slot pipeline (mb_pipe_*) from host buffers: H2D of
    # each slot's samples, the slot, D2H of its LLRs and hard bits, timed on
    # the device by the pipeline's own events
    e2e = None
    if not args.no_e2e:
        pipe = slot.SlotPipeline(cfg, precision=args.precision, sym_batch=args.sym_batch, depth=2,
                                 ns_iters=args.ns_iters)
        if net is not None:
            pipe.set_zf_init(net)
        outs = [pipe.host_outputs() for _ in range(2)]
        for k in range(4):
            t = pipe.submit(iq_host, *outs[k % 2])
        pipe.wait(t)
        if dist:
            dist.barrier()
        pipe.timer_start()
        for k in range(args.steps):
            t = pipe.submit(iq_host, *outs[k % 2])
        pipe.wait(t)
        ems = max_over_ranks(pipe.timer_ms(), dist)
        e2e = {"value": job_value(world, args.steps, ems), "unit": UNIT,
               "h2d_bytes_per_step": pipe.iq_bytes, "d2h_bytes_per_step": pipe.llr_bytes + pipe.hard_bytes,
               "pipeline": "mb_pipe (depth 2): H2D of slot k+1 and D2H of slot k-1 overlap slot k"}
        del pipe

    # short runs of the other measured workloads, so that their numbers come
    # with every default run: the full uplink + downlink slot (256 x 64,
    # 200 consecutive slots, latency percentiles), the 32 uneven cells
    # (autotuned, 50 batched slots) and the LDPC codec on one slot's code
    # blocks; their own --workload lines go further
    configs = None
    if rank == 0 and world == 1 and not args.no_configs:
        f = measure_full(args, n_min=200)
        c = measure_cells(args, steps=50, reps=5)
        lp = measure_ldpc(args)
        configs = {
            "full256x64": {**{k: f[k] for k in ("metric", "value", "unit", "ms_per_step", "latency_us",
                                                   "uplink_evm_db", "downlink", "gpu_launches")},
                           "workload": f["config"]["workload"], "slots": f["steps"]},
            "cells32": {**{k: c[k] for k in ("metric", "value", "unit", "ms_per_step", "autotune",
                                                "one_handle_per_cell", "gpu_launches")},
                        "workload": c["config"]["workload"], "steps": c["steps"]},
            "ldpc256x32": lp}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(cfg, d, args.cpu_seconds)

    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "us_per_slot": 1e3 * ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": MIXED_DTYPE if args.precision == "mixed" else "f32",
            "data": "synthetic (seeded generator, megastation_b200.datagen)",
            "config": workload_config(cfg, args), "clocks": clk, "e2e": e2e,
            "gpu_launches": launches_per_slot * args.steps, "roofline": roof, "cpu_baseline": cpu,
            "plain_fp32": plain, "mixed_exact_init": exact, "zf_init": init_info, "evm_db": evm,
            "hard_bits_vs_plain": hb, "repeat": repeat, "other_workloads": configs,
            "in_flight": inflight,
            "parallelism": f"replicas x{world}"}
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
