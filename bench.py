"""Benchmark: BigWhoop compression hot path on B200 (bwc_compress / bwc_decompress).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--dtype f64|f32] [--size 512]

Workload: the single-large-field configuration -- a 512^3 field (FP64 by default, FP32 with
--dtype f32) from the spectral generator with 8 tanh shock fronts and a constant quarter,
4 CDF 9/7 decomposition levels, codeblocks 32x32x16, quality layers 0.5, 1, 2 and 4 bits per
value.  One step compresses the field (and, for the decompression figure, decompresses the
codestream).  Synthetic data (no public data set exists for this codec); the 1 GiB FP64 input
exceeds the 126 MB L2, so no flush is needed between steps.

value = input GB/s of bwc_compress with the field already in HBM (device pointers in and out);
e2e   = the same call with pinned host buffers (host->device upload and codestream download
        inside the timed region).
Under torchrun every rank compresses its own field (independent replicas, weak scaling); the
time is the maximum over ranks.

--impl reference times the reference's own CPU library (compiled from its sources into
oracle/_ref) with all host threads on the same field and settings, rank 0 only.

cpu_baseline (ours) = the same reference library on the same full field with all host threads
(plus one thread on the central 128^3 cube); its codestream and decompressed field are compared
with this library's byte for byte and bit for bit ("parity_vs_reference").
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "compress/decompress input GB/s at 2 bpv, byte-exact; batched+warm-start vs plain"
RATES = "0.5,1,2,4"
DECOMP = (4, 4, 4, 0)
CODEBLOCKS = (5, 5, 4, 0)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--dtype", default="f64", choices=["f64", "f32"])
    ap.add_argument("--size", type=int, default=512)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true",
                    help="skip the batched-vs-plain comparison on the 64-field uneven batch")
    ap.add_argument("--config", default="single", choices=["single", "combined4d"],
                    help="combined4d: the 384^3 x 8 FP64 advected time series instead")
    return ap.parse_args()


def workload_name(a):
    return (f"single large field: {a.size}^3 {'FP64' if a.dtype == 'f64' else 'FP32'} spectral "
            f"field + 8 tanh shocks + constant quarter, seed 1, 4 levels, cb 32x32x16, layers "
            f"{RATES} bpv")


class ClockSampler:
    """nvidia-smi clock/throttle samples while the timed region runs."""

    def __init__(self, index=0):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}", "--format=csv,noheader",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1].split()[0]))
                mx = float(p[2].split()[0])
            except ValueError:
                continue
            for name, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": ["unsampled"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def make_field(a, device):
    from bigwhoop_b200 import fields
    dt = np.float64 if a.dtype == "f64" else np.float32
    n = a.size
    return fields.shock_field((n, n, n), 1, dtype=dt, device=device)


def dist_setup(a):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(ws, v):
    if ws == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sample_window(n, frac=2):
    """Central (n/frac)^3 cube: it overlaps the constant quarter in the same 1/4 proportion as
    the whole field and crosses the shock fronts like it."""
    s = max(1, n // frac)
    o = (n - s) // 2
    return slice(o, o + s), s


def ref_compress_timed(field_np, prec, threads, rates=RATES, decomp=DECOMP, cb=CODEBLOCKS):
    """One reference bwc_compress (set-up excluded from the time), gain table reset first."""
    from oracle import ref
    ref.set_threads(threads, prec)
    ref.reset_gain_lut(prec)
    rc = ref.RefCompressor(field_np, precision=prec, decomp=decomp, cb=cb, rate=rates)
    try:
        t0 = time.perf_counter()
        cs = rc.compress()
        dt = time.perf_counter() - t0
    finally:
        rc.close()
    return cs, dt


def cpu_baseline(field_np, a, threads=None):
    """The reference CPU library on the same full field and settings with all host threads
    (compress and decompress timed), and with one thread on the central 128^3 cube.  Returns the
    baseline object plus the reference's codestream and decompressed field for the parity
    check."""
    from oracle import ref
    prec = "double" if a.dtype == "f64" else "single"
    threads = threads or os.cpu_count()
    cs, dt = ref_compress_timed(field_np, prec, threads)
    ref.set_threads(threads, prec)
    t0 = time.perf_counter()
    dec = ref.decompress(cs, field_np.shape, field_np.dtype, prec)
    ddt = time.perf_counter() - t0
    w, s1 = sample_window(a.size, 4)
    sub = np.ascontiguousarray(field_np[w, w, w])
    _, dt1 = ref_compress_timed(sub, prec, 1)
    ref.set_threads(threads, prec)
    base = {"value": field_np.nbytes / dt / 1e9, "unit": "GB/s", "cores": threads,
            "kind": "reference",
            "sample": f"the full field ({field_np.nbytes / 2**20:.0f} MiB), same settings, one "
                      f"bwc_compress and one bwc_decompress, {threads} OpenMP threads",
            "decompress_GBps": field_np.nbytes / ddt / 1e9,
            "single_thread": {"value": sub.nbytes / dt1 / 1e9, "unit": "GB/s", "cores": 1,
                              "sample": f"central {s1}^3 cube of the field, same settings"}}
    return base, cs, dec


def run_reference(a):
    """The reference's own CPU library (oracle/_ref, all host threads) on the same field and
    settings as this library's arm: W untimed and K timed bwc_compress calls, rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    prec = "double" if a.dtype == "f64" else "single"
    try:
        import torch
        gpu = torch.cuda.is_available()
    except Exception:
        gpu = False
    if gpu:
        # the same field as the GPU arm, generated on the device, moved to the host
        field = make_field(a, "cuda").cpu().numpy()
        torch.cuda.empty_cache()
        sample = "the full field"
    else:
        # no GPU to evaluate the full-size generator quickly: the central cube of the field
        from bigwhoop_b200 import fields
        w, s = sample_window(a.size)
        dt = np.float64 if a.dtype == "f64" else np.float32
        field = fields.shock_field((s, s, s), 1, dtype=dt)
        sample = f"a {s}^3 field of the same generator (no GPU to generate the full field)"
    field = np.ascontiguousarray(field)
    threads = os.cpu_count()
    times = []
    for i in range(a.warmup + a.steps):
        _, t = ref_compress_timed(field, prec, threads)
        if i >= a.warmup:
            times.append(t)
    tt = float(np.mean(times))
    v = field.nbytes / tt / 1e9
    line = {"metric": METRIC, "value": v, "unit": "GB/s", "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": tt * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if a.dtype == "f64" else "f32",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": workload_name(a), "codec_precision": prec,
                       "rates_bpv": RATES},
            "cpu_baseline": {"value": v, "unit": "GB/s", "cores": threads, "kind": "reference",
                             "sample": f"{sample}, same settings, one bwc_compress per step, "
                                       f"{threads} OpenMP threads"},
            "e2e": {"value": v, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(a):
    import torch
    ws, rank, local = dist_setup(a)
    from bigwhoop_b200 import bwc, ratemodel
    prec = "double" if a.dtype == "f64" else "single"
    # FP64 fields are coded by the double build (the reference's default); FP32 by the single
    field = make_field(a, "cuda").contiguous()
    nbytes = field.numel() * field.element_size()
    dev_out = torch.empty(nbytes + (1 << 20), dtype=torch.uint8, device="cuda")
    host_in = field.cpu().pin_memory()
    host_out = torch.empty(nbytes + (1 << 20), dtype=torch.uint8).pin_memory()
    shape = tuple(field.shape)
    npdt = np.float64 if a.dtype == "f64" else np.float32

    def one(device_resident=True):
        # codestreams depend on the process-wide energy-gain history (every codec setup adds to
        # it, as in the reference); start each step from the same state
        bwc.reset_gain_state(prec)
        if device_resident:
            c = bwc.Compressor(precision=prec, rate=RATES, decomp=DECOMP, codeblocks=CODEBLOCKS,
                               device_ptr=(field.data_ptr(), shape, npdt), out=dev_out.data_ptr())
        else:
            c = bwc.Compressor(precision=prec, rate=RATES, decomp=DECOMP, codeblocks=CODEBLOCKS,
                               device_ptr=(host_in.data_ptr(), shape, npdt),
                               out=host_out.data_ptr())
        torch.cuda.synchronize()
        barrier(ws)
        # bwc_compress returns when the codestream is complete (its own stream synchronised);
        # events on the current stream bracket the call on the device clock
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        n = c.L.bwc_compress(c.codec, c.stream)
        ev1.record()
        torch.cuda.synchronize()
        dt = ev0.elapsed_time(ev1) * 1e-3
        tm = c.timings()
        rc = np.array([ratemodel.stats(c, l) for l in range(len(RATES.split(",")))])
        c.close()
        if n == 0:
            raise RuntimeError("bwc_compress failed")
        one.rate_stats = rc
        return dt, int(n), tm

    for _ in range(a.warmup):
        one(True)
    times, stage = [], []
    with ClockSampler(local) as clocks:
        for _ in range(a.steps):
            dt, ncs, tm = one(True)
            times.append(max_over_ranks(ws, dt))
            stage.append(tm)
    # the host-buffer path gets its own warm-up steps (its first calls set up page-locked paths)
    for _ in range(a.warmup):
        one(False)
    e2e_times, e2e_stage = [], []
    for _ in range(max(1, a.steps)):
        dt, ncs_h, tm_h = one(False)
        e2e_times.append(max_over_ranks(ws, dt))
        e2e_stage.append(tm_h)
    rate_warm = one.rate_stats
    # the same compression with the plain bisection (warm start off), for its tier-2 time
    ratemodel.set_model(None, prec)
    _, ncs_plain, tm_plain = one(True)
    rate_plain = one.rate_stats
    cs_plain = bytes(dev_out[:ncs_plain].cpu().numpy())
    ratemodel.load_default(prec)
    t = float(np.mean(times))
    te = float(np.mean(e2e_times))
    stage = np.mean(np.array(stage), axis=0)
    cs = bytes(host_out[:ncs_h].numpy())
    cs_dev = bytes(dev_out[:ncs].cpu().numpy())

    # decompression (e2e: codestream from host, field back to host)
    dec_out = torch.empty(shape, dtype=field.dtype).pin_memory()
    dtimes = []
    for i in range(a.warmup + a.steps):
        d = bwc.Decompressor(cs, precision=prec, out=dec_out.data_ptr())
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        d.decompress()
        ev1.record()
        torch.cuda.synchronize()
        dtimes.append(ev0.elapsed_time(ev1) * 1e-3)
        dstage = d.timings()
        d.close()
    tdec = float(np.mean(dtimes[a.warmup:]))
    rec = dec_out.numpy().astype(np.float64)
    orig = host_in.numpy().astype(np.float64)
    err = np.abs(rec - orig)
    mse = float(np.mean(err ** 2))
    rng = float(orig.max() - orig.min())
    psnr = 20 * np.log10(rng / (2 * np.sqrt(mse))) if mse > 0 else float("inf")

    # kernels per compression: fill+min/max, normalise, one fused DWT pass per level and the
    # region copies between the ping-pong buffers (before every even level but the first, and
    # after an even number of levels), tier-1 context modelling + MQ coding (per phase),
    # codestream gather
    L = DECOMP[0]
    # (tier-1: one modelling and one MQ launch per phase, stage[11] phases)
    launches = (2 + L + len(range(2, L, 2)) + (1 if L % 2 == 0 else 0)
                + 2 * max(1, int(stage[11]) if len(stage) > 11 else 1) + 1)
    line = None
    if rank == 0:
        total_bytes = nbytes * ws
        value = total_bytes / t / 1e9
        e2e = total_bytes / te / 1e9
        peaks = {}
        pk = os.path.join(HERE, "MEASURED_PEAKS.json")
        if os.path.exists(pk):
            peaks = json.load(open(pk))
        hbm = peaks.get("hbm_gbs", 6650.0)
        clk = clocks.summary()
        sm_hz = (clk.get("sm_mhz") or peaks.get("sm_max_mhz") or 1965.0) * 1e6
        t1_ms = float(stage[3])
        s_bytes = 8 if prec == "double" else 4
        n_vals = field.numel()
        dwt_ms = float(stage[2])
        # DWT algorithmic bytes: one read + one write of each level's region, all axes fused
        alg_dwt = sum(2 * s_bytes * n_vals / 8 ** l for l in range(4))
        t1 = tier1_roofline(stage, dstage, sm_hz, prec)
        line = {
            "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": ws, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": a.dtype, "data": "synthetic",
            "config": {"workload": workload_name(a), "codec_precision": prec,
                       "rates_bpv": RATES, "l2": "input 1 GiB > L2 (no flush needed)"
                       if nbytes > 126e6 else "input smaller than L2"},
            "e2e": {"value": e2e, "unit": "GB/s", "h2d_bytes_per_step": nbytes,
                    "d2h_bytes_per_step": len(cs),
                    "step_ms": [round(x * 1e3, 1) for x in e2e_times],
                    "stages_ms": [round(float(x), 3) for x in np.mean(np.array(e2e_stage), axis=0)[:8]]},
            "decompress": {"value": nbytes / tdec / 1e9, "unit": "GB/s", "kind": "e2e",
                           "stages_ms": [round(float(x), 3) for x in dstage]},
            "stages_ms": {"upload": round(float(stage[0]), 3),
                          "fill_normalise": round(float(stage[1]), 3),
                          "dwt": round(dwt_ms, 3), "tier1": round(t1_ms, 3),
                          "tier1_download": round(float(stage[4]), 3),
                          "tier2_host": round(float(stage[5]), 3),
                          "assembly": round(float(stage[6]), 3)},
            "roofline": t1["roofline"],
            "tier1_kernels": t1["kernels"],
            "roofline_dwt": {"bound": "hbm", "achieved": alg_dwt / (dwt_ms * 1e-3) / 1e9,
                             "peak": hbm, "unit": "GB/s",
                             "frac": alg_dwt / (dwt_ms * 1e-3) / 1e9 / hbm},
            "quality": {"psnr_db": psnr, "max_abs_err": float(err.max()),
                        "codestream_bytes": len(cs), "bpv": len(cs) * 8 / field.numel(),
                        "device_and_host_codestreams_equal": cs == cs_dev},
            "clocks": clk,
            # plus the rate model's forward pass (one launch for all layers) when it predicted
            "gpu_launches": launches + (1 if (rate_warm[:, 3] >= 0).any() else 0),
            "rate_control": {
                "warm_start": "built-in model (bigwhoop_b200/data/pcrd_mlp.npy)",
                "dependent_probe_rounds_per_layer": [int(v) for v in rate_warm[:, 2]],
                "plain_bisection_probes_per_layer": [int(v) for v in rate_plain[:, 1]],
                "tier2_host_ms_warm": round(float(stage[5]), 3),
                "tier2_host_ms_plain": round(float(tm_plain[5]), 3),
                "codestreams_equal": cs_plain == cs_dev},
        }
        if not a.no_batch and ws == 1:
            line["batch"] = batch_compare(prec)
        if not a.no_cpu_baseline and ws == 1:
            base, cs_ref, dec_ref = cpu_baseline(host_in.numpy(), a)
            line["cpu_baseline"] = base
            rec_np = dec_out.numpy()
            line["parity_vs_reference"] = {
                "codestream_identical": cs_ref == cs_dev,
                "codestream_bytes": [len(cs_dev), len(cs_ref)],
                "decompression_bit_identical": bool(np.array_equal(
                    rec_np.view(np.uint64 if rec_np.dtype == np.float64 else np.uint32),
                    dec_ref.view(np.uint64 if dec_ref.dtype == np.float64 else np.uint32))),
                "what": "this library's codestream of the full field (device-resident call) "
                        "against the reference library's, and its decompression of that "
                        "codestream against the reference's decompression"}
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


# Warp instructions issued by each tier-1 kernel at this workload (512^3 FP64, 8192 codeblocks,
# the MQ coder at 16 codeblocks per warp), from the ncu capture named beside it: per coded
# symbol for the encoder's kernels (smsp__inst_executed.sum over the capture's symbol count),
# and the decoder's total for one decompression of the workload's codestream.  The live part of
# the roofline is the symbol count and each kernel's CUDA-event time in this run.
T1_WARP_INSTR = {
    "t1_model_kernel": (2.673, "profiles/t1_kernels_512cube_f64.md"),
    "t1_mq_kernel": (6.010, "profiles/t1_kernels_512cube_f64.md"),
    "t1_decode_kernel": (104.38e9, "profiles/t1_kernels_512cube_f64.md"),
}
SMS = 148


def tier1_roofline(stage, dstage, sm_hz, prec):
    """Tier-1 against its bound, integer instruction issue: symbols per second per kernel and the
    fraction of the GPU's warp-instruction issue slots (148 SMs x 4 schedulers x SM clock) the
    kernel's instructions fill over its measured time.  The MQ coder runs as several launches
    on side streams (one per modelling phase); its figure is per launch: the instructions of
    all launches over the sum of their device times (CUDA events on their own streams)."""
    sym = float(stage[8]) * 1e6 if len(stage) > 8 else 0.0
    model_ms = float(stage[9]) if len(stage) > 9 else 0.0
    mq_ms = float(stage[10]) if len(stage) > 10 else 0.0
    mq_n = int(stage[11]) if len(stage) > 11 else 0
    t1_ms = float(stage[3])
    peak = SMS * 4 * sm_hz
    kernels = {}
    for name, ms, launches in (("t1_model_kernel", model_ms, None),
                               ("t1_mq_kernel", mq_ms, mq_n)):
        ipsym, src = T1_WARP_INSTR[name]
        if ms <= 0 or sym <= 0:
            continue
        k = {"ms": round(ms, 3), "symbols": sym, "Gsymbols_per_s": sym / (ms * 1e-3) / 1e9,
             "warp_instr_per_symbol": ipsym, "instr_source": src,
             "issue_frac": ipsym * sym / (ms * 1e-3) / peak if ipsym else None}
        if launches:
            k["launches"] = launches
            k["ms_per_launch"] = round(ms / launches, 3)
            k["ms"] = round(ms, 3)
            k["timing"] = "sum of the launches' device times; the launches overlap in time"
        else:
            k["timing"] = ("tier-1 start to the end of the last modelling launch (the MQ "
                           "launches of earlier phases run beside it)")
        kernels[name] = k
    dec_ms = float(dstage[3]) if len(dstage) > 3 else 0.0
    dinstr, dsrc = T1_WARP_INSTR["t1_decode_kernel"]
    if dec_ms > 0:
        kernels["t1_decode_kernel"] = {"ms": round(dec_ms, 3), "warp_instr": dinstr,
                                       "instr_source": dsrc,
                                       "issue_frac": dinstr / (dec_ms * 1e-3) / peak
                                       if dinstr else None}
    kernels["tier1_stage"] = {"ms": round(t1_ms, 3), "Gsymbols_per_s":
                              sym / (t1_ms * 1e-3) / 1e9 if t1_ms > 0 else None}
    if "t1_mq_kernel" not in kernels or not kernels["t1_mq_kernel"]["warp_instr_per_symbol"]:
        roof = {"bound": "int_issue", "achieved": None, "peak": peak / 1e12,
                "unit": "Twarp-instr/s", "frac": None, "traffic": None}
    else:
        k = kernels["t1_mq_kernel"]
        ach = k["warp_instr_per_symbol"] * sym / (mq_ms * 1e-3)
        roof = {"bound": "int_issue", "kernel": "t1_mq_kernel", "achieved": ach / 1e12,
                "peak": peak / 1e12, "unit": "Twarp-instr/s", "frac": ach / peak,
                "traffic": None, "symbols_per_s_per_launch": sym / (mq_ms * 1e-3),
                "note": "tier-1 has no HBM or tensor bound: the MQ coder is one dependent chain "
                        "per codeblock, so its launches last as long as their longest chains and "
                        "fill few issue slots; the denominator is the GPU's warp-instruction "
                        "issue rate at the sampled SM clock, the numerator the kernel's "
                        "ncu-counted instructions per symbol times the symbols coded per second "
                        "of launch time in this run",
                "peak_source": "148 SMs x 4 issue slots x sampled SM clock"}
    return {"roofline": roof, "kernels": kernels}


def batch_compare(prec):
    """The uneven batch: 64 fields (seed 2, extents U[33, 300], FP32/FP64, rates 0.25-4 bpv,
    2-4 levels, 32x32x16 codeblocks) from host memory, compressed by 64 plain bwc_compress calls
    (plain bisection) and by one bwc_b200_compress_batch (warm start on), both end to end."""
    import torch
    from bigwhoop_b200 import bwc, fields, ratemodel
    desc = fields.uneven_batch(seed=2, n_fields=64)
    fs = []
    for d in desc:
        f = fields.shock_field(d["shape"], d["seed"], dtype=d["dtype"], slope=d["slope"], device="cuda")
        fs.append(f.cpu().numpy())
    torch.cuda.synchronize()
    total = sum(f.nbytes for f in fs)

    def comp(f, d):
        lv = d["levels"]
        return bwc.Compressor(f, precision=prec, decomp=(lv, lv, lv, 0), codeblocks=(5, 5, 4, 0),
                              rate=str(d["rate"]))

    def plain():
        ratemodel.set_model(None, prec)
        bwc.reset_gain_state(prec)
        out = []
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        ev0.record()
        for f, d in zip(fs, desc):
            c = comp(f, d)
            try:
                out.append(c.compress())
            finally:
                c.close()
        ev1.record()
        torch.cuda.synchronize()
        dt = ev0.elapsed_time(ev1) * 1e-3
        ratemodel.load_default(prec)
        return dt, out

    def batched():
        bwc.reset_gain_state(prec)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        ev0.record()
        comps = [comp(f, d) for f, d in zip(fs, desc)]
        try:
            out = bwc.compress_batch(comps)
        finally:
            for c in comps:
                c.close()
        ev1.record()
        torch.cuda.synchronize()
        return ev0.elapsed_time(ev1) * 1e-3, out

    # warm-ups: both paths meet their launch sizes once (the MQ autotuner times each new
    # codeblock-count class on first use) before they are timed
    batched()
    plain()
    tb, outb = min((batched() for _ in range(2)), key=lambda r: r[0])
    tp, outp = plain()
    tim = bwc.batch_timings(prec)
    return {"workload": "uneven batch: 64 fields, seed 2, extents U[33,300], FP32/FP64, rates "
                        "{0.25..4} bpv, 2-4 levels, cb 32x32x16 (codec precision %s)" % prec,
            "input_bytes": total, "timing": "CUDA events around codec set-up and compression of "
            "all 64 fields (each call returns with its codestream); inputs and codestreams in "
            "host memory",
            "batched_warm_GBps": total / tb / 1e9, "plain_per_field_GBps": total / tp / 1e9,
            "speedup": tp / tb, "codestreams_equal": outb == outp,
            "batched_stages_ms": {"setup_uploads": round(float(tim[0]), 1),
                                  "transform": round(float(tim[1]), 1),
                                  "tier1": round(float(tim[2]), 1),
                                  "tier2_host": round(float(tim[3]), 1),
                                  "gather_outputs": round(float(tim[4]), 1)}}


def run_combined4d(a):
    """The combined large 4D workload: a 384^3 x 8 FP64 spectral field advected by 1.5 cells per
    step with fresh noise (seed 3), 3 spatial and 2 temporal decomposition levels, codeblocks
    32x32x8x2, 6 quality layers 0.25 ... 8 bpv.  Compressed from host memory through the batched
    path with the warm start and through the plain bwc_compress call without it (same bytes),
    then decompressed in full; PSNR and max-abs error against the original.  The reference CPU
    library runs on a bounded sample (the first 2 time steps of a central 192^3 window)."""
    import torch
    from bigwhoop_b200 import bwc, fields, ratemodel
    from oracle import ref
    rates = "0.25,0.5,1,2,4,8"
    kw = dict(precision="double", decomp=(3, 3, 3, 2), codeblocks=(5, 5, 3, 1), rate=rates)
    f = fields.advected_field((8, 384, 384, 384), 3, device="cuda")
    host = f.cpu().pin_memory()
    del f
    torch.cuda.empty_cache()
    arr = host.numpy()
    nbytes = arr.nbytes
    out = torch.empty(nbytes + (1 << 20), dtype=torch.uint8).pin_memory()

    def timed(fn):
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        ev0.record()
        r = fn()
        ev1.record()
        torch.cuda.synchronize()
        return ev0.elapsed_time(ev1) * 1e-3, r

    def batched():
        bwc.reset_gain_state()
        c = bwc.Compressor(arr, out=out.numpy(), **kw)
        try:
            cs = bwc.compress_batch([c])[0]   # bytes: the output buffer is host memory
            st = [ratemodel.stats(c, l) for l in range(6)]
        finally:
            c.close()
        return cs, st

    def plain():
        ratemodel.set_model(None)
        bwc.reset_gain_state()
        c = bwc.Compressor(arr, out=out.numpy(), **kw)
        try:
            cs = c.compress()
            st = [ratemodel.stats(c, l) for l in range(6)]
        finally:
            c.close()
            ratemodel.load_default()
        return cs, st

    timed(batched)   # warm-up
    tb, (cs_b, st_b) = timed(batched)
    tp, (cs_p, st_p) = timed(plain)
    dec = torch.empty(arr.shape, dtype=torch.float64).pin_memory()

    def decompress():
        d = bwc.Decompressor(cs_b, out=dec.data_ptr())
        try:
            d.decompress()
        finally:
            d.close()

    td, _ = timed(decompress)
    err = np.abs(dec.numpy() - arr)
    mse = float(np.mean(err ** 2))
    rng_ = float(arr.max() - arr.min())
    # reference CPU library on a bounded sample
    sub = np.ascontiguousarray(arr[:2, 96:288, 96:288, 96:288])
    threads = os.cpu_count()
    ref.set_threads(threads)
    ref.reset_gain_lut()
    rc = ref.RefCompressor(sub, decomp=(3, 3, 3, 1), cb=(5, 5, 3, 1), rate=rates)
    t0 = time.perf_counter()
    rc.compress()
    tr = time.perf_counter() - t0
    rc.close()
    line = {"metric": METRIC, "value": nbytes / tb / 1e9, "unit": "GB/s", "n_gpus": 1,
            "steps": 1, "warmup": 1, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "combined 4D: 384^3 x 8 FP64 advected spectral field (1.5 "
                                   "cells/step, noise 1e-5, seed 3), decomp 3 spatial + 2 "
                                   "temporal, cb 32x32x8x2, layers " + rates + " bpv",
                       "input_bytes": nbytes},
            "e2e": {"value": nbytes / tb / 1e9, "unit": "GB/s", "h2d_bytes_per_step": nbytes,
                    "d2h_bytes_per_step": len(cs_b)},
            "path": "bwc_b200_compress_batch with the warm start, host buffers",
            "plain_path_GBps": nbytes / tp / 1e9, "codestreams_equal": cs_b == cs_p,
            "decompress_GBps": nbytes / td / 1e9,
            "quality": {"psnr_db": 20 * np.log10(rng_ / (2 * np.sqrt(mse))) if mse > 0 else None,
                        "max_abs_err": float(err.max()), "codestream_bytes": len(cs_b),
                        "bpv": len(cs_b) * 8 / arr.size},
            "rate_control": {"rounds_per_layer_warm": [int(v[2]) for v in st_b],
                             "probes_per_layer_plain": [int(v[1]) for v in st_p]},
            "cpu_baseline": {"value": sub.nbytes / tr / 1e9, "unit": "GB/s", "cores": threads,
                             "kind": "reference",
                             "sample": "time steps 0-1 of the central 192^3 window (113 MiB), "
                                       "temporal decomposition 1 level (2 steps), same other "
                                       "settings"}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    a = parse()
    if a.impl == "reference":
        return run_reference(a)
    if a.config == "combined4d":
        return run_combined4d(a)
    return run_ours(a)


if __name__ == "__main__":
    sys.exit(main())
