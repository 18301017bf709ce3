#!/usr/bin/env python
"""DM-trial x Msamples/s of batched MS-OSM coherent dedispersion + folding.

Workload (one step): 16 MHz complex baseband centred at 1250 MHz (lower edge
1242 MHz), 2^26 complex64 samples carrying an injected pulsar (DM 73.2,
P = 3.1 ms, Gaussian pulse of 3% duty cycle, peak per-sample SNR 0.05, seeded
synthetic data), dedispersed at 256 DM trials uniform over 0-100 pc/cm^3 with
FFT 4096 (MS-OSM, per-bin block delays), |y|^2 detection and folding into
1024 phase bins per trial, all through libmsosm_b200.so.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference|reference-gpu]
                    [--precision fp16|bf16|fp32]
    python bench.py --workload precision-sweep [--seeds 8]

The headline arm (default --precision fp16) runs the inverse transforms on
the tensor cores (tcgen05 f16 GEMMs, f32 accumulation); the plain fused FP32
kernel is timed beside it on the same workload (`fp32_path`), and both
paths' errors against the FP64 oracle are measured on a sample of the
workload (`accuracy_vs_fp64`, in the CPU-baseline leg).

`value`: device time (CUDA events) with the input resident in HBM.  `e2e`:
the same metric through the C ABI with pinned HOST input, the host->device
copy of every step and the device->host read of the folded profiles inside
the timed region.  `--impl reference` times the reference's algorithm in
FP32 on all host cores (oracle/cpu_fp32.py: pocketfft standing in for FFTW,
threads over trials) on a bounded sample; `--impl reference-gpu` times the
reference's own cuFFT classes built for sm_100a (oracle/_ref/ref_gpu_runner)
when present, and the default arm carries that measurement as
`reference_gpu` (run outside its timed region).

`--workload precision-sweep` (not the bench line): a 64 MHz band centred at
1400 MHz, 2^26 samples, 1024 trials over 0-200, FFT 8192, with an injected
pulsar (DM 150, P = 4.7 ms, 2% FWHM, peak SNR 0.05); per precision (FP32
CUDA-core, FP16 and BF16 tensor-core) the device throughput, and for each of
8 signal seeds the series and profile errors against the FP64 oracle on four
sampled trials over the whole signal and the injected pulsar's S/N loss.
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

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BW = 16e6
F0 = 1242e6  # lower band edge: centre 1250 MHz
LOG2_SAMPLES = 26
N_DM = 256
DM_MAX = 100.0
FFTPOINT = 4096
NBINS = 1024
PULSAR = dict(dm=73.2, period=3.1e-3, fwhm=0.03, snr=0.05, seed=0)
METRIC = "DM-trial x Msamples/s (MS-OSM dedispersion + |y|^2 fold, FFT 4096, 256 trials), 1 B200"
UNIT = "DM-trial*Msamples/s"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def workload_config(samples, n_dm, ws):
    return {"workload": "batched multi-DM MS-OSM: 16 MHz @ 1250 MHz, 2^%d complex64 samples, %d DM trials "
                        "0-100 per GPU, FFT %d, fold %d bins" % (int(math.log2(samples)), n_dm, FFTPOINT, NBINS),
            "samples_per_step": samples, "dm_trials_per_gpu": n_dm, "dm_range_per_gpu": [0.0, DM_MAX],
            "fftpoint": FFTPOINT, "fold_bins": NBINS, "detect": "|y|^2", "period_s": PULSAR["period"],
            "injected_dm": PULSAR["dm"],
            "parallelism": f"dm-shard x{ws}" + (" (input broadcast from rank 0, profiles all-gathered)" if ws > 1
                                                 else ""),
            "l2": "inputs larger than L2 (537 MB input, 1.1 GB spectrum ring)"}


def dm_trials(rank, n_dm):
    # weak scaling: rank r owns n_dm trials over [r*100, (r+1)*100]
    from msosm_gpu_b200 import shard
    return shard.weak_trials(rank, n_dm, DM_MAX)


def make_signal(samples, on_gpu=True):
    """The workload's baseband: the library's device simulator (counter-based
    normals, overlap-save dispersion), or for the reference arms the host
    generator (numpy), so that no code of this library runs on their path."""
    t = time.time()
    if on_gpu:
        from msosm_gpu_b200 import simulator as G
        x = G.pulsar_baseband(samples, BW, F0, PULSAR["dm"], PULSAR["period"], PULSAR["fwhm"], PULSAR["snr"],
                              seed=PULSAR["seed"])
    else:
        from msosm_gpu_b200 import simulate as S
        x = S.pulsar_baseband(samples, BW, F0, PULSAR["dm"], PULSAR["period"], PULSAR["fwhm"], PULSAR["snr"],
                              seed=PULSAR["seed"])
    log(f"signal: {samples} samples generated in {time.time() - t:.1f} s ({'device' if on_gpu else 'host'})")
    return x


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str | None):
        self.proc = None
        self.uuid = uuid

    def __enter__(self):
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"]
        if self.uuid:
            cmd += ["-i", self.uuid]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [v.strip() for v in l.split(",")]
            try:
                sm.append(float(f[0]))
                mx = max(mx, float(f[1]))
            except (ValueError, IndexError):
                continue
            for n, v in zip(names, f[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        loaded = [v for v in sm if v > 0.3 * mx] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


class _NoClock:
    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False

    def summary(self):
        return None


# ---------------------------------------------------------------------------
# CPU baseline: the oracle on the host cores
# ---------------------------------------------------------------------------

def cpu_baseline(dms, x, budget_s=12.0):
    """The reference's algorithm in FP32 on all host cores (oracle/cpu_fp32.py:
    forward FFT, per-bin delayed filter product, inverse FFT, discard, |y|^2
    and the Fold_GPU fold; pocketfft standing in for FFTW, threads over
    trials), timed on a bounded sample of the workload."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import cpu_fp32 as C
    threads = os.cpu_count() or 1
    count = 64  # calls of 131k samples: smaller calls leave it bound by per-task overhead
    c = C.MsosmFP32(BW, dms, F0, FFTPOINT, count, period=PULSAR["period"], time_bin=NBINS, threads=threads)
    blk = count * c.M

    def one(k):
        c.filter(x[(k * blk) % (x.size - blk):][:blk])

    t = time.perf_counter()
    one(0)
    first = time.perf_counter() - t
    calls = max(1, min(256, int(budget_s / max(first, 1e-3))))
    t = time.perf_counter()
    for k in range(1, calls + 1):
        one(k)
    el = time.perf_counter() - t
    c.close()
    v = len(dms) * calls * blk / el / 1e6
    return {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{len(dms)} trials x {calls * blk} samples ({calls} calls of {blk}): the reference's "
                      f"MS-OSM in FP32 (oracle/cpu_fp32.py; {C.FFT_LIBRARY}), threads over trials, "
                      f"incl. |y|^2 and the Fold_GPU fold, {el:.1f} s"}


def accuracy_vs_fp64(dms, x, calls=48, count=8):
    """Relative RMS error of both device paths against the FP64 oracle on a
    sample of the workload (the oracle is the checker here): per trial, the
    dedispersed series and the folded |y|^2 profile."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from msosm_gpu_b200 import Dedisperser
    O.lib().orc_set_threads(os.cpu_count() or 1)
    o = O.Dedisp(BW, dms, F0, FFTPOINT, count, threads=os.cpu_count() or 1)
    blk = count * o.M
    nd = int(max(o.Nd))
    devs = {}
    for prec in ("fp16", "bf16", "fp32"):
        dv = Dedisperser(BW, dms, F0, FFTPOINT, count=count, precision=prec)
        dv.fold_init(PULSAR["period"], BW, time_bin=NBINS, discard_Nd=nd, detect="power")
        devs[prec] = dv
    folds = [O.Fold(PULSAR["period"], BW, blk, NBINS) for _ in dms]
    for f in folds:
        f.discard_samples(nd)
    err = {p: np.zeros(len(dms)) for p in devs}
    ref = np.zeros(len(dms))
    for c in range(calls):
        seg = np.ascontiguousarray(x[c * blk:(c + 1) * blk])
        y = o.filter(seg.astype(np.complex128))
        ref += np.sum(np.abs(y) ** 2, axis=1)
        for i, f in enumerate(folds):
            f.fold_data(np.abs(y[i]) ** 2)
        for p, dv in devs.items():
            dv.filter_block(seg)
            err[p] += np.sum(np.abs(dv.get_output().astype(np.complex128) - y) ** 2, axis=1)
    pref = np.stack([f.fold_data_bins() for f in folds])
    out = {"sample": f"{len(dms)} trials x {calls * blk} samples ({calls} calls of {blk}) of the workload's "
                     f"signal; FP64 oracle (oracle/orc.c) as the reference; relative RMS per trial, "
                     f"median and max over trials; profiles folded to {NBINS} bins after discarding {nd} samples"}
    for p, dv in devs.items():
        se = np.sqrt(err[p] / np.maximum(ref, 1e-300))
        prof = dv.get_profiles().astype(np.float64)
        pe = np.sqrt(np.sum((prof - pref) ** 2, axis=1) / np.maximum(np.sum(pref ** 2, axis=1), 1e-300))
        out[p] = {"series_rel_rms_median": float(np.median(se)), "series_rel_rms_max": float(se.max()),
                  "profile_rel_rms_median": float(np.median(pe)), "profile_rel_rms_max": float(pe.max()),
                  "folded_periods": int(dv.folded_periods())}
        dv.close()
    return out


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def fp32_peak_tflops(torch):
    torch.backends.cuda.matmul.allow_tf32 = False
    n = 8192
    a = torch.randn(n, n, device="cuda")
    b = torch.randn(n, n, device="cuda")
    best = 0.0
    for i in range(6):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        torch.cuda.synchronize()
        if i:
            best = max(best, 2 * n ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    del a, b
    return best


# peaks when MEASURED_PEAKS.json (written per machine by the job that runs
# this benchmark) is absent: an earlier measurement on this pool of B200s
FALLBACK_PEAKS = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}


def load_peaks():
    """(peaks, source): the measured copy bandwidth and bf16 GEMM rates of
    this machine, or the fallback figures, labelled as such."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        out = {k: d.get(k) or FALLBACK_PEAKS[k] for k in FALLBACK_PEAKS}
        return out, "measured (MEASURED_PEAKS.json)"
    return dict(FALLBACK_PEAKS), "fallback (MEASURED_PEAKS.json absent): 6.65 TB/s, 1.59 PFLOP/s burst, 1.4 sustained"


def load_traffic():
    p = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    if os.path.exists(p):
        return json.load(open(p))
    return None


def run_ours(args):
    import torch
    import torch.distributed as dist
    from msosm_gpu_b200 import Dedisperser

    ws, rank, local = dist_setup()
    if ws > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    samples = 1 << args.log2_samples
    dms = dm_trials(rank, args.dms)
    x = make_signal(samples)
    peaks, peaks_src = load_peaks()
    fp32 = fp32_peak_tflops(torch)

    # ---- value: input resident in HBM, one call per step -----------------
    blocks = samples // (FFTPOINT // 2)
    xd = torch.from_numpy(x).to(dev)
    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        pass
    from msosm_gpu_b200 import shard

    # N > 1: one stream's trials sharded over the ranks (ShardedDedisperser):
    # rank 0 holds the input, broadcast to the others every call over NCCL
    # (inside the timed region), profiles all-gathered
    all_dms = np.concatenate([dm_trials(r, args.dms) for r in range(ws)])

    def handle(precision, count):
        if ws == 1:
            d = Dedisperser(BW, dms, F0, FFTPOINT, count=count, series=False, precision=precision)
            nd_max = int(d.Nd.max())
        else:
            d = shard.ShardedDedisperser(BW, all_dms, F0, FFTPOINT, count=count, precision=precision, device=dev)
            nd_max = d.max_nd()
        d.fold_init(PULSAR["period"], BW, time_bin=NBINS, discard_Nd=nd_max, detect="power")
        return d, nd_max

    src = xd if rank == 0 else None

    def device_arm(precision, sample_clocks):
        stream = torch.cuda.Stream(dev)
        d, _ = handle(precision, blocks)
        d.set_stream(stream)
        torch.cuda.synchronize()
        for _ in range(args.warmup):
            with torch.cuda.stream(stream):
                d.filter_block(xd if ws == 1 else src)
        torch.cuda.synchronize()
        d.enable_timing(True)
        if ws > 1:
            dist.barrier()
        torch.cuda.synchronize()
        with ClockSampler(uuid) if sample_clocks else _NoClock() as ck:
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                s.record(stream)
                for _ in range(args.steps):
                    d.filter_block(xd if ws == 1 else src)
                e.record(stream)
            torch.cuda.synchronize()
        if ws > 1:
            dist.barrier()
        ms_max = shard.max_over_ranks(s.elapsed_time(e) / args.steps, dev)
        tm = d.timing()
        prof = d.get_profiles()
        d.close()
        return ms_max, tm, prof, ck.summary()

    units = float(args.dms) * samples * ws
    ms_max, tm, prof, clocks = device_arm(args.precision, True)
    value = units / (ms_max * 1e-3) / 1e6
    peak_dm = float(all_dms[int(np.argmax(prof.max(1) - np.median(prof, 1)))])
    other = "fp16" if args.precision == "fp32" else "fp32"
    ms_o, tm_o, _, _ = device_arm(other, False)
    value_other = units / (ms_o * 1e-3) / 1e6

    # ---- e2e: pinned host input through the C ABI, chunked calls -----------
    e_count = min(blocks, 8192)
    calls = blocks // e_count
    de, _ = handle(args.precision, e_count)
    xh = torch.from_numpy(x).pin_memory().numpy()
    chunk = e_count * (FFTPOINT // 2)

    def e2e_step():
        for c in range(calls):
            de.filter_block(xh[c * chunk:(c + 1) * chunk] if rank == 0 or ws == 1 else None)
        return de.get_profiles()

    for _ in range(args.warmup):
        e2e_step()
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    torch.cuda.synchronize()
    e2e_s = (time.perf_counter() - t0) / args.steps
    e2e_v = units / shard.max_over_ranks(e2e_s, dev) / 1e6

    # ---- roofline of the dominant kernel -----------------------------------
    log2n = int(math.log2(FFTPOINT))
    flops_per_sample = 10 * log2n + 16
    launch_samples = float(args.dms) * samples

    def stages(t):
        c = max(t["calls"], 1)
        return {"forward": t["forward_ms"] / c, "dedisp": t["dedisp_ms"] / c, "fold": t["fold_ms"] / c}

    def fp32_roofline(t):
        k_ms = t["dedisp_ms"] / max(t["calls"], 1)
        ach = flops_per_sample * launch_samples / (k_ms * 1e-3) / 1e12
        return {"bound": "fp32", "achieved": ach, "peak": fp32, "unit": "TFLOP/s",
                "frac": ach / fp32 if fp32 else None,
                "kernel": f"dedisp_kernel<{log2n}> (gather x H, FP32 shared-memory inverse FFT, discard, |y|^2, fold)",
                "flops_per_dm_sample": flops_per_sample, "kernel_ms": k_ms,
                "peak_source": "cuBLAS SGEMM 8192^3 measured in this run (MEASURED_PEAKS.json has no FP32 figure)",
                "stage_ms_per_step": stages(t)}

    tr = load_traffic() or {}

    def traffic_of(key):
        b = tr.get(key)
        return b * launch_samples if b else None

    if args.precision in ("fp16", "bf16"):
        k_ms = tm["dedisp_ms"] / max(tm["calls"], 1)
        tpeak = peaks["bf16_tflops_sustained"]
        ach = flops_per_sample * launch_samples / (k_ms * 1e-3) / 1e12
        # executed tensor work: per pair of 4096-point blocks 128x128x128 + 128x64x128 MACs
        exec_tf = 2.0 * (128 * 128 * 128 + 128 * 64 * 128) / 4096.0 * launch_samples / (k_ms * 1e-3) / 1e12
        roofline = {"bound": "tensor", "achieved": ach, "peak": tpeak, "unit": "TFLOP/s", "frac": ach / tpeak,
                    "traffic": traffic_of("tc_bytes_per_dm_sample"),
                    "kernel": "tc_dedisp_kernel (gather x H, inverse FFT as two tcgen05 %s GEMMs + %s twiddle, "
                              "discard, |y|^2, fold)" % (args.precision[:2] + "16", args.precision[:2] + "16"),
                    "flops_per_dm_sample": flops_per_sample, "kernel_ms": k_ms,
                    "executed_tensor_tflops": exec_tf, "executed_tensor_frac": exec_tf / tpeak,
                    "peak_source": peaks_src + ", bf16_tflops_sustained (f16 runs at the bf16 rate; the "
                                   "kernel runs inside a ~100 ms step)",
                    "note": "achieved counts the algorithmic 10 log2 N + 16 flops per DM-trial sample, as the "
                            "FP32 path does; the kernel is bound by CUDA-core issue (gather, twiddle, fold), "
                            "not by the tensor pipe",
                    "stage_ms_per_step": stages(tm)}
        roofline_fp32 = dict(fp32_roofline(tm_o), traffic=traffic_of("bytes_per_dm_sample"))
    else:
        roofline = dict(fp32_roofline(tm), traffic=traffic_of("bytes_per_dm_sample"))
        roofline_fp32 = None
    # issue roofline of the tensor-core kernel: its warp instructions per
    # DM-trial sample (ncu capture) at the measured rate, against 4 issue
    # slots per SM per clock at the SM clock sampled during the run
    roofline_issue = None
    ipd = tr.get("tc_warp_inst_per_dm_sample")
    if args.precision != "fp32" and ipd:
        import torch as _t
        sms = _t.cuda.get_device_properties(dev).multi_processor_count
        mhz = (clocks or {}).get("sm_mhz") or (clocks or {}).get("sm_max_mhz") or 1965.0
        k_ms = tm["dedisp_ms"] / max(tm["calls"], 1)
        ach = ipd * launch_samples / (k_ms * 1e-3)
        pk = 4.0 * sms * mhz * 1e6
        roofline_issue = {"bound": "issue", "achieved": ach, "peak": pk, "unit": "warp instructions/s",
                          "frac": ach / pk, "warp_inst_per_dm_sample": ipd,
                          "note": "the tensor-core kernel is bound by CUDA-core issue (gather, twiddle, fold "
                                  "and their barriers), not by HBM or the tensor pipe; instructions per sample "
                                  "from profiles/roofline_traffic.json"}
    hbm = peaks["hbm_gbs"]
    algo_bytes = 8.0 * samples  # the input, read once for all trials
    roofline_hbm = {"bound": "hbm", "algorithmic_bytes_per_step": algo_bytes,
                    "achieved_gbs": algo_bytes / (ms_max * 1e-3) / 1e9, "peak": hbm, "unit": "GB/s",
                    "peak_source": peaks_src,
                    "note": "the fused path reads the input once for all trials; it is compute-bound"}

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None,
            "dtype": ("%s GEMM operands, f32 accumulation and gather" % (args.precision[:2] + "16")
                      if args.precision != "fp32" else "f32"),
            "data": "synthetic (seeded pulsar + AWGN)",
            "config": dict(workload_config(samples, args.dms, ws), precision=args.precision),
            "e2e": {"value": e2e_v, "unit": UNIT, "h2d_bytes_per_step": int(x.nbytes),
                    "d2h_bytes_per_step": int(prof.nbytes), "ms_per_step": e2e_s * 1e3,
                    "calls_per_step": calls},
            "gpu_launches": int(tm["kernel_launches"]),
            "roofline": roofline, "roofline_hbm": roofline_hbm,
            "clocks": clocks,
            other + "_path": {"value": value_other, "ms_per_step": ms_o, "unit": UNIT,
                              "note": "the same workload through the other precision's fused kernel, timed "
                                      "the same way (value / this = %.3f)" % (value / value_other)},
            "check": {"detected_dm": peak_dm, "injected_dm": PULSAR["dm"]}}
    if roofline_fp32:
        line["roofline_fp32_path"] = roofline_fp32
    if roofline_issue:
        line["roofline_issue"] = roofline_issue
    if rank == 0 and ws == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(dms, x)
        line["accuracy_vs_fp64"] = accuracy_vs_fp64(dms, x)
    if rank == 0 and ws == 1 and not args.no_reference_gpu:
        # the reference's own cuFFT path on this GPU and this signal, after our
        # timed regions (a separate process: its destructors reset the device)
        rg = reference_gpu_measure(samples, args.dms, min(args.steps, 5), x=x, with_series=False)
        if "value" in rg:
            rg["our_e2e_over_this"] = e2e_v / rg["value"]
            rg["our_value_over_this"] = value / rg["value"]
        line["reference_gpu"] = rg
    de.close()
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# precision sweep: 64 MHz band centred at 1400 MHz, FFT 8192 (--fftpoint), 1024 trials
# ---------------------------------------------------------------------------

SWEEP = dict(bw=64e6, f0=1368e6, fftpoint=8192, n_dm=1024, dm_max=200.0, log2_samples=26, nbins=1024,
             pulsar=dict(dm=150.0, period=4.7e-3, fwhm=0.02, snr=0.05), seeds=8,
             sample_dms=(0.0, 60.0, 150.0, 200.0), chunk_blocks=256)
SWEEP_PRECS = ("fp32", "fp16", "bf16")


def profile_snr(p, width):
    """Boxcar matched-filter S/N of a folded profile: the largest circular
    sum of ``width`` bins above the off-pulse mean, over the off-pulse
    standard deviation times sqrt(width); off-pulse = every bin farther than
    two widths from that window."""
    p = np.asarray(p, np.float64)
    n = p.size
    c = np.concatenate([p, p[:width - 1]])
    box = np.convolve(c, np.ones(width), "valid")[:n]
    k = int(np.argmax(box))
    mask = np.ones(n, bool)
    mask[(np.arange(-2 * width, 3 * width) + k) % n] = False
    off = p[mask]
    return float((box[k] - width * off.mean()) / (off.std() * math.sqrt(width)))


def sweep_throughput(x, dms, steps, warmup):
    """Device time of one step (all samples, all trials, fold only) for each
    precision, input resident in HBM."""
    import torch
    from msosm_gpu_b200 import Dedisperser
    cfg = SWEEP
    M = cfg["fftpoint"] // 2
    xd = torch.from_numpy(x).cuda()
    stream = torch.cuda.Stream()
    out = {}
    for prec in SWEEP_PRECS:
        d = Dedisperser(cfg["bw"], dms, cfg["f0"], cfg["fftpoint"], count=x.size // M, series=False,
                        precision=prec)
        d.set_stream(stream)
        d.fold_init(cfg["pulsar"]["period"], cfg["bw"], time_bin=cfg["nbins"], discard_Nd=int(d.Nd.max()),
                    detect="power")
        for _ in range(warmup):
            d.filter_block(xd)
        torch.cuda.synchronize()
        d.enable_timing(True)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            s.record(stream)
            for _ in range(steps):
                d.filter_block(xd)
            e.record(stream)
        torch.cuda.synchronize()
        ms = s.elapsed_time(e) / steps
        tm = d.timing()
        c = max(tm["calls"], 1)
        prof = d.get_profiles()
        width = max(1, int(round(cfg["pulsar"]["fwhm"] * cfg["nbins"])))
        snr = np.array([profile_snr(p, width) for p in prof])
        out[prec] = {"ms_per_step": ms, "value": len(dms) * x.size / (ms * 1e-3) / 1e6,
                     "stage_ms_per_step": {"forward": tm["forward_ms"] / c, "dedisp": tm["dedisp_ms"] / c,
                                           "fold": tm["fold_ms"] / c},
                     "best_trial_dm": float(dms[int(np.argmax(snr))]), "best_trial_snr": float(snr.max())}
        d.close()
    del xd
    return out


def sweep_accuracy(x, seed):
    """Errors of the three device precisions against the FP64 oracle for the
    sampled trials over the whole signal (chunked calls): dedispersed series
    and folded |y|^2 profiles, and the injected pulsar's S/N in each
    precision's profile relative to the oracle's."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from msosm_gpu_b200 import Dedisperser
    cfg = SWEEP
    threads = os.cpu_count() or 1
    O.lib().orc_set_threads(threads)
    dms = np.array(cfg["sample_dms"], np.float32)
    count = cfg["chunk_blocks"]
    o = O.Dedisp(cfg["bw"], dms, cfg["f0"], cfg["fftpoint"], count, threads=threads)
    blk = count * o.M
    nd = int(max(o.Nd))
    devs = {}
    for prec in SWEEP_PRECS:
        dv = Dedisperser(cfg["bw"], dms, cfg["f0"], cfg["fftpoint"], count=count, precision=prec)
        dv.fold_init(cfg["pulsar"]["period"], cfg["bw"], time_bin=cfg["nbins"], discard_Nd=nd, detect="power")
        devs[prec] = dv
    folds = [O.Fold(cfg["pulsar"]["period"], cfg["bw"], blk, cfg["nbins"]) for _ in dms]
    for f in folds:
        f.discard_samples(nd)
    ref2 = np.zeros(len(dms))
    err2 = {p: np.zeros(len(dms)) for p in devs}
    emax = {p: np.zeros(len(dms)) for p in devs}
    calls = x.size // blk
    for c in range(calls):
        seg = np.ascontiguousarray(x[c * blk:(c + 1) * blk])
        y = o.filter(seg.astype(np.complex128))
        ref2 += np.sum(np.abs(y) ** 2, axis=1)
        for i, f in enumerate(folds):
            f.fold_data(np.abs(y[i]) ** 2)
        for p, dv in devs.items():
            dv.filter_block(seg)
            e = np.abs(dv.get_output().astype(np.complex128) - y)
            err2[p] += np.sum(e * e, axis=1)
            emax[p] = np.maximum(emax[p], e.max(axis=1))
    pref = np.stack([f.fold_data_bins() for f in folds])
    width = max(1, int(round(cfg["pulsar"]["fwhm"] * cfg["nbins"])))
    inj = int(np.argmin(np.abs(dms - cfg["pulsar"]["dm"])))
    snr_ref = profile_snr(pref[inj], width)
    rms_ref = np.sqrt(ref2 / (calls * blk))
    res = {"seed": seed, "snr_fp64": snr_ref}
    for p, dv in devs.items():
        prof = dv.get_profiles().astype(np.float64)
        dp = prof - pref
        snr = profile_snr(prof[inj], width)
        res[p] = {"series_rel_rms": (np.sqrt(err2[p] / np.maximum(ref2, 1e-300))).tolist(),
                  "series_max_abs_over_rms": (emax[p] / np.maximum(rms_ref, 1e-300)).tolist(),
                  "profile_rel_rms": (np.sqrt(np.sum(dp ** 2, 1) / np.sum(pref ** 2, 1))).tolist(),
                  "profile_max_abs_over_mean": (np.abs(dp).max(1) / np.abs(pref).mean(1)).tolist(),
                  "snr": snr, "snr_loss": 1.0 - snr / snr_ref}
        dv.close()
    return res


def run_precision_sweep(args):
    from msosm_gpu_b200 import simulator as G
    cfg = SWEEP
    samples = 1 << (args.log2_samples or cfg["log2_samples"])
    n_dm = args.dms or cfg["n_dm"]
    dms = np.linspace(0.0, cfg["dm_max"], n_dm).astype(np.float32)
    pul = cfg["pulsar"]

    def signal(seed):
        t = time.time()
        x = G.pulsar_baseband(samples, cfg["bw"], cfg["f0"], pul["dm"], pul["period"], pul["fwhm"], pul["snr"],
                              seed=seed)
        log(f"seed {seed}: {samples} samples generated in {time.time() - t:.1f} s")
        return x

    x = signal(0)
    thr = sweep_throughput(x, dms, args.steps, args.warmup)
    log("throughput: " + json.dumps(thr))
    seeds = []
    for seed in range(args.seeds):
        if seed:
            x = signal(seed)
        t = time.time()
        seeds.append(sweep_accuracy(x, seed))
        log(f"seed {seed}: accuracy in {time.time() - t:.1f} s: " + json.dumps(seeds[-1]))
    summary = {}
    for p in SWEEP_PRECS:
        def agg(key):
            v = np.array([r[p][key] for r in seeds], np.float64)
            return {"median": float(np.median(v)), "max": float(v.max())} if v.size else None
        summary[p] = {"series_rel_rms": agg("series_rel_rms"),
                      "series_max_abs_over_rms": agg("series_max_abs_over_rms"),
                      "profile_rel_rms": agg("profile_rel_rms"),
                      "profile_max_abs_over_mean": agg("profile_max_abs_over_mean"),
                      "snr_loss": agg("snr_loss"),
                      "throughput": thr[p]["value"], "ms_per_step": thr[p]["ms_per_step"],
                      "speedup_vs_fp32": thr[p]["value"] / thr["fp32"]["value"]}
    line = {"workload": "tensor-core precision sweep: 64 MHz band centred at 1400 MHz (f0 1368 MHz), "
                        "2^%d complex64 samples, %d DM trials 0-%g, FFT %d, fold %d bins"
                        % (int(math.log2(samples)), n_dm, cfg["dm_max"], cfg["fftpoint"], cfg["nbins"]),
            "unit": UNIT, "data": "synthetic (seeded pulsar + AWGN)",
            "pulsar": pul, "seeds": args.seeds, "steps": args.steps, "warmup": args.warmup,
            "precisions": {"fp32": "FP32 CUDA-core inverse FFT (the plain fused path)",
                           "fp16": "tcgen05 f16 operands, f32 accumulation",
                           "bf16": "tcgen05 bf16 operands, f32 accumulation",
                           "split_hi_lo": "not built"},
            "error_reference": "FP64 oracle (oracle/orc.c: the reference algorithm in double precision, "
                               "radix-2 FFT; FFTW is not available)",
            "error_sample": "trials %s over every sample of each seed's signal (calls of %d blocks); series "
                            "error relative to the oracle's RMS, profile error relative to the oracle's "
                            "profile; S/N by a %d-bin boxcar at the trial nearest the injected DM"
                            % (list(cfg["sample_dms"]), cfg["chunk_blocks"],
                               max(1, int(round(pul["fwhm"] * cfg["nbins"])))),
            "throughput_sample": "seed 0, all trials, device time per step (CUDA events), input resident in HBM",
            "summary": summary, "throughput": thr, "per_seed": seeds}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# uneven batch: 64 independent observations, autotuned against fixed choices
# ---------------------------------------------------------------------------

UNEVEN = dict(n_obs=64, log2_len=(20, 25), bws=(4e6, 16e6, 32e6, 64e6), centre=(1100e6, 1500e6),
              trials=(16, 512), dm_max=(20.0, 300.0), period=(1e-3, 1.0), duty=(0.01, 0.10),
              snr=(0.02, 0.2), nbins=256, seed=0)
FIXED = [(2048, "fp32"), (4096, "fp32"), (8192, "fp32"), (16384, "fp32"), (32768, "fp32"), (4096, "fp16"),
         (8192, "fp16"), (16384, "fp16")]


def uneven_observations(n_obs, seed):
    """The observations' parameters: lengths log-uniform 2^20 .. 2^25 (whole
    multiples of 2^15 samples), bandwidth from {4, 16, 32, 64} MHz, centre
    uniform 1100 .. 1500 MHz, trial counts log-uniform 16 .. 512 over
    0 .. DM_max with DM_max uniform 20 .. 300, one pulsar each (period
    log-uniform 1 ms .. 1 s, duty cycle 1 .. 10 %, peak SNR 0.02 .. 0.2, DM
    uniform over the middle 80 % of the range, lowered where the simulator's
    dispersion filter would pass 2^24 points)."""
    from msosm_gpu_b200.autotune import log_uniform
    from msosm_gpu_b200.prepare import nd, osm_min_order
    cfg = UNEVEN
    rng = np.random.default_rng(seed)
    obs = []
    for i in range(n_obs):
        n = int(2 ** rng.uniform(*cfg["log2_len"])) // (1 << 15) * (1 << 15)
        bw = float(cfg["bws"][rng.integers(len(cfg["bws"]))])
        f0 = float(np.float32(rng.uniform(*cfg["centre"]) - bw / 2))
        D = int(round(log_uniform(rng, *cfg["trials"])))
        dm_max = float(rng.uniform(*cfg["dm_max"]))
        dm = float(rng.uniform(0.1, 0.9) * dm_max)
        while 2 * osm_min_order(nd(bw, dm, f0)) > (1 << 24):
            dm *= 0.8
        obs.append(dict(i=i, n=n, bw=bw, f0=f0, trials=D, dm_max=dm_max, dm=dm,
                        period=log_uniform(rng, *cfg["period"]), duty=float(rng.uniform(*cfg["duty"])),
                        snr=float(rng.uniform(*cfg["snr"]))))
    return obs


def uneven_one_launch(obs, tuned, cfg, stream, reps=3):
    """The tuned configuration of every observation as one batch
    (DedispBatch: one persistent launch per tensor-core kernel group, work
    items handed out largest first), against the same handles called back to
    back on the same stream; device-resident inputs, CUDA events, the
    median of `reps` calls each after one warm-up call.  Observations tuned
    to an FFT above one thread block (the FP32 four-step path, above 16384
    points) are left out: a batch runs them in their own launches anyway,
    and their per-trial transform buffers (trials x blocks x FFT points)
    held for all observations at once would not fit the device."""
    import torch
    from msosm_gpu_b200 import DedispBatch, Dedisperser
    from msosm_gpu_b200 import simulator as G
    keep = [k for k, (n, _) in enumerate(tuned) if n <= 16384]
    units = float(sum(obs[k]["trials"] * obs[k]["n"] for k in keep))
    handles, inputs = [], []
    for o, (n, p) in ((obs[k], tuned[k]) for k in keep):
        dms = np.linspace(0.0, o["dm_max"], o["trials"]).astype(np.float32)
        inputs.append(G.pulsar_baseband(o["n"], o["bw"], o["f0"], o["dm"], o["period"], o["duty"], o["snr"],
                                        seed=o["i"], device=torch.device("cuda")))
        d = Dedisperser(o["bw"], dms, o["f0"], n, count=o["n"] // (n // 2), series=False, precision=p)
        d.set_stream(stream)
        d.fold_init(o["period"], o["bw"], time_bin=cfg["nbins"], discard_Nd=int(d.Nd.max()), detect="power")
        handles.append(d)
    torch.cuda.synchronize()

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        out = []
        for _ in range(reps):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                s.record(stream)
                fn()
                e.record(stream)
            torch.cuda.synchronize()
            out.append(s.elapsed_time(e))
        return statistics.median(out)

    def seq():
        for d, x in zip(handles, inputs):
            d.filter_block(x)

    seq_ms = timed(seq)
    b = DedispBatch(handles)
    b.set_stream(stream)
    info = b.info()
    batch_ms = timed(lambda: b.filter_block(inputs))
    b.synchronize()
    b.close()
    for d in handles:
        d.close()
    del inputs
    torch.cuda.empty_cache()
    return {"ms": batch_ms, "value": units / (batch_ms * 1e-3) / 1e6,
            "back_to_back_ms": seq_ms, "back_to_back_value": units / (seq_ms * 1e-3) / 1e6,
            "speedup_vs_back_to_back": seq_ms / batch_ms, "batch": info,
            "observations": len(keep), "left_out_above_16384": len(obs) - len(keep),
            "dm_trial_samples": units,
            "method": "the tuned handles of all observations; one DedispBatch call (one persistent launch per "
                      "tensor-core kernel group, forward transforms per observation) against one filter_block "
                      "call per observation on the same stream; device-resident inputs, CUDA events, median of "
                      "%d calls after a warm-up call" % reps}


def run_uneven_batch(args):
    import torch
    from msosm_gpu_b200 import Dedisperser
    from msosm_gpu_b200 import simulator as G
    from msosm_gpu_b200.autotune import Autotuner, coherence, fixed_choice
    from msosm_gpu_b200.prepare import nd
    cfg = UNEVEN
    obs = uneven_observations(args.obs, cfg["seed"])
    tuner = Autotuner(sample=1 << 21, calls=2)
    stream = torch.cuda.Stream()
    times = []   # per observation: {(fft, prec): ms}
    tuned, tuning_s, detect = [], 0.0, []
    total_units = 0.0
    for o in obs:
        dms = np.linspace(0.0, o["dm_max"], o["trials"]).astype(np.float32)
        t = time.time()
        ch = tuner.tune(o["bw"], dms, o["f0"], period=o["period"], time_bin=cfg["nbins"],
                        min_coherence=args.min_coherence)
        tuning_s += time.time() - t
        tuned.append((ch.fftpoint, ch.precision))
        x = G.pulsar_baseband(o["n"], o["bw"], o["f0"], o["dm"], o["period"], o["duty"], o["snr"], seed=o["i"],
                              device=torch.device("cuda"))
        need = {(ch.fftpoint, ch.precision)} | {fixed_choice(o["bw"], dms, o["f0"], n, p) for n, p in FIXED}
        res = {}
        for n, p in sorted(need):
            d = Dedisperser(o["bw"], dms, o["f0"], n, count=o["n"] // (n // 2), series=False, precision=p)
            d.set_stream(stream)
            d.fold_init(o["period"], o["bw"], time_bin=cfg["nbins"], discard_Nd=int(d.Nd.max()), detect="power")
            torch.cuda.synchronize()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                s.record(stream)
                d.filter_block(x)
                e.record(stream)
            torch.cuda.synchronize()
            res[(n, p)] = s.elapsed_time(e)
            if (n, p) == (ch.fftpoint, ch.precision) and d.folded_periods() >= 8:
                # expected folded S/N: |y|^2 has unit mean and deviation; the
                # pulse adds ~0.75 snr over a duty fraction of the samples
                folded = d.folded_periods() * o["period"] * o["bw"]
                expect = 0.75 * o["snr"] * math.sqrt(folded * o["duty"])
                prof = d.get_profiles().astype(np.float64)
                w = max(1, int(round(o["duty"] * cfg["nbins"])))
                snr = np.array([profile_snr(q, w) for q in prof])
                step = o["dm_max"] / max(o["trials"] - 1, 1)
                # DM resolution: the DM error whose smear across the band is
                # one pulse width (narrow bands and wide pulses resolve DM
                # poorly: S/N is then nearly flat over the trials)
                smear_per_dm = nd(o["bw"], 100.0, o["f0"]) / 100.0 / o["bw"]
                dm_res = o["duty"] * o["period"] / max(smear_per_dm, 1e-30)
                tol = max(1.5 * step, dm_res)
                best = float(dms[int(np.argmax(snr))])
                detect.append({"i": o["i"], "expected_snr": expect, "best_snr": float(snr.max()), "best_dm": best,
                               "dm": o["dm"], "dm_tolerance": tol, "hit": abs(best - o["dm"]) <= tol})
            d.close()
        del x
        times.append(res)
        total_units += o["trials"] * o["n"]
        log(f"obs {o['i']}: n={o['n']} bw={o['bw'] / 1e6:g} D={o['trials']} dm_max={o['dm_max']:.0f} "
            f"tuned={ch.fftpoint}/{ch.precision} " + " ".join(f"{k[0]}/{k[1]}={v:.1f}" for k, v in sorted(res.items())))
    tuned_ms = sum(r[c] for r, c in zip(times, tuned))
    one_launch = uneven_one_launch(obs, tuned, cfg, stream)
    fixed = {}
    for n, p in FIXED:
        ms = 0.0
        for o, r in zip(obs, times):
            dms = np.linspace(0.0, o["dm_max"], o["trials"]).astype(np.float32)
            ms += r[fixed_choice(o["bw"], dms, o["f0"], n, p)]
        fixed[f"{n}/{p}"] = {"ms": ms, "value": total_units / (ms * 1e-3) / 1e6}
    best = max(fixed, key=lambda k: fixed[k]["value"])
    tuned_v = total_units / (tuned_ms * 1e-3) / 1e6
    line = {"workload": "uneven batch: %d independent observations (lengths 2^20-2^25, bandwidth 4/16/32/64 MHz, "
                        "centre 1100-1500 MHz, 16-512 trials over 0-DM_max, DM_max 20-300), one injected pulsar "
                        "each, fold %d bins" % (len(obs), cfg["nbins"]),
            "unit": UNIT, "data": "synthetic (device simulator, seeded)",
            "method": "each observation one filter_block call on device-resident input, CUDA events on the "
                      "handle's stream; fixed configurations raise the FFT to an observation's minimum and "
                      "fall back to FP32 where the tensor path has no kernel; the autotuner times every "
                      "candidate on 2^21 samples of noise per observation shape",
            "total_dm_trial_samples": total_units,
            "tuned": {"ms": tuned_ms, "value": tuned_v,
                      "choices": {f"{n}/{p}": tuned.count((n, p)) for n, p in sorted(set(tuned))}},
            "one_launch": one_launch,
            "fixed": fixed, "best_fixed": best, "tuned_vs_best_fixed": tuned_v / fixed[best]["value"],
            "tuning_s": tuning_s,
            "min_coherence": args.min_coherence,
            "tuned_coherence_min": min(coherence(o["bw"], o["dm_max"], o["f0"], n) for o, (n, _) in zip(obs, tuned)),
            "detected": {"rule": "best-S/N trial within max(1.5 trial steps, the DM error that smears one pulse "
                                 "width across the band) of the injected DM, over observations with >= 8 folded "
                                 "periods and an expected S/N >= 10",
                         "eligible": sum(1 for t in detect if t["expected_snr"] >= 10),
                         "hits": sum(1 for t in detect if t["expected_snr"] >= 10 and t["hit"]),
                         "all": detect},
            "observations": obs}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# streaming to a file: host input in, every trial's uint16 series out
# ---------------------------------------------------------------------------

def run_stream_to_file(args):
    """The reference drivers' output-file use (multiple_dm_concurrent_msosm.cpp):
    pinned host input in calls of `count` blocks, every trial's dedispersed
    series encoded to uint16 and appended to a file by the series writer,
    against the same calls without the writer (wall clock per step, one
    synchronize at the end of each)."""
    import tempfile as _tf

    import torch
    from msosm_gpu_b200 import Dedisperser
    from msosm_gpu_b200.writer import SeriesWriter
    samples = 1 << (args.log2_samples or 24)
    n_dm = args.dms or 16
    count = 256
    dms = np.linspace(0.0, DM_MAX, n_dm).astype(np.float32)
    x = make_signal(samples)
    xh = torch.from_numpy(x).pin_memory().numpy()
    chunk = count * (FFTPOINT // 2)
    calls = samples // chunk
    d = Dedisperser(BW, dms, F0, FFTPOINT, count=count, precision=args.precision)
    import shutil
    need = 2 * n_dm * samples * 4
    tmpdir = None  # the system's temporary directory, or shared memory when it has room
    if os.path.isdir("/dev/shm") and shutil.disk_usage("/dev/shm").free > need:
        tmpdir = "/dev/shm"
    res = {}
    for mode in ("compute", "file"):
        times = []
        for step in range(args.warmup + args.steps):
            fd, path = _tf.mkstemp(suffix=".bin", dir=tmpdir)
            os.close(fd)
            w = SeriesWriter(d, path, kind="uint16", depth=4, threads=4) if mode == "file" else None
            torch.cuda.synchronize()
            t = time.perf_counter()
            for c in range(calls):
                d.filter_block(xh[c * chunk:(c + 1) * chunk])
                if w:
                    w.push()
            nbytes = w.close() if w else 0
            d.synchronize()
            el = time.perf_counter() - t
            os.unlink(path)
            if step >= args.warmup:
                times.append(el)
        s_ = statistics.median(times)
        res[mode] = {"s_per_step": s_, "value": n_dm * samples / s_ / 1e6,
                     "write_gbs": (nbytes / s_ / 1e9) if mode == "file" else None}
    d.close()
    line = {"workload": "stream to file: 16 MHz @ 1250 MHz, 2^%d complex64 samples from pinned host memory in "
                        "calls of %d blocks, %d trials 0-100, FFT %d, every trial's series as uint16 to %s"
                        % (int(math.log2(samples)), count, n_dm, FFTPOINT, tmpdir or "the temp directory"),
            "unit": UNIT, "precision": args.precision, "steps": args.steps, "warmup": args.warmup,
            "bytes_per_step": n_dm * samples * 4, "compute_only": res["compute"], "with_file": res["file"],
            "file_vs_compute": res["file"]["value"] / res["compute"]["value"],
            "method": "wall clock around the calls of one step and the writer's close (all bytes on file)"}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# learned DM proposal: train on simulated pulsars, judge with the full sweep
# ---------------------------------------------------------------------------

def dm_proposal_rows(net, band, n, seed, windows):
    """Searches n observations (half noise only) the three ways: the network's
    logit and offset, and for every pulsar the exhaustive fine sweep (the
    judge) and the fine trials of each window."""
    import torch
    from msosm_gpu_b200 import dm_proposal as P
    from msosm_gpu_b200.simulator import pulsar_baseband
    fine_step = band.dm_max / 4095
    cs = band.dm_max / (band.coarse - 1)
    rng = np.random.default_rng(seed)
    rows = []
    for i in range(n):
        p = P.draw_pulsar(rng, band)
        pulsar = rng.random() >= 0.5
        x = pulsar_baseband(band.samples, band.bw, band.f0, p["dm"], p["period"], p["duty"],
                            p["snr"] if pulsar else 0.0, seed=int(rng.integers(1 << 62)), device=torch.device("cuda"))
        prof = P.fold_trials(x, band, band.coarse_dms, p["period"])
        xin = P.normalise(prof)[None]
        if xin.shape[2] < band.nbins:
            xin = np.repeat(xin, -(-band.nbins // xin.shape[2]), axis=2)[:, :, :band.nbins]
        lg, of = net.forward(np.ascontiguousarray(xin))
        k = P.coarse_peak(prof, p["duty"])
        centres = {"base": k * cs, "net": (k + float(of[0])) * cs}
        r = dict(p, pulsar=bool(pulsar), logit=float(lg[0]), offset=float(of[0]), coarse_peak=k * cs)
        for name, (c, hw) in windows.items():
            lo, hi = max(0.0, centres[c] - hw * cs), min(band.dm_max, centres[c] + hw * cs)
            r[name + "_trials"] = int(np.floor((hi - lo) / fine_step)) + 1
        if pulsar:
            dms, snr = P.fine_search(x, band, p["period"], p["duty"], 0.0, band.dm_max, fine_step)
            r["sweep_snr"], r["sweep_dm"] = float(snr.max()), float(dms[int(np.argmax(snr))])
            for name, (c, hw) in windows.items():
                wd, ws = P.fine_search(x, band, p["period"], p["duty"], centres[c] - hw * cs, centres[c] + hw * cs,
                                       fine_step)
                r[name + "_snr"] = float(ws.max()) if ws.size else 0.0
                r[name + "_found"] = bool(r[name + "_snr"] >= 0.9 * r["sweep_snr"])
        rows.append(r)
        del x
    return rows


def run_dm_proposal(args):
    """Config 5: a 32 MHz band at 1400 MHz, 2^24 samples per observation,
    DM 0-500, period log-uniform 1 ms - 1 s, duty cycle 1-10 %, peak SNR
    0.01-0.2, half the observations noise only; 64 coarse trials folded to
    256 bins feed the network.  Three disjoint sets of seeded observations:
    training, calibration (the detection threshold is fixed here) and test
    (reported).  Each searched observation gets the exhaustive fine sweep
    (4096 trials over 0-500, the judge) for its pulsar; the method without
    the network searches fine trials in a window around the coarse trial of
    highest S/N in every observation; with the network, only observations
    whose logit passes the threshold are searched, around the coarse peak
    moved by the predicted offset.  A pulsar counts as found when the window
    recovers >= 90 % of the sweep's best S/N."""
    from msosm_gpu_b200 import dm_proposal as P
    band = P.Band()
    t = time.time()
    X, lab, tgt, meta = P.simulate_profiles(args.train, band, seed=1)
    gen_s = time.time() - t
    log(f"training set: {args.train} samples in {gen_s:.1f} s ({gen_s / max(args.train, 1) * 1e3:.1f} ms each)")
    net = P.DMProposalNet(band.coarse, band.nbins, 32, 7, 4, max_batch=256, dm_weight=0.25, seed=0)
    t = time.time()
    hist = P.train(net, X, lab, tgt, epochs=args.epochs, batch=256, lr=2e-3, log=log)
    train_s = time.time() - t
    del X
    windows = {"base2": ("base", 2.0), "net2": ("net", 2.0), "net1": ("net", 1.0)}
    t = time.time()
    calib = dm_proposal_rows(net, band, args.calib, 7, windows)
    test = dm_proposal_rows(net, band, args.eval, 11, windows)
    eval_s = time.time() - t
    P.release_handles()

    def detected(rows):
        return [r for r in rows if r["pulsar"] and r["sweep_snr"] >= args.snr_min]

    # the detection threshold, fixed on the calibration set: 0.5 below the
    # lowest logit of a calibration pulsar that the sweep detects and the
    # network's +-2-step window finds (so every such pulsar passes), and
    # never above 0
    cal_found = [r["logit"] for r in detected(calib) if r["net2_found"]]
    tau = min(0.0, min(cal_found) - 0.5) if cal_found else 0.0

    def summary(rows, tau_):
        det = detected(rows)
        gate = lambda r: r["logit"] > tau_  # noqa: E731
        out = {}
        for key, name, use_gate in (("without_network_2steps", "base2", False), ("network_2steps", "net2", True),
                                    ("network_1step", "net1", True)):
            rec = (sum(1 for r in det if r[name + "_found"] and (not use_gate or gate(r))) / len(det)) if det else None
            tr = band.coarse + float(np.mean([r[name + "_trials"] if (not use_gate or gate(r)) else 0 for r in rows]))
            out[key] = {"recall": rec, "trials": tr, "reduction_vs_exhaustive": 4096.0 / tr}
        noise = [r for r in rows if not r["pulsar"]]
        out["noise_flagged"] = (sum(1 for r in noise if gate(r)) / len(noise)) if noise else None
        out["pulsars"] = sum(1 for r in rows if r["pulsar"])
        out["detected_by_sweep"] = len(det)
        out["observations"] = len(rows)
        return out

    line = {"workload": "learned DM proposal: 32 MHz at 1400 MHz, 2^24 samples per observation, DM 0-500, period "
                        "1 ms-1 s, duty 1-10 %, peak SNR 0.01-0.2, half noise only; 64 coarse trials x 256 bins",
            "network": "4 circular conv1d layers (32 channels, kernel 7, ReLU), mean over phase, detection and "
                       "DM-offset heads; bf16 weights, FP32 accumulation; msosm_cnn_* kernels, Adam",
            "train_samples": args.train, "calibration_observations": args.calib, "test_observations": args.eval,
            "noise_fraction": 0.5, "epochs": args.epochs,
            "training_set_seconds": gen_s, "training_seconds": train_s, "search_seconds": eval_s,
            "loss_first_last": [hist[0], hist[-1]] if hist else None, "snr_min": args.snr_min,
            "threshold": {"logit": tau, "rule": "0.5 below the lowest logit among calibration pulsars the sweep "
                                                "detects and the +-2-step network window finds, capped at 0; "
                                                "chosen on the calibration set only"},
            "test": summary(test, tau), "test_at_logit_0": summary(test, 0.0), "calibration": summary(calib, tau),
            "exhaustive_trials": 4096,
            "rule": "a pulsar is found when its fine window recovers >= 90 % of the exhaustive sweep's best S/N; "
                    "recall over the pulsars the sweep detects (S/N >= snr_min); trials per observation include "
                    "the 64 coarse ones",
            "rows": {"calibration": calib, "test": test}}
    print(json.dumps(line), flush=True)
    net.close()


# ---------------------------------------------------------------------------
# single DM: one trial through MS-OSM (FFT 4096) and OSM (FFT 2^18)
# ---------------------------------------------------------------------------

SINGLE = dict(bw=16e6, f0=1242e6, log2_samples=24, fftpoint=4096, osm_fftpoint=1 << 18, nbins=1024,
              pulsar=dict(dm=50.0, period=5e-3, fwhm=0.02, snr=0.1), seed=0, call_log2=21, u16_scale=1000.0)


def run_single_dm(args):
    """One DM trial (16 MHz at 1250 MHz, 2^24 samples, pulsar P = 5 ms, 2 %
    FWHM, peak SNR 0.1, DM 50, seed 0) through the MS-OSM path at FFT 4096
    (FP32 and f16 tensor cores) and the OSM path at FFT 2^18, each folded
    into 1024 bins; the same uint16 input through the reference's own
    MSOSM_GPU_BATCH and OSM_GPU_BATCH (cuFFT, built for sm_100a) on the same
    GPU, timed its own way; every series and profile against the FP64
    oracle over the whole signal."""
    import torch
    from msosm_gpu_b200 import Dedisperser, simulate as S, simulator as G
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    c = SINGLE
    p = c["pulsar"]
    bw, f0, nb = c["bw"], c["f0"], c["nbins"]
    samples = 1 << (args.log2_samples or c["log2_samples"])
    call = min(samples, 1 << c["call_log2"])
    ncalls = samples // call
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    t = time.time()
    x = G.pulsar_baseband(samples, bw, f0, p["dm"], p["period"], p["fwhm"], p["snr"], seed=c["seed"])
    u = S.quantise_uint16(x, c["u16_scale"])
    log(f"signal: {samples} samples in {time.time() - t:.1f} s, quantised to offset-binary uint16 "
        f"({c['u16_scale']:.0f} counts per unit)")
    ud = torch.from_numpy(u.view(np.int32).reshape(-1)).to(dev)
    uh = torch.from_numpy(u.view(np.int32).reshape(-1)).pin_memory().numpy().view(np.uint16).reshape(-1, 2)
    peaks, peaks_src = load_peaks()
    hbm = peaks["hbm_gbs"]
    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        pass
    nd = O.nd(bw, p["dm"], f0)
    paths = {"msosm_fp32": dict(fftpoint=c["fftpoint"], osm=False, precision="fp32"),
             "msosm_fp16": dict(fftpoint=c["fftpoint"], osm=False, precision="fp16"),
             "osm_fp32": dict(fftpoint=c["osm_fftpoint"], osm=True, precision="fp32")}

    def handle(kw, count, series, fold=True):
        d = Dedisperser(bw, [p["dm"]], f0, kw["fftpoint"], count=count, osm=kw["osm"], series=series,
                        precision=kw["precision"])
        if fold:
            d.fold_init(p["period"], bw, time_bin=nb, discard_Nd=nd, detect="power")
        return d

    out = {}
    series_of = {}
    for name, kw in paths.items():
        M = kw["fftpoint"] // 2
        # device value: input resident, the whole signal in one call per step
        # (series materialised and folded)
        stream = torch.cuda.Stream(dev)
        d = handle(kw, samples // M, True)
        d.set_stream(stream)
        for _ in range(args.warmup):
            d.filter_block(ud)
        torch.cuda.synchronize()
        d.enable_timing(True)
        with ClockSampler(uuid) as ck:
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                s.record(stream)
                for _ in range(args.steps):
                    d.filter_block(ud)
                e.record(stream)
            torch.cuda.synchronize()
        ms = s.elapsed_time(e) / args.steps
        tm = d.timing()
        d.close()
        k = max(tm["calls"], 1)
        st = {"forward": tm["forward_ms"] / k, "dedisp": tm["dedisp_ms"] / k, "fold": tm["fold_ms"] / k}
        # algorithmic bytes: uint16 input read once, complex64 series written once
        algo = 12.0 * samples
        kern_ms = st["forward"] + st["dedisp"]
        # e2e through the C ABI from pinned host memory, calls of 2^21 samples:
        # (a) fold only, the profile read back; (b) as the reference's drivers,
        # every call's series copied back to pinned host memory
        de = handle(kw, call // M, False)
        ds = handle(kw, call // M, True)
        # the timed series arm does what the reference's drivers do per call
        # (filter, copy the series back) and no fold
        dsn = handle(kw, call // M, True, fold=False)
        ser = np.empty(call + 1, np.complex64)
        ser = torch.from_numpy(ser.view(np.float32)).pin_memory().numpy().view(np.complex64)
        keep = []

        def e2e_fold():
            for i in range(ncalls):
                de.filter_block(uh[i * call:(i + 1) * call])
            return de.get_profiles()

        def e2e_series(collect=False):
            h = ds if collect else dsn
            for i in range(ncalls):
                h.filter_block(uh[i * call:(i + 1) * call])
                h.get_output(out=ser)
                if collect:
                    keep.append(ser[:-1].copy())

        e2e_series(collect=True)
        series_of[name] = (np.concatenate(keep), ds.get_profiles()[0].copy())
        res = {}
        for key, fn in (("fold", e2e_fold), ("series", e2e_series)):
            for _ in range(args.warmup):
                fn()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(args.steps):
                fn()
            torch.cuda.synchronize()
            res[key] = (time.perf_counter() - t0) / args.steps
        de.close()
        ds.close()
        dsn.close()
        out[name] = {
            "value": samples / (ms * 1e-3) / 1e6, "ms_per_step": ms, "unit": "Msamples/s (1 DM trial)",
            "fftpoint": kw["fftpoint"], "precision": kw["precision"], "clocks": ck.summary(),
            "stage_ms_per_step": st,
            "roofline": {"bound": "hbm", "algorithmic_bytes_per_step": algo,
                         "achieved": algo / (kern_ms * 1e-3) / 1e9, "peak": hbm, "unit": "GB/s",
                         "peak_source": peaks_src,
                         "frac": (algo / (kern_ms * 1e-3) / 1e9 / hbm) if hbm else None,
                         "kernels": "forward + dedispersion kernels (uint16 input read, series written)"},
            "e2e": {"value": samples / res["fold"] / 1e6, "unit": "Msamples/s (1 DM trial)",
                    "ms_per_step": res["fold"] * 1e3, "h2d_bytes_per_step": int(u.nbytes),
                    "d2h_bytes_per_step": nb * 4, "calls_per_step": ncalls},
            "e2e_series": {"value": samples / res["series"] / 1e6, "unit": "Msamples/s (1 DM trial)",
                           "ms_per_step": res["series"] * 1e3, "h2d_bytes_per_step": int(u.nbytes),
                           "d2h_bytes_per_step": 8 * samples, "calls_per_step": ncalls}}
        log(f"{name}: device {out[name]['value']:.0f} Msamples/s, e2e fold {out[name]['e2e']['value']:.0f}, "
            f"e2e series {out[name]['e2e_series']['value']:.0f}")

    # ---- errors against the FP64 oracle over the whole signal -------------
    xin = O.decode_uint16(u)
    for name, kw in paths.items():
        M = kw["fftpoint"] // 2
        o = O.Dedisp(bw, [p["dm"]], f0, kw["fftpoint"], call // M, osm=kw["osm"])
        f = O.Fold(p["period"], bw, call, nb)
        f.discard_samples(nd)
        y, e2, r2 = [], 0.0, 0.0
        ours, prof = series_of[name]
        for i in range(ncalls):
            yi = o.filter(xin[i * call:(i + 1) * call])[0]
            f.fold_data(np.abs(yi) ** 2)
            e2 += float(np.sum(np.abs(ours[i * call:(i + 1) * call] - yi) ** 2))
            r2 += float(np.sum(np.abs(yi) ** 2))
        pr = f.fold_data_bins()
        out[name]["accuracy_vs_fp64"] = {
            "series_rel_rms": math.sqrt(e2 / r2),
            "profile_rel_rms": float(np.sqrt(np.sum((prof - pr) ** 2) / np.sum(pr ** 2))),
            "sample": f"the whole signal ({samples} samples), FP64 oracle (oracle/orc.c)"}
        snr_w = max(1, int(round(p["fwhm"] * nb)))
        out[name]["profile_snr"] = profile_snr(prof, snr_w)

    # ---- the reference's own single-DM classes on the same GPU and input ---
    ref = {"unavailable": "oracle/_ref/ref_gpu_runner not built"}
    if os.path.exists(O.REF_GPU_RUNNER):
        ref = {}
        with tempfile.TemporaryDirectory() as td:
            fin, fout = os.path.join(td, "in.u16"), os.path.join(td, "out.bin")
            u.tofile(fin)
            for name, kind, fp in (("msosm_gpu_batch", "batch", c["fftpoint"]),
                                   ("osm_gpu_batch", "osm", c["osm_fftpoint"])):
                M = fp // 2
                cmd = [O.REF_GPU_RUNNER, "time1", kind, str(fp), str(call // M), str(ncalls),
                       str(max(args.steps, 1)), str(bw), repr(float(p["dm"])), str(f0), fin, fout, "1"]
                r = subprocess.run(cmd, capture_output=True, text=True, timeout=1800)
                if r.returncode != 0:
                    ref[name] = {"unavailable": f"runner exit {r.returncode}: {r.stderr[-300:]}"}
                    continue
                rr = O.read_records(fout)
                rms = float(np.median(rr["ms"]))
                ys = rr["out"].astype(np.float64).view(np.complex128)
                ref[name] = {"e2e": samples / (rms * 1e-3) / 1e6, "unit": "Msamples/s (1 DM trial)",
                             "ms_per_step": rms, "count": call // M, "calls_per_step": ncalls,
                             "method": "std::chrono around filter_block_uint16 + get_output(Complex*) per call "
                                       "and a final synchronize, input and output cudaHostRegister'ed (the "
                                       "reference's single-DM speed tests)"}
                for ours_name in (("msosm_fp32", "msosm_fp16") if kind == "batch" else ("osm_fp32",)):
                    a = series_of[ours_name][0].astype(np.complex128)
                    ref[name]["series_rel_rms_vs_" + ours_name] = float(
                        np.sqrt(np.sum(np.abs(a - ys) ** 2) / np.sum(np.abs(ys) ** 2)))
    line = {"workload": "single-dm", "metric": "Msamples/s of one DM trial (MS-OSM FFT 4096, OSM FFT 2^18, "
                                               "|y|^2 folded to 1024 bins), 1 B200",
            "unit": "Msamples/s", "higher_is_better": True, "steps": args.steps, "warmup": args.warmup,
            "data": "synthetic (seeded pulsar + AWGN from the device simulator, quantised to uint16)",
            "config": {"workload": "single DM: 16 MHz @ 1250 MHz, 2^%d samples, pulsar P 5 ms, FWHM 2 %%, "
                                   "peak SNR 0.1, DM 50, seed 0" % int(math.log2(samples)),
                       "Nd": nd, "delaycount_fft4096": int(O.segmentation(bw, p["dm"], f0, c["fftpoint"] // 2)[0]),
                       "call_samples": call, "fold_bins": nb, "input": "uint16 offset binary"},
            "paths": out, "reference_gpu": ref}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# reference arms
# ---------------------------------------------------------------------------

def run_reference(args):
    ws, rank, _ = dist_setup()
    if rank != 0:
        return
    samples = 1 << args.log2_samples
    dms = dm_trials(0, args.dms)
    x = make_signal(min(samples, 1 << 22), on_gpu=False)
    vals, cb = [], None
    for _ in range(args.warmup + args.steps):
        cb = cpu_baseline(dms, x, budget_s=max(2.0, 60.0 / max(args.steps, 1)))
        vals.append(cb["value"])
    vals = vals[args.warmup:] or vals
    v = statistics.median(vals)
    cb["value"] = v
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded pulsar + AWGN)",
            "config": workload_config(samples, args.dms, ws), "cpu_baseline": cb,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def reference_gpu_measure(samples, n_dm, steps, sweep=False, x=None, with_series=True):
    """The reference's own MSOSM_GPU_DM_concurrent (cuFFT + its kernels,
    built for sm_100a into oracle/_ref/ref_gpu_runner) on this GPU, timed its
    own way: the batched workload in calls of 32 blocks, or with `sweep` the
    precision sweep's 64 MHz / FFT 8192 / DM 0-200 observation in calls of 8
    blocks (the count its ring allows at that depth).  Trials (0, dm_max]:
    the reference leaves its delays uninitialised at DM 0.  Returns a dict
    (or one with "unavailable")."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    if not os.path.exists(O.REF_GPU_RUNNER):
        return {"unavailable": "oracle/_ref/ref_gpu_runner not built"}
    from msosm_gpu_b200 import simulate as S
    if sweep:
        bw, f0, fftpoint, dm_max, count, pul = (SWEEP["bw"], SWEEP["f0"], SWEEP["fftpoint"], SWEEP["dm_max"], 8,
                                                SWEEP["pulsar"])
    else:
        bw, f0, fftpoint, dm_max, count, pul = BW, F0, FFTPOINT, DM_MAX, 32, PULSAR
    dms = ((np.arange(n_dm) + 1) * dm_max / n_dm).astype(np.float32)
    if x is None:
        if sweep:
            x = S.pulsar_baseband(samples, bw, f0, pul["dm"], pul["period"], pul["fwhm"], pul["snr"], seed=0)
        else:
            x = make_signal(samples, on_gpu=False)
    u = S.quantise_uint16(x, 1000.0)
    ncalls = samples // (count * fftpoint // 2)
    res = {}
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "in.u16"), os.path.join(td, "out.bin")
        u.tofile(fin)
        del u
        for with_out in ((0, 1) if with_series else (0,)):
            cmd = [O.REF_GPU_RUNNER, "time", str(fftpoint), str(count), str(ncalls), str(max(steps, 1)),
                   str(with_out), str(bw), str(f0), fin, fout] + [repr(float(v)) for v in dms]
            r = subprocess.run(cmd, capture_output=True, text=True, timeout=1800)
            if r.returncode != 0:
                return {"unavailable": f"runner exit {r.returncode}: {r.stderr[-300:]}"}
            res[with_out] = float(np.median(O.read_records(fout)["ms"]))
    units = float(n_dm) * samples
    out = {"value": units / (res[0] * 1e-3) / 1e6, "unit": UNIT, "ms_per_step": res[0], "steps": steps,
           "dm_range": [float(dms[0]), dm_max], "count": count, "fftpoint": fftpoint,
           "input": "uint16 offset binary (the reference API), pinned host memory",
           "method": "reference MSOSM_GPU_DM_concurrent (cuFFT + its kernels, sm_100a), std::chrono around "
                     "the filter_block_uint16 loop + synchronize, pinned host input (its own drivers' "
                     "method); host copies included; no folding (the reference has none for this class)"}
    if 1 in res:
        out["value_with_series_d2h"] = units / (res[1] * 1e-3) / 1e6
        out["ms_per_step_with_series_d2h"] = res[1]
    return out


def run_reference_gpu(args, sweep=False):
    """`--impl reference-gpu`: reference_gpu_measure as its own line."""
    ws, rank, _ = dist_setup()
    if rank != 0:
        return
    samples = 1 << args.log2_samples
    m = reference_gpu_measure(samples, args.dms, args.steps, sweep=sweep)
    if "unavailable" in m:
        print(json.dumps({"impl": "reference-gpu", "unavailable": m["unavailable"]}))
        return
    metric = ("DM-trial x Msamples/s (MS-OSM dedispersion, FFT %d, %d trials, 64 MHz precision-sweep "
              "observation), 1 B200" % (SWEEP["fftpoint"], args.dms)) if sweep else METRIC
    cfg = (dict(workload="precision-sweep observation: 64 MHz at 1400 MHz, 2^%d samples, %d DM trials, FFT %d"
                         % (args.log2_samples, args.dms, SWEEP["fftpoint"]), samples_per_step=samples)
           if sweep else dict(workload_config(samples, args.dms, 1)))
    print(json.dumps(dict({"impl": "reference-gpu", "metric": metric, "config": cfg}, **m)), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference", "reference-gpu"])
    ap.add_argument("--log2-samples", type=int, default=None, help="default 26 for both workloads")
    ap.add_argument("--dms", type=int, default=None, help="default 256 (batched) or 1024 (precision-sweep)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip the reference's cuFFT path in the default arm's line")
    ap.add_argument("--precision", default="fp16", choices=["fp32", "fp16", "bf16"],
                    help="inverse transforms on the CUDA cores (fp32) or the tensor cores (fp16, bf16)")
    ap.add_argument("--workload", default="batched",
                    choices=["batched", "precision-sweep", "uneven-batch", "stream-to-file", "dm-proposal",
                             "single-dm"],
                    help="batched: the 256-trial 16 MHz workload (the bench line); precision-sweep: the "
                         "64 MHz / FFT 8192 / 1024-trial sweep of the inverse-transform precisions; "
                         "uneven-batch: 64 independent observations, autotuned vs fixed configurations; "
                         "stream-to-file: host input in, every trial's uint16 series written to a file; "
                         "dm-proposal: the learned coarse-DM proposal against the exhaustive fine sweep; "
                         "single-dm: one trial through MS-OSM (FFT 4096) and OSM (FFT 2^18) beside the "
                         "reference's single-DM classes")
    ap.add_argument("--train", type=int, default=20000, help="dm-proposal: training samples")
    ap.add_argument("--epochs", type=int, default=40, help="dm-proposal: training epochs")
    ap.add_argument("--eval", type=int, default=256, help="dm-proposal: test observations (half noise)")
    ap.add_argument("--calib", type=int, default=256,
                    help="dm-proposal: calibration observations (half noise) that fix the detection threshold")
    ap.add_argument("--snr-min", type=float, default=8.0, help="dm-proposal: sweep detection threshold")
    ap.add_argument("--obs", type=int, default=UNEVEN["n_obs"], help="uneven-batch: observations")
    ap.add_argument("--min-coherence", type=float, default=None,
                    help="uneven-batch: the autotuner's floor on MS-OSM coherence with exact dedispersion")
    ap.add_argument("--seeds", type=int, default=SWEEP["seeds"], help="precision-sweep: signal seeds")
    ap.add_argument("--fftpoint", type=int, default=None, choices=[4096, 8192, 16384],
                    help="precision-sweep: FFT size (default 8192; each of these runs on the tensor cores)")
    args = ap.parse_args()
    if args.fftpoint:
        if args.workload != "precision-sweep":
            ap.error("--fftpoint applies to the precision-sweep workload")
        SWEEP["fftpoint"] = args.fftpoint
    if args.workload == "precision-sweep" and args.impl == "reference-gpu":
        args.log2_samples = args.log2_samples or SWEEP["log2_samples"]
        args.dms = args.dms or SWEEP["n_dm"]
        run_reference_gpu(args, sweep=True)
        return
    if args.workload != "batched":
        if args.impl != "ours":
            print(json.dumps({"impl": args.impl, "unavailable": f"the {args.workload} workload has no "
                              "reference arm"}))
            return
        {"precision-sweep": run_precision_sweep, "uneven-batch": run_uneven_batch,
         "stream-to-file": run_stream_to_file, "dm-proposal": run_dm_proposal,
         "single-dm": run_single_dm}[args.workload](args)
        return
    args.log2_samples = args.log2_samples or LOG2_SAMPLES
    args.dms = args.dms or N_DM
    if args.impl == "reference":
        run_reference(args)
    elif args.impl == "reference-gpu":
        run_reference_gpu(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
