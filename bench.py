"""Throughput benchmark of the B200 WiMAX LDPC decoder (one JSON line on rank 0).

Metric: info Gbit/s at FER <= 1e-3, rate 1/2, z = 96 (n = 2304, k = 1152), on
seeded synthetic frames (random info bits, the project's encoder, BPSK, AWGN,
LLR = 2y/sigma^2) generated on the device at Eb/N0 = 2.25 dB, where the plain
normalized min-sum decoder with the reference's cap of 10 iterations has
FER <= 1e-3. A step decodes one batch of 262144 frames (2.4 GB of float32 LLRs,
larger than L2, so no flush is needed between steps). All decoders run on the
same frames: the plain (bit-exact) decoder and the learned min-sum decoder
(8 trained iterations in fp32, run to the same cap of 10 with the last trained
weights), plus the same network in packed binary16 (two frames per thread) as
an extra. `value` is the fp32 learned decoder's when its FER meets the target
and is no worse than the plain decoder's, else the plain one's.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

  value      kernel-only info Gbit/s, LLRs resident in HBM
  e2e        the same metric through the headline decoder's C ABI host call
             (wldpc_lms_decode_host, or wldpc_decode_batch_host for the plain
             one): pinned host LLRs in, posterior + hard bits + status back,
             as the reference's decode(float*) returns them; every decoder
             also reports its own e2e, with and without the posterior
  roofline   the decode kernel against the measured HBM copy bandwidth, and
             the issue-slot roofline that actually binds it
  decoders.*.with_posterior  each decoder again with the float32 posterior
             written back (9n bytes per frame instead of 5n)
  cpu_baseline  the reference's own OpenMP decoder (compiled from its sources)
             on this machine's host cores, on a bounded sample of the workload
  config1    rate 5/6 z=96, 262144 frames at 4 dB, the three decoders
  config2    131072 frames mixed over all 114 codes, one graph launch
  encoder    the dual-diagonal encoder on the headline batch
  single_frame  decode(float*) and BER_runner::run_iteration, one frame per
             call, next to the reference on one core
  waterfall  rate 1/2 z=96 BER/FER sweep (0.1 dB steps, >= 200 bit errors per
             point) with the plain and the fp32 learned decoder: Eb/N0 at BER 1e-5

Multi-GPU: every rank decodes its own shard of frames (weak scaling, no
data-path collective); timing is the max over ranks, counters are summed.
Without torchrun, --gpus N > 1 starts the N ranks itself through
torch.distributed.run. --dry-run --backend gloo runs the rank set-up and the
reductions on CPU with stand-in timings (no GPU, no kernels).
"""
from __future__ import annotations

import argparse
import json
import os
import socket
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "info Gbit/s at FER<=1e-3, learned vs plain min-sum, 1 B200, r1/2 z=96"
RATE, Z = 0, 96
N_BITS, K_BITS = 24 * Z, 12 * Z
FRAMES = 262144
EBNO_DB = 2.25
MAX_ITER = 10
SEED = 20261203
# config 1: the plain decoder's throughput point, rate 5/6 z = 96 at 4 dB
C1_RATE, C1_Z, C1_EBNO = 5, 96, 4.0
C1_K = 20 * C1_Z
# config 2: mixed batch over all 114 codes
MIXED_FRAMES = 131072
WEIGHTS_DIR = os.path.join(ROOT, "wimax_ldpc_lib_b200", "weights")
SECTIONS = ("e2e", "config1", "config2", "encoder", "single_frame", "waterfall")


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def load_profile_value(name, key):
    """a figure recorded from an ncu capture (profiles/<name>, line "key: value ...")."""
    p = os.path.join(ROOT, "profiles", name)
    try:
        for line in open(p):
            if line.startswith(key + ":"):
                return float(line.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
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
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ ranks

def free_port():
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def launch_ranks(args) -> int:
    """--gpus N > 1 without torchrun: start N ranks of this script through
    torch.distributed.run (one process per GPU) and return its exit code."""
    if not args.dry_run and args.impl == "ours":
        import torch
        visible = torch.cuda.device_count()
        if args.gpus > visible:
            print(f"bench.py: --gpus {args.gpus} but only {visible} CUDA device(s) are visible", file=sys.stderr)
            return 2
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
           "--master-addr=127.0.0.1", f"--master-port={free_port()}", os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def dist_setup(backend="nccl"):
    import torch
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        if backend == "nccl":
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    elif backend == "nccl" and torch.cuda.is_available():
        torch.cuda.set_device(local)
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def reduce_step(ms, counters, ws, device):
    """max of the per-rank step time and sum of the per-rank counters; every
    rank calls this at the same point with the same number of counters"""
    import torch
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    c = torch.tensor(counters, dtype=torch.float64, device=device)
    if ws > 1:
        import torch.distributed as dist
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        if counters:
            dist.all_reduce(c)
    return float(t.item()), [float(x) for x in c.tolist()]


def timed_steps(launch, steps, warmup, stream, ws):
    """W untimed launches, then K launches between CUDA events on `stream`,
    bracketed by a barrier and a device synchronize on both sides; returns
    ms per step on this rank"""
    import torch
    for _ in range(warmup):
        launch()
    torch.cuda.synchronize()
    barrier(ws)
    torch.cuda.synchronize()
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(steps):
        launch()
    stop.record(stream)
    torch.cuda.synchronize()
    barrier(ws)
    return start.elapsed_time(stop) / steps


# ---------------------------------------------------------- reference arm

def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_reference_baseline(llr_host, rate=RATE, z=Z, k=K_BITS, seconds=12.0, threads=None):
    """The reference decoder (oracle/_ref, its own sources) with one decoder
    object per OpenMP thread over frames, on a bounded sample of the frames:
    passes over the sample repeat until about `seconds` of CPU work is done."""
    from oracle.oracle import Reference, reference_available
    if not reference_available():
        return None
    ref = Reference()
    threads = threads or os.cpu_count() or 1
    sample = llr_host.shape[0]
    ref.decode(rate, z, llr_host[: min(sample, 4 * threads)], MAX_ITER, threads=threads)
    done, t0 = 0, time.perf_counter()
    while True:
        ref.decode(rate, z, llr_host, MAX_ITER, threads=threads)
        done += sample
        dt = time.perf_counter() - t0
        if dt >= seconds:
            break
    return {"value": done * k / dt / 1e9, "unit": "info Gbit/s", "cores": threads, "kind": "reference",
            "sample": f"{done} frame decodes ({done // sample} passes over the first {sample} frames of the "
                      f"workload), {dt:.1f} s, cap {MAX_ITER}, one decoder per OpenMP thread",
            "cpu": cpu_model()}


def run_reference(args):
    """--impl reference: the reference's CPU decoder on this machine's cores,
    same workload, metric and unit; rank 0 only."""
    import numpy as np
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle.oracle import Oracle, Reference, reference_available
    if not reference_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (reference sources absent)"}))
        return
    threads = os.cpu_count() or 1
    oracle = Oracle()
    ref = Reference()
    # a bounded sample of the same workload: frames per step sized so that the
    # whole run stays within a few minutes
    per_step = max(threads * 16, 2048)
    _, cw, llr, _ = oracle.framegen(RATE, Z, SEED, 0, per_step, EBNO_DB)
    llr = llr.astype(np.float32)
    info = cw[:, :K_BITS]
    for _ in range(args.warmup):
        ref.decode(RATE, Z, llr[: max(threads, 64)], MAX_ITER, threads=threads)
    times, ferr = [], 0
    for _ in range(args.steps):
        t = time.perf_counter()
        _, dec, _ = ref.decode(RATE, Z, llr, MAX_ITER, threads=threads)
        times.append(time.perf_counter() - t)
        ferr += int((dec[:, :K_BITS] != info).any(axis=1).sum())
    total = sum(times)
    value = args.steps * per_step * K_BITS / total / 1e9
    line = {"metric": METRIC, "value": value, "unit": "info Gbit/s", "n_gpus": 0, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": f"plain NMS decode, rate 1/2 z=96, Eb/N0 {EBNO_DB} dB, cap {MAX_ITER}",
                       "frames_per_step": per_step, "decoder": "reference ldpc_decoder::decode (OpenMP)"},
            "fer": ferr / (args.steps * per_step),
            "cpu_baseline": {"value": value, "unit": "info Gbit/s", "cores": threads, "kind": "reference",
                             "sample": f"{per_step} frames per step", "cpu": cpu_model()},
            "e2e": {"value": value, "unit": "info Gbit/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ---------------------------------------------------------------- our arm

def load_weights(rate, z):
    import numpy as np
    p = os.path.join(WEIGHTS_DIR, f"lms_r{rate}_z{z}_T8.json")
    if not os.path.exists(p):
        return None, None
    with open(p) as f:
        meta = json.load(f)
    return meta, np.array(meta["weights"], np.float32)


def make_decoders(wl, rate, z, with_learned=True):
    """plain (bit-exact NMS), learned fp32 and learned packed binary16, all at cap 10"""
    decs = {"plain": wl.Decoder(rate, z, MAX_ITER)}
    meta, w = load_weights(rate, z) if with_learned else (None, None)
    if meta is not None:
        decs["learned"] = wl.LearnedDecoder(rate, z, meta["iterations"], weights=w, cap=MAX_ITER)
        decs["learned_f16x2"] = wl.LearnedDecoder(rate, z, meta["iterations"], weights=w, cap=MAX_ITER,
                                                  precision=wl.LMS_F16X2)
    return decs, meta


KERNELS = {"plain": "tdmp_decode_kernel<{r},{z},NMS>", "learned": "lms_decode_kernel<{r},{z}>",
           "learned_f16x2": "lms16_decode_kernel<{r},{z}>"}
PROFILES = {"plain": "tdmp_nms_r{r}_z{z}.txt", "learned": "lms_r{r}_z{z}.txt", "learned_f16x2": "lms16_r{r}_z{z}.txt"}
DTYPES = {"plain": "f32+f64", "learned": "f32", "learned_f16x2": "f16x2"}


def issue_roofline(profile, frames, ms, clocks, sms):
    """warp-instructions per frame (ncu, same workload) x frames per launch /
    launch time, against 4 issue slots per SM per cycle at the sampled clock"""
    ipf = load_profile_value(profile, "warp_instructions_per_frame")
    if not ipf or not clocks.get("sm_mhz"):
        return None
    ach = ipf * frames / (ms * 1e-3)
    pk = sms * 4 * clocks["sm_mhz"] * 1e6
    return {"bound": "issue", "achieved": ach, "peak": pk, "unit": "warp-instructions/s", "frac": ach / pk,
            "warp_instructions_per_frame": ipf,
            "peak_basis": f"{sms} SMs x 4 schedulers x {clocks['sm_mhz']:.0f} MHz (sampled)"}


def run_dry(args):
    """Rank set-up and reductions only, on CPU (gloo): each rank stands in a
    step time of 1 + rank ms and counters (rank, 1); no GPU, no kernels."""
    ws, rank, _ = dist_setup(args.backend)
    barrier(ws)
    ms, (ferr, frames) = reduce_step(1.0 + rank, [float(rank), 1.0], ws, "cpu")
    barrier(ws)
    if rank == 0:
        print(json.dumps({"metric": METRIC, "dry_run": True, "n_gpus": ws, "backend": args.backend,
                          "ms_per_step": ms, "counters": {"frame_errors": ferr, "ranks": frames},
                          "steps": args.steps, "warmup": args.warmup}))
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_ours(args):
    import numpy as np
    import torch
    import wimax_ldpc_lib_b200 as wl
    wl.lib()                               # fails loudly if the library is missing
    ws, rank, local = dist_setup(args.backend)
    dev = torch.device("cuda", local)
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    frames = args.frames
    n, k = N_BITS, K_BITS
    sections = set(SECTIONS if args.sections == "all" else [s for s in args.sections.split(",") if s])
    peak, peak_kind = load_peaks()

    llr = torch.empty((frames, n), dtype=torch.float32, device=dev)
    info = torch.empty((frames, k), dtype=torch.uint8, device=dev)
    wl.framegen_device(RATE, Z, SEED, rank * frames, frames, EBNO_DB, EBNO_DB, info=info, llr=llr)
    hard = torch.empty((frames, n), dtype=torch.int8, device=dev)
    status = torch.empty(frames, dtype=torch.int32, device=dev)
    stream = torch.cuda.Stream()
    torch.cuda.synchronize()

    decoders, lms_meta = make_decoders(wl, RATE, Z, not args.plain_only)

    def measure(dec, info_t, kbits, nframes):
        ms = timed_steps(lambda: dec.decode_device(llr[:nframes], hard[:nframes], None, status[:nframes],
                                                   stream=stream), args.steps, args.warmup, stream, ws)
        ferr = (hard[:nframes, :kbits].view(torch.uint8) != info_t[:nframes]).any(dim=1).sum().item()
        iters = (status[:nframes] & 0xFFFF).to(torch.float64).sum().item()
        ms, (ferr, iters) = reduce_step(ms, [ferr, iters], ws, dev)
        total = nframes * ws
        return {"value": total * kbits / (ms * 1e-3) / 1e9, "ms_per_step": ms, "fer": ferr / total,
                "frame_errors": int(ferr), "frames": total, "mean_iterations": iters / total}

    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    results = {name: measure(dec, info, k, frames) for name, dec in decoders.items()}
    # the same decodes with the posterior written back as float32 (the
    # reference's decode(float*) leaves it in rx): 9n algorithmic bytes per frame
    post = torch.empty_like(llr)
    for name, dec in decoders.items():
        ms_p = timed_steps(lambda: dec.decode_device(llr, hard, post, status, stream=stream), args.steps,
                           args.warmup, stream, ws)
        ms_p, _ = reduce_step(ms_p, [], ws, dev)
        results[name]["with_posterior"] = {
            "ms_per_step": ms_p, "value": frames * ws * k / (ms_p * 1e-3) / 1e9, "unit": "info Gbit/s",
            "hbm_gbs": frames * 9 * n / (ms_p * 1e-3) / 1e9,
            "note": "float32 posterior written back: 9n bytes per frame (LLR read, posterior and hard bits written)"}
    del post
    clocks = sampler.stop()
    for dec in decoders.values():
        if hasattr(dec, "synchronize"):
            dec.synchronize()

    # the headline decoder: the fp32 learned decoder when it meets the FER
    # target and is no worse than plain, else plain (binary16 is an extra)
    head = "plain"
    L, P = results.get("learned"), results["plain"]
    if L and L["fer"] <= 1e-3 and L["fer"] <= P["fer"]:
        head = "learned"
    R = results[head]
    ms, value = R["ms_per_step"], R["value"]

    # e2e through each decoder's own C ABI host call (pinned host buffers,
    # host<->device copies in the timed region): with the posterior (the
    # reference's decode(float*) semantics) and hard decisions only
    if "e2e" in sections:
        llr_h = torch.empty((frames, n), dtype=torch.float32, pin_memory=True)
        hard_h = torch.empty((frames, n), dtype=torch.int8, pin_memory=True)
        st_h = torch.empty(frames, dtype=torch.int32, pin_memory=True)
        src = llr.cpu()
        e2e_steps = max(1, min(args.steps, 2))

        def host_time(call, refresh):
            if refresh:
                llr_h.copy_(src)
            call()                                             # warm-up
            times = []
            for _ in range(e2e_steps):
                if refresh:
                    llr_h.copy_(src)                           # the decode wrote posteriors back
                torch.cuda.synchronize()
                t = time.perf_counter()
                call()
                times.append(time.perf_counter() - t)
            t_mean, _ = reduce_step(sum(times) / len(times), [], ws, dev)
            return t_mean

        apis = {"plain": ("wldpc_decode_batch_host", "wldpc_decode_batch_host_hard"),
                "learned": ("wldpc_lms_decode_host", "wldpc_lms_decode_host_hard"),
                "learned_f16x2": ("wldpc_lms_decode_host", "wldpc_lms_decode_host_hard")}
        for name, dec in decoders.items():
            t_full = host_time(lambda: dec.decode_host_into(llr_h, hard_h, None, st_h), True)
            llr_h.copy_(src)
            t_hard = host_time(lambda: dec.decode_host_hard_into(llr_h, hard_h, None, st_h), False)
            results[name]["e2e"] = {
                "value": frames * ws * k / t_full / 1e9, "unit": "info Gbit/s",
                "h2d_bytes_per_step": frames * n * 4, "d2h_bytes_per_step": frames * (5 * n + 4),
                "api": apis[name][0] + " (pinned host buffers; posterior, hard bits and status copied back)",
                "timing": f"host wall clock around the synchronous call, mean of {e2e_steps}, max over ranks"}
            results[name]["e2e_hard"] = {
                "value": frames * ws * k / t_hard / 1e9, "unit": "info Gbit/s",
                "h2d_bytes_per_step": frames * n * 4, "d2h_bytes_per_step": frames * (n + 4),
                "api": apis[name][1] + " (pinned host buffers; hard bits and status copied back)"}
        # the headline decoder on pageable buffers, which is what reference callers pass
        pg_llr = src.numpy().copy()
        pg_hard = np.empty((frames, n), np.int8)
        pg_st = np.empty(frames, np.int32)
        dec = decoders[head]

        def pageable_call():
            pg_llr[...] = src.numpy()
            torch.cuda.synchronize()
            t = time.perf_counter()
            dec.decode_host_into(pg_llr, pg_hard, None, pg_st)
            return time.perf_counter() - t
        pageable_call()
        t_pg, _ = reduce_step(pageable_call(), [], ws, dev)
        results[head]["e2e_pageable"] = {"value": frames * ws * k / t_pg / 1e9, "unit": "info Gbit/s",
                                         "api": apis[head][0] + " (pageable numpy buffers)"}
        del llr_h, hard_h, st_h, pg_llr, pg_hard, pg_st
    e2e = results[head].get("e2e")

    bytes_per_launch = frames * 5 * n
    achieved = bytes_per_launch / (ms * 1e-3) / 1e9
    prof = PROFILES[head].format(r=12, z=Z)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": load_profile_value(prof, "traffic_bytes_per_launch_full_batch"), "peak_kind": peak_kind,
                "kernel": KERNELS[head].format(r=RATE, z=Z), "algorithmic_bytes_per_launch": bytes_per_launch,
                "note": "5n bytes per frame (float32 LLR read + int8 hard-decision write); the decoders are "
                        "instruction-issue bound, not HBM-bound: see the issue roofline"}
    iss = issue_roofline(prof, frames, ms, clocks, sms)
    if iss:
        roofline["issue"] = iss
    for name, r in results.items():
        r["hbm_frac"] = frames * 5 * n / (r["ms_per_step"] * 1e-3) / 1e9 / peak
        if "with_posterior" in r:
            r["with_posterior"]["hbm_frac"] = r["with_posterior"]["hbm_gbs"] / peak
        ir = issue_roofline(PROFILES[name].format(r=12, z=Z), frames, r["ms_per_step"], clocks, sms)
        r["issue_frac"] = ir["frac"] if ir else None

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        n_sample = min(frames, 65536)
        cpu = cpu_reference_baseline(llr[:n_sample].cpu().numpy())

    extra = {}
    # config 1: rate 5/6 z = 96 at 4 dB, same frame count (n is the same, so
    # the LLR and hard-decision buffers are reused)
    if "config1" in sections:
        info1 = torch.empty((frames, C1_K), dtype=torch.uint8, device=dev)
        wl.framegen_device(C1_RATE, C1_Z, SEED + 1, rank * frames, frames, C1_EBNO, C1_EBNO, info=info1, llr=llr)
        torch.cuda.synchronize()
        decs1, _ = make_decoders(wl, C1_RATE, C1_Z, not args.plain_only)
        c1 = {}
        for name, dec in decs1.items():
            r = measure(dec, info1, C1_K, frames)
            r["hbm_frac"] = frames * 5 * n / (r["ms_per_step"] * 1e-3) / 1e9 / peak
            ir = issue_roofline(PROFILES[name].format(r=56, z=C1_Z), frames, r["ms_per_step"], clocks, sms)
            r["issue_frac"] = ir["frac"] if ir else None
            r["kernel"] = KERNELS[name].format(r=C1_RATE, z=C1_Z)
            c1[name] = r
            dec.close()
        extra["config1"] = {"workload": f"rate 5/6 z=96 (n=2304, k=1920), {frames} frames per GPU per step, "
                                        f"Eb/N0 {C1_EBNO} dB, cap {MAX_ITER}", "decoders": c1}
        del info1

    # the encoder on the headline batch's info bits (codewords into the
    # hard-decision buffer): k + n bytes per frame
    if "encoder" in sections:
        enc = wl.Encoder(RATE, Z)
        cw = hard.view(torch.uint8)
        ms_e = timed_steps(lambda: enc.encode_device(info, cw, stream=stream), args.steps, args.warmup, stream, ws)
        ms_e, _ = reduce_step(ms_e, [], ws, dev)
        total = frames * ws
        extra["encoder"] = {"kernel": "encode_lanes_kernel<0,96>", "frames": total, "ms_per_step": ms_e,
                            "value": total * k / (ms_e * 1e-3) / 1e9, "unit": "info Gbit/s",
                            "frames_per_s": total / (ms_e * 1e-3),
                            "hbm_gbs": frames * (k + n) / (ms_e * 1e-3) / 1e9,
                            "hbm_frac": frames * (k + n) / (ms_e * 1e-3) / 1e9 / peak,
                            "note": "k + n bytes per frame (byte-per-bit info in, codeword out)"}
        enc.close()

    # config 2: one graph launch over a batch mixing all 114 codes
    if "config2" in sections:
        from wimax_ldpc_lib_b200 import mixed_batch
        variants, offsets, llr_m, cw_m, groups = mixed_batch.build_batch(MIXED_FRAMES, seed=0x311ED + rank,
                                                                         device=dev)
        hard_m = torch.empty(llr_m.numel(), dtype=torch.int8, device=dev)
        status_m = torch.empty(MIXED_FRAMES, dtype=torch.int32, device=dev)
        mixed = wl.MixedDecoder(MAX_ITER)
        mixed.autotune(variants, offsets, llr_m, hard_m, repeats=2)
        threads, layout, chunk, launch = mixed.tuning()
        ms_m = timed_steps(lambda: mixed.decode_device(variants, offsets, llr_m, hard_m, None, status_m,
                                                       stream=stream), args.steps, args.warmup, stream, ws)
        mixed.synchronize()
        info_bits = sum(c * (24 - [12, 8, 8, 6, 6, 4][r]) * z for (r, z), (_, _, c) in groups.items())
        failed = ((status_m >> 16) & 1).sum().item()
        iters = (status_m & 0xFFFF).to(torch.float64).sum().item()
        ms_m, (failed, iters) = reduce_step(ms_m, [failed, iters], ws, dev)
        total = MIXED_FRAMES * ws
        extra["config2"] = {"workload": "131072 frames per GPU, code uniform over the 114 (rate, z), Eb/N0 "
                                        "U[1, 4] dB per frame, cap 10, one CUDA-graph launch",
                            "ms_per_step": ms_m, "value": info_bits * ws / (ms_m * 1e-3) / 1e9,
                            "unit": "info Gbit/s", "autotuned": {"threads": threads, "chunk": chunk,
                                                                "messages": ["registers", "shared"][layout],
                                                                "launch": ["concurrent", "serial"][launch]},
                            "syndrome_failed_fraction": failed / total, "mean_iterations": iters / total}
        ipf = load_profile_value("mixed_decode_131k.txt", "warp_instructions_per_frame")
        if ipf and clocks.get("sm_mhz"):
            extra["config2"]["issue_frac"] = ipf * MIXED_FRAMES / (ms_m * 1e-3) / (sms * 4 * clocks["sm_mhz"] * 1e6)
        mixed.close()
        del variants, offsets, llr_m, cw_m, hard_m, status_m

    # the drop-in per-frame call: ldpc_decoder::decode(float*) is one frame per
    # call through the C ABI (what the facade calls), next to one reference core
    if "single_frame" in sections and rank == 0:
        dec = decoders["plain"]
        one = torch.empty((512, n), dtype=torch.float32, device=dev)
        wl.framegen_device(RATE, Z, SEED + 2, 0, 512, EBNO_DB, EBNO_DB, llr=one)
        src1 = one.cpu().numpy()
        for f in range(16):
            dec.decode(src1[f])
        t = time.perf_counter()
        for f in range(src1.shape[0]):
            dec.decode(src1[f])
        dt = time.perf_counter() - t
        sf = {"api": "wldpc_decoder_decode (one frame per call, synchronous)", "frames": int(src1.shape[0]),
              "frames_per_s": src1.shape[0] / dt, "latency_us": 1e6 * dt / src1.shape[0],
              "info_gbps": src1.shape[0] * k / dt / 1e9}
        from oracle.oracle import Reference, reference_available
        if reference_available():
            ref = Reference()
            ref.decode(RATE, Z, src1[:16], MAX_ITER, threads=1)
            t = time.perf_counter()
            ref.decode(RATE, Z, src1, MAX_ITER, threads=1)
            dt = time.perf_counter() - t
            sf["reference_one_core"] = {"frames_per_s": src1.shape[0] / dt, "latency_us": 1e6 * dt / src1.shape[0],
                                        "info_gbps": src1.shape[0] * k / dt / 1e9}
        # BER_runner::run_iteration, one frame per call (LFSR bits, encode,
        # BPSK + mt19937 noise on the host, decode, error count), both sides
        n_ber = 256
        ber = wl.BERRunner(RATE, Z, 1, MAX_ITER)
        for _ in range(8):
            ber.run_iteration(EBNO_DB)
        t = time.perf_counter()
        for _ in range(n_ber):
            ber.run_iteration(EBNO_DB)
        dt = time.perf_counter() - t
        ber.close()
        sf["ber_runner"] = {"api": "wldpc_ber_runner_run_iteration", "frames": n_ber, "frames_per_s": n_ber / dt,
                            "latency_us": 1e6 * dt / n_ber}
        if reference_available():
            L = ref.lib
            h = L.ref_ber_create(RATE, Z, 1, MAX_ITER)
            for _ in range(8):
                L.ref_ber_run_iteration(h, EBNO_DB)
            t = time.perf_counter()
            for _ in range(n_ber):
                L.ref_ber_run_iteration(h, EBNO_DB)
            dt = time.perf_counter() - t
            L.ref_ber_destroy(h)
            sf["ber_runner"]["reference_one_thread"] = {"frames_per_s": n_ber / dt, "latency_us": 1e6 * dt / n_ber}
        extra["single_frame"] = sf

    # config 4 for the headline code: the full-device waterfall of the plain and
    # the fp32 learned decoder (generation, encoding, channel, decoding and
    # counting on the device), rank 0 only (no collective inside)
    if "waterfall" in sections and rank == 0:
        from wimax_ldpc_lib_b200 import waterfall as wf
        t0 = time.perf_counter()
        wres = {}
        for name in ("plain", "learned"):
            if name not in decoders:
                continue
            pts = wf.sweep(RATE, Z, decoders[name], start=1.6, step=0.1, min_errors=200, max_bits=4e8,
                           stop_ber=1e-6, batch=1 << 17, max_points=12, log=lambda *a: None)
            wres[name] = {"ebno_at_ber_1e-5": wf.ebno_at(pts), "points": len(pts),
                          "frames": sum(p["frames"] for p in pts),
                          "ber": {f"{p['ebno_db']:.1f}": p["ber"] for p in pts},
                          "fer": {f"{p['ebno_db']:.1f}": p["fer"] for p in pts}}
        extra["waterfall"] = {"workload": "rate 1/2 z=96, Eb/N0 from 1.6 dB in 0.1 dB steps until BER < 1e-6, >= 200 "
                                          "info-bit errors (or 4e8 bits) per point, cap 10, all on the device",
                              "decoders": wres, "seconds": time.perf_counter() - t0}

    if rank == 0:
        T = lms_meta["iterations"] if lms_meta else 8
        cfg_dec = {"plain": f"plain NMS TDMP (bit-exact), cap {MAX_ITER}",
                   "learned": f"learned min-sum ({T} trained iterations, fp32), cap {MAX_ITER}",
                   "learned_f16x2": f"learned min-sum ({T} trained iterations, packed binary16, two frames per "
                                    f"thread), cap {MAX_ITER}"}
        line = {"metric": METRIC, "value": value, "unit": "info Gbit/s", "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": DTYPES[head], "data": "synthetic",
                "config": {"workload": f"{cfg_dec[head]} decode, rate 1/2 z=96, {frames} frames per GPU per step, "
                                       f"Eb/N0 {EBNO_DB} dB",
                           "frames_per_gpu": frames, "ebno_db": EBNO_DB, "decoder": head,
                           "l2": "inputs larger than L2 (2.4 GB per GPU), no flush",
                           "parallelism": f"frames sharded over {ws} GPU(s)"},
                "fer": R["fer"], "mean_iterations": R["mean_iterations"], "fer_ok": R["fer"] <= 1e-3,
                "decoders": {name: dict(r, unit="info Gbit/s", config=cfg_dec[name], dtype=DTYPES[name])
                             for name, r in results.items()},
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
                "gpu_launches": args.steps, "clocks": clocks}
        line.update(extra)
        print(json.dumps(line))
    for d in decoders.values():
        d.close()
    if ws > 1:
        torch.distributed.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--frames", type=int, default=FRAMES)
    ap.add_argument("--sections", default="all",
                    help="comma-separated extras to run besides the headline: " + ",".join(SECTIONS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--plain-only", action="store_true")
    ap.add_argument("--backend", default="nccl", choices=["nccl", "gloo"])
    ap.add_argument("--dry-run", action="store_true", help="ranks and reductions only, on CPU (with --backend gloo)")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(launch_ranks(args))
    if args.impl == "reference":
        run_reference(args)
    elif args.dry_run:
        run_dry(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
