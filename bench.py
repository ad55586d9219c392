"""Throughput benchmark of the B200 WiMAX LDPC decoder (one JSON line on rank 0).

Metric: info Gbit/s at FER <= 1e-3, rate 1/2, z = 96 (n = 2304, k = 1152), on
seeded synthetic frames (random info bits, the project's encoder, BPSK, AWGN,
LLR = 2y/sigma^2) generated on the device at Eb/N0 = 2.25 dB, where the plain
normalized min-sum decoder with the reference's cap of 10 iterations has
FER <= 1e-3. A step decodes one batch of 262144 frames (2.4 GB of float32 LLRs,
larger than L2, so no flush is needed between steps). All decoders run on the
same frames: the plain (bit-exact) decoder and, when trained weights are
shipped, the learned min-sum decoder (8 trained iterations, run to the same
cap of 10 with the last trained weights) in fp32 and in packed binary16 (two
frames per thread); `value` is the fastest learned variant's whose FER meets
the target, is no worse than the plain decoder's and that is faster, else the
plain one's; `decoders` reports all three.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

  value      kernel-only info Gbit/s, LLRs resident in HBM
  e2e        the same metric through the C ABI host call of the headline
             decoder (wldpc_lms_decode_host, or wldpc_decode_batch_host for
             the plain one: copy-in, decode, posterior + hard bits copied
             back, as the reference's decode(float*) returns them)
  roofline   the decode kernel against the measured HBM copy bandwidth
  cpu_baseline  the reference's own OpenMP decoder (compiled from its sources)
             on this machine's host cores, on a bounded sample of the workload

Multi-GPU (torchrun): every rank decodes its own shard of frames (weak scaling,
no data-path collective); timing is the max over ranks, FER the sum.
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

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "info Gbit/s at FER<=1e-3, learned vs plain min-sum, 1 B200, r1/2 z=96"
RATE, Z = 0, 96
N_BITS, K_BITS = 24 * Z, 12 * Z
FRAMES = 262144
EBNO_DB = 2.25
MAX_ITER = 10
SEED = 20261203


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


def load_traffic(name):
    """dram bytes per launch of the full batch, from an ncu capture."""
    return load_profile_value(name, "traffic_bytes_per_launch_full_batch")


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


def dist_setup():
    import torch
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    elif torch.cuda.is_available():
        torch.cuda.set_device(local)
    return ws, rank, local


def cpu_reference_baseline(llr_host, seconds=12.0, threads=None):
    """The reference decoder (oracle/_ref, its own sources) with one decoder
    object per OpenMP thread over frames, on a bounded sample of the frames:
    passes over the sample repeat until about `seconds` of CPU work is done."""
    from oracle.oracle import Reference, reference_available
    if not reference_available():
        return None
    ref = Reference()
    threads = threads or os.cpu_count() or 1
    sample = llr_host.shape[0]
    ref.decode(RATE, Z, llr_host[: min(sample, 4 * threads)], MAX_ITER, threads=threads)
    done, t0 = 0, time.perf_counter()
    while True:
        ref.decode(RATE, Z, llr_host, MAX_ITER, threads=threads)
        done += sample
        dt = time.perf_counter() - t0
        if dt >= seconds:
            break
    return {"value": done * K_BITS / dt / 1e9, "unit": "info Gbit/s", "cores": threads, "kind": "reference",
            "sample": f"{done} frame decodes ({done // sample} passes over the first {sample} frames of the "
                      f"workload), {dt:.1f} s, cap {MAX_ITER}, one decoder per OpenMP thread",
            "cpu": cpu_model()}


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


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


LMS_WEIGHTS = os.path.join(ROOT, "wimax_ldpc_lib_b200", "weights", "lms_r0_z96_T8.json")


def run_ours(args):
    import numpy as np
    import torch
    import wimax_ldpc_lib_b200 as wl
    wl.lib()                               # fails loudly if the library is missing
    ws, rank, local = dist_setup()
    dev = torch.device("cuda", local)
    frames = args.frames
    n, k = N_BITS, K_BITS

    llr = torch.empty((frames, n), dtype=torch.float32, device=dev)
    info = torch.empty((frames, k), dtype=torch.uint8, device=dev)
    wl.framegen_device(RATE, Z, SEED, rank * frames, frames, EBNO_DB, EBNO_DB, info=info, llr=llr)
    hard = torch.empty((frames, n), dtype=torch.int8, device=dev)
    status = torch.empty(frames, dtype=torch.int32, device=dev)
    stream = torch.cuda.Stream()
    torch.cuda.synchronize()

    decoders = {"plain": wl.Decoder(RATE, Z, MAX_ITER)}
    lms_meta = None
    if os.path.exists(LMS_WEIGHTS) and not args.plain_only:
        with open(LMS_WEIGHTS) as f:
            lms_meta = json.load(f)
        # the learned decoder at the reference's cap (iterations past the trained
        # ones reuse the last trained weights), compared with plain at cap 10
        decoders["learned"] = wl.LearnedDecoder(RATE, Z, lms_meta["iterations"],
                                                weights=np.array(lms_meta["weights"], np.float32), cap=MAX_ITER)
        # the same network decoded in packed binary16, two frames per thread
        decoders["learned_f16x2"] = wl.LearnedDecoder(RATE, Z, lms_meta["iterations"],
                                                      weights=np.array(lms_meta["weights"], np.float32),
                                                      cap=MAX_ITER, precision=wl.LMS_F16X2)

    def measure(dec):
        for _ in range(args.warmup):
            dec.decode_device(llr, hard, None, status, stream=stream)
        torch.cuda.synchronize()
        if ws > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        start = torch.cuda.Event(enable_timing=True)
        stop = torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for _ in range(args.steps):
            dec.decode_device(llr, hard, None, status, stream=stream)
        stop.record(stream)
        torch.cuda.synchronize()
        if ws > 1:
            torch.distributed.barrier()
        ms = start.elapsed_time(stop) / args.steps
        ferr = (hard[:, :k].view(torch.uint8) != info).any(dim=1).sum().to(torch.float64)
        iters = (status & 0xFFFF).to(torch.float64).sum()
        c = torch.stack([ferr, iters, torch.tensor(ms, dtype=torch.float64, device=dev)])
        if ws > 1:
            torch.distributed.all_reduce(c[:2])
            m = c[2:].clone()
            torch.distributed.all_reduce(m, op=torch.distributed.ReduceOp.MAX)
            c[2] = m[0]
        total = frames * ws
        ms = float(c[2].item())
        return {"value": total * k / (ms * 1e-3) / 1e9, "ms_per_step": ms, "fer": float(c[0].item()) / total,
                "mean_iterations": float(c[1].item()) / total}

    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    results = {name: measure(dec) for name, dec in decoders.items()}
    clocks = sampler.stop()
    for dec in decoders.values():
        if hasattr(dec, "synchronize"):
            dec.synchronize()

    # the headline decoder: the fastest learned variant that meets the FER
    # target, is no worse than plain and is faster, else plain
    head = "plain"
    P = results["plain"]
    for name in ("learned", "learned_f16x2"):
        L = results.get(name)
        if L and L["fer"] <= 1e-3 and L["fer"] <= P["fer"] and L["value"] > results[head]["value"]:
            head = name
    R = results[head]
    ms = R["ms_per_step"]
    value = R["value"]
    dec = decoders[head]

    # e2e through the C ABI host call of the same decoder (pinned host buffers,
    # copies in the timed region)
    e2e = None
    if not args.no_e2e:
        llr_h = torch.empty((frames, n), dtype=torch.float32, pin_memory=True)
        hard_h = torch.empty((frames, n), dtype=torch.int8, pin_memory=True)
        st_h = torch.empty(frames, dtype=torch.int32, pin_memory=True)
        src = llr.cpu()

        def host_call():
            if head == "plain":
                dec.decode_host_into(llr_h, hard_h, None, st_h)
            else:
                wl._check(wl.lib().wldpc_lms_decode_host(dec._h, wl._t_ptr(llr_h), wl._t_ptr(hard_h), None,
                                                         wl._t_ptr(st_h), frames), "lms decode_host")
        e2e_steps = max(1, min(args.steps, 3))
        llr_h.copy_(src)
        host_call()                                            # warm-up
        times = []
        for _ in range(e2e_steps):
            llr_h.copy_(src)                                   # fresh input (decode writes posteriors back)
            torch.cuda.synchronize()
            t = time.perf_counter()
            host_call()
            times.append(time.perf_counter() - t)
        t_e2e = torch.tensor([sum(times) / len(times)], dtype=torch.float64, device=dev)
        if ws > 1:
            torch.distributed.all_reduce(t_e2e, op=torch.distributed.ReduceOp.MAX)
        e2e = {"value": frames * ws * k / float(t_e2e.item()) / 1e9, "unit": "info Gbit/s",
               "h2d_bytes_per_step": frames * n * 4,
               "d2h_bytes_per_step": frames * n * 4 + frames * n + frames * 4,
               "api": ("wldpc_decode_batch_host" if head == "plain" else "wldpc_lms_decode_host") +
                      " (pinned host buffers; posterior, hard bits and status copied back)",
               "timing": "host wall clock around the synchronous call, mean of %d" % e2e_steps}
        del llr_h, hard_h, st_h, src

    peak, peak_kind = load_peaks()
    bytes_per_launch = frames * 5 * n
    achieved = bytes_per_launch / (ms * 1e-3) / 1e9
    prof = {"plain": "tdmp_nms_r12_z96.txt", "learned": "lms_r12_z96.txt",
            "learned_f16x2": "lms16_r12_z96.txt"}[head]
    kernel = {"plain": "tdmp_decode_kernel<0,96,NMS>", "learned": "lms_decode_kernel<0,96>",
              "learned_f16x2": "lms16_decode_kernel<0,96>"}[head]
    traffic = load_traffic(prof)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "peak_kind": peak_kind, "kernel": kernel,
                "algorithmic_bytes_per_launch": bytes_per_launch,
                "note": "5n bytes per frame (float32 LLR read + int8 hard-decision write); the decoders are "
                        "instruction-issue bound, not HBM-bound: see the issue roofline"}
    # issue roofline: warp-instructions per frame (ncu, same workload) x frames
    # per launch / launch time, against 4 issue slots per SM per cycle at the
    # SM clock sampled during the timed region
    ipf = load_profile_value(prof, "warp_instructions_per_frame")
    if ipf and clocks.get("sm_mhz"):
        sms = torch.cuda.get_device_properties(0).multi_processor_count
        ach = ipf * frames / (ms * 1e-3)
        pk = sms * 4 * clocks["sm_mhz"] * 1e6
        roofline["issue"] = {"bound": "issue", "achieved": ach, "peak": pk, "unit": "warp-instructions/s",
                             "frac": ach / pk, "warp_instructions_per_frame": ipf,
                             "peak_basis": f"{sms} SMs x 4 schedulers x {clocks['sm_mhz']:.0f} MHz (sampled)"}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        n_sample = min(frames, 65536)
        cpu = cpu_reference_baseline(llr[:n_sample].cpu().numpy())

    if rank == 0:
        T = lms_meta["iterations"] if lms_meta else 8
        cfg_dec = {"plain": f"plain NMS TDMP (bit-exact), cap {MAX_ITER}",
                   "learned": f"learned min-sum ({T} trained iterations, fp32), cap {MAX_ITER}",
                   "learned_f16x2": f"learned min-sum ({T} trained iterations, packed binary16, two frames per "
                                    f"thread), cap {MAX_ITER}"}
        line = {"metric": METRIC, "value": value, "unit": "info Gbit/s", "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": {"plain": "f32+f64", "learned": "f32", "learned_f16x2": "f16x2"}[head],
                "data": "synthetic",
                "config": {"workload": f"{cfg_dec[head]} decode, rate 1/2 z=96, {frames} frames per GPU per step, "
                                       f"Eb/N0 {EBNO_DB} dB",
                           "frames_per_gpu": frames, "ebno_db": EBNO_DB, "decoder": head,
                           "l2": "inputs larger than L2 (2.4 GB per GPU), no flush",
                           "parallelism": f"frames sharded over {ws} GPU(s)"},
                "fer": R["fer"], "mean_iterations": R["mean_iterations"], "fer_ok": R["fer"] <= 1e-3,
                "decoders": {name: dict(r, unit="info Gbit/s", config=cfg_dec[name]) for name, r in results.items()},
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
                "gpu_launches": args.steps, "clocks": clocks}
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
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--plain-only", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
