"""Mixed-code batches: building them on the device, and the mixed-batch benchmark.

  python -m wimax_ldpc_lib_b200.mixed_batch [--frames 131072] [--steps 10] [--sweep] [--tuning T,L,C,P]

The workload draws every frame's code uniformly over the 114 (rate, z) codes
and its Eb/N0 uniformly in [1, 4] dB; rate 3/4B frames are random codewords
from the null space of H (it has no dual-diagonal encoder), the others come
from the encoder. Frames are stored back to back (frame f at offset[f]) and
presented to the decoder in a random order. The benchmark autotunes the
persistent decoder, times one-graph-launch decodes with CUDA events, and
times the same frames decoded code by code with the (rate, z)-specialised
kernels for comparison; both must agree bit for bit. --sweep also times every
candidate of the autotuner's space (CTA threads x message layout x chunk x
launch policy) and reports the table; --tuning T,L,C,P skips the autotuner
and uses that candidate (threads, layout 0 = registers / 1 = shared, chunk,
launch 0 = concurrent / 1 = serial).
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

import wimax_ldpc_lib_b200 as wl  # noqa: E402


def build_batch(frames, seed=0x311ED, ebno=(1.0, 4.0), device="cuda", codes=None):
    """Returns (variants u8, offsets i64, llr f32, codewords u8, groups) on the device;
    groups[(rate, z)] = (frame ids in decode order, packed start, count)."""
    import torch
    rng = np.random.default_rng(seed)
    codes = codes or [(r, z) for r in range(6) for z in wl.Z_VALUES]
    pick = rng.integers(0, len(codes), frames)
    order = rng.permutation(frames)                 # decode order differs from storage order
    counts = np.bincount(pick, minlength=len(codes))
    ns = np.array([24 * z for _, z in codes])
    total = int((counts * ns).sum())
    llr = torch.empty(total, dtype=torch.float32, device=device)
    cw = torch.empty(total, dtype=torch.uint8, device=device)
    variants = np.empty(frames, np.uint8)
    offsets = np.empty(frames, np.int64)
    groups = {}
    start = 0
    first = 0
    for ci, (rate, z) in enumerate(codes):
        c = int(counts[ci])
        if c == 0:
            continue
        n = 24 * z
        seg_llr = llr[start:start + c * n].view(c, n)
        seg_cw = cw[start:start + c * n].view(c, n)
        if rate == 4:
            wl.framegen_nullspace_device(rate, z, seed, first, c, ebno[0], ebno[1], codeword=seg_cw, llr=seg_llr)
        else:
            wl.framegen_device(rate, z, seed, first, c, ebno[0], ebno[1], codeword=seg_cw, llr=seg_llr)
        ids = order[np.flatnonzero(pick == ci)]     # these decode positions hold this code's frames
        variants[ids] = wl.variant(rate, z)
        offsets[ids] = start + np.arange(c) * n
        groups[(rate, z)] = (ids, start, c)
        start += c * n
        first += c
    return (torch.from_numpy(variants).to(device), torch.from_numpy(offsets).to(device), llr, cw, groups)


def decode_by_code(groups, llr, hard, status_by_frame, max_iter=10, stream=None):
    """The specialised per-(rate, z) decoders, one launch per code."""
    import torch
    # the per-code status buffers and the scatter into frame order run on the
    # decoding stream, so nothing reads a status before its decode wrote it
    with torch.cuda.stream(stream if stream is not None else torch.cuda.current_stream()):
        for (rate, z), (ids, start, c) in groups.items():
            n = 24 * z
            dec = wl.Decoder(rate, z, max_iter)
            st = torch.empty(c, dtype=torch.int32, device=llr.device)
            dec.decode_device(llr[start:start + c * n].view(c, n), hard[start:start + c * n].view(c, n), None, st,
                              stream=torch.cuda.current_stream())
            status_by_frame[torch.from_numpy(ids).to(llr.device)] = st


def main():
    import torch
    ap = argparse.ArgumentParser()
    ap.add_argument("--frames", type=int, default=131072)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--out", default=None, help="also write the JSON result to this file")
    ap.add_argument("--sweep", action="store_true", help="time every tuning candidate")
    ap.add_argument("--tuning", default=None,
                    help="threads,layout,chunk,launch[,rows per thread] instead of the autotuner")
    ap.add_argument("--z", type=int, nargs="*", default=None, help="only these z values")
    ap.add_argument("--rates", type=int, nargs="*", default=None, help="only these rates")
    args = ap.parse_args()
    codes = [(r, z) for r in (args.rates if args.rates else range(6)) for z in (args.z if args.z else wl.Z_VALUES)]
    variants, offsets, llr, cw, groups = build_batch(args.frames, codes=codes)
    hard = torch.empty(llr.numel(), dtype=torch.int8, device="cuda")
    status = torch.empty(args.frames, dtype=torch.int32, device="cuda")
    mixed = wl.MixedDecoder(10)
    stream = torch.cuda.Stream()
    table = []
    if args.sweep:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for threads in (96, 192):
            for rows in (1, 2):
                for layout in (wl.MIXED_MSG_REGISTERS, wl.MIXED_MSG_SHARED):
                    for chunk in (8, 16, 32, 64):
                        for launch in (wl.MIXED_CONCURRENT, wl.MIXED_SERIAL):
                            mixed.set_tuning(threads, layout, chunk, launch)
                            mixed.set_rows_per_thread(rows)
                            mixed.decode_device(variants, offsets, llr, hard, None, status, stream=stream)
                            e0.record(stream)
                            for _ in range(3):
                                mixed.decode_device(variants, offsets, llr, hard, None, status, stream=stream)
                            e1.record(stream)
                            torch.cuda.synchronize()
                            mixed.synchronize()
                            ms = e0.elapsed_time(e1) / 3
                            table.append({"threads": threads, "rows_per_thread": rows,
                                          "messages": ["registers", "shared"][layout], "chunk": chunk,
                                          "launch": ["concurrent", "serial"][launch], "ms": ms})
                            print(f"sweep: {threads:3d} threads, {rows} row{'s' if rows > 1 else ' '} per thread, "
                                  f"messages in {table[-1]['messages']:9s}, chunk {chunk:2d}, "
                                  f"{table[-1]['launch']:10s}: {ms:7.3f} ms")
    if args.tuning:
        vals = [int(x) for x in args.tuning.split(",")]
        mixed.set_tuning(*vals[:4])
        mixed.set_rows_per_thread(vals[4] if len(vals) > 4 else 1)
        best = None
    else:
        best = mixed.autotune(variants, offsets, llr, hard, repeats=3)
    threads, layout, chunk, launch = mixed.tuning()
    rows = mixed.rows_per_thread()
    for _ in range(3):
        mixed.decode_device(variants, offsets, llr, hard, None, status, stream=stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        mixed.decode_device(variants, offsets, llr, hard, None, status, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize()
    mixed.synchronize()
    ms_mixed = e0.elapsed_time(e1) / args.steps
    hard_ref = torch.empty_like(hard)
    status_ref = torch.empty_like(status)
    for _ in range(2):
        decode_by_code(groups, llr, hard_ref, status_ref, stream=stream)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        decode_by_code(groups, llr, hard_ref, status_ref, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_split = e0.elapsed_time(e1) / args.steps
    same_hard = bool(torch.equal(hard, hard_ref))
    same_status = bool(torch.equal(status, status_ref))
    info_bits = sum(c * (24 - [12, 8, 8, 6, 6, 4][r]) * z for (r, z), (_, _, c) in groups.items())
    fer_frames = float(((status >> 16) & 1).double().mean().item())
    res = {"workload": f"mixed batch: code uniform over {len(codes)} (rate, z), Eb/N0 U[1, 4] dB, cap 10",
                      "frames": args.frames, "info_bits_per_batch": info_bits,
                      "mixed": {"ms": ms_mixed, "info_gbps": info_bits / (ms_mixed * 1e-3) / 1e9,
                                "threads": threads, "rows_per_thread": rows, "chunk": chunk,
                                "messages": ["registers", "shared"][layout],
                                "launch": ["concurrent", "serial"][launch], "autotune_best_ms": best},
                      "per_code_launches": {"ms": ms_split, "info_gbps": info_bits / (ms_split * 1e-3) / 1e9,
                                            "launches": len(groups)},
                      "bit_exact_match": same_hard and same_status,
                      "hard_bits_match": same_hard, "status_match": same_status, "syndrome_failed_fraction": fer_frames,
                      "mean_iterations": float((status & 0xFFFF).double().mean().item()),
                      "device": torch.cuda.get_device_name(0), "sweep": table}
    print(json.dumps(res))
    if args.out:
        os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
        with open(args.out, "w") as f:
            json.dump(res, f, indent=1)


if __name__ == "__main__":
    main()
