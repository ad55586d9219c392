"""Evaluates trained learned min-sum weights against the plain decoder and
records where they ship.

  python -m wimax_ldpc_lib_b200.eval_lms weights/lms_r0_z96_T8.json [--frames 1048576]
  python -m wimax_ldpc_lib_b200.eval_lms --transfer [--frames 262144]

For every Eb/N0 point (default 1.0 to 3.0 dB in 0.25 dB steps) it generates
held-out frames on the device (a seed and frame counters disjoint from
training), decodes the same frames with the learned decoder at its trained cap T and at
the reference's cap 10 (iterations past T reuse the last trained weights),
the learned decoder in packed binary16 at cap 10 (`learned10_f16x2`, where the
weights are in its range), and with the plain normalized min-sum at caps T and
10, and records FER, info
BER, mean iterations and kernel-only info Gbit/s (CUDA events). The learned
weights ship at a point and cap when their frame errors on those frames are
no more than the plain decoder's at the same cap and they need fewer
iterations on average (plain min-sum stays the yardstick and the fallback). The
table is written back into the weight file under "evaluation".

--transfer evaluates every code without weights of its own (the 19 z values
of each rate other than the trained z = 48 and z = 96) with the weights
trained at the nearest z of the same rate -- the weights are per (iteration,
layer, base column), so they apply to any z -- by the same rule, and writes
weights/lms_transfer.json (which learned_weights() reads to say where a
transferred table ships).
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

EVAL_SEED = 0xE7A1


def evaluate(meta, frames=1 << 20, batch=1 << 18, points=None, log=print):
    import torch
    rate, z, T = meta["rate"], meta["z"], meta["iterations"]
    info_ = wl.code_info(rate, z)
    n, k = info_.n, info_.k
    lo = meta.get("training", {}).get("ebno_db", [1.0, 3.0])[0]
    points = points or [lo + 0.25 * i for i in range(9)]
    batch = min(batch, frames)
    # 3/4B has no encoder: frames are null-space codewords and errors count over all n bits
    kk = n if rate == 4 else k
    w = np.array(meta["weights"], np.float32)
    decs = {"learned": wl.LearnedDecoder(rate, z, T, weights=w),
            "learned10": wl.LearnedDecoder(rate, z, T, weights=w, cap=10),
            f"plain{T}": wl.Decoder(rate, z, T), "plain10": wl.Decoder(rate, z, 10)}
    if np.abs(w[0]).max() <= 2.0 and w[1].min() >= 0.0 and w[1].max() <= 1024.0:
        decs["learned10_f16x2"] = wl.LearnedDecoder(rate, z, T, weights=w, cap=10, precision=wl.LMS_F16X2)
    llr = torch.empty((batch, n), dtype=torch.float32, device="cuda")
    info = torch.empty((batch, kk), dtype=torch.uint8, device="cuda")
    hard = torch.empty((batch, n), dtype=torch.int8, device="cuda")
    st = torch.empty(batch, dtype=torch.int32, device="cuda")
    stream = torch.cuda.Stream()
    rows = []
    for p_i, eb in enumerate(points):
        acc = {name: {"frame_errors": 0, "bit_errors": 0, "iterations": 0.0, "ms": 0.0} for name in decs}
        done = 0
        while done < frames:
            nb = min(batch, frames - done)
            first = (1 << 40) + p_i * (1 << 32) + done
            if rate == 4:
                wl.framegen_nullspace_device(rate, z, EVAL_SEED, first, nb, eb, eb, codeword=info[:nb], llr=llr[:nb],
                                             stream=stream)
            else:
                wl.framegen_device(rate, z, EVAL_SEED, first, nb, eb, eb, info=info[:nb], llr=llr[:nb], stream=stream)
            for name, dec in decs.items():
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                dec.decode_device(llr[:nb], hard[:nb], None, st[:nb], stream=stream)
                e1.record(stream)
                torch.cuda.synchronize()
                err = hard[:nb, :kk].view(torch.uint8) != info[:nb]
                a = acc[name]
                a["frame_errors"] += int(err.any(dim=1).sum().item())
                a["bit_errors"] += int(err.sum().item())
                a["iterations"] += float((st[:nb] & 0xFFFF).double().sum().item())
                a["ms"] += e0.elapsed_time(e1)
            done += nb
        row = {"ebno_db": eb, "frames": frames}
        for name, a in acc.items():
            row[name] = {"fer": a["frame_errors"] / frames, "frame_errors": a["frame_errors"],
                         "ber": a["bit_errors"] / (frames * kk), "mean_iterations": a["iterations"] / frames,
                         "info_gbps": frames * k / (a["ms"] * 1e-3) / 1e9}
        L, L10, P8, P = row["learned"], row["learned10"], row[f"plain{T}"], row["plain10"]
        row["ship_cap10"] = bool(L10["frame_errors"] <= P["frame_errors"] and
                                 L10["mean_iterations"] < P["mean_iterations"])
        row[f"ship_cap{T}"] = bool(L["frame_errors"] <= P8["frame_errors"] and
                                   L["mean_iterations"] < P8["mean_iterations"])
        if "learned10_f16x2" in row:
            H = row["learned10_f16x2"]
            row["ship_cap10_f16x2"] = bool(H["frame_errors"] <= P["frame_errors"] and
                                           H["mean_iterations"] < P["mean_iterations"])
        rows.append(row)
        log(f"{eb:5.2f} dB | learned{T} FER {L['fer']:.2e} it {L['mean_iterations']:.2f} {L['info_gbps']:.1f} Gb/s "
            f"| plain{T} FER {P8['fer']:.2e} it {P8['mean_iterations']:.2f} | learned10 FER {L10['fer']:.2e} "
            f"it {L10['mean_iterations']:.2f} {L10['info_gbps']:.1f} Gb/s | plain10 FER {P['fer']:.2e} "
            f"it {P['mean_iterations']:.2f} {P['info_gbps']:.1f} Gb/s | ship@10 {row['ship_cap10']} "
            f"ship@{T} {row[f'ship_cap{T}']}")
        if "learned10_f16x2" in row:
            H = row["learned10_f16x2"]
            log(f"{'':5s}    | learned10 f16x2 FER {H['fer']:.2e} it {H['mean_iterations']:.2f} "
                f"{H['info_gbps']:.1f} Gb/s | ship@10 {row['ship_cap10_f16x2']}")
    return rows


def transfer(frames, out, log=print):
    """Every (rate, z) without trained weights, with the nearest trained z's table."""
    import time
    import torch
    res = {"format": "wimax_ldpc_lib_b200 learned-weight transfer evaluation v1", "seed": EVAL_SEED,
           "frames_per_point": frames, "device": torch.cuda.get_device_name(0),
           "rule": "weights trained at the nearest z of the same rate; ship at a point and cap where learned frame "
                   "errors <= plain frame errors at that cap on the same held-out frames and learned mean "
                   "iterations < plain mean iterations", "codes": []}
    t0 = time.time()
    for rate in range(6):
        for z in wl.Z_VALUES:
            meta, _, src_z = wl.learned_weights(rate, z, evaluated_only=False)
            if meta is None or src_z == z:
                continue
            m = dict(meta, z=z)
            rows = evaluate(m, frames, batch=frames, log=lambda *a: None)
            ship10 = sum(r["ship_cap10"] for r in rows)
            ship16 = sum(r.get("ship_cap10_f16x2", False) for r in rows)
            res["codes"].append({"rate": rate, "z": z, "source_z": src_z,
                                 "source": f"lms_r{rate}_z{src_z}_T{meta['iterations']}.json",
                                 "ships_cap10": ship10, "ships_cap10_f16x2": ship16, "points": rows})
            P = rows[len(rows) // 2]
            log(f"rate {wl.RATE_NAMES[rate]:5s} z={z:2d} from z={src_z}: ships at {ship10}/{len(rows)} points "
                f"(binary16 {ship16}); mid point {P['ebno_db']:.2f} dB learned10 FER {P['learned10']['fer']:.2e} "
                f"it {P['learned10']['mean_iterations']:.2f} vs plain10 {P['plain10']['fer']:.2e} "
                f"it {P['plain10']['mean_iterations']:.2f}")
            res["seconds"] = round(time.time() - t0, 1)
            with open(out, "w") as f:
                json.dump(res, f)
    print(f"wrote {out}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("weights", nargs="?")
    ap.add_argument("--frames", type=int, default=None)
    ap.add_argument("--points", type=float, nargs="*", default=None)
    ap.add_argument("--transfer", action="store_true", help="evaluate the codes without weights of their own")
    ap.add_argument("--out", default=None, help="where to write the weight file with its evaluation "
                                                "(default: in place)")
    args = ap.parse_args()
    if args.transfer:
        transfer(args.frames or (1 << 18), args.out or os.path.join(HERE, "weights", "lms_transfer.json"))
        return
    if not args.weights:
        ap.error("a weight file, or --transfer")
    args.frames = args.frames or (1 << 20)
    with open(args.weights) as f:
        meta = json.load(f)
    rows = evaluate(meta, args.frames, points=args.points)
    import torch
    meta["evaluation"] = {"seed": EVAL_SEED, "frames_per_point": args.frames, "device": torch.cuda.get_device_name(0),
                          "rule": "ship at a cap where learned frame errors <= plain frame errors at that cap on "
                                  "the same held-out frames and learned mean iterations < plain mean iterations "
                                  "(fp32 and, at cap 10, packed binary16)",
                          "points": rows}
    out = args.out or args.weights
    with open(out, "w") as f:
        json.dump(meta, f)
    print(f"evaluation written into {out}")


if __name__ == "__main__":
    main()
