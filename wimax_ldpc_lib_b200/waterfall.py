"""Full-device BER / FER waterfalls and the reference's two sweep procedures.

  python -m wimax_ldpc_lib_b200.waterfall --z 96 48 [--rates 0 1 2 3 4 5] [--out results/waterfall.json]

Writes the JSON result and the same points as CSV beside it (results/waterfall.csv).

Frames are generated, encoded, modulated, corrupted and decoded on the
device (framegen, or null-space codewords for 3/4B, which has no
dual-diagonal encoder). For every (rate, z) and decoder (plain normalized
min-sum, cap 10; the learned min-sum, cap 10, in fp32 and in packed binary16,
where trained weights for that code are shipped) the Eb/N0 sweep starts at --start dB and steps by 0.1 dB;
each point runs batches until at least 200 information-bit errors (or a bit
budget) and the sweep stops once BER < 1e-6. Reported per point: FER, info
BER, the reference BER_runner's BER (codeword-bit errors over info bits,
reference lib/BER_runner.cc:148-160,198-199), mean iterations and
kernel-only info Gbit/s; per code: the Eb/N0 at BER 1e-5 (log-linear
interpolation).

The reference's own sweep procedures, restated on this frame source:
* ber_example_point: BER_example's budget (reference lib/BER_example.cc:142-169):
  a pilot of 46080/n frames, then 10*floor(3.912/BER) bits more (3.912e8 when
  the pilot saw no error), converted to frames by dividing by n, counters not
  reset in between;
* capacity_search: Capacity_example's search (reference
  lib/Capacity_plot_example.cc:91,150-186): from 0.25 dB in 0.01 dB steps, the
  first Eb/N0 at which 3.912/1e-5 bits (divided by n, plus one frame) pass
  without a single bit error.
Noise comes from the device generator (Philox), not the reference's mt19937
stream, so values agree statistically, not frame for frame.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

import wimax_ldpc_lib_b200 as wl  # noqa: E402

SEED = 0x3A7EF
RATE_NAMES = wl.RATE_NAMES


class FrameSource:
    """Device frames of one code: LLRs, transmitted codewords (info bits are the
    first k codeword bits for the encoder; for 3/4B the comparison covers all n)."""

    def __init__(self, rate, z, batch, seed=SEED):
        import torch
        self.rate, self.z, self.batch, self.seed = rate, z, batch, seed
        ci = wl.code_info(rate, z)
        self.n, self.k = ci.n, ci.k
        self.llr = torch.empty((batch, self.n), dtype=torch.float32, device="cuda")
        self.cw = torch.empty((batch, self.n), dtype=torch.uint8, device="cuda")
        self.counter = 0

    def next(self, frames, ebno):
        f = min(frames, self.batch)
        if self.rate == 4:
            wl.framegen_nullspace_device(self.rate, self.z, self.seed, self.counter, f, ebno, ebno,
                                         codeword=self.cw[:f], llr=self.llr[:f])
        else:
            wl.framegen_device(self.rate, self.z, self.seed, self.counter, f, ebno, ebno,
                               codeword=self.cw[:f], llr=self.llr[:f])
        self.counter += f
        return f


def run_frames(src, dec, ebno, frames):
    """Decodes `frames` fresh frames; returns counters and kernel milliseconds."""
    import torch
    hard = torch.empty((src.batch, src.n), dtype=torch.int8, device="cuda")
    st = torch.empty(src.batch, dtype=torch.int32, device="cuda")
    tot = {"frames": 0, "frame_errors": 0, "info_bit_errors": 0, "cw_bit_errors": 0, "iterations": 0, "ms": 0.0}
    done = 0
    while done < frames:
        f = src.next(frames - done, ebno)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        dec.decode_device(src.llr[:f], hard[:f], None, st[:f])
        e1.record()
        torch.cuda.synchronize()
        diff = hard[:f].view(torch.uint8) != src.cw[:f]
        info = diff[:, :src.k] if src.rate != 4 else diff
        tot["frames"] += f
        tot["frame_errors"] += int(info.any(dim=1).sum().item())
        tot["info_bit_errors"] += int(info.sum().item())
        tot["cw_bit_errors"] += int(diff.sum().item())
        tot["iterations"] += int((st[:f] & 0xFFFF).sum().item())
        tot["ms"] += e0.elapsed_time(e1)
        done += f
    return tot


def sweep(rate, z, dec, start=0.5, step=0.1, min_errors=200, max_bits=2e10, stop_ber=1e-6, batch=1 << 17,
          max_points=60, log=print):
    src = FrameSource(rate, z, batch)
    k_eff = src.k if rate != 4 else src.n
    points = []
    eb = start
    for _ in range(max_points):
        tot = {"frames": 0, "frame_errors": 0, "info_bit_errors": 0, "cw_bit_errors": 0, "iterations": 0, "ms": 0.0}
        while tot["info_bit_errors"] < min_errors and tot["frames"] * k_eff < max_bits:
            need = batch if tot["frames"] else max(4096, min(batch, int(2e6 // k_eff)))
            t = run_frames(src, dec, eb, need)
            for key in tot:
                tot[key] += t[key]
        bits = tot["frames"] * k_eff
        p = {"ebno_db": round(eb, 4), "frames": tot["frames"], "fer": tot["frame_errors"] / tot["frames"],
             "ber": tot["info_bit_errors"] / bits, "bit_errors": tot["info_bit_errors"],
             "ber_reference_definition": tot["cw_bit_errors"] / (tot["frames"] * src.k),
             "mean_iterations": tot["iterations"] / tot["frames"],
             "info_gbps": tot["frames"] * src.k / (tot["ms"] * 1e-3) / 1e9}
        points.append(p)
        log(f"  {RATE_NAMES[rate]:5s} z={z} {eb:5.2f} dB  FER {p['fer']:.3e}  BER {p['ber']:.3e}  "
            f"it {p['mean_iterations']:.2f}  {p['info_gbps']:.1f} Gb/s  ({tot['frames']} frames)")
        if p["ber"] < stop_ber:
            break
        eb += step
    return points


def ebno_at(points, target=1e-5):
    """Eb/N0 where BER crosses target (log-linear interpolation), or None."""
    for a, b in zip(points, points[1:]):
        if a["ber"] >= target > b["ber"] and b["ber"] > 0:
            la, lb = math.log10(a["ber"]), math.log10(b["ber"])
            return a["ebno_db"] + (math.log10(target) - la) / (lb - la) * (b["ebno_db"] - a["ebno_db"])
        if a["ber"] >= target and b["ber"] == 0:
            return b["ebno_db"]
    return None


def pilot_frames(n):
    """BER_example's pilot run: 46080 bits in whole frames (reference lib/BER_example.cc:142-150)."""
    return max(1, 46080 // n)


def ber_example_frames(pilot_ber, n):
    """Frames of BER_example's main run after a pilot that measured pilot_ber:
    10 * floor(3.912 / BER) bits, or floor(3.912 / 1e-8) bits when the pilot
    saw no error, in whole frames (reference lib/BER_example.cc:152-166)."""
    bits = math.floor(3.912 / 1e-8) if pilot_ber == 0.0 else 10 * math.floor(3.912 / pilot_ber)
    return bits // n


def capacity_frames(n):
    """Frames per Eb/N0 step of the capacity search: 3.912 / 1e-5 bits over
    n, plus one (reference lib/Capacity_plot_example.cc:150-160)."""
    return int(3.912 / 0.00001) // n + 1


def ber_example_point(rate, z, dec, ebno):
    """BER_example's procedure at one Eb/N0 (reference lib/BER_example.cc:142-169)."""
    src = FrameSource(rate, z, 1 << 17)
    tot = run_frames(src, dec, ebno, pilot_frames(src.n))
    ber = tot["cw_bit_errors"] / (tot["frames"] * src.k)
    t2 = run_frames(src, dec, ebno, ber_example_frames(ber, src.n))
    for key in tot:
        tot[key] += t2[key]
    return tot["cw_bit_errors"] / (tot["frames"] * src.k), tot["frames"]


def capacity_search(rate, z, dec, start=0.25, step=0.01, max_steps=2000):
    """Capacity_example's search (reference lib/Capacity_plot_example.cc:91,150-186)."""
    src = FrameSource(rate, z, 1 << 16)
    frames = capacity_frames(src.n)
    eb = start
    for _ in range(max_steps):
        tot = run_frames(src, dec, eb, frames)
        if tot["cw_bit_errors"] == 0:
            return round(eb, 4)
        eb += step
    return None


CSV_FIELDS = ["rate", "z", "decoder", "ebno_db", "frames", "fer", "ber", "bit_errors", "ber_reference_definition",
              "mean_iterations", "info_gbps"]


def write_csv(res, path):
    """One line per (code, decoder, Eb/N0 point): the sweep as a table, in
    place of the reference's MathGL plots."""
    with open(path, "w") as f:
        f.write(",".join(CSV_FIELDS) + "\n")
        for e in res["codes"]:
            for name, d in e["decoders"].items():
                for p in d["points"]:
                    row = {"rate": e["rate"], "z": e["z"], "decoder": name, **p}
                    f.write(",".join(str(row[k]) for k in CSV_FIELDS) + "\n")


def save(res, out):
    os.makedirs(os.path.dirname(os.path.abspath(out)), exist_ok=True)
    with open(out, "w") as f:
        json.dump(res, f, indent=1)
    write_csv(res, os.path.splitext(out)[0] + ".csv")


def learned_weights(rate, z):
    p = os.path.join(HERE, "weights", f"lms_r{rate}_z{z}_T8.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        return json.load(f)


def main():
    import torch
    ap = argparse.ArgumentParser()
    ap.add_argument("--z", type=int, nargs="+", default=[96, 48])
    ap.add_argument("--rates", type=int, nargs="+", default=[0, 1, 2, 3, 4, 5])
    ap.add_argument("--start", type=float, default=None)
    ap.add_argument("--max-bits", type=float, default=2e10)
    ap.add_argument("--capacity", action="store_true", help="also run the capacity search (plain decoder)")
    ap.add_argument("--out", default=os.path.join(os.path.dirname(HERE), "results", "waterfall.json"))
    args = ap.parse_args()
    starts = {0: 0.75, 1: 1.5, 2: 1.5, 3: 2.0, 4: 2.0, 5: 2.75}
    res = {"device": torch.cuda.get_device_name(0), "seed": SEED, "rule": "0.1 dB steps, >= 200 info-bit errors or "
           f"{args.max_bits:.0e} bits per point, stop at BER < 1e-6; cap 10", "codes": []}
    t0 = time.time()
    for z in args.z:
        for rate in args.rates:
            entry = {"rate": RATE_NAMES[rate], "rate_enum": rate, "z": z, "n": 24 * z, "decoders": {}}
            decs = {"plain": wl.Decoder(rate, z, 10)}
            meta = learned_weights(rate, z)
            if meta is not None:
                w = np.array(meta["weights"], np.float32)
                decs["learned"] = wl.LearnedDecoder(rate, z, meta["iterations"], weights=w, cap=10)
                if np.abs(w[0]).max() <= 2.0 and w[1].min() >= 0.0 and w[1].max() <= 1024.0:
                    decs["learned_f16x2"] = wl.LearnedDecoder(rate, z, meta["iterations"], weights=w, cap=10,
                                                              precision=wl.LMS_F16X2)
            for name, dec in decs.items():
                print(f"{RATE_NAMES[rate]} z={z} {name}")
                pts = sweep(rate, z, dec, start=args.start if args.start is not None else starts[rate],
                            max_bits=args.max_bits)
                entry["decoders"][name] = {"points": pts, "ebno_at_ber_1e-5": ebno_at(pts)}
            if args.capacity and rate != 4:
                entry["capacity_search_ebno_db"] = capacity_search(rate, z, decs["plain"])
            res["codes"].append(entry)
            res["seconds"] = round(time.time() - t0, 1)
            save(res, args.out)   # after every code, so a partial sweep is kept
    print("Eb/N0 at BER 1e-5:")
    for e in res["codes"]:
        print(f"  {e['rate']:5s} z={e['z']:3d}  " + "  ".join(
            f"{k}: {v['ebno_at_ber_1e-5'] if v['ebno_at_ber_1e-5'] is None else round(v['ebno_at_ber_1e-5'], 3)}"
            for k, v in e["decoders"].items()))
    print(f"wrote {args.out}")


if __name__ == "__main__":
    main()
