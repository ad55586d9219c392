"""Trains the learned min-sum decoder on the GPU and writes its weight file.

  python -m wimax_ldpc_lib_b200.train_lms --rate 0 --z 96 --iterations 8 \
      --steps 20000 --batch 4096 --ebno 1.0 3.0 --lr 1e-3 --out weights/lms_r0_z96_T8.json

Everything runs in the library (wldpc_lms_train): frames are generated on the
device from fresh counters every step (random info bits, the encoder, BPSK,
AWGN at an Eb/N0 drawn uniformly per frame), the project's forward/backward
kernels compute the BCE loss and its gradient, and the Adam kernel updates
the weights. The weights start at the normalized min-sum constants
(a = 0.815, b = 0). The output is JSON: the weight table
(2 x T x 12 x 24: a then b, [iteration][layer][base column]) and the run's
settings and loss curve.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

import wimax_ldpc_lib_b200 as wl  # noqa: E402


def train(rate, z, iterations, steps, batch, ebno_lo, ebno_hi, lr, seed, chunk=500, log=print):
    lms = wl.LearnedDecoder(rate, z, iterations)
    curve, t0 = [], time.time()
    done = 0
    while done < steps:
        k = min(chunk, steps - done)
        hist = lms.train(k, batch, ebno_lo, ebno_hi, seed, first_frame=done * batch, lr=lr)
        done += k
        curve.append([done, float(hist.mean())])
        log(f"step {done:6d}  loss {hist.mean():.5f}  ({time.time() - t0:.1f} s)")
    return lms, curve, time.time() - t0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--rate", type=int, default=0)
    ap.add_argument("--z", type=int, default=96)
    ap.add_argument("--iterations", type=int, default=8)
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--ebno", type=float, nargs=2, default=[1.0, 3.0])
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=0x5EED1)
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    import torch
    assert torch.cuda.is_available(), "training runs on the GPU"
    lms, curve, secs = train(args.rate, args.z, args.iterations, args.steps, args.batch, args.ebno[0],
                             args.ebno[1], args.lr, args.seed)
    out = args.out or os.path.join(HERE, "weights", f"lms_r{args.rate}_z{args.z}_T{args.iterations}.json")
    os.makedirs(os.path.dirname(out), exist_ok=True)
    meta = {"format": "wimax_ldpc_lib_b200 learned min-sum weights v1",
            "rate": args.rate, "z": args.z, "iterations": args.iterations,
            "model": "message = s * max(a[t,i,c] * min - b[t,i,c], 0), layered, fp32",
            "training": {"steps": args.steps, "batch": args.batch, "ebno_db": args.ebno, "lr": args.lr,
                         "optimizer": "Adam(0.9, 0.999, 1e-8)", "seed": args.seed,
                         "loss": "mean BCE over iterations, bits and frames", "seconds": round(secs, 1),
                         "device": torch.cuda.get_device_name(0)},
            "loss_curve": curve,
            "weights": lms.get_weights().tolist()}
    with open(out, "w") as f:
        json.dump(meta, f)
    print(f"wrote {out}")


if __name__ == "__main__":
    main()
