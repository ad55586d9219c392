"""Trains the learned min-sum decoder on the GPU and writes its weight file.

  python -m wimax_ldpc_lib_b200.train_lms --rate 0 --z 96 --iterations 8 \
      --steps 20000 --batch 4096 --ebno 1.0 3.0 --lr 1e-3 --out weights/lms_r0_z96_T8.json

Data-parallel over N GPUs (each rank --batch frames per step, gradients
all-reduced over NCCL, identical Adam steps on every rank):

  torchrun --nproc-per-node N -m wimax_ldpc_lib_b200.train_lms --batch 2048 ...

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


def train_data_parallel(model, steps, batch, ebno_lo, ebno_hi, lr, seed, rank, world, all_reduce, new_buffer,
                        chunk=500, log=print):
    """Data-parallel training over `world` ranks (one GPU each). At step s rank
    r draws frames [(s * world + r) * batch, ... + batch) -- so the job's
    step covers the same frames as one process with world * batch frames --,
    computes their gradient, the ranks' gradients are summed by `all_reduce`
    (in place) and divided by `world`, and every rank applies the same Adam
    step, so the replicas stay identical. `model` has grad_size / step_grad /
    apply_grad (LearnedDecoder); `new_buffer(n)` makes a float32 buffer of n
    values that step_grad, all_reduce and apply_grad accept."""
    grad, loss = new_buffer(model.grad_size()), new_buffer(1)
    curve, acc, t0 = [], 0.0, time.time()
    for s in range(steps):
        model.step_grad(batch, ebno_lo, ebno_hi, seed, (s * world + rank) * batch, grad, loss)
        all_reduce(grad)
        grad /= world
        all_reduce(loss)
        model.apply_grad(grad, lr)
        acc += float(loss[0]) / world
        if (s + 1) % chunk == 0 or s + 1 == steps:
            n = (s % chunk) + 1
            curve.append([s + 1, acc / n])
            if rank == 0:
                log(f"step {s + 1:6d}  loss {acc / n:.5f}  ({time.time() - t0:.1f} s, {world} ranks)")
            acc = 0.0
    return curve, time.time() - t0


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
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = 0
    if world > 1:
        # torchrun: one rank per GPU, gradients all-reduced over NCCL; --batch is per rank
        import datetime
        import torch.distributed as dist
        rank, local = int(os.environ["RANK"]), int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        lms = wl.LearnedDecoder(args.rate, args.z, args.iterations)
        curve, secs = train_data_parallel(lms, args.steps, args.batch, args.ebno[0], args.ebno[1], args.lr, args.seed,
                                          rank, world, lambda t: dist.all_reduce(t),
                                          lambda n: torch.zeros(n, dtype=torch.float32, device="cuda"))
        dist.barrier()
        dist.destroy_process_group()
        if rank != 0:
            return
    else:
        lms, curve, secs = train(args.rate, args.z, args.iterations, args.steps, args.batch, args.ebno[0],
                                 args.ebno[1], args.lr, args.seed)
    out = args.out or os.path.join(HERE, "weights", f"lms_r{args.rate}_z{args.z}_T{args.iterations}.json")
    os.makedirs(os.path.dirname(out), exist_ok=True)
    meta = {"format": "wimax_ldpc_lib_b200 learned min-sum weights v1",
            "rate": args.rate, "z": args.z, "iterations": args.iterations,
            "model": "message = s * max(a[t,i,c] * min - b[t,i,c], 0), layered, fp32",
            "training": {"steps": args.steps, "batch": args.batch * world, "ranks": world,
                         "ebno_db": args.ebno, "lr": args.lr,
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
