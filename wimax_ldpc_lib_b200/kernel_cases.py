"""Runs each kernel of the library once on one seeded case of a chosen size,
for profilers (ncu: every launch below is one capture) and quick timing.

  python -m wimax_ldpc_lib_b200.kernel_cases [--frames F] [--cases decode,encode,train,syndrome,bits,lfsr,nullspace]

  decode     F frames of rate 1/2 z = 96 at 2.25 dB and of rate 5/6 z = 96 at
             4 dB (framegen_kernel), each decoded once by the plain decoder
             (tdmp_decode_kernel), the learned decoder with its shipped
             weights (lms_decode_kernel) and the same weights in packed
             binary16 (lms16_decode_kernel), cap 10
  encode     F rate 1/2 z = 96 info words (encode_lanes_kernel)

  train      one Adam step of the learned decoder's training (rate 1/2,
             z = 96, F/16 frames generated on the device): framegen_kernel,
             lms_train_kernel, lms_reduce_adam_kernel
  syndrome   compute_syndrome over F host frames of rate 1/2 z = 96 hard bits
             (syndrome_lanes_kernel, reference lib/ldpc_decoder.cc:67-104)
  bits       decode(int8_t*) over F host frames of +-1 hard bits with 50 flips
             (bits_to_llr_kernel, then the decoder; reference
             lib/ldpc_decoder.cc:108-118)
  lfsr       BER_runner's info-bit stream, F * 1152 bits (lfsr_bits_kernel,
             reference lib/BER_runner.cc:124-146)
  nullspace  F random rate 3/4B z = 96 codewords from the null space of H
             with AWGN (framegen_nullspace_kernel)

Every case prints its wall time; kernels run on the default stream.
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

import wimax_ldpc_lib_b200 as wl  # noqa: E402

CASES = ("decode", "encode", "train", "syndrome", "bits", "lfsr", "nullspace")


def main():
    import torch
    ap = argparse.ArgumentParser()
    ap.add_argument("--frames", type=int, default=65536)
    ap.add_argument("--cases", default=",".join(CASES))
    ap.add_argument("--seed", type=int, default=12345)
    args = ap.parse_args()
    torch.cuda.set_device(0)
    F = args.frames
    rng = np.random.default_rng(args.seed)
    for case in [c for c in args.cases.split(",") if c]:
        t0 = time.perf_counter()
        if case == "decode":
            extra = []
            for rate, ebno in ((0, 2.25), (5, 4.0)):
                n = 24 * 96
                llr = torch.empty((F, n), dtype=torch.float32, device="cuda")
                hard = torch.empty((F, n), dtype=torch.int8, device="cuda")
                st = torch.empty(F, dtype=torch.int32, device="cuda")
                wl.framegen_device(rate, 96, args.seed, 0, F, ebno, ebno, llr=llr)
                meta, w, _ = wl.learned_weights(rate, 96)
                decs = [wl.Decoder(rate, 96, 10),
                        wl.LearnedDecoder(rate, 96, meta["iterations"], weights=w, cap=10),
                        wl.LearnedDecoder(rate, 96, meta["iterations"], weights=w, cap=10, precision=wl.LMS_F16X2)]
                for dec in decs:
                    dec.decode_device(llr, hard, None, st)
                    torch.cuda.synchronize()
                    extra.append(f"{(st & 0xFFFF).float().mean().item():.2f}")
            extra = "mean iterations " + " ".join(extra)
        elif case == "encode":
            enc = wl.Encoder(0, 96)
            info = torch.from_numpy(rng.integers(0, 2, (F, enc.k), dtype=np.uint8)).cuda()
            cw = torch.empty((F, enc.n), dtype=torch.uint8, device="cuda")
            enc.encode_device(info, cw)
            torch.cuda.synchronize()
            extra = f"codeword weight {cw.float().mean().item():.3f}"
        elif case == "train":
            lms = wl.LearnedDecoder(0, 96, 8)
            hist = lms.train(1, max(64, F // 16), 1.0, 3.0, args.seed)
            extra = f"loss {hist[0]:.5f}"
        elif case in ("syndrome", "bits"):
            dec = wl.Decoder(0, 96, 10)
            n = dec.n
            if case == "syndrome":
                bits = rng.integers(0, 2, (F, n), dtype=np.int8)
                out = dec.syndrome_host(bits)
                extra = f"mean failing rows {out.mean():.1f}"
            else:
                enc = wl.Encoder(0, 96)
                info = torch.from_numpy(rng.integers(0, 2, (F, dec.k), dtype=np.uint8)).cuda()
                cw = torch.empty((F, n), dtype=torch.uint8, device="cuda")
                enc.encode_device(info, cw)
                torch.cuda.synchronize()
                bits = cw.cpu().numpy().astype(np.int8)
                flips = rng.integers(0, n, (F, 50))
                np.put_along_axis(bits, flips, 1 - np.take_along_axis(bits, flips, 1), 1)
                dec_bits, ne = dec.decode_bits_host(bits)
                extra = f"frames still failing {int(ne.sum())}"
        elif case == "lfsr":
            out = torch.empty(F * 1152, dtype=torch.uint8, device="cuda")
            wl.lfsr_bits_device(0, out)
            torch.cuda.synchronize()
            extra = f"ones {out[:115200].sum().item()}"
        elif case == "nullspace":
            n = 24 * 96
            cw = torch.empty((F, n), dtype=torch.uint8, device="cuda")
            llr = torch.empty((F, n), dtype=torch.float32, device="cuda")
            wl.framegen_nullspace_device(4, 96, args.seed, 0, F, 3.0, 3.0, codeword=cw, llr=llr)
            torch.cuda.synchronize()
            extra = f"mean codeword weight {cw.float().mean().item():.3f}"
        else:
            raise SystemExit(f"unknown case {case}; choose from {', '.join(CASES)}")
        print(f"{case}: {time.perf_counter() - t0:.3f} s ({extra})")


if __name__ == "__main__":
    main()
