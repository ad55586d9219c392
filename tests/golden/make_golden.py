"""Generates the golden fixtures in this folder from the reference itself.

Run in a checkout where the reference sources are available (default
/root/reference) after ``make -C oracle ref``; the reference is compiled from
its own unmodified sources by oracle/Makefile into oracle/_ref/. Inputs come
from tests/inputs.py (bit-reproducible everywhere), so the fixtures store only
per-frame digests of the reference's outputs plus small scalars:

  decode_golden.json   TDMP decoder (NMS / OMS / MS builds): per frame the
                       digest of (posterior float32 bytes, hard bits), the
                       return value and the iteration count (by the
                       smaller-cap recipe of oracle/ref_harness.cc)
  encode_golden.json   encoder outputs for all 114 (rate, z)
  tables_golden.json   digests of the expanded check-node tables, D and X
  misc_golden.json     int8 decode adapter, compute_syndrome and BER_runner
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from oracle.oracle import MS, NMS, OMS, Oracle, Reference  # noqa: E402
import inputs  # noqa: E402

Z_ALL = list(range(24, 97, 4))


def decode_case(ref, rate, z, llr, max_iter, with_iters=True):
    post, dec, ret = ref.decode(rate, z, llr, max_iter)
    case = {"digests": inputs.frame_digests(post, dec), "ret": ret.astype(int).tolist()}
    if with_iters:
        it = ref.iterations(rate, z, llr, cap=max_iter)
        case["iters"] = it.astype(int).tolist()   # cap+1 marks "not converged within cap"
    return case


def main():
    oracle = Oracle()
    refs = {NMS: Reference(NMS), OMS: Reference(OMS), MS: Reference(MS)}
    dec = {"cases": []}
    # the 1024-frame rate-1/2 z=24 workload at 2.0 dB, cap 10
    info, cw, llr = inputs.frames(oracle, 0, 24, 1024, 2.0, seed=1000)
    c = decode_case(refs[NMS], 0, 24, llr, 10)
    c.update(name="r12_z24_2dB", kind="awgn", rate=0, z=24, frames=1024, ebno=2.0, seed=1000, max_iter=10, mode=NMS)
    dec["cases"].append(c)
    # all 114 variants, 16 frames each
    for rate in range(6):
        for z in Z_ALL:
            eb = inputs.SWEEP_EBNO[rate]
            seed = 2000 + 100 * rate + z
            info, cw, llr = inputs.frames(oracle, rate, z, 16, eb, seed=seed)
            c = decode_case(refs[NMS], rate, z, llr, 10)
            c.update(name=f"sweep_r{rate}_z{z}", kind="awgn", rate=rate, z=z, frames=16, ebno=eb, seed=seed,
                     max_iter=10, mode=NMS)
            dec["cases"].append(c)
    # the other two flavours
    for mode in (OMS, MS):
        for (rate, z) in [(0, 24), (0, 96), (2, 60), (5, 96), (4, 44)]:
            eb = inputs.SWEEP_EBNO[rate]
            seed = 5000 + 100 * rate + z + 7 * mode
            info, cw, llr = inputs.frames(oracle, rate, z, 32, eb, seed=seed)
            c = decode_case(refs[mode], rate, z, llr, 10, with_iters=False)
            c.update(name=f"mode{mode}_r{rate}_z{z}", kind="awgn", rate=rate, z=z, frames=32, ebno=eb, seed=seed,
                     max_iter=10, mode=mode)
            dec["cases"].append(c)
    # edge cases at several caps
    for kind in ["zeros", "ties", "huge", "valid", "noise"]:
        for (rate, z) in [(0, 24), (5, 96), (3, 52)]:
            for max_iter in (0, 1, 10):
                seed = 7000 + 13 * rate + z
                llr = inputs.edge_llr(kind, rate, z, 24, seed, oracle)
                c = decode_case(refs[NMS], rate, z, llr, max_iter, with_iters=max_iter > 0)
                c.update(name=f"edge_{kind}_r{rate}_z{z}_cap{max_iter}", kind=kind, rate=rate, z=z, frames=24,
                         seed=seed, max_iter=max_iter, mode=NMS)
                dec["cases"].append(c)
    with open(os.path.join(HERE, "decode_golden.json"), "w") as f:
        json.dump(dec, f, separators=(",", ":"))

    enc = {"cases": []}
    for rate in range(6):
        for z in Z_ALL:
            n, m, k = inputs.code_dims(rate, z)
            seed = 9000 + 100 * rate + z
            u = inputs.info_bits(seed, 4, k)
            u[0, :4] = [2, 5, 255, 1]     # non-0/1 bytes pass through the systematic copy
            cwr = refs[NMS].encode(rate, z, u)
            enc["cases"].append({"rate": rate, "z": z, "seed": seed, "frames": 4,
                                 "digests": [inputs.digest(cwr[f]) for f in range(4)]})
    with open(os.path.join(HERE, "encode_golden.json"), "w") as f:
        json.dump(enc, f, separators=(",", ":"))

    tab = {"cases": []}
    for rate in range(6):
        for z in Z_ALL:
            t = refs[NMS].checknode_table(rate, z)
            ci = refs[NMS].code_info(rate, z)
            tab["cases"].append({"rate": rate, "z": z, "rows": int(t.shape[0]), "cols": int(t.shape[1]),
                                 "D": ci["D"], "X": ci["X"], "N": ci["N"], "M": ci["M"],
                                 "digest": inputs.digest(t.astype("<i2"))})
    with open(os.path.join(HERE, "tables_golden.json"), "w") as f:
        json.dump(tab, f, separators=(",", ":"))

    misc = {"decode_bits": [], "syndrome": [], "ber_runner": []}
    for (rate, z) in [(0, 24), (0, 96), (5, 96), (1, 40)]:
        n, m, k = inputs.code_dims(rate, z)
        seed = 11000 + 100 * rate + z
        u = inputs.info_bits(seed, 16, k)
        cwr = refs[NMS].encode(rate, z, u).astype(np.int8)
        flips = inputs.raw(seed + 1, 16 * 8).reshape(16, 8) % np.uint64(n)
        bits = cwr.copy()
        for f in range(16):
            for v in flips[f]:
                bits[f, int(v)] ^= 1
        bits[0, :3] = [3, -1, 2]            # odd bytes: XOR semantics of the reference
        d, ret = refs[NMS].decode_bits(rate, z, bits, 10)
        misc["decode_bits"].append({"rate": rate, "z": z, "seed": seed, "digests": [inputs.digest(d[f]) for f in range(16)],
                                    "ret": ret.astype(int).tolist()})
        misc["syndrome"].append({"rate": rate, "z": z, "seed": seed,
                                 "count": refs[NMS].syndrome(rate, z, bits, False).astype(int).tolist(),
                                 "early": refs[NMS].syndrome(rate, z, bits, True).astype(int).tolist()})
    L = refs[NMS].lib
    for (rate, z, eb, iters) in [(0, 24, 1.5, 40), (0, 96, 1.75, 20), (5, 48, 3.5, 30), (2, 72, 2.25, 20)]:
        h = L.ref_ber_create(rate, z, 1, 10)
        bers = [L.ref_ber_run_iteration(h, eb) for _ in range(iters)]
        misc["ber_runner"].append({"rate": rate, "z": z, "ebno": eb, "iters": iters, "ber": bers,
                                   "bits": int(L.ref_ber_bits(h)), "errors": int(L.ref_ber_errors(h)),
                                   "cw_len": int(L.ref_ber_codeword_len(h)),
                                   "dw_len": int(L.ref_ber_dataword_len(h))})
        L.ref_ber_destroy(h)
    with open(os.path.join(HERE, "misc_golden.json"), "w") as f:
        json.dump(misc, f, separators=(",", ":"))
    print("golden fixtures written")


if __name__ == "__main__":
    main()
