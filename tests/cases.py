"""Rebuilds the inputs of a golden decode case (see tests/golden/make_golden.py)."""
import numpy as np

import inputs


def case_llr(oracle, case) -> np.ndarray:
    if case["kind"] == "awgn":
        _, _, llr = inputs.frames(oracle, case["rate"], case["z"], case["frames"], case["ebno"], case["seed"])
        return llr
    return inputs.edge_llr(case["kind"], case["rate"], case["z"], case["frames"], case["seed"], oracle)


def expected_iters(case):
    """iterations as the decoder reports them: cap+1 in the fixture means 'ran to the cap'."""
    cap = case["max_iter"]
    return [min(i, cap) for i in case["iters"]]
