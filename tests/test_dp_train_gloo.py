"""Data-parallel training of the learned min-sum on CPU: two gloo ranks run
train_lms.train_data_parallel with half the batch each; the gradient of a
rank's frames comes from the oracle's restated forward/backward (standing in
for wldpc_lms_step_grad) and Adam is restated in numpy (standing in for
wldpc_lms_apply_grad). Both ranks end with identical weights, equal to one
process training on the whole batch."""
import os
import socket

import numpy as np
import torch
import torch.multiprocessing as mp

RATE, Z, T, BATCH, STEPS, SEED, LR = 0, 24, 2, 4, 3, 41, 1e-2


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


class OracleModel:
    """grad_size / step_grad / apply_grad of LearnedDecoder, on the oracle."""

    def __init__(self, oracle):
        self.o = oracle
        self.w = np.zeros((2, T, 12, 24), np.float32)
        self.w[0] = 0.815
        self.m = np.zeros(self.w.size)
        self.v = np.zeros(self.w.size)
        self.t = 0

    def grad_size(self):
        return self.w.size

    def step_grad(self, batch, lo, hi, seed, first, grad, loss):
        _, cw, llr, _ = self.o.framegen(RATE, Z, seed, first, batch, lo, hi)
        l, g = self.o.learned_loss_grad(RATE, Z, T, self.w, llr.astype(np.float32), cw)
        grad.copy_(torch.from_numpy(g))
        loss[0] = l

    def apply_grad(self, grad, lr):
        g = grad.numpy()
        self.t += 1
        self.m = 0.9 * self.m + 0.1 * g
        self.v = 0.999 * self.v + 0.001 * g * g
        mh = self.m / (1 - 0.9 ** self.t)
        vh = self.v / (1 - 0.999 ** self.t)
        self.w = (self.w.reshape(-1) - lr * mh / (np.sqrt(vh) + 1e-8)).astype(np.float32).reshape(self.w.shape)


def _run(oracle, rank, world, batch, all_reduce):
    from wimax_ldpc_lib_b200.train_lms import train_data_parallel
    model = OracleModel(oracle)
    curve, _ = train_data_parallel(model, STEPS, batch, 1.5, 2.5, LR, SEED, rank, world, all_reduce,
                                   lambda n: torch.zeros(n, dtype=torch.float64), chunk=STEPS, log=lambda *_: None)
    return model.w, curve


def _worker(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from oracle.oracle import Oracle
    w, curve = _run(Oracle(), rank, world, BATCH // world, lambda t: dist.all_reduce(t))
    out.put((rank, w, curve))
    dist.destroy_process_group()


def test_two_ranks_match_one_process(oracle):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict((r, (w, c)) for r, w, c in (q.get(timeout=180) for _ in procs))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    w_one, curve_one = _run(oracle, 0, 1, BATCH, lambda t: None)
    assert np.array_equal(res[0][0], res[1][0])                      # replicas identical
    assert not np.array_equal(w_one[0], np.float32(0.815) * np.ones_like(w_one[0]))   # it trained
    np.testing.assert_allclose(res[0][0], w_one, rtol=0, atol=1e-6)  # same frames, same steps
    assert abs(res[0][1][-1][1] - curve_one[-1][1]) <= 1e-9 * max(1.0, abs(curve_one[-1][1]))
