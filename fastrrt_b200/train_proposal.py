"""Trains the learned expansion proposal on the planner's own solves and
saves its weights (npz of w1, b1, w2, b2, w3, b3).

    python -m fastrrt_b200.train_proposal [--plans N] [--epochs E] [--out PATH]

Training rows come from seeded batched requests (mixed 128 / 256 / 512
frames, 5-30% obstacles, seeds from 500000 on, disjoint from the evaluation
seeds), half of them the single-instance 256 x 256 layout; the network is
trained by the library's own GPU kernels.  With --rounds 2 a second set of
requests (new seeds) is solved with the first network attached and the
final network is trained on the rows of both.
"""
import argparse
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_WEIGHTS = os.path.join(HERE, "proposal_weights.npz")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--plans", type=int, default=16384)
    ap.add_argument("--epochs", type=int, default=12)
    ap.add_argument("--batch", type=int, default=512)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--c0-share", type=float, default=0.5)
    ap.add_argument("--rounds", type=int, default=2)
    ap.add_argument("--out", default=DEFAULT_WEIGHTS)
    a = ap.parse_args()
    import torch

    from . import proposal as P
    t0 = time.time()
    X, L, solved = P.collect_dataset(a.plans, seed0=500_000, max_rows=2_000_000, c0_share=a.c0_share)
    t1 = time.time()
    net = P.ProposalNet(seed=a.seed, max_batch=a.batch)
    loss = net.train(X, L, len(L), epochs=a.epochs, batch=a.batch, lr=a.lr, seed=a.seed)
    for r in range(1, a.rounds):
        X2, L2, s2 = P.collect_dataset(a.plans, seed0=500_000 + r * 10_000_000, max_rows=2_000_000,
                                       c0_share=a.c0_share, net=net)
        X, L = torch.cat([X, X2]), torch.cat([L, L2])
        solved += s2
        net = P.ProposalNet(seed=a.seed + r, max_batch=a.batch)
        loss = net.train(X, L, len(L), epochs=a.epochs, batch=a.batch, lr=a.lr, seed=a.seed + r)
    t2 = time.time()
    ws = net.get_weights()
    np.savez_compressed(a.out, **{k: w for k, w in zip(["w1", "b1", "w2", "b2", "w3", "b3"], ws)},
                        rows=len(L), plans=a.plans * a.rounds, solved=solved, loss=loss)
    print(f"rows {len(L)} from {solved} solved of {a.plans * a.rounds} plans ({t1 - t0:.1f} s), "
          f"trained {a.epochs} epochs in {t2 - t1:.1f} s, last-batch loss {loss:.3f} -> {a.out}")


def load(net, path=DEFAULT_WEIGHTS):
    """loads saved weights into a ProposalNet; False when the file is absent"""
    if not os.path.exists(path):
        return False
    d = np.load(path)
    net.set_weights([d[k] for k in ["w1", "b1", "w2", "b2", "w3", "b3"]])
    return True


if __name__ == "__main__":
    main()
