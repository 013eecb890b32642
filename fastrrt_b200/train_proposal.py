"""Trains the learned expansion proposal on the planner's own solves and
saves its weights (npz of w1, b1, w2, b2, w3, b3).

    python -m fastrrt_b200.train_proposal [--plans N] [--epochs E] [--source S] [--rows R]
                                          [--batch B] [--out PATH]

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
    ap.add_argument("--source", default="paths", choices=("paths", "nodes", "both"),
                    help="rows: expansions on validated paths, every accepted expansion, or both")
    ap.add_argument("--rows", type=int, default=2_000_000, help="rows collected per round at most")
    ap.add_argument("--out", default=DEFAULT_WEIGHTS)
    a = ap.parse_args()
    import torch

    from . import proposal as P
    t0 = time.time()
    X, L, solved = P.collect_dataset(a.plans, seed0=500_000, max_rows=a.rows, c0_share=a.c0_share,
                                     source=a.source)
    t1 = time.time()
    train_s, trained_rows = 0.0, 0

    def train(seed):
        nonlocal train_s, trained_rows
        net = P.ProposalNet(seed=seed, max_batch=a.batch)
        torch.cuda.synchronize()
        ts = time.time()
        loss = net.train(X, L, len(L), epochs=a.epochs, batch=a.batch, lr=a.lr, seed=seed)
        torch.cuda.synchronize()
        train_s += time.time() - ts
        trained_rows += (len(L) // a.batch) * a.batch * a.epochs
        return net, loss

    net, loss = train(a.seed)
    for r in range(1, a.rounds):
        X2, L2, s2 = P.collect_dataset(a.plans, seed0=500_000 + r * 10_000_000, max_rows=a.rows,
                                       c0_share=a.c0_share, net=net, source=a.source)
        X, L = torch.cat([X, X2]), torch.cat([L, L2])
        solved += s2
        net, loss = train(a.seed + r)
    t2 = time.time()
    rows_per_s = trained_rows / max(train_s, 1e-9)
    tflops = rows_per_s * P.TRAIN_FLOP_PER_ROW / 1e12
    ws = net.get_weights()
    np.savez_compressed(a.out, **{k: w for k, w in zip(["w1", "b1", "w2", "b2", "w3", "b3"], ws)},
                        rows=len(L), plans=a.plans * a.rounds, solved=solved, loss=loss, source=a.source,
                        batch=a.batch, epochs=a.epochs, train_s=train_s, train_rows_per_s=rows_per_s,
                        train_tflops=tflops)
    print(f"rows {len(L)} ({a.source}) from {solved} solved of {a.plans * a.rounds} plans "
          f"({t1 - t0:.1f} s to collect the first round), trained {a.epochs} epochs per round in "
          f"{train_s:.1f} s ({rows_per_s:.3g} rows/s, {tflops:.1f} TFLOP/s), last-batch loss {loss:.3f} "
          f"-> {a.out}; {t2 - t0:.1f} s in all")


def load(net, path=DEFAULT_WEIGHTS):
    """loads saved weights into a ProposalNet; False when the file is absent"""
    if not os.path.exists(path):
        return False
    d = np.load(path)
    net.set_weights([d[k] for k in ["w1", "b1", "w2", "b2", "w3", "b3"]])
    return True


if __name__ == "__main__":
    main()
