"""Trains the learned Richardson-Lucy proposal (libapr_b200.learned) on plain
GPU RL trajectories of seeded deconvolution volumes and writes its weights.

    python -m libapr_b200.train_proposal [--volumes 200] [--shape 128,512,512]
                                        [--lr 1e-3] [--out libapr_b200/data/rl_proposal_cnn.npz]

Volume v uses seed 10000 + 2 v (evaluation uses other seeds).  From each
volume's RL trajectory (u_0 = 1) the pairs (u_i, u_{i+10}) for i in
PAIR_ITERATIONS train the network, one Adam step per pair.
"""
import argparse
import json
import os
import sys
import time

PAIR_ITERATIONS = (10, 20, 40, 80, 160, 320)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--volumes", type=int, default=200)
    ap.add_argument("--shape", default="128,512,512")
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--max-minutes", type=float, default=30.0)
    ap.add_argument("--out", default=None)
    ap.add_argument("--log", default=None)
    args = ap.parse_args(argv)
    import torch
    from libapr_b200 import learned as Lr
    shape = tuple(int(v) for v in args.shape.split(","))
    net = Lr.ProposalCNN(seed=args.seed)
    out = args.out or Lr.WEIGHTS_FILE
    t0 = time.time()
    log = []
    for v in range(args.volumes):
        apr, raw, psf, _ = Lr.deconvolution_workload(shape, seed=10000 + 2 * v)
        P = raw.numel()
        u = torch.empty(P, dtype=torch.float32, device="cuda")
        done = 0
        losses = []
        for i in PAIR_ITERATIONS:
            Lr.rl_iterations(apr, raw, u, psf, i - done, resume=done > 0)
            u0 = u.clone()
            Lr.rl_iterations(apr, raw, u, psf, 10, resume=True)
            done = i + 10
            losses.append(net.train_step(apr, raw, u0, u, psf, lr=args.lr))
        rec = {"volume": v, "particles": P, "loss": losses, "seconds": time.time() - t0}
        log.append(rec)
        print(json.dumps(rec), flush=True)
        del apr
        if (v + 1) % 10 == 0 or v + 1 == args.volumes:
            net.save(out)
        if time.time() - t0 > 60 * args.max_minutes:
            print("time limit reached after %d volumes" % (v + 1), flush=True)
            break
    net.save(out)
    if args.log:
        with open(args.log, "w") as f:
            json.dump(log, f)
    return 0


if __name__ == "__main__":
    sys.exit(main())
