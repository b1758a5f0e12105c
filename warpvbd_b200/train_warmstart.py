"""Train the warm-start network on the GPU and save it.

    python -m warpvbd_b200.train_warmstart [--out PATH] [--seed S] [--epochs E] [--lr LR]

Generates about 8.2M samples from seeded plain-VBD rollouts of 1000 steps,
every 25th step recorded (cantilever and mass-spring environments -- cubes of
7-15 voxels under columns of 5-30, the range of the benchmark batch -- E
log-uniform in [1e5, 1e7] Pa, nu in [0.30, 0.48], random gravity direction
per batch, N(0, 0.1^2) m/s initial velocity noise), trains the MLP for 24
epochs with the project's CUDA kernels and writes the model
(parameters and normalisation) (default: warpvbd_b200/data/warmstart_mlp.npz).  Prints a JSON
summary with the dataset size, the training loss curve, R^2 and timings.
"""
import argparse
import json
import time

from . import warmstart as ws


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=ws.DEFAULT_WEIGHTS)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--epochs", type=int, default=24)
    ap.add_argument("--batches", type=int, default=6)
    ap.add_argument("--envs", type=int, default=24)
    ap.add_argument("--steps", type=int, default=1000, help="steps per rollout")
    ap.add_argument("--every", type=int, default=25, help="record every n-th step")
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--batch", type=int, default=4096, help="minibatch size")
    ap.add_argument("--fine", action="store_true",
                    help="include 1 m cantilevers of 40 and 80 voxels in the rollouts")
    ap.add_argument("--target-tol", type=float, default=None,
                    help="solve the recorded steps to this tolerance for their targets")
    ap.add_argument("--cube", type=int, nargs=2, default=(7, 15),
                    help="mass-spring cube edge range (voxels, inclusive)")
    ap.add_argument("--column", type=int, nargs=2, default=(5, 30),
                    help="mass-spring column length range (voxels, inclusive)")
    args = ap.parse_args()
    import torch
    t0 = time.perf_counter()
    X, Y = ws.rollout_dataset(seed=args.seed, n_batches=args.batches,
                              envs_per_batch=args.envs, steps=args.steps,
                              record_every=args.every, fine=args.fine,
                              target_tol=args.target_tol, cube=tuple(args.cube),
                              column=tuple(args.column))
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    model, info = ws.train_warmstart(X, Y, epochs=args.epochs, batch=args.batch, lr=args.lr,
                                     seed=args.seed)
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    ws.save(args.out, model, {"loss": info["loss"], "r2": info["r2"],
                               "samples": info["samples"], "seed": args.seed})
    print(json.dumps({"samples": info["samples"], "loss": info["loss"], "r2": info["r2"],
                      "rollout_s": t1 - t0, "train_s": t2 - t1, "out": args.out}))


if __name__ == "__main__":
    main()
