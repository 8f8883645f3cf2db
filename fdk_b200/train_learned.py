"""Train and evaluate the learned residual row filter on the C5 workload.

    python -m fdk_b200.train_learned [--n-train 2000] [--epochs 20] [--n-test 200]
                                      [--loss-region volume|fov] [--time-limit S]
                                      [--out fdk_b200/weights/residual_c5.npz]
    python -m fdk_b200.train_learned --eval-only [--out weights.npz]   # held-out result only

Writes the trained parameters (npz) and prints one JSON line with the held-out result: MSE of
plain Hann-ramp FDK, of the learned filter, and of the gated choice (the learned reconstruction
kept only where it beats plain FDK against the phantom), plus the training history.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

from fdk_b200 import learned  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n-train", type=int, default=2000)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--n-test", type=int, default=200)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--time-limit", type=float, default=None, help="stop training after this many seconds")
    ap.add_argument("--schedule", default="cosine", choices=["constant", "cosine"])
    ap.add_argument("--input-window", default=None, help="ramp window of the network's input rows (default: hann)")
    ap.add_argument("--batch", type=int, default=1, help="phantoms per Adam step (gradients averaged)")
    ap.add_argument("--loss-region", default="volume", choices=["volume", "fov"],
                    help="voxels of the training loss: the whole cube or the fully sampled field of view")
    ap.add_argument("--eval-only", action="store_true", help="evaluate the weights at --out, no training")
    ap.add_argument("--out", default=os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights",
                                                  "residual_c5.npz"))
    args = ap.parse_args()
    log = lambda *a: print(*a, file=sys.stderr, flush=True)  # noqa: E731
    t0 = time.time()
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)

    window = args.input_window or "hann"
    if args.eval_only:
        w = np.load(args.out)
        window = str(w["input_window"]) if "input_window" in w else window
        ev = learned.evaluate(w["params"], args.n_test, input_window=None if window == "hann" else window)
        print(json.dumps({"weights": os.path.relpath(args.out), "input_window": window, "eval": ev}), flush=True)
        return

    def checkpoint(ep, params, hist):
        np.savez(args.out, params=params, history=np.asarray(hist), steps=(ep + 1) * (args.n_train // args.batch),
                 input_window=window)

    tr = learned.train(args.n_train, args.epochs, args.lr, log=log, time_limit_s=args.time_limit, on_epoch=checkpoint,
                       schedule=args.schedule, input_window=args.input_window, batch=args.batch,
                       loss_region=args.loss_region)
    np.savez(args.out, params=tr["params"], history=np.asarray(tr["history"]), steps=tr["steps"], input_window=window)
    ev = learned.evaluate(tr["params"], args.n_test, input_window=args.input_window)
    out = {"workload": "C5: 256^3, 90 views of 256^2, I0=1e4, mu=0.02/mm", "n_train": args.n_train,
           "schedule": args.schedule, "input_window": window, "lr": args.lr, "batch": args.batch,
           "loss_region": args.loss_region,
           "epochs_requested": args.epochs, "epochs_run": len(tr["history"]), "steps": tr["steps"],
           "stopped_early": tr["stopped_early"], "train_seconds": tr["seconds"], "history": tr["history"],
           "eval": ev, "total_seconds": time.time() - t0, "weights": os.path.relpath(args.out)}
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
