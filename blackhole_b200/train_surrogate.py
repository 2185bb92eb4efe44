"""Train the learned transfer function on rays the integrator traces.

    python -m blackhole_b200.train_surrogate --frames 4096 --size 128 \
        --epochs 16 --out blackhole_b200/data/surrogate_c4.npz

Training set: n_frames frames of size x size pixels over alpha, beta in
[-15, 15] M with a random sub-pixel shift, spin a ~ U[0, 0.998] and
inclination ~ U[5, 89] deg per frame (per-frame seeds), observer r = 1000 M,
traced by the mixed-precision DP45 tracer (rtol 1e-8) with two disk
crossings recorded; 4096 frames of 128^2 are 2^26 rays. A held-out set of
frames with other seeds measures class accuracy, the fraction of pixels
above the confidence gate and the error of the first-hit radius.
"""
from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np
import torch

from . import surrogate as S


def evaluate(net: S.Surrogate, data: S.RaySet, min_conf: float = 0.99) -> dict:
    head = net.forward(data.inputs)
    t = data.targets
    cls = t[:, 0].long()
    used = cls >= 0
    p = torch.softmax(head[:, 0:3], dim=1)
    conf, pred = p.max(1)
    ok = used & (pred == cls)
    gate = conf >= min_conf
    disk = used & (cls == 1) & (pred == 1)
    r_rel = (torch.exp(head[disk, 3] + 2) - torch.exp(t[disk, 2] + 2)).abs() / torch.exp(t[disk, 2] + 2)
    g_rel = (head[disk, 9] - t[disk, 8]).abs() / (t[disk, 8] + 1)
    esc = used & (cls == 2) & (pred == 2)
    th_err = (head[esc, 10].clamp(-1, 1).acos() - t[esc, 9].clamp(-1, 1).acos()).abs()
    return {
        "accuracy": float(ok.sum() / used.sum()),
        "confident_fraction": float((gate & used).sum() / used.sum()),
        "confident_accuracy": float((ok & gate).sum() / max(1, int((gate & used).sum()))),
        "r1_rel_median": float(r_rel.median()) if r_rel.numel() else None,
        "r1_rel_p99": float(torch.quantile(r_rel[:100000], 0.99)) if r_rel.numel() else None,
        "g_rel_median": float(g_rel.median()) if g_rel.numel() else None,
        "theta_inf_median": float(th_err.median()) if th_err.numel() else None,
    }


def main(argv=None) -> dict:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--frames", type=int, default=4096)
    ap.add_argument("--size", type=int, default=128)
    ap.add_argument("--epochs", type=float, default=16.0)
    ap.add_argument("--batch", type=int, default=16384)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--holdout-frames", type=int, default=64)
    ap.add_argument("--out", default="blackhole_b200/data/surrogate_c4.npz")
    ap.add_argument("--log", default=None, help="JSON lines log file")
    ap.add_argument("--source-commit", default=None,
                    help="git commit of the sources, for the manifest (default: asked of git)")
    a = ap.parse_args(argv)

    t0 = time.time()
    data = S.generate_rays(a.frames, a.size, seed=a.seed)
    hold = S.generate_rays(a.holdout_frames, a.size, seed=a.seed + 1000003)
    torch.cuda.synchronize()
    t_data = time.time() - t0
    net = S.Surrogate(max_batch=a.batch, seed=a.seed)
    logf = open(a.log, "w") if a.log else None

    def log(rec):
        line = json.dumps(rec)
        print(line, flush=True)
        if logf:
            logf.write(line + "\n")
            logf.flush()

    log({"event": "data", "rays": int(data.inputs.shape[0]), "holdout": int(hold.inputs.shape[0]), "seconds": t_data})
    t1 = time.time()
    steps_per_epoch = data.inputs.shape[0] // a.batch
    S.train(net, data, epochs=a.epochs, batch=a.batch, lr=a.lr, seed=a.seed, log_every=max(1, steps_per_epoch),
            log=lambda r: log({"event": "train", **r}))
    torch.cuda.synchronize()
    t_train = time.time() - t1
    if net.device_error() != 0:
        raise RuntimeError("a surrogate kernel reported a timed-out wait")
    ev = evaluate(net, hold)
    rec = {"event": "done", "train_seconds": t_train, "epochs": a.epochs, "batch": a.batch, **ev}
    log(rec)
    net.save(a.out, manifest={
        "seed": a.seed,
        "git_commit": a.source_commit,
        "train": {"epochs": a.epochs, "batch": a.batch, "lr": a.lr, "optimizer": "Adam, cosine learning rate",
                  "train_seconds": t_train},
        "data": {"frames": a.frames, "size": a.size, "holdout_frames": a.holdout_frames,
                 "window_M": 15.0, "spin": [0.0, 0.998], "theta_obs_deg": [5.0, 89.0], "r_obs": 1000.0,
                 "tracer": "mixed-precision DP45 rtol 1e-8, 2 crossings", "seed": a.seed},
        "holdout": ev,
    })
    if logf:
        logf.close()
    return rec


if __name__ == "__main__":
    main()
