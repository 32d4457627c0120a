"""Train the learned gas optics on the GPU and write its weights.

    python -m ccpp_physics_b200.train_surrogate [--samples 20000000] [--epochs 100]
                                                [--out ccpp_physics_b200/data/lw_surrogate_weights.npz]

Training data: `--samples` layer samples (whole 127-layer columns of the
synthetic profile generator, seed 101) labelled by the library's plain FP64
setcoef + taumol (rrtmg_lw_gpu_gas_optics).  Training: the library's own
tcgen05 forward/backward kernels and Adam (rrtmg_lw_gpu_surrogate_train),
batch 8,192, learning rate 3e-3 decaying (cosine) to 1e-5, optical-depth
errors weighted by 1/(1 + 1.66 tau).  The weights file also records the
per-epoch loss, the training time and the sample count.
"""
from __future__ import annotations

import argparse
import time

import numpy as np


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--samples", type=int, default=20_000_000)
    ap.add_argument("--epochs", type=int, default=100)
    ap.add_argument("--lr", type=float, default=3e-3)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--out", default=None)
    args = ap.parse_args(argv)
    import torch
    from . import rrtmg_lw as lw
    from . import surrogate as sg
    rc, msg = lw.rlwinit(device=0)
    if rc:
        raise SystemExit(msg)
    t0 = time.time()
    feats, targ = sg.make_dataset(args.samples, seed=101)
    norm = sg.normalisation(feats, targ)
    y = sg.normalise_targets(targ, norm)
    del targ
    torch.cuda.synchronize()
    t_data = time.time() - t0
    sg.init(norm, seed=args.seed)
    t0 = time.time()
    losses = sg.train(feats, y, epochs=args.epochs, batch=8192, lr=args.lr, lr_final=1e-5, tau_weight=True)
    torch.cuda.synchronize()
    t_train = time.time() - t0
    out = args.out or sg.WEIGHTS_PATH
    sg.save(out, losses=losses, train_seconds=np.float64(t_train), data_seconds=np.float64(t_data),
            samples=np.int64(feats.shape[0]), epochs=np.int64(args.epochs), batch=np.int64(8192),
            samples_per_second=np.float64(feats.shape[0] * args.epochs / t_train))
    print(f"trained {feats.shape[0]} samples x {args.epochs} epochs in {t_train:.1f} s "
          f"({feats.shape[0] * args.epochs / t_train / 1e6:.1f} M samples/s), final loss {losses[-1]:.3e} -> {out}")


if __name__ == "__main__":
    main()
