"""Trains the proposal network on the GPU and writes its parameters.

    python -m cumulus3d_b200.train_proposal [--scenes 600] [--steps 6000] [--out cumulus3d_b200/weights/proposal_aerial.npz]

Training set: `--scenes` seeded crop scenes (256×256 reference crops of the 1920×1080 aerial formation, 4 source
windows each) labelled by the engine's own 6-iteration plain PatchStereo; AdamW, batch 8, lr 1e-3 (1e-4 for the last
quarter of the steps), weight decay 1e-4.  Reports the held-out gain (agreement with the plain 6-iteration result after
1 iteration from random vs learned init) at the end.
"""
from __future__ import annotations

import argparse
import json
import pathlib
import time

from . import proposal


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--scenes", type=int, default=600)
    ap.add_argument("--steps", type=int, default=6000)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=1000)
    ap.add_argument("--out", type=pathlib.Path, default=proposal.DEFAULT_WEIGHTS)
    ap.add_argument("--report", type=pathlib.Path, default=None)
    a = ap.parse_args(argv)
    t0 = time.time()
    data = proposal.make_training_set(a.scenes, seed=a.seed)
    t_data = time.time() - t0
    print(f"training set: {a.scenes} scenes, valid label fraction {data.valid_fraction:.3f}, {t_data:.1f}s", flush=True)
    net = proposal.ProposalNet(0, seed=1)
    t1 = time.time()
    k = (3 * a.steps) // 4
    losses = proposal.train(net, data, k, a.batch, a.lr, seed=1)
    losses += proposal.train(net, data, a.steps - k, a.batch, a.lr * 0.1, seed=2)
    t_train = time.time() - t1
    meta = {"scenes": a.scenes, "steps": a.steps, "batch": a.batch, "lr": a.lr, "seed": a.seed,
            "final_loss": sum(losses[-50:]) / max(len(losses[-50:]), 1)}
    net.save(a.out, meta)
    gain = proposal.evaluate_gain(net, n_scenes=8, iters=1)
    rep = {**meta, "valid_fraction": data.valid_fraction, "seconds_data": t_data, "seconds_train": t_train,
           "ms_per_step": 1e3 * t_train / a.steps, "first_loss": sum(losses[:20]) / 20, "heldout": gain}
    print(json.dumps(rep), flush=True)
    if a.report:
        a.report.write_text(json.dumps(rep, indent=1))
    net.close()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
