"""Training and evaluation of the learned candidate sifter on pipeline candidates.

    python -m pirate_b200.sifter_study [--config rank16|small] [--train N] [--test N] [--out results.json]

Events come from pirate_b200.sifter.CandidateGenerator (pulses from pirate's simpulse model, N(0,1)
noise, RFI) run through the dedispersion pipeline; the training events and the held-out test events
use different seeds (different noise, pulse bank, RFI draws). The sifter is trained by its own CUDA
kernels on the candidates that passed the 6-sigma threshold, then scored on the test events. Reported:
recall of the test pulses at several false-alarm fractions of the test negatives (noise and RFI
events), for the sifter's logit and for the plain threshold's peak SNR, overall and per negative kind.
"""

import argparse
import json
import time

import numpy as np

import pirate_b200 as pb
from pirate_b200 import sifter as S


def config(name):
    """rank16: the benchmark's rank-16 pipeline (16384 channels, 5 primary trees, 2048-sample chunks,
    float16 storage), 8 beams per batch. small: rank 12 from 2048 channels, 1024-sample chunks."""
    def prim(rank, n, wt_time):
        return [dict(num_early_triggers=0, max_width=32, dm_downsampling=0, time_downsampling=0,
                     wt_dm_downsampling=2 ** ((rank - (1 if i else 0)) // 2), wt_time_downsampling=wt_time)
                for i in range(n)]
    if name == "rank16":
        rank, nfreq, nt = 16, 16384, 2048
    else:
        rank, nfreq, nt = 12, 2048, 1024
    return dict(zone_nfreq=[nfreq], zone_freq_edges=[400.0, 800.0], time_sample_ms=1.0, toplevel_tree_rank=rank,
                time_samples_per_chunk=nt, dtype="float16", frequency_subband_counts=[0, 0, 0, 0, 1],
                primary_trees=prim(rank, 5, 64), beams_per_gpu=8, beams_per_batch=8, num_active_batches=1,
                future_write_max_samples=0, max_gpu_clag=10000)


def dm_range(cfg):
    """DMs whose full-band sweep (4.148806e6 ms MHz^2 cm^3/pc x DM x (400^-2 - 800^-2)) stays within 95%
    of a chunk, so that a pulse fits in its event's two chunks."""
    per_dm = 4.148806e6 * (400.0 ** -2 - 800.0 ** -2) / cfg["time_sample_ms"]
    hi = 0.95 * cfg["time_samples_per_chunk"] / per_dm
    return (0.2 * hi, hi)


def study(cfg, n_train, n_test, epochs=40, batch=256, lr=2e-3, nbank=64, seed=0, log=None, fars=(1e-2, 1e-3, 1e-4)):
    import torch
    t0 = time.time()
    dr = dm_range(cfg)
    tr = S.CandidateGenerator(cfg, seed=seed + 1, nbank=nbank, dm_range=dr, log=log).generate(n_train)
    t1 = time.time()
    te = S.CandidateGenerator(cfg, seed=seed + 2, nbank=nbank, dm_range=dr, log=log).generate(n_test)
    t2 = time.time()
    sf = S.Sifter(device=0, max_batch=512, seed=seed + 7)
    v = tr["valid"] == 1
    hist = sf.fit(torch.from_numpy(tr["patch"][v]).cuda(), tr["label"][v], epochs=epochs, batch=batch, lr=lr, log=log)
    t3 = time.time()
    logit = sf.forward(torch.from_numpy(te["patch"]).cuda()).cpu().numpy().astype(np.float64)
    score = np.where(te["valid"] == 1, logit, -np.inf)
    peak = np.where(te["valid"] == 1, te["peak"].astype(np.float64), -np.inf)
    pos, neg = te["label"] == 1, te["label"] == 0
    res = dict(config=cfg, dm_range=list(dr), n_train=int(n_train), n_test=int(n_test),
               train_valid=int(v.sum()), test_positives=int(pos.sum()), test_negatives=int(neg.sum()),
               test_negatives_by_kind={"noise": int((te["kind"] == 1).sum()), "rfi": int((te["kind"] == 2).sum())},
               test_positives_with_candidate=int((pos & (te["valid"] == 1)).sum()),
               loss_history=[float(x) for x in hist],
               seconds=dict(generate_train=t1 - t0, generate_test=t2 - t1, train=t3 - t2), recall={})
    for far in fars:
        rs = S.recall_at_far(score[pos], score[neg], far)
        rt = S.recall_at_far(peak[pos], peak[neg], far)
        res["recall"]["%g" % far] = dict(sifter=rs[0], sifter_false_alarms=rs[2], threshold=rt[0],
                                         threshold_false_alarms=rt[2], allowed_false_alarms=int(np.floor(far * neg.sum())))
    # Per negative kind (noise-only negatives: the threshold's home ground).
    for kind, k in (("noise", 1), ("rfi", 2)):
        nk = te["kind"] == k
        rs = S.recall_at_far(score[pos], score[nk], 1e-2)
        rt = S.recall_at_far(peak[pos], peak[nk], 1e-2)
        res["recall"]["1e-2_vs_%s_only" % kind] = dict(sifter=rs[0], threshold=rt[0])
    return res, sf


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", default="rank16", choices=["rank16", "small"])
    ap.add_argument("--train", type=int, default=40000)
    ap.add_argument("--test", type=int, default=20000)
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--out", default=None)
    ap.add_argument("--weights", default=None, help="write the trained parameters (npz)")
    args = ap.parse_args()
    res, sf = study(config(args.config), args.train, args.test, epochs=args.epochs, log=lambda s: print(s, flush=True))
    txt = json.dumps(res, indent=1)
    print(txt)
    if args.out:
        with open(args.out, "w") as f:
            f.write(txt)
    if args.weights:
        np.savez_compressed(args.weights, params=sf.get_params())


if __name__ == "__main__":
    main()
