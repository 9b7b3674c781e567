"""Generates the committed golden fixtures of tests/golden. Run in a checkout that has pirate's
source tree available (its path is the required first argument):

    python tests/golden/make_golden.py PIRATE_SRC

  example_plan_trees.json  config + per-tree plan fields of pirate's configs/example_dedispersion_plan.yml
                           (the plan pirate's own 'show_dedisperser' printed for configs/dedispersion/chord_sb2_et.yml)
  toy_fp32.npz             seeded inputs/weights and the fp32 oracle's outputs on a small config
"""

import json
import os
import sys

import numpy as np
import yaml

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

import helpers as H  # noqa: E402


def example_plan(src):
    with open(os.path.join(src, "configs", "dedispersion", "chord_sb2_et.yml")) as f:
        cfg = yaml.safe_load(f)
    with open(os.path.join(src, "configs", "example_dedispersion_plan.yml")) as f:
        plan = yaml.safe_load(f)
    keys = ["ndm_out", "nt_out", "dm_min", "dm_max", "trigger_frequency", "primary_tree_index",
            "early_trigger_level", "amb_rank", "dd_rank", "nt_ds", "max_width", "dm_downsampling",
            "time_downsampling", "Dcore", "nprofiles", "wt_dm_downsampling", "wt_time_downsampling",
            "ndm_wt", "nt_wt", "frequency_subband_counts"]
    out = dict(config=cfg, stage1_dd_rank=plan["stage1_dd_rank"], stage1_amb_rank=plan["stage1_amb_rank"],
               trees=[{k: t[k] for k in keys} for t in plan["trees"]])
    with open(os.path.join(HERE, "example_plan_trees.json"), "w") as f:
        json.dump(out, f, indent=1)


def toy():
    prim = [dict(num_early_triggers=0, max_width=8, dm_downsampling=0, time_downsampling=0, wt_dm_downsampling=8,
                 wt_time_downsampling=16),
            dict(num_early_triggers=1, max_width=4, dm_downsampling=0, time_downsampling=0, wt_dm_downsampling=8,
                 wt_time_downsampling=16)]
    cfg = H.toy_config(rank=7, nfreq=200, nt=128, subbands=[2, 2, 1], beams_per_gpu=2, beams_per_batch=1,
                       primary_trees=prim)
    xs = H.make_inputs(cfg, 2, seed=2024)
    orc, _ = H.run_oracle(cfg, xs[:0], [])
    ws = H.make_weights(orc, seed=7)
    _, res = H.run_oracle(cfg, xs, ws, 1, 32)
    d = dict(config=json.dumps(cfg), nseq=len(xs), ntrees=orc.ntrees)
    for s, x in enumerate(xs):
        d["x%d" % s] = x
        for i in range(orc.ntrees):
            d["max_%d_%d" % (s, i)] = res[s][0][i]
            d["arg_%d_%d" % (s, i)] = res[s][1][i]
    for i, w in enumerate(ws):
        d["w%d" % i] = w
    np.savez_compressed(os.path.join(HERE, "toy_fp32.npz"), **d)


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit("usage: python tests/golden/make_golden.py PIRATE_SRC")
    src = sys.argv[1]
    example_plan(src)
    toy()
    print("wrote", os.listdir(HERE))
