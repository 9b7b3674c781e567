"""Generates tests/golden/avar_golden.npz: pirate's own analytic peak-finding variances
(pirate_frb/slow_avar/PfVariance.py: PfAvarApproximation, pure numpy) on small plans, and a strided
sample of them on the benchmark's full rank-16 plan, as fixtures for pirate_b200.PfAvarApproximation
and GpuDedisperser.fill_analytic_weights.

    python tests/golden/make_avar_golden.py PIRATE_SRC      (the pirate source tree, required)

pirate's python package cannot be imported as a whole here (its compiled extension is not built), so
the two pure-numpy modules are loaded from their files with small stand-ins for the two names they
import from the rest of the package (integer_log2, and constants.max_pf_width = 32 from
include/pirate/constants.hpp). The plan they see is this repository's DedispersionPlan (its tree
fields are pinned against pirate's example plan by the other fixtures), seen through the attribute
names pirate's python uses.
"""

import importlib.util
import json
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import helpers as H  # noqa: E402
import pirate_b200 as pb  # noqa: E402


def load_slow_avar(src):
    pkg = types.ModuleType("pirate_frb")
    pkg.__path__ = []
    utils = types.ModuleType("pirate_frb.utils")

    def integer_log2(n):
        n = int(n)
        if n <= 0 or (n & (n - 1)):
            raise ValueError(n)
        return n.bit_length() - 1

    utils.integer_log2 = integer_log2
    pyb = types.ModuleType("pirate_frb.pirate_pybind11")
    pyb.constants = types.SimpleNamespace(max_pf_width=32)
    sub = types.ModuleType("pirate_frb.slow_avar")
    sub.__path__ = []
    sys.modules.update({"pirate_frb": pkg, "pirate_frb.utils": utils, "pirate_frb.pirate_pybind11": pyb,
                        "pirate_frb.slow_avar": sub})
    mods = {}
    for name in ("SparseTile", "PfVariance"):
        full = "pirate_frb.slow_avar." + name
        spec = importlib.util.spec_from_file_location(full, os.path.join(src, "pirate_frb", "slow_avar", name + ".py"))
        m = importlib.util.module_from_spec(spec)
        sys.modules[full] = m
        spec.loader.exec_module(m)
        mods[name] = m
    return mods["PfVariance"]


def plan_view(plan):
    """This repository's plan under the attribute names pirate's python plan has."""
    trees = []
    for t in plan.trees:
        fs = types.SimpleNamespace(pf_rank=t.pf_rank, N=t.nsubbands, n_to_flo=list(t.n_to_flo), n_to_fhi=list(t.n_to_fhi))
        pf = types.SimpleNamespace(wt_dm_downsampling=t.wt_dm_downsampling)
        trees.append(types.SimpleNamespace(total_rank=t.total_rank, frequency_subbands=fs, pf=pf,
                                           nprofiles=t.nprofiles, primary_tree_index=t.primary_tree_index))
    cfg = types.SimpleNamespace(make_channel_map=plan.config.make_channel_map)
    return types.SimpleNamespace(nfreq=plan.nfreq, ntrees=plan.ntrees, trees=trees, config=cfg)


def pt(et, w, wt_dm, wt_t=16):
    return dict(num_early_triggers=et, max_width=w, dm_downsampling=0, time_downsampling=0,
                wt_dm_downsampling=wt_dm, wt_time_downsampling=wt_t)


# (name, config): small plans covering early triggers, downsampled primary trees (upper-half delays),
# several zones, more input channels than tree channels and the reverse, subbands, and widths to 32.
CASES = [
    ("toy_r8", H.toy_config(rank=8, nfreq=300, nt=512)),
    ("r6_zones", H.toy_config(rank=6, nfreq=None, nt=512, subbands=[1, 1, 1], zone_nfreq=[400, 250, 350],
                              zone_freq_edges=[400.0, 500.0, 650.0, 800.0],
                              primary_trees=[pt(0, 16, 8), pt(1, 8, 8), pt(0, 4, 4)])),
    ("r9_w32", H.toy_config(rank=9, nfreq=200, nt=1024, subbands=[0, 1, 1, 1], zone_nfreq=[120, 80],
                            zone_freq_edges=[300.0, 550.0, 800.0],
                            primary_trees=[pt(0, 32, 64, 64), pt(2, 16, 32), pt(0, 8, 16)])),
    ("r5_full_wt", H.toy_config(rank=5, nfreq=40, nt=256, subbands=[1],
                                primary_trees=[pt(0, 8, 32), pt(1, 4, 4)])),
]


# The benchmark's plan at full size: rank 16 from 16384 channels over 400-800 MHz, 5 primary trees
# (widths to 32, weight downsampling 64), full-band search, float16 storage. Its per-channel variances
# come from FULL_SEED; the fixture keeps every FULL_STRIDE-th variance of each tree (flat index).
FULL = dict(zone_nfreq=[16384], zone_freq_edges=[400.0, 800.0], time_sample_ms=1.0, toplevel_tree_rank=16,
            time_samples_per_chunk=2048, dtype="float16", frequency_subband_counts=[0, 0, 0, 0, 1],
            primary_trees=[pt(0, 32, 64, 64) for _ in range(5)], beams_per_gpu=1, beams_per_batch=1,
            num_active_batches=1, future_write_max_samples=0, max_gpu_clag=10000)
FULL_SEED = 7
FULL_STRIDE = 13


def full_freq_variances(nfreq):
    return np.random.default_rng(FULL_SEED).uniform(0.5, 1.5, nfreq)


def main():
    if len(sys.argv) < 2:
        sys.exit("usage: python tests/golden/make_avar_golden.py PIRATE_SRC")
    src = sys.argv[1]
    PV = load_slow_avar(src)
    rng = np.random.default_rng(2024)
    out = {}
    plan = pb.DedispersionPlan(pb.DedispersionConfig.from_dict(FULL))
    ref = PV.PfAvarApproximation(plan_view(plan), full_freq_variances(plan.nfreq))
    out["full_r16/config"] = np.frombuffer(json.dumps(FULL).encode(), dtype=np.uint8)
    for i, v in enumerate(ref.tree_variance):
        out["full_r16/tree%d_strided" % i] = np.asarray(v, dtype=np.float64).ravel()[::FULL_STRIDE].copy()
    print("full_r16", plan.ntrees, "trees", [v.shape for v in ref.tree_variance])
    for name, cfg in CASES:
        plan = pb.DedispersionPlan(pb.DedispersionConfig.from_dict(cfg))
        fv = plan.config.make_random_freq_variances(rng=rng)
        fv = fv * rng.uniform(0.5, 1.5, size=fv.shape)       # per-channel variation on top of the zones
        ref = PV.PfAvarApproximation(plan_view(plan), fv)
        out[name + "/config"] = np.frombuffer(json.dumps(cfg).encode(), dtype=np.uint8)
        out[name + "/freq_variances"] = fv
        for i, v in enumerate(ref.tree_variance):
            out["%s/tree%d" % (name, i)] = np.asarray(v, dtype=np.float64)
        print(name, plan.ntrees, "trees", [v.shape for v in ref.tree_variance])
    np.savez_compressed(os.path.join(HERE, "avar_golden.npz"), **out)


if __name__ == "__main__":
    main()
