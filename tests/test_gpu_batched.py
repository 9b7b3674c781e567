"""Many beams with uneven plans in one replayed CUDA graph (pirate_b200.BatchedDedisperser, C ABI
pb2_batched_*): groups of different tree ranks, numbers of primary trees and beam counts run one chunk
each per graph launch; every group's float32 outputs must equal the fp32 oracle's (which restates
pirate's ReferenceDedisperser) bit for bit, before and after the autotuner has changed the schedule."""

import numpy as np
import pytest

import helpers as H

pytestmark = pytest.mark.gpu

GROUPS = [   # (rank, nfreq, primary trees as (early triggers, max width), beams, subbands)
    (8, 640, [(0, 16), (1, 8)], 2, [0, 1, 1]),
    (9, 300, [(1, 32), (0, 8), (0, 4)], 1, [1, 1, 1]),
    (10, 1024, [(0, 32)], 3, [0, 0, 1]),
]


def _cfgs(dtype="float32"):
    out = []
    for rank, nfreq, pts, beams, sb in GROUPS:
        prim = H._prim(rank, [(e, w, 0) for e, w in pts], 16)
        out.append(H.toy_config(rank=rank, nfreq=nfreq, nt=512, dtype=dtype, subbands=sb, beams_per_gpu=beams,
                                beams_per_batch=beams, primary_trees=prim))
    return out


def _run(bd, cfgs, xs, nchunks):
    import torch
    res = []
    for c in range(nchunks):
        for g, cfg in enumerate(cfgs):
            bd.input(g).copy_(torch.from_numpy(xs[g][c]).to(bd.device))
        bd.step()
        torch.cuda.synchronize()
        res.append([([m.float().cpu().numpy().astype(np.float64) for m in bd.outputs(g).out_max],
                     [a.cpu().numpy().view(np.uint32).copy() for a in bd.outputs(g).out_argmax]) for g in range(len(cfgs))])
    return res


def test_batched_graph_matches_oracle_and_autotune(pb2lib):
    pb = pb2lib
    cfgs = _cfgs()
    nchunks = 5
    plans = [pb.DedispersionPlan(pb.DedispersionConfig.from_dict(c)) for c in cfgs]
    bd = pb.BatchedDedisperser(plans, cuda_device_id=0)
    bd.allocate()
    xs, ores = [], []
    for g, cfg in enumerate(cfgs):
        x = H.make_inputs(cfg, nchunks, seed=40 + g)
        orc, _ = H.run_oracle(cfg, [], [])
        ws = H.make_weights(orc, seed=50 + g)
        for i, w in enumerate(ws):
            bd.fill_all_weights(g, i, w)
        _, r = H.run_oracle(cfg, x, ws, 1, 32)
        xs.append(x)
        ores.append(r)

    def check(res, what):
        for c in range(nchunks):
            for g in range(len(cfgs)):
                for i in range(len(ores[g][c][0])):
                    assert np.array_equal(res[c][g][0][i], ores[g][c][0][i]), (what, c, g, i, "out_max")
                    assert np.array_equal(res[c][g][1][i], ores[g][c][1][i]), (what, c, g, i, "out_argmax")

    check(_run(bd, cfgs, xs, nchunks), "default schedule")
    nk = bd.kernels_per_step()
    assert nk >= 1 + sum(1 + len(c["primary_trees"]) for c in cfgs)
    rec = bd.autotune(reps=2)
    assert "chosen" in rec and len(rec["chosen"]["groups"]) == len(cfgs)
    check(_run(bd, cfgs, xs, nchunks), "autotuned schedule")
    # every schedule choice gives the same bits
    bd.set_schedule([False] * 3, [True] * 3, [256] * 3, concurrent=False)
    bd.reset()
    check(_run(bd, cfgs, xs, nchunks), "serial, unmerged, general peak finder")
