"""GpuDedisperser.fill_analytic_weights (src_lib/GpuDedisperser.cpp:1162-1238) on the GPU. The
weights it writes are checked through the dedisperser's outputs: with float32 storage they are
bitwise those of the oracle run with weights 1/sqrt(float32(variance)) of PfAvarApproximation,
replicated over every weight slot, beam and weight-time index."""

import numpy as np
import pytest

import helpers as H

pytestmark = pytest.mark.gpu


def _analytic_weights(pb, plan, fv, nbatches_wt):
    """Host weights (nbatches_wt, B, ndm_wt, nt_wt, P, N) that fill_analytic_weights should write
    (pirate: PeakFindingKernelParams::fill_host_weights with randomize=false,
    src_lib/PeakFindingKernel.cu:606-692)."""
    a = pb.PfAvarApproximation(plan, fv)
    ws = []
    for t, v in zip(plan.trees, a.tree_variance):
        base = (1.0 / np.sqrt(v.astype(np.float32).astype(np.float64))).astype(np.float32)   # (N, D, P)
        w = np.transpose(base, (1, 2, 0))                                                   # (D, P, N)
        w = np.broadcast_to(w[:, None], (t.ndm_wt, t.nt_wt, t.nprofiles, t.nsubbands))
        ws.append(np.ascontiguousarray(np.broadcast_to(w, (nbatches_wt, plan.beams_per_batch) + w.shape)))
    return ws


def _run(pb, cfg, xs, fv, nbatches_wt):
    import torch
    plan = pb.DedispersionPlan(pb.DedispersionConfig.from_dict(cfg))
    dd = pb.GpuDedisperser(plan, cuda_device_id=0, num_consumers=1, nbatches_wt=nbatches_wt)
    dd.allocate()
    dd.fill_analytic_weights(fv)
    res = []
    for x in xs:
        with dd.get_input() as arr:
            arr.copy_(torch.from_numpy(x).to(arr.device))
        with dd.get_output(0, sync=True) as out:
            res.append(([m.float().cpu().numpy().astype(np.float64) for m in out.out_max],
                        [a.cpu().numpy().view(np.uint32).copy() for a in out.out_argmax]))
    torch.cuda.synchronize()
    return plan, res


def test_fill_analytic_weights_vs_oracle(pb2lib):
    cfg = H.toy_config(rank=8, nfreq=300, nt=512, beams_per_gpu=4, beams_per_batch=2)
    plan = pb2lib.DedispersionPlan(pb2lib.DedispersionConfig.from_dict(cfg))
    rng = np.random.default_rng(17)
    fv = rng.uniform(0.2, 3.0, plan.nfreq)
    xs = H.make_inputs(cfg, 2, seed=17)
    ws = _analytic_weights(pb2lib, plan, fv, nbatches_wt=2)
    _, ores = H.run_oracle(cfg, xs, ws)
    _, g = _run(pb2lib, cfg, xs, fv, nbatches_wt=2)
    for seq in range(len(xs)):
        for i in range(plan.ntrees):
            assert np.array_equal(g[seq][0][i], ores[seq][0][i]), "seq %d tree %d out_max" % (seq, i)
            assert np.array_equal(g[seq][1][i], ores[seq][1][i]), "seq %d tree %d out_argmax" % (seq, i)


def test_fill_analytic_weights_errors(pb2lib):
    """Before allocate(): an error. A bad freq_variances array: an error that stops the dedisperser,
    so that its next call fails too (pirate's stoppable-object rule, notes/stoppable_class.md)."""
    cfg = H.toy_config(rank=6, nfreq=100, nt=256)
    plan = pb2lib.DedispersionPlan(pb2lib.DedispersionConfig.from_dict(cfg))
    dd = pb2lib.GpuDedisperser(plan, cuda_device_id=0, num_consumers=1)
    with pytest.raises(RuntimeError, match="allocate"):
        dd.fill_analytic_weights(np.ones(plan.nfreq))
    dd = pb2lib.GpuDedisperser(plan, cuda_device_id=0, num_consumers=1)
    dd.allocate()
    bad = np.ones(plan.nfreq)
    bad[3] = -1.0
    with pytest.raises(RuntimeError, match="freq_variances"):
        dd.fill_analytic_weights(bad)
    with pytest.raises(RuntimeError):
        dd.fill_analytic_weights(np.ones(plan.nfreq))
