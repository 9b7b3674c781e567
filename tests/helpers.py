"""Shared helpers for the parity tests: seeded inputs/weights, runs of the CUDA path through the
public API, and runs of the CPU oracle on identical inputs."""

import numpy as np

import oracle as O


def toy_config(rank=8, nfreq=640, nt=256, dtype="float32", subbands=(2, 2, 1), beams_per_gpu=2,
               beams_per_batch=1, num_active_batches=1, primary_trees=None, zone_nfreq=None,
               zone_freq_edges=None):
    if primary_trees is None:
        primary_trees = [
            dict(num_early_triggers=0, max_width=16, dm_downsampling=0, time_downsampling=0,
                 wt_dm_downsampling=16, wt_time_downsampling=16),
            dict(num_early_triggers=1, max_width=8, dm_downsampling=0, time_downsampling=0,
                 wt_dm_downsampling=16, wt_time_downsampling=16),
        ]
    return dict(zone_nfreq=list(zone_nfreq or [nfreq]), zone_freq_edges=list(zone_freq_edges or [400.0, 800.0]),
                time_sample_ms=1.0, toplevel_tree_rank=rank, time_samples_per_chunk=nt, dtype=dtype,
                frequency_subband_counts=list(subbands), primary_trees=primary_trees,
                beams_per_gpu=beams_per_gpu, beams_per_batch=beams_per_batch,
                num_active_batches=num_active_batches, future_write_max_samples=0, max_gpu_clag=10000)


def quantize(x, dtype):
    """Rounds float32 data to the storage dtype and back (what the GPU path sees)."""
    import torch
    t = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float32))
    return t.to(getattr(torch, dtype)).to(torch.float32).numpy()


def make_inputs(cfg, nchunks, seed, pulse=None):
    """Seeded N(0,1) inputs, one (B, nfreq, nt) array per (chunk, batch) in seq_id order."""
    rng = np.random.default_rng(seed)
    B = cfg["beams_per_batch"]
    nb = cfg["beams_per_gpu"] // B
    F = sum(cfg["zone_nfreq"])
    T = cfg["time_samples_per_chunk"]
    xs = []
    for s in range(nchunks * nb):
        x = rng.standard_normal((B, F, T)).astype(np.float32)
        xs.append(quantize(x, cfg["dtype"]))
    return xs


def make_weights(orc, seed, nbatches_wt=1, kind="random"):
    rng = np.random.default_rng(seed + 1000)
    ws = []
    for i in range(orc.ntrees):
        shp = orc.wt_shape(i)
        if kind == "random":
            w = np.stack([O.random_weights(shp, rng) for _ in range(nbatches_wt)])
        else:
            w = np.stack([O.bare_weights(shp, orc.trees[i]["nprofiles"]) for _ in range(nbatches_wt)])
        ws.append(w)
    return ws


def run_gpu(pb, cfg, xs, weights, nbatches_wt=1):
    """Runs the CUDA path through pirate_b200.GpuDedisperser; returns per-seq (out_max, out_argmax) lists."""
    import torch
    plan = pb.DedispersionPlan(pb.DedispersionConfig.from_dict(cfg))
    dd = pb.GpuDedisperser(plan, cuda_device_id=0, num_consumers=1, nbatches_wt=nbatches_wt)
    dd.allocate()
    for i, w in enumerate(weights):
        dd.fill_all_weights(i, w)
    tdt = getattr(torch, cfg["dtype"])
    res = []
    for seq, x in enumerate(xs):
        with dd.get_input() as arr:
            arr.copy_(torch.from_numpy(x).to(tdt).to(arr.device))
        with dd.get_output(0, sync=True) as out:
            res.append(([m.float().cpu().numpy().astype(np.float64) for m in out.out_max],
                        [a.cpu().numpy().view(np.uint32).copy() for a in out.out_argmax]))
    torch.cuda.synchronize()
    return plan, dd, res


def run_oracle(cfg, xs, weights, sophistication=1, real_bits=32, keep=None):
    orc = O.OracleDedisperser(cfg, sophistication, real_bits)
    nb = cfg["beams_per_gpu"] // cfg["beams_per_batch"]
    res = []
    for seq, x in enumerate(xs):
        ib = seq % nb
        wts = [w[seq % w.shape[0]] for w in weights]
        m, a = orc.dedisperse(ib, x, wts)
        extra = keep(orc, seq) if keep else None
        res.append((m, a, extra))
    return orc, res
