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


# (rank, nfreq, nt, subbands, primary trees as (num_early_triggers, max_width), beams_per_gpu, beams_per_batch)
PARITY_CASES = [
    (6, 100, 128, [1], [(0, 4)], 1, 1),
    (8, 640, 256, [2, 2, 1], [(0, 16), (1, 8)], 2, 1),
    (9, 300, 256, [1, 1, 1], [(1, 32), (0, 8), (1, 2)], 2, 2),
    (10, 1024, 512, [0, 0, 1], [(0, 32), (0, 16), (0, 8)], 1, 1),
    (11, 2000, 256, [3, 5, 3, 1], [(2, 8), (1, 4)], 4, 2),
    (7, 50, 128, [1, 1], [(0, 1), (0, 2)], 3, 1),
    # explicit output time downsampling (third entry): 16 and 32 (saturated boxcar levels, partial
    # 32-output tiles), 64, 2 and 1
    (8, 256, 512, [0, 1, 1], [(0, 32, 16), (0, 16, 32)], 2, 1),
    (7, 128, 512, [1, 1], [(0, 8, 64), (0, 4, 2), (0, 2, 1)], 1, 1),
]


def case_config(case, dtype="float32"):
    rank, nfreq, nt, sb, pts, bpg, bpb = case
    prim = []
    for ip, pt in enumerate(pts):
        net, w = pt[:2]
        tds = pt[2] if len(pt) > 2 else 0
        prim.append(dict(num_early_triggers=net, max_width=w, dm_downsampling=0, time_downsampling=tds,
                         wt_dm_downsampling=2 ** ((rank - (1 if ip else 0) - net) // 2), wt_time_downsampling=max(16, tds)))
    return toy_config(rank=rank, nfreq=nfreq, nt=nt, dtype=dtype, subbands=sb, beams_per_gpu=bpg,
                      beams_per_batch=bpb, num_active_batches=1, primary_trees=prim)


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


# ---- Fixture cases pinned to pirate's own reference dedisperser (tests/golden/make_ref_golden.py) ----

def _prim(rank, pts, wt_time=16):
    prim = []
    for ip, (net, w, tds) in enumerate(pts):
        prim.append(dict(num_early_triggers=net, max_width=w, dm_downsampling=0, time_downsampling=tds,
                         wt_dm_downsampling=2 ** ((rank - (1 if ip else 0) - net) // 2),
                         wt_time_downsampling=max(wt_time, tds)))
    return prim


def pirate_fixture_cases():
    """Cases whose outputs from pirate's ReferenceDedisperser are committed as fixtures. Each entry:
    name, cfg, nchunks, input seed, weight seed, weight kind ('random' or 'bare'), extras."""
    cases = []
    for k, c in enumerate(PARITY_CASES):
        cases.append(dict(name="parity%d_r%d" % (k, c[0]), cfg=case_config(c), nchunks=5,
                          seed=c[0] * 7 + c[2], wseed=c[0], wkind="random", extra=None))
    cases.append(dict(name="nan_r8", cfg=case_config(PARITY_CASES[1]), nchunks=3, seed=5, wseed=2,
                      wkind="random", extra="nan"))
    # The reference's own CPU-runnable case: rank 10 from 1024 channels, one tree, widths 1-8, no
    # subbands, 4 chunks of 2048 samples, one dispersed boxcar pulse (width 4, amplitude 1 per channel).
    cases.append(dict(name="rank10_pulse", cfg=toy_config(rank=10, nfreq=1024, nt=2048, subbands=[0, 0, 0, 1],
                                                         beams_per_gpu=1, beams_per_batch=1,
                                                         primary_trees=_prim(10, [(0, 8, 0)], 64)),
                      nchunks=4, seed=1010, wseed=0, wkind="bare", extra="pulse"))
    # Five primary trees at rank 12, run until the longest delay lines of every tree have wrapped
    # (tree 4's longest lag is 2^11 samples of 16-fold downsampled time, 64 chunks of 512).
    cases.append(dict(name="rank12_5trees_wrap", cfg=toy_config(rank=12, nfreq=2048, nt=512, subbands=[0, 0, 0, 0, 1],
                                                               beams_per_gpu=1, beams_per_batch=1,
                                                               primary_trees=_prim(12, [(0, 32, 0)] * 5, 16)),
                      nchunks=68, seed=1212, wseed=12, wkind="random", extra=None))
    # Rank 16 (stage ranks 8 + 8) with an early trigger, two chunks.
    cases.append(dict(name="rank16_et", cfg=toy_config(rank=16, nfreq=4096, nt=2048, subbands=[0, 2, 0, 0, 1],
                                                      beams_per_gpu=1, beams_per_batch=1,
                                                      primary_trees=_prim(16, [(1, 32, 0)], 64)),
                      nchunks=2, seed=16, wseed=16, wkind="random", extra=None))
    # Rank 16, one primary tree, 34 chunks of 2048: the longest stage-1 -> stage-2 delay lines (2^16
    # samples, 32 chunks) wrap inside the compared run. Compared on the GPU only (the CPU oracle needs
    # minutes for it).
    cases.append(dict(name="rank16_wrap", cfg=toy_config(rank=16, nfreq=4096, nt=2048, subbands=[0, 0, 0, 0, 1],
                                                        beams_per_gpu=1, beams_per_batch=1,
                                                        primary_trees=_prim(16, [(0, 32, 0)], 64)),
                      nchunks=34, seed=1616, wseed=17, wkind="random", extra=None, cpu=False))
    return cases


def fixture_inputs(case):
    """The seeded inputs of a fixture case, in seq_id order (float32, exactly representable in the
    case's storage dtype)."""
    cfg = case["cfg"]
    xs = make_inputs(cfg, case["nchunks"], seed=case["seed"])
    if case["extra"] == "nan":
        rng = np.random.default_rng(17)
        for x in xs:
            x[rng.random(x.shape) < 2e-4] = np.nan
        nb = cfg["beams_per_gpu"] // cfg["beams_per_batch"]
        xs[nb][:, :, 100:104] = np.nan
    elif case["extra"] == "pulse":
        # Dispersed boxcar: arrival t0 + k_DM * DM * (nu^-2 - nu_hi^-2) per channel (k_DM = 4.148806e6
        # ms MHz^2 cm^3 / pc), DM = 30 pc/cm^3, inside tree 0's range (full-band delay 583 of 1024 samples).
        F = sum(cfg["zone_nfreq"])
        T = cfg["time_samples_per_chunk"]
        lo, hi = cfg["zone_freq_edges"][0], cfg["zone_freq_edges"][-1]
        nu = lo + (np.arange(F) + 0.5) * (hi - lo) / F
        delay_ms = 4.148806e6 * 30.0 * (nu ** -2 - hi ** -2)
        t0 = 3000
        full = np.concatenate(xs, axis=2)   # (B, F, nchunks*T)
        for f in range(F):
            a = t0 + int(round(delay_ms[f] / cfg["time_sample_ms"]))
            full[:, f, a:a + 4] += 1.0
        xs = [np.ascontiguousarray(full[:, :, c * T:(c + 1) * T]) for c in range(case["nchunks"])]
    return xs


def fixture_weights(case, orc):
    return make_weights(orc, seed=case["wseed"], kind=case["wkind"])


def output_digest(out_max, out_argmax):
    """sha256 of one tree's outputs as little-endian float32 and uint32 bytes."""
    import hashlib
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(out_max, dtype="<f4").tobytes())
    h.update(np.ascontiguousarray(out_argmax, dtype="<u4").tobytes())
    return h.hexdigest()


def inputs_digest(xs):
    import hashlib
    h = hashlib.sha256()
    for x in xs:
        h.update(np.ascontiguousarray(x, dtype="<f4").tobytes())
    return h.hexdigest()


def pulse_fixture_cases():
    """SinglePulse cases whose construction by pirate's simpulse.cpp is committed as fixtures: channel
    edges (regular and irregular), per-channel variances and the pulse parameters (dispersion,
    scattering, intrinsic width, spectral index, arrival before and after zero, subband restriction)."""
    out = []
    pars = [
        dict(dm=50.0, sm=0.0, intrinsic_width=1e-3, spectral_index=0.0, undispersed_arrival_time_sec=0.2,
             time_sample_ms=1.0, snr=20.0),
        dict(dm=300.0, sm=2.0, intrinsic_width=3e-4, spectral_index=-1.5, undispersed_arrival_time_sec=-0.5,
             time_sample_ms=0.983, snr=12.0),
        dict(dm=0.0, sm=0.5, intrinsic_width=0.0, spectral_index=2.0, undispersed_arrival_time_sec=1.0,
             time_sample_ms=2.0, snr=50.0),
        dict(dm=1200.0, sm=0.1, intrinsic_width=5e-3, spectral_index=0.7, undispersed_arrival_time_sec=0.0,
             time_sample_ms=1.0, snr=8.0, subband_freq_lo_MHz=520.0, subband_freq_hi_MHz=610.0),
        dict(dm=700.0, sm=4.0, intrinsic_width=2e-3, spectral_index=-0.5, undispersed_arrival_time_sec=0.37,
             time_sample_ms=1.0, snr=30.0, internal_nt=512),
    ]
    for k, p in enumerate(pars):
        rng = np.random.default_rng(500 + k)
        nfreq = 256 if k == 4 else 64
        if k % 2 == 0:
            edges = np.linspace(400.0, 800.0, nfreq + 1)
        else:
            df = rng.uniform(0.2, 1.8, nfreq)
            edges = 400.0 + 400.0 * np.concatenate([[0.0], np.cumsum(df)]) / df.sum()
        var = rng.uniform(0.5, 2.0, nfreq)
        out.append(dict(name="pulse%d" % k, params=p, edges=edges, var=var))
    return out
