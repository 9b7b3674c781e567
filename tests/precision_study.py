"""Precision study of the storage dtypes: float32, float16 and bfloat16 storage (all with fp32
arithmetic) against the FP64 oracle of the same plan, on N(0,1) noise with a heavy-tailed RFI mix.

    python tests/precision_study.py [--rank 16] [--nfreq 16384] [--beams 8] [--chunks 16]
                                    [--workers W] [--json out.json]

Input per beam (seeded by beam and chunk, so every process regenerates it identically):
  - N(0,1) samples in every channel;
  - narrowband RFI: 1% of the channels (fixed per beam) carry a 10 sigma sinusoid in time, period
    log-uniform in 4..1024 samples, random phase;
  - zero-DM broadband spikes: each time sample, with probability 1e-3, gets +20 sigma in every channel.
The plan is the benchmark's tree layout at the given rank: 5 primary trees (time downsampling 1-16),
widths to 32, full-band search, bare unit-variance weights, so out_max is in noise sigma.

The GPU runs the float32 input through each storage dtype (the input is rounded to the storage dtype
on the way in, as a user of that plan would store it); the FP64 oracle runs on the float32 input. So
the errors include the input's rounding to the storage dtype.

Reported per dtype, over every output cell (beam, tree, coarse dm, output time) of every chunk:
  - max and RMS |GPU - FP64| in sigma, overall and per magnitude class of the FP64 value
    (|ref| <= 10 sigma: noise and ordinary candidates; 10-100; > 100: RFI-dominated);
  - max relative error |GPU - FP64| / max(1, |ref|);
  - output cells where the GPU value is not finite;
  - trigger-index agreement: the fraction of cells whose GPU token equals the FP64 oracle's, overall
    and among cells with ref >= 6 sigma; and for every disagreement the margin it implies: the FP64
    value of the oracle's trial minus the FP64 value of the GPU's trial (re-evaluated with the
    oracle's eval_tokens). A disagreement is consistent with the error bound when that margin is at
    most twice the largest error seen at that magnitude.

The GPU pass runs first (one beam and one dtype at a time) and keeps its outputs in memory-mapped
files; then one spawned process per beam runs the FP64 oracle and compares.
"""

import argparse
import json
import math
import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(HERE))

DTYPES = ("float32", "float16", "bfloat16")
CLASSES = ((0.0, 10.0), (10.0, 100.0), (100.0, math.inf))
RFI_FRACTION, RFI_SIGMA = 0.01, 10.0
SPIKE_RATE, SPIKE_SIGMA = 1e-3, 20.0
TRIGGER_SIGMA = 6.0


def study_config(rank, nfreq, nt=2048):
    prim = [dict(num_early_triggers=0, max_width=32, dm_downsampling=0, time_downsampling=0,
                 wt_dm_downsampling=64, wt_time_downsampling=64) for _ in range(5)]
    return dict(zone_nfreq=[nfreq], zone_freq_edges=[400.0, 800.0], time_sample_ms=1.0,
                toplevel_tree_rank=rank, time_samples_per_chunk=nt, dtype="float32",
                frequency_subband_counts=[0, 0, 0, 0, 1], primary_trees=prim,
                beams_per_gpu=1, beams_per_batch=1, num_active_batches=1,
                future_write_max_samples=0, max_gpu_clag=10000)


def rfi_chunk(beam, chunk, nfreq, nt, seed=2025):
    """(1, nfreq, nt) float32 input of one beam and chunk: noise + narrowband sinusoids + spikes."""
    beam_rng = np.random.default_rng([seed, beam])
    nrfi = max(1, int(round(RFI_FRACTION * nfreq)))
    chans = beam_rng.choice(nfreq, nrfi, replace=False)
    periods = np.exp(beam_rng.uniform(np.log(4.0), np.log(1024.0), nrfi))
    phases = beam_rng.uniform(0.0, 2 * np.pi, nrfi)
    rng = np.random.default_rng([seed, beam, chunk])
    x = rng.standard_normal((nfreq, nt), dtype=np.float32)
    t = np.arange(chunk * nt, (chunk + 1) * nt, dtype=np.float64)
    x[chans] += (RFI_SIGMA * np.sin(2 * np.pi * t[None, :] / periods[:, None] + phases[:, None])).astype(np.float32)
    spikes = rng.random(nt) < SPIKE_RATE
    x[:, spikes] += np.float32(SPIKE_SIGMA)
    return x[None]


def gpu_pass(cfg, beams, chunks, outdir, log=print):
    """Runs every beam through the three storage dtypes (one dedisperser at a time); writes out_max
    (float32) and tokens per (dtype, beam) as (chunks, cells) memory-mapped .npy files in outdir."""
    import gc
    import torch
    import oracle as O
    import pirate_b200 as pb
    for beam in range(beams):
        xs = [rfi_chunk(beam, ch, cfg["zone_nfreq"][0], cfg["time_samples_per_chunk"]) for ch in range(chunks)]
        for dt in DTYPES:
            plan = pb.DedispersionPlan(pb.DedispersionConfig.from_dict(dict(cfg, dtype=dt)))
            dd = pb.GpuDedisperser(plan, cuda_device_id=0, num_consumers=1)
            dd.allocate()
            for i, t in enumerate(plan.trees):
                shp = (1, t.ndm_wt, t.nt_wt, t.nprofiles, t.nsubbands)
                dd.fill_all_weights(i, O.bare_weights(shp, t.nprofiles)[None])
            n = sum(t.ndm_out * t.nt_out for t in plan.trees)
            mx = np.lib.format.open_memmap(os.path.join(outdir, "%s_b%d_max.npy" % (dt, beam)), "w+", np.float32, (chunks, n))
            tk = np.lib.format.open_memmap(os.path.join(outdir, "%s_b%d_tok.npy" % (dt, beam)), "w+", np.uint32, (chunks, n))
            for ch in range(chunks):
                with dd.get_input() as arr:
                    arr.copy_(torch.from_numpy(xs[ch]).to(arr.device))
                with dd.get_output(0, sync=True) as out:
                    mx[ch] = np.concatenate([m.float().cpu().numpy().ravel() for m in out.out_max])
                    tk[ch] = np.concatenate([a.cpu().numpy().view(np.uint32).ravel() for a in out.out_argmax])
            mx.flush()
            tk.flush()
            nbytes = dd.device_bytes()
            del dd, mx, tk
            gc.collect()
            torch.cuda.synchronize()
            log("gpu pass: beam %d %s done (%.1f GB on the device)" % (beam, dt, nbytes / 1e9))


def _empty_stats():
    return dict(n=0, nonfinite=0, max_abs=0.0, sum_sq=0.0, max_rel=0.0,
                cls=[dict(n=0, max_abs=0.0, sum_sq=0.0) for _ in CLASSES],
                tok_equal=0, trig_n=0, trig_equal=0, mism_gaps=[])


def compare_beam(args):
    """FP64 oracle for one beam, compared with the GPU outputs of every dtype. Runs in a spawned
    process."""
    cfg, beam, chunks, outdir = args
    import oracle as O
    orc = O.OracleDedisperser(cfg, 1, 64)
    ws = [O.bare_weights(orc.wt_shape(i), orc.trees[i]["nprofiles"]) for i in range(orc.ntrees)]
    shapes = [orc.out_shape(i) for i in range(orc.ntrees)]
    sizes = [int(np.prod(s)) for s in shapes]
    offs = np.concatenate([[0], np.cumsum(sizes)])
    maps = {dt: (np.load(os.path.join(outdir, "%s_b%d_max.npy" % (dt, beam)), mmap_mode="r"),
                 np.load(os.path.join(outdir, "%s_b%d_tok.npy" % (dt, beam)), mmap_mode="r")) for dt in DTYPES}
    st = {dt: _empty_stats() for dt in DTYPES}
    for ch in range(chunks):
        x = rfi_chunk(beam, ch, cfg["zone_nfreq"][0], cfg["time_samples_per_chunk"])
        om, oa = orc.dedisperse(0, x, ws)
        ref = np.concatenate([m.ravel() for m in om])
        rtok = np.concatenate([a.ravel() for a in oa])
        aref = np.abs(ref)
        for dt in DTYPES:
            s = st[dt]
            g = maps[dt][0][ch].astype(np.float64)
            gt = maps[dt][1][ch]
            fin = np.isfinite(g)
            s["n"] += g.size
            s["nonfinite"] += int((~fin).sum())
            err = np.abs(g - ref)[fin]
            a = aref[fin]
            s["max_abs"] = max(s["max_abs"], float(err.max(initial=0.0)))
            s["sum_sq"] += float((err ** 2).sum())
            s["max_rel"] = max(s["max_rel"], float((err / np.maximum(1.0, a)).max(initial=0.0)))
            for k, (lo, hi) in enumerate(CLASSES):
                sel = (a > lo) & (a <= hi) if k else (a <= hi)
                c = s["cls"][k]
                c["n"] += int(sel.sum())
                if sel.any():
                    c["max_abs"] = max(c["max_abs"], float(err[sel].max()))
                    c["sum_sq"] += float((err[sel] ** 2).sum())
            eq = gt == rtok
            s["tok_equal"] += int(eq.sum())
            trig = ref >= TRIGGER_SIGMA
            s["trig_n"] += int(trig.sum())
            s["trig_equal"] += int((eq & trig).sum())
            if not eq.all():
                # FP64 value of each GPU trial (eval_tokens on the chunk just dedispersed)
                ev = np.concatenate([orc.eval_tokens(i, gt[offs[i]:offs[i + 1]].reshape(shapes[i]), ws[i]).ravel()
                                     for i in range(orc.ntrees)])
                idx = np.nonzero(~eq)[0]
                for j in idx:
                    s["mism_gaps"].append((float(ref[j]), float(ref[j] - ev[j])))
    return beam, st


def merge(parts):
    out = {}
    for dt in DTYPES:
        m = _empty_stats()
        for st in parts:
            s = st[dt]
            for k in ("n", "nonfinite", "sum_sq", "tok_equal", "trig_n", "trig_equal"):
                m[k] += s[k]
            m["max_abs"] = max(m["max_abs"], s["max_abs"])
            m["max_rel"] = max(m["max_rel"], s["max_rel"])
            for c, cs in zip(m["cls"], s["cls"]):
                c["n"] += cs["n"]
                c["max_abs"] = max(c["max_abs"], cs["max_abs"])
                c["sum_sq"] += cs["sum_sq"]
            m["mism_gaps"] += s["mism_gaps"]
        nf = m["n"] - m["nonfinite"]
        gaps = m["mism_gaps"]
        # a disagreement is consistent when its margin is at most twice the largest error of its class
        bound = [2 * c["max_abs"] for c in m["cls"]]

        def klass(v):
            a = abs(v)
            return 0 if a <= 10.0 else (1 if a <= 100.0 else 2)

        worst = max((g / max(bound[klass(r)], 1e-300) for r, g in gaps), default=0.0)
        out[dt] = dict(
            cells=m["n"], nonfinite=m["nonfinite"],
            max_abs_sigma=m["max_abs"], rms_sigma=math.sqrt(m["sum_sq"] / max(nf, 1)), max_rel=m["max_rel"],
            classes=[dict(range_sigma=[lo, None if math.isinf(hi) else hi], cells=c["n"], max_abs_sigma=c["max_abs"],
                          rms_sigma=math.sqrt(c["sum_sq"] / max(c["n"], 1))) for (lo, hi), c in zip(CLASSES, m["cls"])],
            token_agreement=m["tok_equal"] / max(m["n"], 1),
            trigger_cells=m["trig_n"], trigger_agreement=m["trig_equal"] / max(m["trig_n"], 1),
            disagreements=len(gaps), max_margin_sigma=max((g for _, g in gaps), default=0.0),
            max_margin_over_bound=worst)
    return out


def run(rank, nfreq, beams, chunks, workers=None, log=print):
    import multiprocessing as mp
    cfg = study_config(rank, nfreq)
    with tempfile.TemporaryDirectory(prefix="pb2_precision_") as outdir:
        t0 = time.time()
        gpu_pass(cfg, beams, chunks, outdir, log)
        t1 = time.time()
        if workers is None:
            workers = min(beams, os.cpu_count() or 1)
            try:
                import psutil
                per = 3.2e9 * 2 ** (rank - 12) * 1.05 + 2e9     # FP64 oracle footprint, measured 44 GB at rank 16
                workers = max(1, min(workers, int(psutil.virtual_memory().available * 0.8 // per)))
            except ImportError:
                pass
        ctx = mp.get_context("spawn")
        with ctx.Pool(workers) as pool:
            parts = [st for _, st in pool.imap_unordered(compare_beam, [(cfg, b, chunks, outdir) for b in range(beams)])]
        t2 = time.time()
    res = merge(parts)
    meta = dict(rank=rank, nfreq=nfreq, beams=beams, chunks=chunks, nt=cfg["time_samples_per_chunk"], trees=5,
                workers=workers, gpu_seconds=round(t1 - t0, 1), oracle_seconds=round(t2 - t1, 1),
                rfi=dict(narrowband_fraction=RFI_FRACTION, narrowband_sigma=RFI_SIGMA, spike_rate=SPIKE_RATE,
                         spike_sigma=SPIKE_SIGMA))
    return dict(meta=meta, dtypes=res)


def table(r):
    m = r["meta"]
    lines = ["rank %d, %d channels, %d beams x %d chunks of %d samples, 5 trees; %d oracle processes"
             % (m["rank"], m["nfreq"], m["beams"], m["chunks"], m["nt"], m["workers"]), "",
             "| storage | max abs err (sigma) | RMS err (sigma) | max err, ref within 10 sigma | max err, 10-100 | max err, over 100 "
             "| max rel err | non-finite | token agreement | agreement, ref>=6 sigma | disagreements | max margin (sigma) "
             "| margin / bound |",
             "|---|---|---|---|---|---|---|---|---|---|---|---|---|"]
    for dt, d in r["dtypes"].items():
        c = d["classes"]
        lines.append("| %s | %.3g | %.3g | %.3g | %.3g | %.3g | %.3g | %d | %.6f | %.6f (%d cells) | %d | %.3g | %.3g |" % (
            dt, d["max_abs_sigma"], d["rms_sigma"], c[0]["max_abs_sigma"], c[1]["max_abs_sigma"], c[2]["max_abs_sigma"],
            d["max_rel"], d["nonfinite"], d["token_agreement"], d["trigger_agreement"], d["trigger_cells"],
            d["disagreements"], d["max_margin_sigma"], d["max_margin_over_bound"]))
    return "\n".join(lines)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--rank", type=int, default=16)
    ap.add_argument("--nfreq", type=int, default=16384)
    ap.add_argument("--beams", type=int, default=8)
    ap.add_argument("--chunks", type=int, default=16)
    ap.add_argument("--workers", type=int, default=None)
    ap.add_argument("--json", default=None)
    a = ap.parse_args()
    r = run(a.rank, a.nfreq, a.beams, a.chunks, a.workers, log=lambda s: print(s, flush=True))
    print(table(r))
    if a.json:
        with open(a.json, "w") as f:
            json.dump(r, f, indent=1)


if __name__ == "__main__":
    main()
