"""Benchmark of the B200 dedispersion path.

Workload (a 'step' = one 2048-sample chunk of every beam): rank-16 tree (65536 tree channels) gridded
from 16384 frequency channels over 400-800 MHz, 5 primary trees (time downsampling 1..16), peak
finding up to width 32 per tree (64 samples in primary tree 1), full-band search (subband counts
[0,0,0,0,1]), float16 storage with float32 arithmetic, 1 ms samples, seeded N(0,1) inputs.

Metric: real-time beams per B200 = beams * chunk_seconds / seconds_per_chunk (pirate's definition,
src_lib/GpuDedisperser.cpp:1598,1676). Prints one JSON line.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--beams B] [--dtype float16] [--impl reference]

Multi-GPU: the path shards by beam with no exchange step, so N GPUs run N independent replicas
(one process per GPU under torchrun; run without torchrun, --gpus N > 1 launches torchrun itself);
value = all ranks' beams over the max-over-ranks time.

Also reported on one GPU: the plain fp32 path (one beam, float32 storage and input, no batching;
the benchmark plan with fp32 storage) as 'plain_fp32', and the number of beams whose lag state fits in HBM as
'capacity_beams'.
"""

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CHUNK = 2048
SAMPLE_MS = 1.0
CHUNK_SECONDS = CHUNK * SAMPLE_MS * 1e-3
METRIC = "real-time beams/B200 (rank 16, fp16)"
L2_BYTES = 126 * 2 ** 20


def bench_config(beams, dtype, rank=16, npri=5, nfreq=16384, streams=1):
    """streams > 1: the beams form that many batches, one per compute stream (num_active_batches)."""
    prim = [dict(num_early_triggers=0, max_width=32, dm_downsampling=0, time_downsampling=0,
                 wt_dm_downsampling=64, wt_time_downsampling=64) for _ in range(npri)]
    return dict(zone_nfreq=[nfreq], zone_freq_edges=[400.0, 800.0], time_sample_ms=SAMPLE_MS,
                toplevel_tree_rank=rank, time_samples_per_chunk=CHUNK, dtype=dtype,
                frequency_subband_counts=[0, 0, 0, 0, 1], primary_trees=prim,
                beams_per_gpu=beams, beams_per_batch=beams // streams, num_active_batches=streams,
                future_write_max_samples=0, max_gpu_clag=10000)


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while the timed region runs."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []          # (host time, csv line)
        self.window = None       # (start, end) host times of the timed region

    def __enter__(self):
        """Starts sampling every 50 ms and waits (up to 3 s) for the first sample."""
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            t0 = time.time()
            while not self.lines and time.time() - t0 < 3.0:
                time.sleep(0.01)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def mark(self, start, end):
        self.window = (start, end)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lines = self.lines
        if self.window:
            # samples taken during the timed region (the one just after it if the region was shorter
            # than the sampling interval)
            inside = [ln for t, ln in lines if self.window[0] <= t <= self.window[1] + 0.06]
            lines = inside or [ln for t, ln in lines if t >= self.window[0]][:1]
        else:
            lines = [ln for _, ln in lines]
        for ln in lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for n, v in zip(names, parts[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def run_ours(args, rank, world):
    import numpy as np
    import torch
    import pirate_b200 as pb
    from pirate_b200 import replicas

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    cfg = bench_config(args.beams, args.dtype, args.rank, args.npri, args.nfreq, args.streams)
    plan = pb.DedispersionPlan(pb.DedispersionConfig.from_dict(cfg))
    dd = pb.GpuDedisperser(plan, cuda_device_id=dev, num_consumers=1)
    nbat = args.streams   # batches per chunk
    dd.allocate()
    tdt = getattr(torch, args.dtype)

    # Unit-variance ("bare") peak-finding weights: out_max in sigma for N(0,1) input.
    for i, t in enumerate(plan.trees):
        var = [1.0]
        for l in range((t.nprofiles - 1) // 3):
            var += [2.0 ** (l + 1), 1.5 * 2.0 ** l, 2.5 * 2.0 ** l]
        w = (1.0 / np.sqrt(np.array(var))).astype(np.float32)
        arr = np.empty((dd.nbatches_wt, plan.beams_per_batch, t.ndm_wt, t.nt_wt, t.nprofiles, t.nsubbands), np.float32)
        arr[...] = w[None, None, None, None, :, None]
        dd.fill_all_weights(i, arr)

    stream = torch.cuda.current_stream()
    gen = torch.Generator(device="cuda")
    gen.manual_seed(1234 + rank)
    seq = [0]
    B, F, T = plan.beams_per_batch, plan.nfreq, plan.nt_in

    def quantized_input(device):
        """pirate's raw input format: int4 samples (two per byte, low nibble first) with one fp16
        (scale, offset) pair per 256 samples. N(0,1) data quantized with scale 0.5 (range +-3.5 sigma),
        1% of samples flagged missing (-8)."""
        x = torch.randn((B, F, T), generator=gen, device="cuda", dtype=torch.float32)
        v = torch.clamp(torch.round(x * 2.0), -7, 7).to(torch.int32)
        v[torch.rand((B, F, T), generator=gen, device="cuda") < 0.01] = -8
        nib = (v & 0xf).to(torch.uint8)
        data = (nib[..., 0::2] | (nib[..., 1::2] << 4)).contiguous()
        so = torch.empty((B, F, T // 256, 2), dtype=torch.float16, device="cuda")
        so[..., 0] = 0.5
        so[..., 1] = 0.0
        return data.to(device), so.to(device)

    dq_data, dq_so = quantized_input("cuda")

    # The consumer acquires and releases outputs on its own stream (as pirate's timing loop does on its
    # kernel-timer stream): on the input stream, the next chunk's launch would wait for this chunk's
    # outputs, leaving a gap between consecutive chunks' kernels.
    out_dev = torch.cuda.Stream()

    def step_device():
        """One chunk of all beams (nbat batches); the int4 input stays resident in the input slots."""
        s0 = seq[0]
        for s in range(s0, s0 + nbat):
            d, so = dd.acquire_input_int4(s, stream)
            if s < nbat:
                d.copy_(dq_data)
                so.copy_(dq_so)
            dd.release_input_and_launch_dd_kernels(s, stream)
        for s in range(s0, s0 + nbat):
            dd.acquire_output(0, s, out_dev)
            dd.release_output(0, s, out_dev)
        seq[0] += nbat

    for _ in range(args.warmup):
        step_device()
    torch.cuda.synchronize()
    replicas.barrier()
    torch.cuda.synchronize()

    # Timed region: K steps bracketed by events on the caller stream (the headline).
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev) as clk:
        h0 = time.time()
        e0.record(stream)
        for _ in range(args.steps):
            step_device()
        stream.wait_stream(out_dev)   # the last chunk's outputs consumed
        e1.record(stream)
        torch.cuda.synchronize()
        clk.mark(h0, time.time())
    ms = replicas.max_over_ranks(e0.elapsed_time(e1))
    replicas.barrier()
    ms_per_step = ms / args.steps
    # A second timed region of K steps with CUDA events around every kernel class on the dedisperser's
    # compute stream (the roofline's per-kernel durations). The events between the kernels cost about
    # 2-3% of a step, so they stay out of the headline region.
    torch.cuda.synchronize()
    dd.enable_timing(True)
    k0 = torch.cuda.Event(enable_timing=True)
    k1 = torch.cuda.Event(enable_timing=True)
    k0.record(stream)
    for _ in range(args.steps):
        step_device()
    stream.wait_stream(out_dev)
    k1.record(stream)
    torch.cuda.synchronize()
    ktimes = dd.kernel_times()
    dd.enable_timing(False)
    kms_per_step = replicas.max_over_ranks(k0.elapsed_time(k1)) / args.steps
    replicas.barrier()

    # End to end through the public API, as pirate's timing loop (GpuDedisperser::time,
    # src_lib/GpuDedisperser.cpp:1584-1680) runs it: per step, the int4 data and scales/offsets go from
    # pinned host memory to the acquired input slot on a copy stream, the kernels run, and (beyond
    # pirate's loop) every tree's out_max and out_argmax come back to pinned host memory on a third
    # stream. The copies overlap the previous chunk's kernels.
    h_data = torch.empty(dq_data.shape, dtype=torch.uint8, pin_memory=True)
    h_so = torch.empty(dq_so.shape, dtype=torch.float16, pin_memory=True)
    h_data.copy_(dq_data.cpu())
    h_so.copy_(dq_so.cpu())
    copy_stream = torch.cuda.Stream()
    out_stream = torch.cuda.Stream()
    torch.cuda.synchronize()
    outs_host = None
    h2d = (h_data.numel() + h_so.numel() * 2) * nbat
    d2h = 0
    esize = torch.tensor([], dtype=tdt).element_size()
    for t in plan.trees:
        d2h += args.beams * t.ndm_out * t.nt_out * (esize + 4)

    def step_e2e():
        nonlocal outs_host
        s0 = seq[0]
        for s in range(s0, s0 + nbat):
            d, so = dd.acquire_input_int4(s, copy_stream)
            with torch.cuda.stream(copy_stream):
                d.copy_(h_data, non_blocking=True)
                so.copy_(h_so, non_blocking=True)
            dd.release_input_and_launch_dd_kernels(s, copy_stream)
        for s in range(s0, s0 + nbat):
            o = dd.acquire_output(0, s, out_stream)
            if outs_host is None:
                outs_host = [[(torch.empty(m.shape, dtype=m.dtype, pin_memory=True),
                               torch.empty(a.shape, dtype=a.dtype, pin_memory=True)) for m, a in zip(o.out_max, o.out_argmax)]
                             for _ in range(nbat)]
            with torch.cuda.stream(out_stream):
                for (hm, ha), m, a in zip(outs_host[s - s0], o.out_max, o.out_argmax):
                    hm.copy_(m, non_blocking=True)
                    ha.copy_(a, non_blocking=True)
            dd.release_output(0, s, out_stream)
        seq[0] += nbat

    e2e_steps = max(4, min(args.steps, 32))
    for _ in range(3):
        step_e2e()
    torch.cuda.synchronize()
    replicas.barrier()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(copy_stream)
    for _ in range(e2e_steps):
        step_e2e()
    f1.record(out_stream)
    torch.cuda.synchronize()
    ems = replicas.max_over_ranks(f0.elapsed_time(f1))

    # pirate's own timing loop through the C ABI (GpuDedisperser::time: int4 batches from pinned host
    # memory, kernels, output consumed): beams_per_batch * chunk seconds over the interval between
    # consecutive batches' completions, median after 2 * nbat warm-up iterations (rank 0's GPU).
    torch.cuda.synchronize()
    nit = max(4 * nbat + 2, min(args.steps, 40))
    rtb = dd.time(nit)
    time_loop = float(np.median(rtb[2 * nbat + 1:]))
    seq[0] += nit

    # Beams whose state fits in this GPU's HBM at this plan: total memory over the device bytes per beam.
    per_beam = dd.device_bytes() / float(args.beams)
    capacity_beams = int(torch.cuda.get_device_properties(dev).total_memory // per_beam)

    alg = [x * nbat for x in dd.algorithmic_bytes()]   # per step: every batch of the chunk
    # The gridding class reads int4 data and scales/offsets instead of storage-dtype samples.
    alg[0] += float(args.beams) * plan.nfreq * (plan.nt_in / 2 + plan.nt_in / 256 * 4 - plan.nt_in * esize)
    return dict(plan=plan, dd=dd, ms_per_step=ms_per_step, e2e_ms_per_step=ems / e2e_steps, ktimes=ktimes,
                kms_per_step=kms_per_step, time_loop=time_loop, time_loop_iters=nit,
                alg=alg, clocks=clk.summary(), h2d=h2d, d2h=d2h, device_bytes=dd.device_bytes(),
                kernels_per_batch=dd.kernels_per_batch() * nbat, capacity_beams=capacity_beams,
                bytes_per_beam=per_beam)


def uneven_groups(scale):
    """The uneven workload: tree ranks 12, 14, 16 in proportions 1:1:2 (64 beams at scale 1),
    downsampling depths (primary trees) 3, 4, 5 spread over each rank's beams, 2048-sample chunks,
    float16 storage; channels = 2^rank / 4 (the benchmark's 16384 channels for rank 16)."""
    out = []
    for rank, nbeams in ((12, 16), (14, 16), (16, 32)):
        n = max(3, int(round(nbeams * scale)))
        split = [n - 2 * (n // 3), n // 3, n // 3]
        for depth, k in zip((3, 4, 5), split):
            if k:
                out.append((rank, depth, k))
    return out


def group_config(rank, depth, beams, dtype="float16", max_gpu_clag=10000):
    prim = [dict(num_early_triggers=0, max_width=32, dm_downsampling=0, time_downsampling=0,
                 wt_dm_downsampling=2 ** ((rank - (1 if i else 0)) // 2), wt_time_downsampling=64) for i in range(depth)]
    return dict(zone_nfreq=[2 ** rank // 4], zone_freq_edges=[400.0, 800.0], time_sample_ms=SAMPLE_MS,
                toplevel_tree_rank=rank, time_samples_per_chunk=CHUNK, dtype=dtype,
                frequency_subband_counts=[0, 0, 0, 0, 1], primary_trees=prim, beams_per_gpu=beams,
                beams_per_batch=beams, num_active_batches=1, future_write_max_samples=0, max_gpu_clag=max_gpu_clag)


def run_batched(scale, steps, reps=3):
    """The uneven workload (beams of ranks 12/14/16, one replayed CUDA graph per chunk, autotuned schedule): returns
    the real-time beams, ms per step and the record. Inputs are N(0,1) float16 noise resident in every
    group's input slot."""
    import torch
    import pirate_b200 as pb
    groups = uneven_groups(scale)
    plans = [pb.DedispersionPlan(pb.DedispersionConfig.from_dict(group_config(r, d, b))) for r, d, b in groups]
    bd = pb.BatchedDedisperser(plans, cuda_device_id=int(os.environ.get("LOCAL_RANK", "0")))
    bd.allocate()
    for g, p in enumerate(plans):
        bd.fill_analytic_weights(g, np.ones(p.nfreq))
        bd.input(g).normal_()
    torch.cuda.synchronize()
    rec = bd.autotune(reps=reps)
    for g in range(len(plans)):
        bd.input(g).normal_()
    torch.cuda.synchronize()
    for _ in range(3):
        bd.step()
    ms = bd.time_steps(steps)
    nbeams = sum(b for _, _, b in groups)
    res = dict(value=round(nbeams * CHUNK_SECONDS / (ms * 1e-3), 2), unit="beams", ms_per_step=round(ms, 4), beams=nbeams,
               groups=[dict(rank=r, primary_trees=d, beams=b) for r, d, b in groups],
               device_bytes=bd.device_bytes(), kernels_per_step=bd.kernels_per_step(),
               autotune=dict(chosen=rec["chosen"], candidates=len(rec["candidates"])))
    del bd
    torch.cuda.empty_cache()
    return res


def run_spill(steps, beams=8, clag=2, sweep=True):
    """The benchmark plan with delay lines more than 'clag' chunks deep in pinned host memory (g2h/h2g
    copy kernels every chunk): real-time beams, device and host bytes."""
    import torch
    import pirate_b200 as pb
    cfg = bench_config(beams, "float16")
    cfg["max_gpu_clag"] = clag
    plan = pb.DedispersionPlan(pb.DedispersionConfig.from_dict(cfg))
    dd = pb.GpuDedisperser(plan, cuda_device_id=int(os.environ.get("LOCAL_RANK", "0")), num_consumers=1)
    dd.allocate()
    dd.fill_analytic_weights(np.ones(plan.nfreq))
    stream = torch.cuda.current_stream()
    seq = [0]

    def step():
        s = seq[0]
        a = dd.acquire_input(s, stream)
        if s == 0:
            a.normal_()
        dd.release_input_and_launch_dd_kernels(s, stream)
        dd.acquire_output(0, s, stream)
        dd.release_output(0, s, stream)
        seq[0] += 1
    for _ in range(3):
        step()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    res = dict(value=round(beams * CHUNK_SECONDS / (ms * 1e-3), 2), unit="beams", ms_per_step=round(ms, 4), beams=beams,
               max_gpu_clag=clag, device_bytes=dd.device_bytes(), host_bytes=dd.host_bytes(),
               device_bytes_per_beam=round(dd.device_bytes() / beams / 1e9, 3))
    # Beams whose state fits at this max_gpu_clag: the fewer of what the GPU's HBM and the host's
    # memory hold (device and host bytes per beam).
    try:
        import psutil
        host_total = psutil.virtual_memory().total
        hbm = torch.cuda.get_device_properties(torch.cuda.current_device()).total_memory
        per_dev, per_host = dd.device_bytes() / beams, dd.host_bytes() / beams
        res["capacity_beams"] = int(min(hbm // per_dev, host_total // per_host if per_host else hbm // per_dev))
        res["capacity_note"] = ("min(HBM %.0f GB / %.2f GB per beam, host memory %.0f GB / %.2f GB per beam)"
                                % (hbm / 1e9, per_dev / 1e9, host_total / 1e9, per_host / 1e9))
    except Exception:
        pass
    del dd
    torch.cuda.empty_cache()
    if sweep:
        res["capacity_by_clag"] = spill_capacity()
    return res


def spill_capacity(clags=(1, 2, 4, 8, 16, 32)):
    """Beams whose state fits in HBM plus host memory, for several max_gpu_clag values: device and
    host bytes of a one-beam dedisperser of the benchmark plan (an upper bound per beam, fixed buffers
    included), the fewer of HBM / device bytes and host memory / host bytes."""
    import torch
    import psutil
    import pirate_b200 as pb
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    hbm = torch.cuda.get_device_properties(dev).total_memory
    host = psutil.virtual_memory().total
    out = []
    for clag in clags:
        cfg = bench_config(1, "float16")
        cfg["max_gpu_clag"] = clag
        dd = pb.GpuDedisperser(pb.DedispersionPlan(pb.DedispersionConfig.from_dict(cfg)), cuda_device_id=dev, num_consumers=1)
        dd.allocate()
        d, h = dd.device_bytes(), dd.host_bytes()
        del dd
        torch.cuda.empty_cache()
        out.append({"max_gpu_clag": clag, "device_gb_per_beam": round(d / 1e9, 3), "host_gb_per_beam": round(h / 1e9, 3),
                    "beams": int(min(hbm // d, host // h if h else hbm // d))})
    return out


def run_sifter(steps, beams=8, n_train=6144, n_test=3072):
    """The learned candidate sifter: trained by its own kernels on candidates of the small pipeline
    (rank 12, 5 primary trees; sifter_study.config('small')), recall at false-alarm fractions of the
    held-out negatives against the plain threshold; then the candidate stage (per-beam peaks, patches,
    MLP) attached to the benchmark workload, its device time per step (CUDA events)."""
    import torch
    import pirate_b200 as pb
    from pirate_b200 import sifter_study as SS
    res, sf = SS.study(SS.config("small"), n_train, n_test, epochs=40, fars=(1e-2, 1e-3))
    cfg = bench_config(beams, "float16")
    plan = pb.DedispersionPlan(pb.DedispersionConfig.from_dict(cfg))
    dd = pb.GpuDedisperser(plan, cuda_device_id=int(os.environ.get("LOCAL_RANK", "0")), num_consumers=1)
    dd.allocate()
    dd.fill_analytic_weights(np.ones(plan.nfreq))
    dd.enable_sifter(6.0, sf)
    stream = torch.cuda.current_stream()
    seq = [0]

    def step():
        s = seq[0]
        a = dd.acquire_input(s, stream)
        if s == 0:
            a.normal_()
        dd.release_input_and_launch_dd_kernels(s, stream)
        dd.acquire_output(0, s, stream)
        dd.release_output(0, s, stream)
        seq[0] += 1
    for _ in range(3):
        step()
    torch.cuda.synchronize()
    dd.enable_timing(True)
    for _ in range(steps):
        step()
    kt = dd.kernel_times()
    dd.enable_timing(False)
    tot = sum(v[0] for v in kt.values())
    out = dict(recall=res["recall"], test_positives=res["test_positives"], test_negatives=res["test_negatives"],
               train_candidates=res["train_valid"], workload="rank 12 from 2048 channels, 5 primary trees, 1024-sample chunks, "
               "float16; pulses (simpulse model), noise and RFI events",
               candidate_stage_ms_per_step=round(kt["sifter"][0] / steps, 4),
               candidate_stage_share=round(kt["sifter"][0] / tot, 4) if tot else None,
               candidate_stage_config="benchmark workload, %d beams: per-beam peaks, 9x32x6 patches, MLP on the tensor cores" % beams)
    del dd, sf
    torch.cuda.empty_cache()
    return out


def run_plain_fp32(args, steps):
    """The plain fp32 GPU path (the benchmark plan's shape): one beam, float32 storage, float32 N(0,1)
    input resident in the input slot (no int4 input, no batching), same plan otherwise. Returns
    (real-time beams, ms per step)."""
    import torch
    import pirate_b200 as pb
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    cfg = bench_config(1, "float32", args.rank, args.npri, args.nfreq)
    plan = pb.DedispersionPlan(pb.DedispersionConfig.from_dict(cfg))
    dd = pb.GpuDedisperser(plan, cuda_device_id=dev, num_consumers=1)
    dd.allocate()
    import numpy as np
    for i, t in enumerate(plan.trees):
        arr = np.ones((dd.nbatches_wt, 1, t.ndm_wt, t.nt_wt, t.nprofiles, t.nsubbands), np.float32)
        dd.fill_all_weights(i, arr)
    stream = torch.cuda.current_stream()
    g = torch.Generator(device="cuda")
    g.manual_seed(99)
    x = torch.randn((1, plan.nfreq, plan.nt_in), generator=g, device="cuda", dtype=torch.float32)
    seq = [0]
    out = torch.cuda.Stream()   # outputs consumed on their own stream, as in the headline loop

    def step():
        s = seq[0]
        a = dd.acquire_input(s, stream)
        if s == 0:
            a.copy_(x)
        dd.release_input_and_launch_dd_kernels(s, stream)
        dd.acquire_output(0, s, out)
        dd.release_output(0, s, out)
        seq[0] += 1

    for _ in range(3):
        step()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        step()
    stream.wait_stream(out)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    del dd
    torch.cuda.empty_cache()
    return CHUNK_SECONDS / (ms * 1e-3), ms


def cpu_kind():
    """'reference' when pirate's own reference CPU sources were compiled as oracle/_ref (travels with
    the repository as a built file), else 'port' (the oracle's restatement)."""
    return "reference" if os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libpirate_ref.so")) else "port"


def cpu_sample(nchunks=1, dtype="float16", kind=None):
    """Times pirate's CPU ReferenceDedisperser (sophistication 1: two-stage trees with lagged
    downsampling, pirate's GPU algorithm) on one beam of the bench workload, single-threaded: pirate's
    own code from oracle/_ref when it is built, else the oracle's fp32 restatement of it. The int4 chunk
    is dequantized first (ReferenceDequantizationKernel's arithmetic), as pirate's timing loop does.
    Returns seconds per chunk."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle
    kind = kind or cpu_kind()
    cfg = bench_config(1, "float32")
    cfg["dtype"] = dtype if dtype != "bfloat16" else "float16"   # same plan shapes as the GPU run
    if kind == "reference":
        import pirate_ref
        ref = pirate_ref.PirateReferenceDedisperser(cfg, sophistication=1)
        shapes = [(1, t["ndm_wt"], t["nt_wt"], t["nprofiles"], t["N"]) for t in ref.trees]
        ws = [oracle.bare_weights(sh, t["nprofiles"]) for sh, t in zip(shapes, ref.trees)]
        run = lambda x: ref.dedisperse(x, ws)   # noqa: E731
    else:
        orc = oracle.OracleDedisperser(cfg, 1, 32)
        ws = [oracle.bare_weights(orc.wt_shape(i), orc.trees[i]["nprofiles"]) for i in range(orc.ntrees)]
        run = lambda x: orc.dedisperse(0, x, ws)   # noqa: E731
    # The same int4 input format as the GPU run, dequantized (ReferenceDequantizationKernel) and then
    # dedispersed, as pirate's timing loop does per chunk.
    rng = np.random.default_rng(0)
    v = np.clip(np.round(rng.standard_normal((1, 16384, CHUNK)) * 2.0), -7, 7).astype(np.int64)
    v[rng.random(v.shape) < 0.01] = -8
    nib = (v & 0xf).astype(np.uint8)
    data = (nib[..., 0::2] | (nib[..., 1::2] << 4)).astype(np.uint8)
    so = np.zeros((1, 16384, CHUNK // 256, 2), np.float16)
    so[..., 0] = 0.5
    t0 = time.time()
    for _ in range(nchunks):
        x = oracle.dequantize(data, so, 1, 16384, CHUNK)
        run(x)
    return (time.time() - t0) / nchunks


def _cpu_worker(q, nchunks, dtype):
    q.put(cpu_sample(nchunks, dtype))


def run_reference(args, rank, world):
    """The reference arm: pirate's CPU ReferenceDedisperser on the host cores, one beam per process
    (about 24 GB each at rank 16): pirate's own sources compiled as oracle/_ref, or, where that build is
    absent, the oracle's restatement."""
    if rank != 0:
        return None
    import multiprocessing as mp
    ncores = os.cpu_count() or 1
    try:
        avail = os.sysconf("SC_AVPHYS_PAGES") * os.sysconf("SC_PAGE_SIZE")
    except Exception:
        avail = 64 << 30
    nproc = int(max(1, min(ncores, avail // (24 << 30))))
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    t0 = time.time()
    ps = [ctx.Process(target=_cpu_worker, args=(q, 1, args.dtype)) for _ in range(nproc)]
    for p in ps:
        p.start()
    per = [q.get() for _ in ps]
    for p in ps:
        p.join()
    wall = time.time() - t0
    sec = max(per)
    value = nproc * CHUNK_SECONDS / sec
    return dict(value=value, sec=sec, nproc=nproc, wall=wall)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--beams", type=int, default=8)
    ap.add_argument("--streams", type=int, default=1, help="compute streams (num_active_batches); beams split into that many batches")
    ap.add_argument("--no-plain-fp32", action="store_true")
    ap.add_argument("--no-streams-leg", action="store_true", help="skip the two-compute-stream leg")
    ap.add_argument("--no-batched", action="store_true", help="skip the uneven-workload batched leg")
    ap.add_argument("--no-spill", action="store_true", help="skip the host-spill leg")
    ap.add_argument("--no-sifter", action="store_true", help="skip the learned-sifter leg")
    ap.add_argument("--batched-scale", type=float, default=0.5, help="the uneven workload's 64 beams x this")
    ap.add_argument("--dtype", default="float16", choices=["float16", "bfloat16", "float32"])
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    # Smaller workloads, for profiler captures only (the headline workload is the default).
    ap.add_argument("--rank", type=int, default=16)
    ap.add_argument("--npri", type=int, default=5)
    ap.add_argument("--nfreq", type=int, default=16384)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.streams < 1 or args.beams % args.streams:
        sys.exit("bench.py: --beams must be a multiple of --streams")

    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # One process per GPU: relaunch under torchrun (rendezvous on 127.0.0.1).
        import socket
        with socket.socket() as sk:
            sk.bind(("127.0.0.1", 0))
            port = sk.getsockname()[1]
        cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", str(args.gpus),
               "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
        sys.exit(subprocess.call(cmd))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world != args.gpus:
        sys.exit("bench.py: --gpus %d but WORLD_SIZE=%d" % (args.gpus, world))
    cfg_json = {"workload": "rank-16 tree, 16384 channels 400-800 MHz, 5 primary trees (time downsampling 1-16), "
                            "2048-sample chunks, widths to 32 per tree, full-band search",
                "beams_per_gpu": args.beams, "beams_per_batch": args.beams // args.streams,
                "compute_streams": args.streams, "chunk_samples": CHUNK, "sample_ms": SAMPLE_MS,
                "storage": args.dtype, "parallelism": "replicas x%d (beams shard, no collective)" % args.gpus,
                "l2": "inputs and lag state exceed L2 (126 MB) every step",
                "input": "int4 samples + fp16 (scale, offset) per 256 samples (pirate's raw format), "
                         "dequantized inside the gridding kernel"}

    if args.impl == "reference":
        if world > 1:
            import torch.distributed as dist
            dist.init_process_group("gloo")
        r = run_reference(args, rank, world)
        if rank == 0:
            line = {"metric": METRIC, "value": r["value"], "unit": "beams", "impl": "reference", "n_gpus": args.gpus,
                    "steps": 1, "warmup": 0, "ms_per_step": r["sec"] * 1e3, "higher_is_better": True,
                    "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic N(0,1)",
                    "config": cfg_json,
                    "cpu_baseline": {"value": r["value"], "unit": "beams", "cores": r["nproc"], "kind": cpu_kind(),
                                     "sample": "1 chunk of 1 beam per process, %d processes (int4 dequantization, then pirate's "
                                               "ReferenceDedisperser sophistication 1, %s)" % (
                                                   r["nproc"], "pirate's own code, oracle/_ref" if cpu_kind() == "reference"
                                                   else "the oracle's fp32 restatement")},
                    "e2e": {"value": r["value"], "unit": "beams", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
            print(json.dumps(line), flush=True)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    r = run_ours(args, rank, world)
    peak, peak_kind = load_peaks()
    from pirate_b200.replicas import real_time_beams
    value = real_time_beams(args.beams, world, r["ms_per_step"] * 1e-3, CHUNK_SECONDS)
    e2e = real_time_beams(args.beams, world, r["e2e_ms_per_step"] * 1e-3, CHUNK_SECONDS)

    classes = ["grid_lds", "sifter", "stage1", "stage2", "pf"]
    kt = r["ktimes"]
    tot_ms = sum(kt[c][0] for c in classes)
    dom = max(classes, key=lambda c: kt[c][0])
    nsteps = args.steps
    dom_ms_per_step = kt[dom][0] / nsteps
    dom_launches_per_step = kt[dom][1] / nsteps
    dom_bytes = r["alg"][classes.index(dom)]
    achieved = dom_bytes / (dom_ms_per_step * 1e-3) / 1e9
    # DRAM traffic per launch of the dominant kernel: the ncu-measured ratio of DRAM bytes
    # (dram__bytes_read.sum + dram__bytes_write.sum) to algorithmic bytes on a capture of the same
    # kernel, times this workload's algorithmic bytes per launch (profiles/traffic.json).
    traffic = None
    dom_bytes_per_launch = dom_bytes / dom_launches_per_step if dom_launches_per_step else None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath) and dom_bytes_per_launch:
        try:
            with open(tpath) as f:
                tj = json.load(f)
            if dom in tj and tj[dom].get("dram_over_alg"):
                traffic = round(tj[dom]["dram_over_alg"] * dom_bytes_per_launch)
        except Exception:
            traffic = None
    alg_total = sum(r["alg"])
    # Stage 2 and peak finding counted together as pirate's fused CoalescedDdKernel2
    # (src_lib/CoalescedDdKernel2.cu:128-135): the stage-1 delay lines read once plus the outputs, which
    # equals the peak finder's algorithmic bytes (its subband-row reads are the same count of samples);
    # the subband rows' HBM round trip between the two kernels counts as overhead here.
    t_cdd2 = (kt["stage2"][0] + kt["pf"][0]) / nsteps
    cdd2 = None
    if t_cdd2 > 0:
        a_cdd2 = r["alg"][classes.index("pf")] / (t_cdd2 * 1e-3) / 1e9
        cdd2 = {"achieved": round(a_cdd2, 1), "peak": peak, "unit": "GB/s", "frac": round(a_cdd2 / peak, 4),
                "ms_per_step": round(t_cdd2, 4), "algorithmic_bytes_per_step": r["alg"][classes.index("pf")]}
    e2e_alg_gbs = alg_total / (r["ms_per_step"] * 1e-3) / 1e9

    line = None
    if rank == 0:
        line = {"metric": METRIC, "value": round(value, 2), "unit": "beams", "n_gpus": world, "steps": nsteps,
                "warmup": args.warmup, "ms_per_step": round(r["ms_per_step"], 4), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic N(0,1), seeded",
                "config": cfg_json,
                "e2e": {"value": round(e2e, 2), "unit": "beams", "h2d_bytes_per_step": int(r["h2d"]),
                        "d2h_bytes_per_step": int(r["d2h"]), "ms_per_step": round(r["e2e_ms_per_step"], 4)},
                "gpu_launches": int(r["kernels_per_batch"] * nsteps),
                "roofline": {"bound": "hbm", "kernel": dom, "launches_per_step": dom_launches_per_step,
                             "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                             "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
                             "traffic": traffic, "algorithmic_bytes_per_launch": dom_bytes_per_launch,
                             "algorithmic_bytes_per_step": dom_bytes},
                "kernels": {c: {"ms_per_step": round(kt[c][0] / nsteps, 4), "share": round(kt[c][0] / tot_ms, 4) if tot_ms else None,
                                "alg_GBps": round(r["alg"][i] / (kt[c][0] / nsteps * 1e-3) / 1e9, 1) if kt[c][0] else None}
                            for i, c in enumerate(classes)},
                "time_loop": {"value": round(r["time_loop"], 2), "unit": "beams", "iterations": r["time_loop_iters"],
                              "note": "pirate's GpuDedisperser::time loop (pb2_dd_time) on one GPU: int4 input copied from "
                                      "pinned host memory every batch, median over iterations"},
                "cdd2_model": cdd2,
                "kernel_timing": {"ms_per_step": round(r["kms_per_step"], 4), "steps": nsteps,
                                  "note": "per-kernel-class CUDA events in a second timed region of the same K steps"},
                "pipeline_alg_GBps": round(e2e_alg_gbs, 1),
                "device_bytes": r["device_bytes"],
                "clocks": r["clocks"]}
        line["capacity_beams"] = r["capacity_beams"]
        line["capacity_note"] = ("beams whose lag state and buffers fit in this GPU's HBM (%.2f GB per beam); "
                                 "the real-time figure above is throughput" % (r["bytes_per_beam"] / 1e9))
    if world == 1:
        # free the headline run's device memory before the other legs
        import gc
        import torch
        r.pop("dd", None)
        gc.collect()
        torch.cuda.empty_cache()
    if world == 1 and args.streams == 1 and args.beams % 2 == 0 and not args.no_streams_leg:
        # The same workload as two batches of beams on two compute streams (num_active_batches 2): the
        # batches' kernels overlap, filling each other's partial waves. Reported beside the headline,
        # whose per-kernel event timing needs one stream.
        import copy
        a2 = copy.copy(args)
        a2.streams, a2.steps = 2, max(10, min(args.steps, 30))
        r2 = run_ours(a2, rank, world)
        r2.pop("dd", None)
        gc.collect()
        torch.cuda.empty_cache()
        line["two_streams"] = {"value": round(real_time_beams(args.beams, world, r2["ms_per_step"] * 1e-3, CHUNK_SECONDS), 2),
                               "e2e": round(real_time_beams(args.beams, world, r2["e2e_ms_per_step"] * 1e-3, CHUNK_SECONDS), 2),
                               "ms_per_step": round(r2["ms_per_step"], 4), "steps": a2.steps,
                               "config": "%d beams as 2 batches of %d on 2 compute streams" % (args.beams, args.beams // 2)}
    if world == 1 and not args.no_plain_fp32:
        pv, pms = run_plain_fp32(args, max(10, min(args.steps, 30)))
        line["plain_fp32"] = {"value": round(pv, 2), "unit": "beams", "ms_per_step": round(pms, 4),
                              "config": "1 beam, float32 storage, float32 input resident on the device, no batching"}
        line["vs_plain_fp32"] = round(value / pv, 3)
    if world == 1 and not args.no_batched:
        line["batched_uneven"] = run_batched(args.batched_scale, max(10, min(args.steps, 30)))
        line["batched_uneven"]["note"] = ("the uneven workload at %g x its 64 beams: the full 64 need about 300 GB of lag "
                                        "state (fp16), more than this GPU's HBM plus host memory" % args.batched_scale)
    if world == 1 and not args.no_spill:
        line["spill"] = run_spill(max(5, min(args.steps, 10)))
        # the same at the max_gpu_clag that fits the most beams (the sweep above): fewer, deeper rows spilled
        deep = run_spill(max(5, min(args.steps, 10)), clag=32, sweep=False)
        line["spill"]["max_gpu_clag_32"] = {k: deep[k] for k in ("value", "ms_per_step", "device_bytes_per_beam", "capacity_beams")
                                            if k in deep}
    if world == 1 and not args.no_sifter:
        line["sifter"] = run_sifter(max(5, min(args.steps, 20)))
    if rank == 0:
        if not args.no_cpu_baseline and world == 1:
            kind = cpu_kind()
            sec = cpu_sample(1, args.dtype, kind)
            line["cpu_baseline"] = {"value": round(CHUNK_SECONDS / sec, 4), "unit": "beams", "cores": 1, "kind": kind,
                                    "sample": "1 chunk of 1 beam, %.1f s: int4 dequantization, then pirate's ReferenceDedisperser "
                                              "sophistication 1 (%s)" % (sec, "pirate's own code, oracle/_ref" if kind == "reference"
                                                                        else "the oracle's fp32 restatement")}
        print(json.dumps(line), flush=True)

    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
