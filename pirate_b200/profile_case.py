"""A small rank-14 pipeline for kernel captures: 4096 channels (400-800 MHz), 5 primary trees, 2048-sample
chunks, 8 beams in one batch, float16, host spill of every row whose lag reaches 2 chunks
(`max_gpu_clag` 1), and the candidate stage with an untrained sifter at 6 sigma. It holds about 5 GB on
the device and 5 GB of mapped host memory, so profilers can replay its kernels.

    python -m pirate_b200.profile_case [--chunks 6] [--clag 1] [--no-sifter]
"""

import argparse

import numpy as np


def config(clag=1):
    prim = [dict(num_early_triggers=0, max_width=32, dm_downsampling=0, time_downsampling=0,
                 wt_dm_downsampling=2 ** ((14 - (1 if i else 0)) // 2), wt_time_downsampling=64)
            for i in range(5)]
    return dict(zone_nfreq=[4096], zone_freq_edges=[400.0, 800.0], time_sample_ms=1.0, toplevel_tree_rank=14,
                time_samples_per_chunk=2048, dtype="float16", frequency_subband_counts=[0, 0, 0, 0, 1],
                primary_trees=prim, beams_per_gpu=8, beams_per_batch=8, num_active_batches=1,
                future_write_max_samples=0, max_gpu_clag=clag)


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--chunks", type=int, default=6)
    ap.add_argument("--clag", type=int, default=1, help="max_gpu_clag (10000: no host spill)")
    ap.add_argument("--no-sifter", action="store_true")
    a = ap.parse_args(argv)
    import torch
    import pirate_b200 as pb
    from pirate_b200 import sifter as S
    plan = pb.DedispersionPlan(pb.DedispersionConfig.from_dict(config(a.clag)))
    dd = pb.GpuDedisperser(plan, cuda_device_id=0, num_consumers=1)
    dd.allocate()
    dd.fill_analytic_weights(np.ones(plan.nfreq))
    if not a.no_sifter:
        dd.enable_sifter(6.0, S.Sifter(device=0, max_batch=64, seed=1))
    print("device GB %.2f, host GB %.2f" % (dd.device_bytes() / 1e9, dd.host_bytes() / 1e9), flush=True)
    for _ in range(a.chunks):
        with dd.get_input() as x:
            x.normal_()
        with dd.get_output(0, sync=True):
            pass
    torch.cuda.synchronize()
    print("ok")


if __name__ == "__main__":
    main()
