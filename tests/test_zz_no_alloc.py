"""The allocation-free entry point pb2_dedisperse_chunk_noalloc (include/pirate_b200.h).

It serves callers that cannot call cudaMalloc, such as real-time threads that must not stall on
cudaMalloc's device-wide synchronization, or code inside a framework whose memory pool must own
every device allocation. It dedisperses one chunk as the first chunk of a fresh stream with all
scratch in a fixed static device array. Its outputs must equal, bit for bit (the float32 tolerance
of the other parity tests), those of the allocating GpuDedisperser entry points on chunk 0 of a new
dedisperser, on two calls in a row (the scratch array keeps the previous call's contents, so the
second call checks that it is cleared). This file is collected last on purpose."""

import ctypes

import numpy as np
import pytest

import helpers as H

pytestmark = pytest.mark.gpu


def _noalloc(pb, plan, x, ws, outs_max, outs_arg, stream):
    L = pb.lib()
    f = L.pb2_dedisperse_chunk_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_void_p),
                  ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p]
    n = plan.ntrees
    wp = (ctypes.c_void_p * n)(*[w.data_ptr() for w in ws])
    mp = (ctypes.c_void_p * n)(*[m.data_ptr() for m in outs_max])
    ap = (ctypes.c_void_p * n)(*[a.data_ptr() for a in outs_arg])
    return f(plan._h, x.data_ptr(), wp, mp, ap, stream.cuda_stream)


@pytest.mark.parametrize("dtype,beams", [("float32", 1), ("float16", 2)])
def test_noalloc_matches_gpu_dedisperser(pb2lib, dtype, beams):
    """float32 with one beam, and float16 (the benchmark's storage) with two beams per batch, so that
    the per-beam strides of every scratch region are exercised. Both entry points run the same kernels
    on the same inputs, so even float16 outputs must agree bit for bit."""
    import torch
    pb = pb2lib
    cfg = H.toy_config(rank=8, nfreq=640, nt=256, dtype=dtype, subbands=[2, 2, 1], beams_per_gpu=beams,
                       beams_per_batch=beams)
    plan = pb.DedispersionPlan(pb.DedispersionConfig.from_dict(cfg))
    orc, _ = H.run_oracle(cfg, [], [])
    ws_host = H.make_weights(orc, seed=5)
    dev = torch.device("cuda:0")
    stream = torch.cuda.current_stream()
    ws_dev = [torch.from_numpy(w[0]).to(dev) for w in ws_host]
    tdt = getattr(torch, dtype)
    outs_max = [torch.empty(orc.out_shape(i), dtype=tdt, device=dev) for i in range(plan.ntrees)]
    outs_arg = [torch.empty(orc.out_shape(i), dtype=torch.int32, device=dev) for i in range(plan.ntrees)]

    for call in range(2):
        x = H.make_inputs(cfg, 1, seed=100 + call)[0]
        # Existing entry points: chunk 0 of a fresh GpuDedisperser.
        _, _, ref = H.run_gpu(pb, cfg, [x], ws_host)
        xd = torch.from_numpy(x).to(dev).to(tdt)
        for m, a in zip(outs_max, outs_arg):
            m.fill_(123.0)
            a.fill_(-7)
        rc = _noalloc(pb, plan, xd, ws_dev, outs_max, outs_arg, stream)
        assert rc == 0, pb.lib().pb2_last_error().decode()
        torch.cuda.synchronize()
        for i in range(plan.ntrees):
            got_m = outs_max[i].cpu().numpy().astype(np.float64)
            got_a = outs_arg[i].cpu().numpy().view(np.uint32)
            assert np.array_equal(got_m, ref[0][0][i]), "call %d tree %d: out_max differs" % (call, i)
            assert np.array_equal(got_a, ref[0][1][i]), "call %d tree %d: out_argmax differs" % (call, i)


def test_noalloc_rejects_large_plan(pb2lib):
    import torch
    pb = pb2lib
    prim = [dict(num_early_triggers=0, max_width=32, dm_downsampling=0, time_downsampling=0,
                 wt_dm_downsampling=64, wt_time_downsampling=64)]
    cfg = H.toy_config(rank=16, nfreq=16384, nt=2048, subbands=[0, 0, 0, 0, 1], beams_per_gpu=1,
                       beams_per_batch=1, primary_trees=prim)
    plan = pb.DedispersionPlan(pb.DedispersionConfig.from_dict(cfg))
    dev = torch.device("cuda:0")
    dummy = torch.zeros(16, device=dev)
    rc = _noalloc(pb, plan, dummy, [dummy] * plan.ntrees, [dummy] * plan.ntrees, [dummy] * plan.ntrees,
                  torch.cuda.current_stream())
    assert rc != 0
    assert "PB2_NOALLOC_SCRATCH_BYTES" in pb.lib().pb2_last_error().decode()
