"""int4 input (pirate's raw format; GpuDequantizationKernel, src_lib/GpuDequantizationKernel.cu):
the standalone dequantization kernel against the oracle's restatement of
ReferenceDequantizationKernel::apply, and the dedisperser's fused int4 input path against
"dequantize, then dedisperse" and against the oracle dedisperser."""

import numpy as np
import pytest

import helpers as H
import oracle as O

pytestmark = pytest.mark.gpu


def _to_device(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("dtype", ["float32", "float16", "bfloat16"])
def test_dequantize_kernel(pb2lib, dtype):
    """fp32 output bit for bit equal to the oracle; fp16/bf16 output = the oracle's fp32 value rounded
    once to nearest (even), bit for bit. Includes the -8 'missing' sentinel."""
    import torch
    rng = np.random.default_rng(21)
    B, F, T = 2, 5, 768
    data, so = O.random_quantized(rng, B, F, T)
    ref = O.dequantize(data, so, B, F, T)
    out = torch.empty((B, F, T), dtype=getattr(torch, dtype), device="cuda")
    pb2lib.dequantize(out, _to_device(so), _to_device(data))
    torch.cuda.synchronize()
    want = torch.from_numpy(ref).to(getattr(torch, dtype))   # round-to-nearest-even on the host
    bits = torch.int32 if dtype == "float32" else torch.int16
    assert torch.equal(out.cpu().view(bits), want.view(bits))


def test_dequantize_rejects_bad_shapes(pb2lib):
    import torch
    out = torch.empty((1, 2, 300), dtype=torch.float32, device="cuda")
    with pytest.raises(RuntimeError):
        pb2lib.dequantize(out, torch.empty((1, 2, 1, 2), dtype=torch.float16, device="cuda"),
                          torch.empty((1, 2, 150), dtype=torch.uint8, device="cuda"))


def _run_int4(pb, cfg, qs, weights, fused):
    """Runs the dedisperser on int4 chunks qs = [(data, scales_offsets)], either through the fused
    int4 input path or through pirate_b200.dequantize into the ordinary input buffer."""
    import torch
    plan = pb.DedispersionPlan(pb.DedispersionConfig.from_dict(cfg))
    dd = pb.GpuDedisperser(plan, cuda_device_id=0, num_consumers=1)
    dd.allocate()
    for i, w in enumerate(weights):
        dd.fill_all_weights(i, w)
    res = []
    for data, so in qs:
        if fused:
            with dd.get_input_int4() as (d, s):
                d.copy_(_to_device(data))
                s.copy_(_to_device(so))
        else:
            with dd.get_input() as x:
                pb.dequantize(x, _to_device(so), _to_device(data))
        with dd.get_output(0, sync=True) as out:
            res.append(([m.float().cpu().numpy().astype(np.float64) for m in out.out_max],
                        [a.cpu().numpy().view(np.uint32).copy() for a in out.out_argmax]))
    torch.cuda.synchronize()
    return res


def _quantized_chunks(cfg, nchunks, seed):
    rng = np.random.default_rng(seed)
    B, F, T = cfg["beams_per_batch"], sum(cfg["zone_nfreq"]), cfg["time_samples_per_chunk"]
    nb = cfg["beams_per_gpu"] // B
    return [O.random_quantized(rng, B, F, T) for _ in range(nchunks * nb)]


def _int4_cfg(dtype):
    prim = [dict(num_early_triggers=0, max_width=16, dm_downsampling=0, time_downsampling=0,
                 wt_dm_downsampling=16, wt_time_downsampling=16),
            dict(num_early_triggers=1, max_width=8, dm_downsampling=0, time_downsampling=0,
                 wt_dm_downsampling=16, wt_time_downsampling=16)]
    return H.toy_config(rank=8, nfreq=300, nt=512, dtype=dtype, subbands=[2, 2, 1], beams_per_gpu=2,
                        beams_per_batch=1, primary_trees=prim)


@pytest.mark.parametrize("dtype", ["float32", "float16", "bfloat16"])
def test_int4_fused_equals_dequantize_then_dedisperse(pb2lib, dtype):
    cfg = _int4_cfg(dtype)
    qs = _quantized_chunks(cfg, 3, seed=9)
    orc, _ = H.run_oracle(cfg, [], [])
    ws = H.make_weights(orc, seed=9)
    a = _run_int4(pb2lib, cfg, qs, ws, fused=True)
    b = _run_int4(pb2lib, cfg, qs, ws, fused=False)
    for seq in range(len(qs)):
        for i in range(len(a[seq][0])):
            assert np.array_equal(a[seq][0][i], b[seq][0][i]), "seq %d tree %d out_max" % (seq, i)
            assert np.array_equal(a[seq][1][i], b[seq][1][i]), "seq %d tree %d out_argmax" % (seq, i)


def test_int4_fp32_vs_oracle(pb2lib):
    """float32 plan fed int4 chunks: bit for bit equal to the oracle dedisperser on the oracle's
    dequantized input."""
    cfg = _int4_cfg("float32")
    qs = _quantized_chunks(cfg, 3, seed=10)
    B, F, T = cfg["beams_per_batch"], sum(cfg["zone_nfreq"]), cfg["time_samples_per_chunk"]
    xs = [O.dequantize(d, s, B, F, T) for d, s in qs]
    orc, _ = H.run_oracle(cfg, [], [])
    ws = H.make_weights(orc, seed=10)
    _, ores = H.run_oracle(cfg, xs, ws, 1, 32)
    g = _run_int4(pb2lib, cfg, qs, ws, fused=True)
    for seq in range(len(qs)):
        for i in range(orc.ntrees):
            assert np.array_equal(g[seq][0][i], ores[seq][0][i]), "seq %d tree %d out_max" % (seq, i)
            assert np.array_equal(g[seq][1][i], ores[seq][1][i]), "seq %d tree %d out_argmax" % (seq, i)


@pytest.mark.parametrize("nfreq,npri", [(300, 5), (900, 5), (2000, 2)])
def test_int4_lookup_tables_vs_oracle(pb2lib, nfreq, npri):
    """The gridding kernel's per-warp int4 lookup tables: 16-sample windows (5 primary trees: two scale
    blocks per warp), channel pairs whose input rows exceed the tables mixed with pairs that fit
    (900 channels), and pairs that never fit (2000). float32 is bitwise the oracle; float16 equals the
    separate dequantization kernel followed by the dedisperser."""
    prim = H._prim(8, [(0, 16, 0)] + [(0, 8, 0)] * (npri - 1), wt_time=16)
    for dtype in ("float32", "float16"):
        cfg = H.toy_config(rank=8, nfreq=nfreq, nt=1024, dtype=dtype, subbands=[2, 2, 1], beams_per_gpu=2,
                           beams_per_batch=1, primary_trees=prim)
        qs = _quantized_chunks(cfg, 2, seed=nfreq)
        orc, _ = H.run_oracle(cfg, [], [])
        ws = H.make_weights(orc, seed=11)
        g = _run_int4(pb2lib, cfg, qs, ws, fused=True)
        if dtype == "float32":
            B, F, T = cfg["beams_per_batch"], sum(cfg["zone_nfreq"]), cfg["time_samples_per_chunk"]
            xs = [O.dequantize(d, s, B, F, T) for d, s in qs]
            _, want = H.run_oracle(cfg, xs, ws, 1, 32)
        else:
            want = _run_int4(pb2lib, cfg, qs, ws, fused=False)
        for seq in range(len(qs)):
            for i in range(orc.ntrees):
                assert np.array_equal(g[seq][0][i], want[seq][0][i]), (dtype, seq, i)
                assert np.array_equal(g[seq][1][i], want[seq][1][i]), (dtype, seq, i)
