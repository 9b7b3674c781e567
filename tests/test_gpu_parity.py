"""Parity of the CUDA dedispersion path (through the public GpuDedisperser API, i.e. the C ABI)
with the CPU oracle restating pirate's ReferenceDedisperser, on identical seeded inputs.

float32 plans must match the fp32 oracle bit for bit (out_max) and token for token (out_argmax):
the kernels perform the oracle's exact sequence of fp32 operations. float16/bfloat16 storage plans
are compared with the FP64 oracle on the same (quantized) inputs, in units of the output sigma
(bare unit-variance weights), and their tokens are checked by re-evaluating them in the oracle
(ReferencePeakFindingKernel::eval_tokens, src_lib/PeakFindingKernel.cu:467)."""

import numpy as np
import pytest

import helpers as H
import oracle as O

pytestmark = pytest.mark.gpu

FP32_CASES = H.PARITY_CASES


def _cfg(case, dtype="float32"):
    return H.case_config(case, dtype)


@pytest.mark.parametrize("case", FP32_CASES, ids=lambda c: "r%d_f%d_t%d" % (c[0], c[1], c[2]))
def test_fp32_bitwise(pb2lib, case):
    cfg = _cfg(case)
    nb = cfg["beams_per_gpu"] // cfg["beams_per_batch"]
    nchunks = 5
    xs = H.make_inputs(cfg, nchunks, seed=case[0] * 7 + case[2])
    orc, _ = H.run_oracle(cfg, xs[:0], [])  # shapes only
    ws = H.make_weights(orc, seed=case[0], nbatches_wt=1)
    _, ores = H.run_oracle(cfg, xs, ws, 1, 32)
    plan, dd, gres = H.run_gpu(pb2lib, cfg, xs, ws)
    for seq in range(nchunks * nb):
        for i in range(orc.ntrees):
            gm, ga = gres[seq][0][i], gres[seq][1][i]
            om, oa = ores[seq][0][i], ores[seq][1][i]
            assert gm.shape == om.shape
            if not np.array_equal(gm, om):
                d = np.abs(gm - om)
                pytest.fail("seq %d tree %d: out_max differs at %d/%d entries, max |diff| %.3g" % (seq, i, (d > 0).sum(), d.size, d.max()))
            if not np.array_equal(ga, oa):
                pytest.fail("seq %d tree %d: out_argmax differs at %d/%d entries" % (seq, i, (ga != oa).sum(), ga.size))


@pytest.mark.parametrize("case", [FP32_CASES[1], FP32_CASES[6]], ids=["r8_tds4", "r8_tds16_32"])
def test_fp32_nan_inputs(pb2lib, case):
    """Inputs with NaN samples: NaN propagates through the trees; the peak finder ignores NaN trials
    (the reference's strict '>' never takes one) and reports -1e30 / token 0xffffffff where every trial
    is NaN. float32 outputs and tokens must still match the oracle exactly."""
    cfg = _cfg(case)
    nb = cfg["beams_per_gpu"] // cfg["beams_per_batch"]
    nchunks = 3
    xs = H.make_inputs(cfg, nchunks, seed=5)
    rng = np.random.default_rng(17)
    for x in xs:
        x[rng.random(x.shape) < 2e-4] = np.nan
    xs[nb][:, :, 100:104] = np.nan   # a NaN burst in every channel: some outputs see only NaN trials
    orc, _ = H.run_oracle(cfg, xs[:0], [])
    ws = H.make_weights(orc, seed=2, nbatches_wt=1)
    _, ores = H.run_oracle(cfg, xs, ws, 1, 32)
    plan, dd, gres = H.run_gpu(pb2lib, cfg, xs, ws)
    nan_trials = 0
    for seq in range(nchunks * nb):
        for i in range(orc.ntrees):
            gm, ga = gres[seq][0][i], gres[seq][1][i]
            om, oa = ores[seq][0][i], ores[seq][1][i]
            nan_trials += int((oa == 0xffffffff).sum())
            assert np.array_equal(gm, om, equal_nan=True), "seq %d tree %d: out_max differs" % (seq, i)
            assert np.array_equal(ga, oa), "seq %d tree %d: out_argmax differs at %d entries" % (seq, i, (ga != oa).sum())
    assert not np.isnan(np.concatenate([r.ravel() for s in ores for r in s[0]])).any()
    assert nan_trials > 0   # the burst left outputs without a winning trial


LOWP_CASES = [
    ("float16", (8, 640, 256, [2, 2, 1], [(0, 16), (1, 8)], 2, 1), 1e-2),
    ("bfloat16", (8, 640, 256, [2, 2, 1], [(0, 16), (1, 8)], 2, 1), 6e-2),
    ("float16", (10, 1024, 512, [0, 0, 1], [(0, 32), (0, 16), (0, 8)], 1, 1), 1e-2),
]


@pytest.mark.parametrize("dtype,case,tol", LOWP_CASES, ids=lambda v: str(v) if isinstance(v, str) else None)
def test_lowp_vs_fp64(pb2lib, dtype, case, tol):
    """Max |error| of fp16/bf16-storage outputs against the FP64 oracle, in sigma, within 'tol'."""
    cfg = _cfg(case, dtype)
    nb = cfg["beams_per_gpu"] // cfg["beams_per_batch"]
    nchunks = 4
    xs = H.make_inputs(cfg, nchunks, seed=11)
    orc64 = None
    orc, _ = H.run_oracle(cfg, xs[:0], [], 1, 64)
    ws = H.make_weights(orc, seed=3, kind="bare")
    orc64, ores = H.run_oracle(cfg, xs, ws, 1, 64, keep=lambda o, s: None)
    plan, dd, gres = H.run_gpu(pb2lib, cfg, xs, ws)
    worst = 0.0
    for seq in range(nchunks * nb):
        for i in range(orc.ntrees):
            gm, om = gres[seq][0][i], ores[seq][0][i]
            worst = max(worst, float(np.abs(gm - om).max()))
    assert worst <= tol, "max |gpu - fp64 oracle| = %.3g sigma > %.3g" % (worst, tol)
    # Tokens: the trial each GPU token names must evaluate (in the oracle) to the oracle's max within tol.
    last = len(xs) - 1
    for i in range(orc.ntrees):
        ev = orc64.eval_tokens(i, gres[last][1][i], ws[i][0])
        assert np.abs(ev - ores[last][0][i]).max() <= 2 * tol


def test_fp32_bitwise_rank16(pb2lib):
    """Maximum tree rank (16): stage ranks 8+8 (the 4+4 register-tree split) and buffers whose sizes
    end on page boundaries; two chunks bitwise against the fp32 oracle."""
    prim = [dict(num_early_triggers=1, max_width=32, dm_downsampling=0, time_downsampling=0,
                 wt_dm_downsampling=64, wt_time_downsampling=64)]
    cfg = H.toy_config(rank=16, nfreq=4096, nt=2048, dtype="float32", subbands=[0, 2, 0, 0, 1],
                       beams_per_gpu=1, beams_per_batch=1, primary_trees=prim)
    xs = H.make_inputs(cfg, 2, seed=16)
    orc, _ = H.run_oracle(cfg, xs[:0], [])
    ws = H.make_weights(orc, seed=16)
    _, ores = H.run_oracle(cfg, xs, ws, 1, 32)
    _, _, gres = H.run_gpu(pb2lib, cfg, xs, ws)
    for seq in range(len(xs)):
        for i in range(orc.ntrees):
            assert np.array_equal(gres[seq][0][i], ores[seq][0][i]), "seq %d tree %d out_max" % (seq, i)
            assert np.array_equal(gres[seq][1][i], ores[seq][1][i]), "seq %d tree %d out_argmax" % (seq, i)


def test_fp32_small_output_trees_share_warps(pb2lib):
    """Rank 14, 5 primary trees, peak-finding downsampling 16: the two most downsampled trees have 16 and
    8 output times per chunk, and their peak finder runs 2 and 4 coarse DMs per warp (16 and 8 lanes
    each). Two beams, three chunks, NaN planted in one beam: bitwise the fp32 oracle."""
    import bench
    cfg = bench.bench_config(2, "float32", 14, 5, 4096)
    plan = pb2lib.DedispersionPlan(pb2lib.DedispersionConfig.from_dict(cfg))
    assert [t.nt_out for t in plan.trees][-2:] == [16, 8]
    xs = H.make_inputs(cfg, 3, seed=14)
    xs[1][1, 100:140, 500:520] = np.nan
    orc, _ = H.run_oracle(cfg, xs[:0], [])
    ws = H.make_weights(orc, seed=14)
    _, ores = H.run_oracle(cfg, xs, ws, 1, 32)
    _, _, gres = H.run_gpu(pb2lib, cfg, xs, ws)
    for seq in range(len(xs)):
        for i in range(orc.ntrees):
            assert np.array_equal(gres[seq][0][i], ores[seq][0][i], equal_nan=True), "seq %d tree %d out_max" % (seq, i)
            assert np.array_equal(gres[seq][1][i], ores[seq][1][i]), "seq %d tree %d out_argmax" % (seq, i)


@pytest.mark.parametrize("dtype", ["float32", "float16"])
def test_benchmark_config_full_size(pb2lib, dtype):
    """The benchmark's workload at full size, one beam, two chunks, fed pirate's raw int4 input
    through the fused dequantizing input path: rank-16 tree from 16384 channels, 5 primary trees
    (time downsampling 1-16), widths to 32, full-band search. float32 storage: bitwise equal to the fp32
    oracle on the dequantized input. float16 storage (the benchmark's): within the fp16 tolerance
    of 1e-2 sigma (bare weights), and every GPU token re-evaluates in the oracle to within 2e-2."""
    import torch
    import bench
    cfg = bench.bench_config(1, dtype)
    rng = np.random.default_rng(77)
    B, F, T = 1, 16384, cfg["time_samples_per_chunk"]
    qs = [O.random_quantized(rng, B, F, T) for _ in range(2)]
    xs = [O.dequantize(d, s, B, F, T) for d, s in qs]
    orc = O.OracleDedisperser(cfg, 1, 32)         # one instance: about 20 GB of lag state at rank 16
    ws = [O.bare_weights(orc.wt_shape(i), orc.trees[i]["nprofiles"])[None] for i in range(orc.ntrees)]
    ores = [orc.dedisperse(0, x, [w[0] for w in ws]) for x in xs]
    plan = pb2lib.DedispersionPlan(pb2lib.DedispersionConfig.from_dict(cfg))
    dd = pb2lib.GpuDedisperser(plan, cuda_device_id=0, num_consumers=1)
    dd.allocate()
    for i, w in enumerate(ws):
        dd.fill_all_weights(i, w)
    for seq, (d, s) in enumerate(qs):
        with dd.get_input_int4() as (dq, sq):
            dq.copy_(torch.from_numpy(d).cuda())
            sq.copy_(torch.from_numpy(s).cuda())
        with dd.get_output(0, sync=True) as out:
            for i in range(orc.ntrees):
                gm = out.out_max[i].float().cpu().numpy().astype(np.float64)
                ga = out.out_argmax[i].cpu().numpy().view(np.uint32)
                om, oa = ores[seq][0][i], ores[seq][1][i]
                if dtype == "float32":
                    assert np.array_equal(gm, om), "seq %d tree %d out_max" % (seq, i)
                    assert np.array_equal(ga, oa), "seq %d tree %d out_argmax" % (seq, i)
                else:
                    err = float(np.abs(gm - om).max())
                    assert err <= 1e-2, "seq %d tree %d: max |gpu - oracle| = %.3g sigma" % (seq, i, err)
                    if seq == len(qs) - 1:
                        ev = orc.eval_tokens(i, ga, ws[i][0])
                        assert np.abs(ev - om).max() <= 2e-2, "tree %d: tokens" % i
