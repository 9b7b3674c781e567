"""Host spill of the stage-1 delay lines (pirate's MegaRingbuf host zones and g2h/h2g copies,
src_lib/MegaRingbuf.cpp:155-183, src_lib/GpuDedisperser.cpp:628-707): with a small max_gpu_clag, rows
whose readers are more than that many chunks behind live in pinned host memory and move through the
g2h/h2g copy kernels every chunk. The outputs must not change: float32 storage stays bit for bit equal
to the fp32 oracle, and float16 storage to the same plan without spill."""

import numpy as np
import pytest

import helpers as H

pytestmark = pytest.mark.gpu


def _cfg(rank, nfreq, nt, sb, pts, bpg, bpb, clag, dtype="float32"):
    c = H.toy_config(rank=rank, nfreq=nfreq, nt=nt, dtype=dtype, subbands=sb, beams_per_gpu=bpg, beams_per_batch=bpb,
                     primary_trees=H._prim(rank, pts, 16))
    c["max_gpu_clag"] = clag
    return c


CASES = [
    # rank, nfreq, nt, subbands, trees (early triggers, width, time ds), beams, beams/batch, max_gpu_clag, chunks
    (10, 1024, 64, [0, 0, 1], [(0, 16, 0)], 2, 1, 1, 24),
    (9, 300, 128, [1, 1, 1], [(1, 16, 0), (0, 8, 0)], 2, 2, 0, 12),
    (11, 2000, 256, [0, 1, 0, 1], [(0, 32, 0), (0, 16, 0), (0, 8, 0)], 1, 1, 2, 14),
]


@pytest.mark.parametrize("case", CASES, ids=["r10_t64", "r9_et", "r11_3trees"])
def test_spill_fp32_bitwise(pb2lib, case):
    rank, nfreq, nt, sb, pts, bpg, bpb, clag, nchunks = case
    cfg = _cfg(rank, nfreq, nt, sb, pts, bpg, bpb, clag)
    nb = bpg // bpb
    xs = H.make_inputs(cfg, nchunks, seed=rank + nt)
    orc, _ = H.run_oracle(cfg, [], [])
    ws = H.make_weights(orc, seed=rank)
    _, ores = H.run_oracle(cfg, xs, ws, 1, 32)
    plan, dd, gres = H.run_gpu(pb2lib, cfg, xs, ws)
    assert dd.host_bytes() > 0, "nothing was spilled"
    ref = pb2lib.GpuDedisperser(pb2lib.DedispersionPlan(pb2lib.DedispersionConfig.from_dict(dict(cfg, max_gpu_clag=10000))),
                                cuda_device_id=0, num_consumers=1)
    ref.allocate()
    assert dd.device_bytes() < ref.device_bytes()
    for seq in range(nchunks * nb):
        for i in range(orc.ntrees):
            assert np.array_equal(gres[seq][0][i], ores[seq][0][i]), (seq, i, "out_max")
            assert np.array_equal(gres[seq][1][i], ores[seq][1][i]), (seq, i, "out_argmax")


def test_spill_fp16_matches_resident(pb2lib):
    """The benchmark's tree layout at rank 12 (5 primary trees, float16 storage), 40 chunks: spilled
    (max_gpu_clag 2) and fully resident runs give identical bytes."""
    cfg = _cfg(12, 2048, 1024, [0, 0, 0, 0, 1], [(0, 32, 0)] * 5, 2, 2, 2, dtype="float16")
    xs = H.make_inputs(cfg, 40, seed=3)
    orc, _ = H.run_oracle(cfg, [], [])
    ws = H.make_weights(orc, seed=3)
    _, dd, g1 = H.run_gpu(pb2lib, cfg, xs, ws)
    assert dd.host_bytes() > 0
    _, dd0, g0 = H.run_gpu(pb2lib, dict(cfg, max_gpu_clag=10000), xs, ws)
    assert dd0.host_bytes() == 0
    for seq in range(len(xs)):
        for i in range(len(g0[seq][0])):
            assert np.array_equal(g1[seq][0][i], g0[seq][0][i]), (seq, i)
            assert np.array_equal(g1[seq][1][i], g0[seq][1][i]), (seq, i)
