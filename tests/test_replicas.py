"""Multi-GPU replicas (one process per GPU, beams sharded, no data exchange) exercised on CPU with
gloo, world size 2: the timing bookkeeping (barrier, max over ranks, whole-job metric) and the claim
it rests on, that a beam's outputs do not depend on which process or batch dedisperses it."""

import os
import socket

import numpy as np
import pytest

import helpers as H
import oracle as O


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _cfg(beams_per_gpu):
    return H.toy_config(rank=7, nfreq=200, nt=256, dtype="float32", subbands=[2, 2, 1],
                        beams_per_gpu=beams_per_gpu, beams_per_batch=1)


NCHUNKS = 2


def _beam_input(beam, chunk):
    """Seeded N(0,1) input of one beam and chunk, a function of the global beam id only."""
    cfg = _cfg(1)
    rng = np.random.default_rng(1000 * beam + chunk)
    return rng.standard_normal((1, sum(cfg["zone_nfreq"]), cfg["time_samples_per_chunk"])).astype(np.float32)


def _weights():
    orc = O.OracleDedisperser(_cfg(1), 1, 32)
    return H.make_weights(orc, seed=5)


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    import datetime
    import torch.distributed as dist
    from pirate_b200 import replicas
    try:
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
        r, w = replicas.rank_world()
        lo, hi = replicas.beam_range(1, r)
        orc = O.OracleDedisperser(_cfg(1), 1, 32)
        ws = _weights()
        replicas.barrier()
        outs = []
        for c in range(NCHUNKS):
            for b in range(lo, hi):
                m, a = orc.dedisperse(0, _beam_input(b, c), [x[0] for x in ws])
                outs.append((b, c, [np.asarray(v).copy() for v in m], [np.asarray(v).copy() for v in a]))
        # a rank-dependent "duration": every rank must see the slowest one
        slowest = replicas.max_over_ranks(1.5 + r)
        replicas.barrier()
        gathered = [None] * w
        dist.all_gather_object(gathered, outs)
        dist.destroy_process_group()
        q.put((r, w, slowest, gathered if r == 0 else None, None))
    except Exception as e:  # reported to the parent, which fails the test
        q.put((rank, world, None, None, repr(e)))


def test_beam_range_and_metric():
    from pirate_b200 import replicas
    assert replicas.beam_range(4, 0) == (0, 4)
    assert replicas.beam_range(4, 3) == (12, 16)
    with pytest.raises(ValueError):
        replicas.beam_range(0, 1)
    # 4 beams per GPU on 8 GPUs, slowest rank 8 ms per 2.048 s chunk
    assert replicas.real_time_beams(4, 8, 8e-3, 2.048) == pytest.approx(32 * 256.0)
    with pytest.raises(ValueError):
        replicas.real_time_beams(4, 1, 0.0, 2.048)
    # without a process group: identity and no-op
    assert replicas.max_over_ranks(3.25) == 3.25
    replicas.barrier()


def test_two_gloo_ranks_shard_beams():
    import multiprocessing as mp
    O.build()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = [q.get(timeout=300) for _ in ps]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    errs = [e for *_, e in res if e]
    assert not errs, errs
    assert sorted(r for r, *_ in res) == [0, 1]
    assert all(s == 2.5 for _, _, s, _, _ in res)
    gathered = next(g for _, _, _, g, _ in res if g is not None)

    # One process serving both beams (beams_per_gpu 2, one beam per batch) gives the same outputs.
    cfg2 = _cfg(2)
    xs = [_beam_input(b, c) for c in range(NCHUNKS) for b in range(2)]
    _, ref = H.run_oracle(cfg2, xs, _weights())
    by_key = {(b, c): (m, a) for outs in gathered for b, c, m, a in outs}
    assert len(by_key) == 2 * NCHUNKS
    for seq in range(len(xs)):
        b, c = seq % 2, seq // 2
        m, a = by_key[(b, c)]
        for i in range(len(m)):
            assert np.array_equal(m[i], ref[seq][0][i]), "beam %d chunk %d tree %d out_max" % (b, c, i)
            assert np.array_equal(a[i], ref[seq][1][i]), "beam %d chunk %d tree %d out_argmax" % (b, c, i)


def test_reference_arm_non_zero_rank_does_no_work():
    """Under torchrun the reference arm runs on rank 0 only; the other ranks return at once."""
    import argparse
    import bench
    args = argparse.Namespace(dtype="float16")
    assert bench.run_reference(args, 1, 2) is None
