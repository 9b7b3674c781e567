"""GpuDedisperser ordering, back-pressure and error semantics, after pirate's GpuDedisperser
(include/pirate/Dedisperser.hpp:158-219, src_lib/GpuDedisperser.cpp:796-808, 1078-1081) and its
"stoppable" error model (notes/stoppable_class.md): any failing entry point stops the object and every
later call rethrows the stored error.

Every wait here is on the host and bounded (the release timeout of the dedisperser, a thread join with a
timeout): no GPU-side wait is left without its event having been recorded."""

import threading
import time

import numpy as np
import pytest

import helpers as H

pytestmark = pytest.mark.gpu


def _small(pb, **kw):
    cfg = H.toy_config(rank=8, nfreq=640, nt=256, subbands=[2, 2, 1], beams_per_gpu=kw.pop("beams_per_gpu", 2),
                       beams_per_batch=kw.pop("beams_per_batch", 1), num_active_batches=kw.pop("num_active_batches", 1))
    plan = pb.DedispersionPlan(pb.DedispersionConfig.from_dict(cfg))
    dd = pb.GpuDedisperser(plan, cuda_device_id=0, **kw)
    dd.allocate()
    return cfg, plan, dd


def _launch(dd, seq, x=None):
    import torch
    a = dd.acquire_input(seq)
    if x is not None:
        a.copy_(torch.from_numpy(x).to(a.device).to(a.dtype))
    dd.release_input_and_launch_dd_kernels(seq)


def _stopped(dd):
    with pytest.raises(RuntimeError):
        dd.acquire_input(0)


def test_wrong_seq_id_raises_and_stops(pb2lib):
    _, _, dd = _small(pb2lib)
    with pytest.raises(RuntimeError, match="expected seq_id=0"):
        dd.acquire_input(1)
    # stopped: even the right call now rethrows the stored error
    with pytest.raises(RuntimeError, match="expected seq_id=0, got 1"):
        dd.acquire_input(0)


def test_release_input_before_acquire(pb2lib):
    _, _, dd = _small(pb2lib)
    with pytest.raises(RuntimeError, match="release_input_and_launch_dd_kernels"):
        dd.release_input_and_launch_dd_kernels(0)
    _stopped(dd)


def test_double_acquire_output(pb2lib):
    _, _, dd = _small(pb2lib, synchronous=False, nbatches_out=2)
    _launch(dd, 0)
    dd.acquire_output(0, 0)
    with pytest.raises(RuntimeError, match="expected seq_id=1, got 0"):
        dd.acquire_output(0, 0)
    _stopped(dd)


def test_release_output_before_acquire(pb2lib):
    _, _, dd = _small(pb2lib)
    _launch(dd, 0)
    with pytest.raises(RuntimeError, match="release_output"):
        dd.release_output(0, 0)
    _stopped(dd)


def test_acquire_output_not_launched(pb2lib):
    """acquire_output waits for the launch (another thread's), bounded by the release timeout."""
    _, _, dd = _small(pb2lib, release_timeout_ms=200)
    t0 = time.time()
    with pytest.raises(RuntimeError, match="has not been launched within 200 ms"):
        dd.acquire_output(0, 0)
    assert time.time() - t0 < 10.0
    _stopped(dd)


def test_synchronous_consumer_must_release_first(pb2lib):
    _, _, dd = _small(pb2lib, synchronous=True, nbatches_out=2)
    _launch(dd, 0)
    _launch(dd, 1)
    dd.acquire_output(0, 0)
    with pytest.raises(RuntimeError, match="synchronous consumer"):
        dd.acquire_output(0, 1)
    _stopped(dd)


def test_stop_then_calls_raise(pb2lib):
    _, _, dd = _small(pb2lib)
    _launch(dd, 0)
    dd.stop()
    with pytest.raises(RuntimeError, match="after stop"):
        dd.acquire_output(0, 0)


def test_consumer_that_never_releases(pb2lib):
    """Output slots are reused every nbatches_out batches: launching seq_id = nbatches_out waits for the
    consumer's release of seq_id 0, which never comes; the call fails after the release timeout (and
    stops the object) instead of overwriting outputs the consumer still holds."""
    _, _, dd = _small(pb2lib, synchronous=False, nbatches_out=2, release_timeout_ms=300)
    _launch(dd, 0)
    _launch(dd, 1)
    dd.acquire_output(0, 0)
    dd.acquire_output(0, 1)
    dd.acquire_input(2)
    t0 = time.time()
    with pytest.raises(RuntimeError, match="has not released seq_id=0"):
        dd.release_input_and_launch_dd_kernels(2)
    dt = time.time() - t0
    assert 0.25 <= dt < 10.0, dt
    _stopped(dd)


def _weights(cfg, seed, nbatches_wt):
    orc, _ = H.run_oracle(cfg, [], [])
    return orc, H.make_weights(orc, seed=seed, nbatches_wt=nbatches_wt)


def test_backpressure_waits_for_a_late_consumer(pb2lib):
    """A consumer thread holds seq_id 0 for 0.5 s; the producer's launch of seq_id 2 (nbatches_out = 2)
    returns only after that release, and every output the consumer reads equals the fp32 oracle."""
    cfg, plan, dd = _small(pb2lib, synchronous=False, nbatches_out=2, release_timeout_ms=20000)
    orc, ws = _weights(cfg, 3, dd.nbatches_wt)
    for i, w in enumerate(ws):
        dd.fill_all_weights(i, w)
    nchunks = 3
    xs = H.make_inputs(cfg, nchunks, seed=8)
    _, ores = H.run_oracle(cfg, xs, ws, 1, 32)
    got, errors = {}, []
    released0 = []

    def consumer():
        try:
            for seq in range(len(xs)):
                out = dd.acquire_output(0, seq, sync=True)
                got[seq] = ([m.float().cpu().numpy().astype(np.float64) for m in out.out_max],
                            [a.cpu().numpy().view(np.uint32).copy() for a in out.out_argmax])
                if seq == 0:
                    time.sleep(0.5)
                    released0.append(time.time())
                dd.release_output(0, seq)
        except Exception as e:   # reported below
            errors.append(e)

    th = threading.Thread(target=consumer)
    _launch(dd, 0, xs[0])
    _launch(dd, 1, xs[1])
    th.start()
    t_launched = []
    for seq in range(2, len(xs)):
        _launch(dd, seq, xs[seq])
        t_launched.append(time.time())
    th.join(timeout=60)
    assert not th.is_alive()
    assert not errors, errors
    assert released0 and t_launched[0] >= released0[0] - 0.01
    for seq in range(len(xs)):
        for i in range(orc.ntrees):
            assert np.array_equal(got[seq][0][i], ores[seq][0][i]), (seq, i)
            assert np.array_equal(got[seq][1][i], ores[seq][1][i]), (seq, i)


def test_two_batches_two_consumers(pb2lib):
    """Two beam batches per chunk (num_active_batches 2), nbatches_out 2, two non-synchronous
    consumers that release in different orders: every consumer sees, for every seq_id, the fp32
    oracle's outputs bit for bit."""
    cfg, plan, dd = _small(pb2lib, beams_per_gpu=4, beams_per_batch=2, num_active_batches=2, synchronous=False,
                           nbatches_out=2, num_consumers=2, release_timeout_ms=20000)
    orc, ws = _weights(cfg, 4, dd.nbatches_wt)
    for i, w in enumerate(ws):
        dd.fill_all_weights(i, w)
    nchunks = 3
    xs = H.make_inputs(cfg, nchunks, seed=9)
    _, ores = H.run_oracle(cfg, xs, ws, 1, 32)
    held = {0: [], 1: []}
    for seq, x in enumerate(xs):
        _launch(dd, seq, x)
        for c in (0, 1):
            out = dd.acquire_output(c, seq, sync=True)
            held[c].append(seq)
            assert out.ibeam == (seq % 2) * 2 and out.ichunk_zero_based == seq // 2
            for i in range(orc.ntrees):
                m = out.out_max[i].float().cpu().numpy().astype(np.float64)
                a = out.out_argmax[i].cpu().numpy().view(np.uint32)
                assert np.array_equal(m, ores[seq][0][i]), (c, seq, i)
                assert np.array_equal(a, ores[seq][1][i]), (c, seq, i)
        # consumer 0 releases at once; consumer 1 keeps one batch and releases it one step later
        dd.release_output(0, held[0].pop(0))
        if len(held[1]) == 2:
            dd.release_output(1, held[1].pop(0))
    while held[1]:
        dd.release_output(1, held[1].pop(0))


def test_batches_overlap_on_two_compute_streams(pb2lib):
    """Three beam batches per chunk on two compute streams (num_active_batches 2), every batch of a chunk
    launched before any output is read, so consecutive chunks of one batch alternate streams and the
    batches of a chunk overlap on the GPU. Outputs equal the fp32 oracle bit for bit, and each beam's
    candidate peak (per-stream reduction scratch) is its largest output over the trees."""
    import torch
    cfg, plan, dd = _small(pb2lib, beams_per_gpu=6, beams_per_batch=2, num_active_batches=2, synchronous=False,
                           nbatches_out=6, release_timeout_ms=20000)
    assert dd.num_compute_streams == 2
    orc, ws = _weights(cfg, 5, dd.nbatches_wt)
    for i, w in enumerate(ws):
        dd.fill_all_weights(i, w)
    dd.enable_sifter(threshold=1e30)
    nchunks, nb = 3, 3
    xs = H.make_inputs(cfg, nchunks, seed=10)
    _, ores = H.run_oracle(cfg, xs, ws, 1, 32)
    for ichunk in range(nchunks):
        seqs = range(ichunk * nb, (ichunk + 1) * nb)
        for seq in seqs:
            _launch(dd, seq, xs[seq])
        for seq in seqs:
            out = dd.acquire_output(0, seq, sync=True)
            assert out.ibeam == (seq % nb) * 2 and out.ichunk_zero_based == ichunk
            best = np.full(2, -np.inf)
            for i in range(orc.ntrees):
                m = out.out_max[i].float().cpu().numpy().astype(np.float64)
                a = out.out_argmax[i].cpu().numpy().view(np.uint32)
                assert np.array_equal(m, ores[seq][0][i]), (seq, i)
                assert np.array_equal(a, ores[seq][1][i]), (seq, i)
                best = np.maximum(best, m.reshape(2, -1).max(axis=1))
            peak = out.candidates["peak"].cpu().numpy().astype(np.float64)
            assert np.array_equal(peak, best), seq
            assert not out.candidates["valid"].cpu().numpy().any()
            dd.release_output(0, seq)
    torch.cuda.synchronize()


def _time_cfg(**kw):
    return H.toy_config(rank=8, nfreq=300, nt=512, dtype="float16", subbands=[2, 2, 1], beams_per_gpu=4,
                        beams_per_batch=2, num_active_batches=kw.pop("num_active_batches", 2))


def test_time_loop(pb2lib):
    """pirate's GpuDedisperser.time: int4 batches from pinned host memory through the public entry
    points, on two compute streams. Every iteration after the first reports a positive, finite real-time
    beam count; the cursors advance, so the streaming API carries on from seq_id = niterations, and the
    pybind11 surface runs the same loop."""
    import torch
    cfg = _time_cfg()
    plan = pb2lib.DedispersionPlan(pb2lib.DedispersionConfig.from_dict(cfg))
    dd = pb2lib.GpuDedisperser(plan, cuda_device_id=0, num_consumers=1)
    dd.allocate()
    dd.fill_analytic_weights(np.ones(plan.nfreq))
    rtb = dd.time(12)
    assert rtb.shape == (12,) and rtb[0] == 0
    assert np.all(np.isfinite(rtb[1:])) and np.all(rtb[1:] > 0)
    with dd.get_input() as x:          # seq_id 12
        x.zero_()
    with dd.get_output(0, sync=True) as out:
        assert out.ichunk_zero_based == 6 and out.ibeam == 0
    torch.cuda.synchronize()

    from pirate_b200 import _pirate_b200_pybind as pyb
    c = pyb.DedispersionConfig.from_yaml_string(pb2lib.DedispersionConfig.from_dict(cfg).to_yaml_string())
    d2 = pyb.GpuDedisperser(pyb.DedispersionPlan(c), cuda_device_id=0, num_consumers=1)
    d2.allocate()
    r2 = np.array(d2.time(6))
    assert r2[0] == 0 and np.all(r2[1:] > 0)


def test_time_loop_preconditions(pb2lib):
    """time() needs one consumer and more than 2 * num_active_batches iterations; a failing call stops
    the dedisperser, as pirate's entry points do."""
    cfg = _time_cfg()
    plan = pb2lib.DedispersionPlan(pb2lib.DedispersionConfig.from_dict(cfg))
    dd = pb2lib.GpuDedisperser(plan, cuda_device_id=0, num_consumers=2)
    dd.allocate()
    with pytest.raises(RuntimeError, match="num_consumers == 1"):
        dd.time(8)
    dd = pb2lib.GpuDedisperser(plan, cuda_device_id=0, num_consumers=1)
    dd.allocate()
    with pytest.raises(RuntimeError, match="niterations"):
        dd.time(4)
    _stopped(dd)
